"""Benchmark: vrad's lighting stage on the seeded 8x8 room grid, LDR and HDR.

One step = the lighting stage of one map in both ranges, as the reference
runs it with -both (vrad_light_pass_ranges_device), from the uploaded world
to the LIGHTING and LIGHTING_HDR lumps:
  direct  the fused direct gather over every light sample of the map (for
          each of its 5.68 M samples, every light of its cluster's list in
          gather order: shadow segments to 64 point and spot lights, the
          sun's sky test and 162 sky-ambient directions, traced in-kernel;
          one traversal lights both ranges), then each range's four
          supersampling passes;
  bounce  the transfer build once (every candidate patch pair's ray traced,
          form factors, scales), then per range the patches' direct light
          and the radiosity bounces to the stop threshold (0.1, the
          configuration's);
  final   per range the luxel radial filters of the direct and the bounced
          light, RGBE encode, medians, into its lump.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --workload seam     # the IRayTracer seam alone, rays in HBM
    python bench.py --workload transfer-cache   # the transfer cache's store and hit

Prints one JSON line (rank 0).  `value` is rays/s (the rays the reference
traces for the stage, over the device-timed step, all ranks) with the world
resident in HBM; `e2e` is the same through the C ABI's host-buffer entry
points with the inputs built, the scene, world and bounce uploaded and both
lumps read back inside every step.  `--impl reference` times the
reference's algorithm (the oracle's restatement) on the host cores.
Under torchrun each rank lights its own map (seed + rank): whole maps per
GPU, no data-path exchange; the batched workload deals its maps to the ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "vrad lighting stage rays/s (8x8 room grid, LDR+HDR, 1 B200)"
UNIT = "rays/s"
BYTES_PER_RAY = 28.0 + 0.125        # 28-byte ray record in, one hit bit out
CONFIG_SEED = 1
BOUNCE_THRESHOLD = 0.1      # the configuration's stop threshold (the reference's own default is 1.0)
MAX_BOUNCES = 100           # Radiosity.BounceAsync's default bounce limit


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--side", type=int, default=8, help=argparse.SUPPRESS)
    ap.add_argument("--workload", default="stage", choices=["stage", "seam", "ambient", "forward", "transfer-cache"])
    ap.add_argument("--ambient-samples", type=int, default=131072, help=argparse.SUPPRESS)
    ap.add_argument("--no-e2e", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-cpu", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-learned", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-batch", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-ambient", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--batch-maps", type=int, default=32, help=argparse.SUPPRESS)
    ap.add_argument("--batch-workers", type=int, default=4, help=argparse.SUPPRESS)
    return ap.parse_args()


def world_for(side: int, seed: int = CONFIG_SEED):
    from hl2sdk_tools_sharp_b200 import roomgrid as rg
    if side == 16:
        return rg.generate(rg.config_large(seed))
    cfg = rg.config_8x8(seed) if side == 8 else rg.config_3x3(seed)
    if side not in (3, 8):
        cfg.side = side
    return rg.generate(cfg)


def device_rays(world, device):
    """The full direct-light ray set, built on the device with torch, in
    face-coherent order (see workload.direct_rays)."""
    from hl2sdk_tools_sharp_b200 import workload as wl
    return wl.direct_rays_device(world, wl.luxel_samples(world), device)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        for r in rows:
            for name, col in (("hw_slowdown", 5), ("hw_thermal_slowdown", 6), ("sw_thermal_slowdown", 7),
                              ("sw_power_cap", 8)):
                if r[col].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_setup(gpus: int, backend: str = "nccl"):
    """One process per GPU (torchrun's environment); the process group is
    only the barrier and the max-over-ranks time: the ranks are replicas,
    each lighting its own map, with no data-path exchange."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        import torch
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_value(units_per_rank: float, ms_per_step: float, world: int) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return world * units_per_rank / (ms_per_step / 1000.0)


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def host_sample(rays: dict, total: int, cap: int = 16_000_000) -> dict:
    """Every k-th ray of each kind (the same k for all), at most `cap` rays,
    copied to host memory; the CPU leg samples within this."""
    stride = max(1, -(-total // cap))
    return {k: rays[k][::stride].cpu().numpy() for k in ("light", "sun", "sky")}


def cpu_reference(world_map, rays_np: dict, total: int, budget_s: float = 20.0):
    """The reference's algorithm on the host: the restated KD build and
    packet walk (oracle), all host threads, on a bounded sample of each ray
    kind in proportion to the full workload."""
    from oracle import oracle as O
    threads = O.default_threads()
    tree = O.kd_build(world_map.tri_verts, world_map.tri_ids)
    pool = sum(len(v) for v in rays_np.values())
    # Calibrate on a small sample, then size the timed sample to the budget.
    def run(frac):
        n = 0
        t0 = time.perf_counter()
        for kind, rays in rays_np.items():
            k = max(64, int(len(rays) * frac))
            sel = rays[:: max(1, len(rays) // k)][:k]
            flags = 0 if kind == "light" else O.SKY_PASS
            O.kd_trace(tree, sel, flags=flags, threads=threads)
            n += len(sel)
        return n, time.perf_counter() - t0
    n, dt = run(min(1.0, 2e5 / pool))
    frac = min(1.0, (2e5 / pool) * budget_s / max(dt, 1e-3))
    n, dt = run(frac)
    return {"value": n / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} rays ({100.0 * n / total:.2f}% of each ray kind, strided) of the "
                      f"8x8 direct-light workload; restated KD build + 4-ray packet walk"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import torch
    w = world_for(args.side)
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    rays = device_rays(w, dev)
    total = sum(int(rays[k].shape[0]) for k in ("light", "sun", "sky"))
    rays_np = host_sample(rays, total)
    vals, walls = [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        cb = cpu_reference(w, rays_np, total, budget_s=max(3.0, 60.0 / max(1, args.warmup + args.steps)))
        if i >= args.warmup:
            vals.append(cb["value"])
            walls.append(time.perf_counter() - t0)
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.median(walls),
        "seconds_per_full_step_extrapolated": total / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded room grid)",
        "config": {"workload": "8x8 room grid direct-lighting rays (light + sun + 162-dir sky)",
                   "rays_per_step": total, "seed": CONFIG_SEED},
        "cpu_baseline": {**cb, "value": value},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main_seam(args):
    import torch
    from hl2sdk_tools_sharp_b200 import tracer as T
    rank, world_size, local = dist_setup(args.gpus)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)

    w = world_for(args.side)
    tr = T.CudaRayTracer(T.make_triangles(w.tri_verts, w.tri_ids), device=local)
    info = tr.scene_info()
    rays = device_rays(w, device)
    kinds = [("light", T.RayTraceOptions.stock_exact()),
             ("sun", T.RayTraceOptions(0.0, sky_does_not_block=True)),
             ("sky", T.RayTraceOptions(0.0, sky_does_not_block=True))]
    bits = {k: torch.zeros((rays[k].shape[0] + 63) // 64 + 1, dtype=torch.int64, device=device)
            for k, _ in kinds}
    total = sum(rays[k].shape[0] for k, _ in kinds)

    def step():
        for k, o in kinds:
            tr.trace_visibility(rays[k], bits[k], o)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()

    # Spot-check the resident results against the oracle on a sample.
    check = None
    if rank == 0 and not args.no_cpu:
        from oracle import oracle as O
        tris = O.prepare_triangles(w.tri_verts, w.tri_ids)
        bad = 0
        checked = 0
        for k, o in kinds:
            n = rays[k].shape[0]
            idx = np.arange(0, n, max(1, n // 20000))[:20000]
            sel = rays[k][torch.from_numpy(idx).to(device)].cpu().numpy()
            _, _, bb = O.brute_trace(tris, sel, flags=O.SKY_PASS if o.sky_does_not_block else 0)
            want = O.bits_to_bool(bb, len(sel))
            allbits = bits[k].cpu().numpy().view(np.uint64)
            got = O.bits_to_bool(allbits, n)[idx]
            bad += int((got != want).sum())
            checked += len(sel)
        check = {"rays": checked, "mismatches": bad}

    # Timed region: K steps, events on the launching (current) stream.
    stream = torch.cuda.current_stream(device)
    barrier(world_size)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps)]
    with ClockSampler(local) as clocks:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for s in range(args.steps):
            ev[2 * s].record(stream)
            step()
            ev[2 * s + 1].record(stream)
        t1.record(stream)
        torch.cuda.synchronize()
    barrier(world_size)
    elapsed_ms = t0.elapsed_time(t1)
    elapsed_ms = max_over_ranks(elapsed_ms, world_size)
    per_step = [ev[2 * s].elapsed_time(ev[2 * s + 1]) for s in range(args.steps)]
    ms_per_step = elapsed_ms / args.steps
    value = world_size * total / (ms_per_step / 1000.0)

    # Per-kind kernel times (one launch per kind) for the roofline.
    kt = {}
    for k, o in kinds:
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(3):
            tr.trace_visibility(rays[k], bits[k], o)
        b.record(stream)
        torch.cuda.synchronize()
        kt[k] = a.elapsed_time(b) / 3.0

    # End to end through the host-buffer C ABI: pinned host rays in, bits out.
    e2e = None
    if not args.no_e2e:
        host = {k: torch.empty(rays[k].shape, dtype=torch.float32, pin_memory=True) for k, _ in kinds}
        hbits = {k: torch.zeros(((rays[k].shape[0] + 63) // 64,), dtype=torch.int64, pin_memory=True)
                 for k, _ in kinds}
        for k, _ in kinds:
            host[k].copy_(rays[k])
        hv = {k: host[k].numpy().view(T.RAY_DTYPE).reshape(-1) for k, _ in kinds}
        hb = {k: hbits[k].numpy().view(np.uint64) for k, _ in kinds}
        def e2e_step():
            for k, o in kinds:
                tr.trace_visibility(hv[k], hb[k], o)
        e2e_step()
        torch.cuda.synchronize()
        barrier(world_size)
        t = time.perf_counter()
        e2e_steps = max(1, min(args.steps, 3))
        for _ in range(e2e_steps):
            e2e_step()
        e2e_s = (time.perf_counter() - t) / e2e_steps
        e2e_s = max_over_ranks(e2e_s, world_size)
        e2e = {"value": world_size * total / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(sum(host[k].numel() * 4 for k, _ in kinds)),
               "d2h_bytes_per_step": int(sum(8 * ((rays[k].shape[0] + 63) // 64) for k, _ in kinds))}
        del host, hbits

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu:
        cpu = cpu_reference(w, host_sample(rays, total), total, budget_s=15.0)

    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))

    # The learned warm start: a network trained on the device on plain
    # bounce solutions of eight small seeded maps (2 to 6 rooms a side),
    # then this map bounced from its guess, against the plain bounce.
    learned = None
    if rank == 0 and not args.no_learned:
        from hl2sdk_tools_sharp_b200 import learned as LN
        t = time.perf_counter()
        lx, lt = LN.collect([LN.training_config(k) for k in range(8)], threshold=BOUNCE_THRESHOLD)
        collect_s = time.perf_counter() - t
        net = LN.Network(stage.tracer, seed=7)
        ta, tb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ta.record(stream)
        loss = LN.train(net, lx, lt, steps=3000)
        tb.record(stream)
        torch.cuda.synchronize()
        train_ms = ta.elapsed_time(tb)
        stage.set_bounce_model(net)
        warm_lump, _, _ = stage.light_pass()
        bw = stage.bounce_stats()
        stage.set_bounce_model(None)
        hx, ht = stage.bounce_features()
        for _ in range(3):
            net.forward(hx)
        ta.record(stream)
        for _ in range(10):
            y = net.forward(hx)
        tb.record(stream)
        torch.cuda.synchronize()
        fwd_ms = ta.elapsed_time(tb) / 10
        flops = 2.0 * (32 * 128 + 128 * 128 + 128 * 8) * len(hx)
        tpeak = float(peaks.get("bf16_tflops", 1590.0))
        learned = {"plain_bounces": int(bst.bounces), "warm_bounces": int(bw.bounces),
                   "plain_bounce_ms": statistics.median([p[2] for p in phases]), "warm_bounce_ms": bw.bounce_ms,
                   "iteration_ratio": bst.bounces / max(1, bw.bounces),
                   "lightmap_within_1_lsb": LN.within_one_lsb(warm_lump, lump_host),
                   "guess_abs_error_log1p": float((y - ht).abs().mean().item()),
                   "training": {"maps": 8, "rows": int(len(lx)), "steps": 3000, "batch": 32768,
                                "collect_s": collect_s, "train_ms": train_ms, "final_loss": loss},
                   "roofline": {"bound": "tensor", "kernel": "k_mlp_forward_tc (tcgen05.mma kind::f16, bf16 in, fp32 in TMEM)",
                                "achieved": flops / (fwd_ms / 1000.0) / 1e12, "peak": tpeak, "unit": "TFLOP/s",
                                "frac": flops / (fwd_ms / 1000.0) / 1e12 / tpeak, "rows": int(len(hx)),
                                "ms": fwd_ms, "flops_per_row": flops / len(hx)}}
        net.close()
    sky_ms = kt["sky"]
    achieved = BYTES_PER_RAY * rays["sky"].shape[0] / (sky_ms / 1000.0) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None,
                "kernel": "k_trace<kModeSkyPass> (sky segments)",
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded room grid, rays built on the device)",
            "config": {"workload": "8x8 room grid direct-lighting rays (light + sun + 162-dir sky)",
                       "side": args.side, "seed": CONFIG_SEED, "luxels": rays["luxels"],
                       "triangles": info.triangles, "rays_per_step": total,
                       "rays": {k: int(rays[k].shape[0]) for k, _ in kinds},
                       "l2": "inputs larger than L2 (rays ~%.1f GB per step)" % (28 * total / 1e9),
                       "parallelism": f"replicas{world_size}"},
            "e2e": e2e,
            "gpu_launches": 3 * args.steps,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "kernel_ms": kt,
            "step_ms": per_step,
            "bvh": {"nodes": info.bvh_nodes, "leaves": info.bvh_leaves, "max_leaf": info.max_leaf, "depth": info.bvh_depth,
                    "build_ms": info.build_ms, "pad": info.box_pad},
            "check": check,
            "learned": learned,
        }
        print(json.dumps(line), flush=True)
    tr.close()
    if world_size > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def oracle_faces_sample(world, inp, stride: int, phase: int = 0):
    """Every `stride`-th face (from `phase`) with its samples, renumbered,
    for the CPU legs."""
    sel = np.arange(phase % max(1, stride), len(inp.faces), max(1, stride))
    ff = inp.face_first
    parts = [inp.samples[ff[f]:ff[f + 1]] for f in sel]
    counts = np.array([len(p) for p in parts])
    first = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    samples = np.concatenate(parts).copy()
    samples["face"] = np.repeat(np.arange(len(sel)), counts)
    index = np.concatenate([np.arange(ff[f], ff[f + 1]) for f in sel])
    return sel, samples, first, index


def cpu_direct(world, inp, lights, tree, budget_s: float, phase: int = 0):
    """The reference's direct gather for one range (its light list) on the
    host: the restated KD walk and four-sample-group gather with its
    supersampling passes, all host threads, on a strided sample of faces
    sized to about budget_s.  (samples/s, segments/s, description)."""
    from oracle import oracle as O
    threads = O.default_threads()

    def run(stride, ph):
        sel, samples, first, _ = oracle_faces_sample(world, inp, stride, ph)
        t0 = time.perf_counter()
        _, rays = O.direct(tree, inp.faces[sel], samples, first, lights, inp.cluster_offsets, inp.cluster_lights,
                           inp.sky_directions, inp.sun_jitter, inp.sun_samples, inp.sun_angular_extent,
                           threads=threads, count_rays=True, verts=inp.verts)
        return rays, len(samples), time.perf_counter() - t0, len(sel)
    rays, n, dt, nf = run(max(1, len(inp.faces) // 64), phase)
    stride = max(1, int(len(inp.faces) / max(1.0, nf * budget_s / max(dt, 1e-3))))
    rays, n, dt, nf = run(stride, phase)
    return n / dt, rays / dt, f"{nf} of {len(inp.faces)} faces (every {stride}th), {n} samples, {rays} segments"


def cpu_transfers(ob, budget_s: float = 10.0, phase: int = 0):
    """The transfer build restated (candidate walk, KD-traced rays, form
    factors) on a strided sample of receivers: (transfer rays/s, description)."""
    patches, _ = ob.patches()
    leaves = np.flatnonzero(patches["child1"] == -1)

    def run(stride, ph):
        sub = leaves[ph % stride::stride]
        ob.forget_transfers()
        t0 = time.perf_counter()
        _, _, _, rays = ob.transfers(sub)
        return rays, time.perf_counter() - t0, len(sub)
    rays, dt, n = run(max(1, len(leaves) // 400), 1)
    stride = max(1, int(len(leaves) / max(1.0, n * budget_s / max(dt, 1e-3))))
    rays, dt, n = run(stride, phase)
    return rays / dt, f"{n} of {len(leaves)} receivers (every {stride}th), {rays} transfer rays"


def world_and_inputs(side, seed=CONFIG_SEED):
    """The map and the stage's inputs for both ranges, through the library's
    host builders (the native sample builder)."""
    from hl2sdk_tools_sharp_b200 import lighting as L
    w = world_for(side, seed)
    return w, L.prepare(w, hdr=True)


def reference_inputs(world):
    """The same inputs built without the CUDA library: faces and both light
    lists by the host layer's pure-Python builders, samples by the oracle's
    FaceSampleBuilder restatement (bit-identical to the native builder,
    tests/test_lighting_cpu.py)."""
    from hl2sdk_tools_sharp_b200 import lighting as L, workload as wl
    from oracle import oracle as O
    faces, verts = L.faces_of(world)
    raw, first = O.build_samples(faces, verts)
    lights, off, flat = L.build_lights(world)
    lights_hdr, _, _ = L.build_lights(world, hdr=True)
    return L.LightingInputs(faces, verts, raw.view(L.SAMPLE_DTYPE), first, lights, off, flat,
                            wl.ambient_directions().astype(np.float32), np.zeros((0, 3), np.float32),
                            lights_hdr=lights_hdr)


def oracle_bounce(world, inp, tree=None, bounces=MAX_BOUNCES, threshold=BOUNCE_THRESHOLD):
    """The oracle's bounce over the world (patches built, nothing traced)."""
    from hl2sdk_tools_sharp_b200 import lighting as L
    from oracle import oracle as O
    tree = tree if tree is not None else O.kd_build(world.tri_verts, world.tri_ids)
    off, lst = L.pvs_lists(world)
    return O.Bounce(tree, inp.faces, inp.verts, inp.samples, inp.face_first, L.face_reflectivity(world), off, lst,
                    bounces=bounces, threshold=threshold)


WORKLOAD = ("8x8 room grid lighting stage, LDR and HDR ranges: per range the direct gather (64 point/spot "
            "lights, sun, 162-dir sky, 4 supersampling passes), the bounce (patch light, radiosity to threshold "
            "0.1) and the final pass into LIGHTING / LIGHTING_HDR; one transfer build for both ranges")


WORKLOAD_LARGE = ("16x16 room grid lighting stage (the large configuration without displacements or ambient "
                  "occlusion), LDR and HDR ranges: per range the direct gather (256 point/spot lights, a sun of 256 "
                  "jittered rays, 162-dir sky, 4 supersampling passes), the bounce (patch light, radiosity to "
                  "threshold 0.1) and the final pass into LIGHTING / LIGHTING_HDR; one transfer build for both ranges")


def stage_config(args):
    """The workload's defining keys, the same in both arms."""
    work = WORKLOAD_LARGE if args.side == 16 else (WORKLOAD if args.side == 8 else f"{args.side}x{args.side} "
                                                   "room grid lighting stage, LDR and HDR ranges")
    return {"workload": work, "side": args.side, "seed": CONFIG_SEED, "ranges": "LDR+HDR",
            "bounce_threshold": BOUNCE_THRESHOLD, "max_bounces": MAX_BOUNCES,
            "l2": "no L2 flush: the 0.3 GB sample set and 5 GB of candidate pairs exceed L2",
            "parallelism": f"replicas{args.gpus} (one map per rank, seed {CONFIG_SEED} + rank)"}


def run_reference_stage(args):
    """The reference's algorithm on the host cores (the oracle, a C++
    restatement of the reference's C#, which cannot run here), all host
    threads, on the GPU arm's workload.  Set-up (untimed): the inputs
    without the CUDA library, the KD tree, both ranges' full direct gather,
    the full transfer build, and each range's bounce and final pass timed
    whole once.  Each step then times a bounded sample of the ray-tracing
    parts (both ranges' direct gathers on a strided face sample, the
    transfer build on a strided receiver sample); value = the stage's rays
    over the stage seconds those rates and the whole-pass timings give.
    ms_per_step is the wall time a step took."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O
    t_setup = time.perf_counter()
    w = world_for(args.side)
    inp = reference_inputs(w)
    threads = O.default_threads()
    tree = O.kd_build(w.tri_verts, w.tri_ids)
    ranges = {"ldr": inp.lights, "hdr": inp.lights_hdr}
    light, direct_rays = {}, {}
    for r, lights in ranges.items():
        light[r], direct_rays[r] = O.direct(tree, inp.faces, inp.samples, inp.face_first, lights, inp.cluster_offsets,
                                            inp.cluster_lights, inp.sky_directions, inp.sun_jitter, inp.sun_samples,
                                            inp.sun_angular_extent, threads=threads, count_rays=True,
                                            verts=inp.verts)
    ob = oracle_bounce(w, inp, tree)
    t = time.perf_counter()
    t_off, t_src, t_w, transfer_rays = ob.transfers()
    transfer_full_s = time.perf_counter() - t
    whole = {}
    for r in ranges:
        t = time.perf_counter()
        _, _, nb, _ = ob.run(light[r])
        bounce_s = time.perf_counter() - t
        t = time.perf_counter()
        ob.final(light[r])
        whole[r] = {"bounces": int(nb), "bounce_s": bounce_s, "final_s": time.perf_counter() - t}
    setup_s = time.perf_counter() - t_setup
    rays_per_step = int(direct_rays["ldr"] + direct_rays["hdr"] + transfer_rays)
    vals, walls, stages = [], [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        rates = {r: cpu_direct(w, inp, lights, tree, 0.5, phase=i) for r, lights in ranges.items()}
        t_rate, t_sample = cpu_transfers(ob, budget_s=0.6, phase=i)
        wall = time.perf_counter() - t0
        stage_s = (sum(len(inp.samples) / rates[r][0] for r in ranges) + transfer_rays / t_rate
                   + sum(whole[r]["bounce_s"] + whole[r]["final_s"] for r in ranges))
        if i >= args.warmup:
            vals.append(rays_per_step / stage_s)
            walls.append(wall)
            stages.append(stage_s)
    value = statistics.median(vals)
    sample = (f"per step: LDR gather {rates['ldr'][2]}; HDR gather {rates['hdr'][2]}; transfer build {t_sample}; "
              f"the bounce and final pass of each range timed whole once at set-up "
              f"(LDR {whole['ldr']['bounces']} bounces {whole['ldr']['bounce_s']:.2f} s + final "
              f"{whole['ldr']['final_s']:.2f} s, HDR {whole['hdr']['bounces']} bounces "
              f"{whole['hdr']['bounce_s']:.2f} s + final {whole['hdr']['final_s']:.2f} s)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.median(walls),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded room grid)",
        "config": stage_config(args),
        "stage_s_extrapolated": statistics.median(stages),
        "rays_per_step": rays_per_step,
        "setup_s": setup_s, "transfer_build_whole_s": transfer_full_s,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def deal_maps(weights, world: int) -> list:
    """Whole maps dealt to `world` ranks, largest first, each to the rank
    with the least weight so far (LPT); ties to the lowest rank.  Returns
    each rank's map indices in dealing order."""
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in sorted(range(len(weights)), key=lambda k: (-weights[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += weights[i]
    return out


def batched_run(args, device_index: int, rank: int = 0, world: int = 1) -> dict:
    """The batched workload: `batch_maps` seeded room grids, sides drawn
    from 2..10 rooms, each bounced to the 8x8 map's threshold, lit by the
    native batch runner (host buffers in and out, every map's scene, world
    and bounce uploaded inside the timed run).  Across ranks the maps are
    dealt whole (deal_maps, weighted by rooms), with no exchange: each rank
    lights its share, and the job takes the slowest rank's time.  The
    autotuner picks the gather's launch shape and the maps in flight on the
    first eight maps of the share; one warm-up run, then the timed run, then
    the same maps on one worker."""
    from hl2sdk_tools_sharp_b200 import batch as B, roomgrid as rg
    out = {}
    try:
        t = time.perf_counter()
        cfgs = [rg.config_batch(i, seed=CONFIG_SEED) for i in range(args.batch_maps)]
        mine = deal_maps([c.side ** 2 for c in cfgs], world)[rank]
        cfgs = [cfgs[i] for i in mine]
        maps = [B.map_inputs(rg.generate(c), bounces=MAX_BOUNCES, threshold=BOUNCE_THRESHOLD) for c in cfgs]
        prep_s = time.perf_counter() - t
        with B.LightingBatch(workers=args.batch_workers, device=device_index) as batch:
            workers, block, tune = batch.autotune(maps[:min(8, len(maps))])
            warm, _ = batch.run(maps)
            results, st = batch.run(maps)
            one, st1 = batch.run(maps, workers=1)
        same = all(np.array_equal(a.lighting, b.lighting) and np.array_equal(a.lighting, c.lighting)
                   for a, b, c in zip(results, warm, one))
        out = {"maps": len(maps), "map_indices": mine, "sides": [c.side for c in cfgs],
               "rooms": int(sum(c.side ** 2 for c in cfgs)),
               "triangles": int(sum(len(m.triangles) for m in maps)),
               "samples": int(sum(len(m.inputs.samples) for m in maps)),
               "workers": st.workers, "threads_per_cta": st.block, "autotune_s": tune,
               "seconds": st.seconds, "busy_seconds": st.busy_seconds, "one_worker_s": st1.seconds,
               "rays": int(st.rays), "rays_per_s": st.rays / st.seconds, "luxels": int(st.luxels),
               "luxels_per_s": st.luxels / st.seconds, "lighting_bytes": int(st.lighting_bytes),
               "map_s": {"min": min(r.seconds for r in results), "max": max(r.seconds for r in results)},
               "lumps_equal_across_runs": bool(same), "host_prep_s": prep_s,
               "note": "wall clock of vrad_batch_run: per map the scene, world and bounce uploads from host "
                       "arrays, the light pass, the lump read back to host memory; host_prep_s (the maps' "
                       "generation in Python) is outside it"}
    except Exception as exc:  # reported in the line; the headline still prints
        out = {"error": f"{type(exc).__name__}: {exc}"}
    # Every rank takes the same collective steps, with or without an error.
    secs = out.get("seconds", 0.0)
    job_s = max_over_ranks(secs, world)
    job_rays = sum_over_ranks(out.get("rays", 0), world)
    if world > 1:
        out = {"rank0": out, "ranks": world, "job_seconds": job_s, "job_rays": int(job_rays),
               "job_rays_per_s": job_rays / job_s if job_s > 0 else None,
               "split": "whole maps per rank, dealt largest first by rooms; no collective on the data path"}
    return out


# Per launch DRAM traffic of the dominant kernels, from one ncu capture each
# (dram__bytes_read.sum + dram__bytes_write.sum over the units that launch
# processed), scaled by the units a full launch processes.  The captures
# and their commands: profiles/k_transfer_4x4_roomgrid.md,
# profiles/k_direct_4x4_roomgrid.md.
TRAFFIC_PER_TRANSFER_RAY = (92441088 + 49963008) / 19922134.0


def lockdown_ambient_lumps(seed: int = 3) -> dict:
    """dm_lockdown's geometry lumps (the committed fixture) with a seeded
    synthetic lighting lump, texture reflectivities and a sky ambient light:
    the fixture keeps the map's geometry, not its 6 MB lighting."""
    from hl2sdk_tools_sharp_b200 import ambient as A, bsp as B
    from tests.golden import fixtures as F
    lumps = dict(F.lockdown_lumps())
    rng = np.random.default_rng(seed)
    faces = np.frombuffer(lumps[B.LUMP_FACES][1], B.FACE)
    texinfo = np.frombuffer(lumps[B.LUMP_TEXINFO][1], B.TEXINFO)
    ntex = int(texinfo["texdata"].max()) + 1
    td = np.zeros(ntex, A.TEXDATA)
    td["reflectivity"] = rng.uniform(0.05, 0.9, (ntex, 3)).astype(np.float32)
    styles = (faces["styles"] != 255).sum(1)
    size = (faces["lm_size"][:, 0].astype(np.int64) + 1) * (faces["lm_size"][:, 1] + 1) * 4 * np.maximum(styles, 1)
    end = int(np.max(np.where(faces["lightofs"] >= 0, faces["lightofs"] + 4 * size, 0)))
    light = rng.integers(0, 256, end + 64, dtype=np.uint8)
    light[3::4] = rng.integers(-9, 3, len(light[3::4])).astype(np.int8).view(np.uint8)
    wl = np.zeros(2, A.WORLDLIGHT)
    wl["type"] = (1, A.EMIT_SKYAMBIENT)
    wl["intensity"][1] = (0.25, 0.5, 0.75)
    lumps[B.LUMP_TEXDATA] = (0, td.tobytes())
    lumps[B.LUMP_LIGHTING] = (1, light.tobytes())
    lumps[A.LUMP_WORLDLIGHTS] = (0, wl.tobytes())
    return lumps


def ambient_run(args, samples: int = 131072) -> dict:
    """The leaf ambient ray cubes (vrad_ambient_cubes) on dm_lockdown's
    geometry: `samples` seeded points in its open leaves, 162 rays each,
    timed on the device (inputs resident) and end to end through the host
    call; the first 2,048 cubes checked against the oracle, which is also
    timed on a bounded sample on the host's cores."""
    import torch
    from hl2sdk_tools_sharp_b200 import ambient as A, bsp as B
    lumps = lockdown_ambient_lumps()
    leaves = np.frombuffer(lumps[B.LUMP_LEAFS][1], B.LEAF_V0 if lumps[B.LUMP_LEAFS][0] == 0 else B.LEAF_V1)
    open_ = leaves[(leaves["contents"] & A.CONTENTS_SOLID) == 0]
    rng = np.random.default_rng(17)
    pick = open_[rng.integers(0, len(open_), samples)]
    u = rng.uniform(0.02, 0.98, (samples, 3))
    pos = (pick["mins"] + u * (pick["maxs"].astype(np.float64) - pick["mins"])).astype(np.float32)
    out = {"workload": f"dm_lockdown geometry ({len(np.frombuffer(lumps[B.LUMP_NODES][1], B.NODE))} nodes, "
                       f"{len(np.frombuffer(lumps[B.LUMP_FACES][1], B.FACE))} faces), seeded synthetic lighting, "
                       f"{samples} seeded points in open leaves x 162 rays",
           "samples": samples, "rays": samples * A.DIRECTIONS}
    with A.CudaAmbientSampler(lumps) as s:
        stream = torch.cuda.current_stream()
        d_pos = torch.from_numpy(pos).cuda()
        d_out = torch.empty((samples, A.SIDES, 3), dtype=torch.float32, device="cuda")
        for _ in range(2):
            s.cubes_device(d_pos, out=d_out, stream=stream.cuda_stream)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 5
        a.record(stream)
        for _ in range(reps):
            s.cubes_device(d_pos, out=d_out, stream=stream.cuda_stream)
        b.record(stream)
        torch.cuda.synchronize()
        s.status()
        ms = a.elapsed_time(b) / reps
        t = time.perf_counter()
        host = s.cubes(pos)
        e2e_s = time.perf_counter() - t
    out.update({"ms": ms, "rays_per_s": out["rays"] / (ms / 1000.0), "samples_per_s": samples / (ms / 1000.0),
                "e2e": {"s": e2e_s, "rays_per_s": out["rays"] / e2e_s, "h2d_bytes": int(pos.nbytes),
                        "d2h_bytes": int(host.nbytes)},
                "gpu_launches_per_call": 2 * ((samples + 16383) // 16384)})
    if not args.no_cpu:
        from oracle import oracle as O
        geom = B.trace_geometry(lumps)
        r = A.ambient_range(lumps, False)
        check = 2048
        threads = O.default_threads()
        t = time.perf_counter()
        want = O.ambient_cubes(geom, r.faces, r.lighting, A.anorms(), float(A.cone_tan()), r.sky_ambient,
                               pos[:check], threads=threads)
        cpu_s = time.perf_counter() - t
        out["check"] = {"samples": check,
                        "mismatched_samples": int((host[:check].view(np.uint32) != want.view(np.uint32))
                                                  .any(axis=(1, 2)).sum())}
        out["cpu_baseline"] = {"kind": "port", "cores": threads, "sample": f"{check} samples x 162 rays",
                               "rays_per_s": check * A.DIRECTIONS / cpu_s}
    return out


def recheck_run(world, stride: int = 7) -> dict:
    """The FP64 recheck (vrad_trace_visibility_recheck) over the light rays
    of every `stride`-th luxel of the map (point, spot and sun segments;
    the sky pass-through mode is outside the recheck): how many rays the
    FP32 values flag, their FP64 classes, and the FP32/FP64 disagreements."""
    from hl2sdk_tools_sharp_b200 import tracer as T, workload as wl
    s = wl.luxel_samples(world, stride=stride)
    rays = np.ascontiguousarray(wl.direct_rays(world, s, ambient=False).light)
    with T.CudaRayTracer(T.make_triangles(world.tri_verts, world.tri_ids)) as tr:
        t = time.perf_counter()
        vis, _, st = tr.visibility_recheck(rays, T.RayTraceOptions.stock_exact())
        wall = time.perf_counter() - t
    st.update({"sample": f"light rays of every {stride}th luxel", "blocked": int(vis.sum()), "call_s": wall,
               "flag_margin": 1e-3, "fp64_margin": 1e-6})
    return st


def main_stage(args):
    import torch
    from hl2sdk_tools_sharp_b200 import lighting as L, tracer as T
    rank, world_size, local = dist_setup(args.gpus)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)

    # Weak scaling over whole maps: rank r lights its own map (seed + r),
    # no data-path exchange (rank 0's is the single-GPU workload).
    w, inp = world_and_inputs(args.side, CONFIG_SEED + rank)
    n = len(inp.samples)
    refl = L.face_reflectivity(w)
    pvs_off, pvs_list = L.pvs_lists(w)
    tris = T.make_triangles(w.tri_verts, w.tri_ids)
    stage = L.LightingStage(w, inp, device=local)
    stage.upload_bounce(refl, pvs_off, pvs_list, bounces=MAX_BOUNCES, threshold=BOUNCE_THRESHOLD)
    info = stage.tracer.scene_info()
    block, tune_ms = stage.autotune()                # picks the launch shape (untimed)
    # Ray counts: each range lit alone (the reference's passes: each range
    # traces its own direct segments, the first builds the transfers), and
    # both at once (what one step traces: the first gather round once).
    _, _, _, st_l, bs_l = stage.light_pass_ranges(L.RANGE_LDR)
    _, _, _, st_h, _ = stage.light_pass_ranges(L.RANGE_HDR)
    ldr_host, hdr_host, _, pstats, bst = stage.light_pass_ranges()
    transfer_rays = int(bst[0].transfer_rays)
    rays_per_step = int(st_l.visibility_rays + st_l.sky_rays + st_h.visibility_rays + st_h.sky_rays) + transfer_rays
    traced_per_step = int(pstats.visibility_rays + pstats.sky_rays) + transfer_rays
    luxels = int(pstats.luxels)
    nbytes = len(ldr_host)
    d_ldr = torch.empty(nbytes, dtype=torch.uint8, device=device)
    d_hdr = torch.empty(nbytes, dtype=torch.uint8, device=device)
    d_out = torch.empty(n * 4, dtype=torch.float32, device=device)
    for _ in range(max(3, args.warmup)):
        stage.light_pass_ranges_device(d_ldr, d_hdr)
    torch.cuda.synchronize()

    check = None
    cpu_parts = {}
    if rank == 0 and not args.no_cpu:
        # Parity on this run's own output: per range a strided sample of
        # faces through the oracle's direct gather, a sample of receivers
        # through its transfer build, and each whole lump through its bounce
        # and final pass fed the device's sample light and transfers (each
        # pinned by those samples); the bounce and final pass timed here are
        # the CPU baseline's.
        from oracle import oracle as O
        tree = O.kd_build(w.tri_verts, w.tri_ids)
        got = {"ldr": stage.pass_sample_light(L.RANGE_LDR), "hdr": stage.pass_sample_light(L.RANGE_HDR)}
        got = {r: np.concatenate([v["lighting"], v["direct_sun_amount"][:, None]], 1) for r, v in got.items()}
        t_off, t_rec = stage.transfers()
        sel, samples, first, index = oracle_faces_sample(w, inp, 97)
        check = {"samples": int(len(index))}
        for r, lights in (("ldr", inp.lights), ("hdr", inp.lights_hdr)):
            want = O.direct(tree, inp.faces[sel], samples, first, lights, inp.cluster_offsets,
                            inp.cluster_lights, inp.sky_directions, inp.sun_jitter, inp.sun_samples,
                            inp.sun_angular_extent, verts=inp.verts)
            check[f"{r}_mismatches"] = int((got[r][index].view(np.uint32) != want.view(np.uint32)).any(1).sum())
        ob = oracle_bounce(w, inp, tree)
        patches, _ = ob.patches()
        leaves = np.flatnonzero(patches["child1"] == -1)
        sub = leaves[::max(1, len(leaves) // 200)]
        o_off, o_src, o_w, _ = ob.transfers(sub)
        tr_bad = 0
        for p in sub:
            a, b = t_off[p], t_off[p + 1]
            c, d = o_off[p], o_off[p + 1]
            tr_bad += int(not (np.array_equal(t_rec["patch"][a:b], o_src[c:d])
                               and np.array_equal(t_rec["weight"][a:b].view(np.uint32), o_w[c:d].view(np.uint32))))
        check.update({"receivers": int(len(sub)), "receiver_mismatches": tr_bad})
        ob.set_transfers(t_off, t_rec["patch"], t_rec["weight"])
        for r, lump in (("ldr", ldr_host), ("hdr", hdr_host)):
            t = time.perf_counter()
            _, _, o_bounces, _ = ob.run(got[r])
            cpu_parts[f"bounce_{r}_s"] = time.perf_counter() - t
            t = time.perf_counter()
            lump_want, _ = ob.final(got[r])
            cpu_parts[f"final_{r}_s"] = time.perf_counter() - t
            check[f"{r}_bounces"] = int(bst[0 if r == "ldr" else 1].bounces)
            check[f"{r}_oracle_bounces"] = int(o_bounces)
            check[f"{r}_lump_words"] = int(len(lump_want) // 4)
            check[f"{r}_lump_mismatches"] = int((lump.view(np.uint32) != lump_want.view(np.uint32)).sum())
        del t_rec

    stream = torch.cuda.current_stream(device)
    barrier(world_size)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps)]
    phases = []
    with ClockSampler(local) as clocks:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for s_ in range(args.steps):
            ev[2 * s_].record(stream)
            stage.light_pass_ranges_device(d_ldr, d_hdr)
            ev[2 * s_ + 1].record(stream)
            b = stage.bounce_stats_ranges()
            phases.append((b[0].patch_light_ms + b[1].patch_light_ms, b[0].transfer_ms,
                           b[0].bounce_ms + b[1].bounce_ms, b[0].bounces, b[1].bounces))
        t1.record(stream)
        torch.cuda.synchronize()
    barrier(world_size)
    elapsed_ms = max_over_ranks(t0.elapsed_time(t1), world_size)
    per_step = [ev[2 * k].elapsed_time(ev[2 * k + 1]) for k in range(args.steps)]
    ms_per_step = elapsed_ms / args.steps
    job_rays = sum_over_ranks(rays_per_step, world_size)
    value = job_rays / (ms_per_step / 1000.0)
    # End to end through the host-buffer C ABI, every step: the stage's
    # inputs built on the host (faces, the samples by the native builder,
    # both ranges' light lists from the entities), the scene (intersection
    # form and BVH), the world and the bounce uploaded, and both ranges lit
    # with their lumps read back into pinned memory.
    e2e = None
    if not args.no_e2e:
        from hl2sdk_tools_sharp_b200 import workload as wl
        out_ldr = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True).numpy()
        out_hdr = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True).numpy()
        sample_buf = np.empty(n + 64, L.SAMPLE_DTYPE)   # reused from map to map
        parts = {"inputs": [], "upload_scene": [], "upload_world": [], "upload_bounce": [], "light_pass": []}
        h2d = []

        def e2e_step():
            t0 = time.perf_counter()
            i2 = L.prepare(w, hdr=True, sample_out=sample_buf)
            faces, verts, samples, lights, lights_hdr = i2.faces, i2.verts, i2.samples, i2.lights, i2.lights_hdr
            off, flat = i2.cluster_offsets, i2.cluster_lights
            t1 = time.perf_counter()
            stage.tracer.upload_scene(tris)
            t2 = time.perf_counter()
            stage.upload_world(i2)
            t3 = time.perf_counter()
            stage.upload_bounce(refl, pvs_off, pvs_list, bounces=MAX_BOUNCES, threshold=BOUNCE_THRESHOLD)
            t4 = time.perf_counter()
            stage.light_pass_ranges(ldr=out_ldr, hdr=out_hdr)
            t5 = time.perf_counter()
            for k, a, b in (("inputs", t0, t1), ("upload_scene", t1, t2), ("upload_world", t2, t3),
                            ("upload_bounce", t3, t4), ("light_pass", t4, t5)):
                parts[k].append(b - a)
            h2d.append(tris.nbytes + faces.nbytes + verts.nbytes + samples.nbytes + lights.nbytes + lights_hdr.nbytes
                       + off.nbytes + flat.nbytes + i2.sun_jitter.nbytes + refl.nbytes + pvs_off.nbytes
                       + pvs_list.nbytes)
        e2e_step()
        barrier(world_size)
        t = time.perf_counter()
        e2e_steps = max(1, min(args.steps, 3))
        for _ in range(e2e_steps):
            e2e_step()
        e2e_s = max_over_ranks((time.perf_counter() - t) / e2e_steps, world_size)
        e2e = {"value": job_rays / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d[-1]),
               "d2h_bytes_per_step": int(2 * nbytes), "stage_s": e2e_s,
               "parts_s": {k: statistics.median(v[1:]) for k, v in parts.items()},
               "step_parts_s": [[round(parts[k][i], 4) for k in parts] for i in range(1, len(parts["light_pass"]))],
               "note": "per step: the inputs built on the host (faces, samples, both light lists), the scene "
                       "upload with its BVH build, the world and bounce uploads with all their host set-up, "
                       "both ranges lit and their lumps read back"}
        if not (np.array_equal(out_ldr, ldr_host) and np.array_equal(out_hdr, hdr_host)):
            e2e["mismatch_vs_device"] = True

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu:
        from oracle import oracle as O
        tree = O.kd_build(w.tri_verts, w.tri_ids)
        ob = oracle_bounce(w, inp, tree)
        r_l = cpu_direct(w, inp, inp.lights, tree, 6.0)
        r_h = cpu_direct(w, inp, inp.lights_hdr, tree, 6.0, phase=1)
        t_rate, t_sample = cpu_transfers(ob, budget_s=12.0)
        cparts = {"direct_ldr": n / r_l[0], "direct_hdr": n / r_h[0], "transfers": transfer_rays / t_rate,
                  **{k: v for k, v in cpu_parts.items()}}
        stage_s = sum(cparts.values())
        cpu = {"value": rays_per_step / stage_s, "unit": UNIT, "cores": O.default_threads(), "kind": "port",
               "sample": (f"LDR gather: {r_l[2]}; HDR gather: {r_h[2]}; transfer build: {t_sample} "
                          f"({t_rate:.3g} rays/s); each range's bounce (patch light and bounces over the device's "
                          f"transfers) and final pass timed whole"),
               "stage_s": stage_s, "parts_s": cparts}

    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))

    # The learned warm start (LDR range): a network trained on the device on
    # plain bounce solutions of 32 seeded maps (2 to 8 rooms a side), then
    # this map and three held-out maps bounced from its guess, against the
    # plain bounce, with each held-out map's guess error and contraction.
    learned = None
    if rank == 0 and not args.no_learned:
        from hl2sdk_tools_sharp_b200 import learned as LN
        train_maps = 32
        t = time.perf_counter()
        lx, lt = LN.collect([LN.training_config(k) for k in range(train_maps)], threshold=BOUNCE_THRESHOLD)
        collect_s = time.perf_counter() - t
        net = LN.Network(stage.tracer, seed=7)
        ta, tb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ta.record(stream)
        loss = LN.train(net, lx, lt, steps=3000)
        tb.record(stream)
        torch.cuda.synchronize()
        train_ms = ta.elapsed_time(tb)
        plain_lump, _, _ = stage.light_pass()
        bp = stage.bounce_stats()
        stage.set_bounce_model(net)
        warm_lump, _, _ = stage.light_pass()
        bw = stage.bounce_stats()
        stage.set_bounce_model(None)
        hx, ht = stage.bounce_features()
        for _ in range(3):
            net.forward(hx)
        ta.record(stream)
        for _ in range(10):
            y = net.forward(hx)
        tb.record(stream)
        torch.cuda.synchronize()
        fwd_ms = ta.elapsed_time(tb) / 10
        flops = 2.0 * (32 * 128 + 128 * 128 + 128 * 8) * len(hx)
        tpeak = float(peaks.get("bf16_tflops", 1590.0))
        guess = y.float().expm1().clamp_min(0)
        conv = ht.float().expm1()
        t = time.perf_counter()
        held_out = LN.evaluate(net, [LN.heldout_config(k) for k in range(3)], threshold=BOUNCE_THRESHOLD)
        held_s = time.perf_counter() - t
        learned = {"range": "LDR", "plain_bounces": int(bp.bounces), "warm_bounces": int(bw.bounces),
                   "eps": float((guess - conv).abs().mean() / conv.abs().mean()),
                   "held_out": held_out, "held_out_s": held_s,
                   "plain_bounce_ms": bp.bounce_ms, "warm_bounce_ms": bw.bounce_ms,
                   "iteration_ratio": bp.bounces / max(1, bw.bounces),
                   "lightmap_within_1_lsb": LN.within_one_lsb(warm_lump, plain_lump),
                   "guess_abs_error_log1p": float((y - ht).abs().mean().item()),
                   "training": {"maps": train_maps, "rows": int(len(lx)), "steps": 3000, "batch": 32768,
                                "collect_s": collect_s, "train_ms": train_ms, "final_loss": loss},
                   "roofline": {"bound": "tensor", "kernel": "k_mlp_forward_tc (tcgen05.mma kind::f16, bf16 in, fp32 in TMEM)",
                                "achieved": flops / (fwd_ms / 1000.0) / 1e12, "peak": tpeak, "unit": "TFLOP/s",
                                "frac": flops / (fwd_ms / 1000.0) / 1e12 / tpeak, "rows": int(len(hx)),
                                "ms": fwd_ms, "flops_per_row": flops / len(hx)}}
        net.close()
    batched = None
    if not args.no_batch:
        batched = batched_run(args, local, rank, world_size)
    leaf_ambient = ambient_run(args) if rank == 0 and not args.no_ambient else None
    recheck = recheck_run(w) if rank == 0 and not args.no_ambient else None
    # The dominant phases on the launching stream: both ranges' direct
    # gather (the two-range first round and each range's supersampling
    # passes), timed by a host-buffer pass, and the transfer build (its
    # phase events in every timed step).
    dms = []
    for _ in range(3):
        _, _, _, ps, _ = stage.light_pass_ranges(ldr=ldr_host.copy(), hdr=hdr_host.copy())
        dms.append(ps.direct_ms)
    direct_ms = statistics.median(dms)
    transfer_ms = statistics.median([p[1] for p in phases])
    direct_rays = int(pstats.visibility_rays + pstats.sky_rays)
    if direct_ms >= transfer_ms:
        alg_bytes = 28.0 * direct_rays + 48.0 * n
        kernel, kernel_ms = "k_direct (both ranges' gather + traversal) and the supersampling passes", direct_ms
        alg_note = "28 B per traced segment + 16 B sample in + 2 x 16 B values out"
        traffic = None
    else:
        alg_bytes = 28.0 * transfer_rays + 8.0 * bst[0].transfers
        kernel, kernel_ms = "transfer build (k_candidates + k_transfer + compaction)", transfer_ms
        alg_note = "28 B per candidate ray + 8 B per transfer written"
        traffic = TRAFFIC_PER_TRANSFER_RAY * transfer_rays
    achieved = alg_bytes / (kernel_ms / 1000.0) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": kernel, "kernel_ms": kernel_ms, "algorithmic_bytes": alg_note,
                "algorithmic_bytes_per_launch": alg_bytes,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_transfer launch on "
                                  "the 4x4 map (profiles/k_transfer_4x4_roomgrid.md), per transfer ray, times this "
                                  "launch's transfer rays",
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "direct_ms": direct_ms, "transfer_build_ms": transfer_ms}
    nb_l = int(statistics.median([p[3] for p in phases]))
    nb_h = int(statistics.median([p[4] for p in phases]))
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded room grid)",
            "config": stage_config(args),
            "counts": {"samples": n, "faces": int(len(inp.faces)), "triangles": info.triangles,
                       "lights": int(len(inp.lights)), "rays_per_step": rays_per_step,
                       "rays_traced_per_step": traced_per_step,
                       "direct_rays_ldr": int(st_l.visibility_rays + st_l.sky_rays),
                       "direct_rays_hdr": int(st_h.visibility_rays + st_h.sky_rays),
                       "transfer_rays": transfer_rays, "transfers": int(bst[0].transfers),
                       "patches": int(bst[0].patches), "receivers": int(bst[0].receivers),
                       "luxels": luxels, "lighting_bytes_per_range": nbytes,
                       "bounces_ldr": nb_l, "bounces_hdr": nb_h,
                       "job_rays_per_step": job_rays},
            "rays_note": ("rays_per_step counts what the reference traces for the stage: each range's direct "
                          "segments (it lights the ranges in two passes) and one transfer build; one step here "
                          "traces rays_traced_per_step (the two ranges' first gather round share one traversal)"),
            "samples_per_s": world_size * n / (ms_per_step / 1000.0),
            "luxels_per_s": world_size * 2 * luxels / (ms_per_step / 1000.0),
            "stage_s": ms_per_step / 1000.0,
            "phase_ms": {"direct_both_ranges": direct_ms, "patch_light": statistics.median([p[0] for p in phases]),
                         "transfers": transfer_ms, "bounces": statistics.median([p[2] for p in phases])},
            "e2e": e2e,
            # Per step (the ncu launch list in profiles/): the two-range
            # gather 1; per range its supersampling (1 + 4 per pass run),
            # patch light 2, final 4, per bounce the gather, the 8 tree
            # levels of CollectLight and the totals; the transfer build 16
            # (candidates, rays, count, write, slices, their scans and sort).
            "gpu_launches": (1 + (1 + 4 * int(st_l.extra_passes_run)) + (1 + 4 * int(st_h.extra_passes_run))
                             + 2 * (2 + 4) + 16 + 10 * (nb_l + nb_h)) * args.steps,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "step_ms": per_step,
            "bvh": {"nodes": info.bvh_nodes, "leaves": info.bvh_leaves, "max_leaf": info.max_leaf,
                    "depth": info.bvh_depth, "build_ms": info.build_ms, "pad": info.box_pad},
            "autotune": {"threads_per_cta": block, "ms": tune_ms},
            "check": check,
            "learned": learned,
            "batched": batched,
            "leaf_ambient": leaf_ambient,
            "fp64_recheck": recheck,
        }
        print(json.dumps(line), flush=True)
    stage.close()
    if world_size > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def forward_run(rows: int = 999080, reps: int = 20) -> dict:
    """The learned warm start's tcgen05 forward alone on `rows` seeded rows
    (the 8x8 map's receiver count by default), timed on the device."""
    import torch
    from hl2sdk_tools_sharp_b200 import learned as LN, tracer as T
    with T.CudaRayTracer(T.make_triangles(np.zeros((1, 9), np.float32), np.zeros(1, np.int32))) as tr:
        net = LN.Network(tr, seed=7)
        g = torch.Generator(device="cuda")
        g.manual_seed(3)
        x = torch.randn((rows, LN.INPUTS), device="cuda", generator=g).to(torch.bfloat16).contiguous()
        y = torch.empty((rows, LN.OUTPUTS), device="cuda")
        for _ in range(3):
            net.forward(x, out=y)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            net.forward(x, out=y)
        b.record()
        torch.cuda.synchronize()
        net.status()
        ms = a.elapsed_time(b) / reps
        net.close()
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    flops = 2.0 * (32 * 128 + 128 * 128 + 128 * 8) * rows
    tf = flops / (ms / 1000.0) / 1e12
    peak = float(peaks.get("bf16_tflops", 1590.0))
    return {"kernel": "k_mlp_forward_tc", "rows": rows, "ms": ms, "achieved_tflops": tf, "peak_tflops": peak,
            "frac": tf / peak, "peak_source": "measured" if "bf16_tflops" in peaks else "fallback"}


def transfer_cache_run(args, reps: int = 3) -> dict:
    """The transfer cache on the map of --side (default 8x8): the store
    (vrad_transfer_export: the set put in patch order and shuffled into
    planes on the device, deflated on the host's threads) and the hit
    (vrad_transfer_install: inflated on the host's threads, decoded and put
    in receiver order on the device, sliced for the gather), each timed
    around its blocking library call (best of `reps`), beside the transfer
    build they stand in for; then a pass lit with the installed set checked
    against one that built its own."""
    from hl2sdk_tools_sharp_b200 import lighting as L, transfer_cache as C
    w, inp = world_and_inputs(args.side, CONFIG_SEED)
    refl = L.face_reflectivity(w)
    pvs_off, pvs_list = L.pvs_lists(w)
    with L.LightingStage(w, inp) as st:
        st.upload_bounce(refl, pvs_off, pvs_list, bounces=MAX_BOUNCES, threshold=BOUNCE_THRESHOLD)
        ldr, hdr, _, _, bst = st.light_pass_ranges()
        build_ms, total = float(bst[0].transfer_ms), int(bst[0].transfers)
        store = []
        for _ in range(reps):
            t = {}
            idx, packed = C.export(st, timing=t)
            store.append(t["abi_s"])
    packed_bytes = int(sum(memoryview(p).nbytes for p in packed))
    with L.LightingStage(w, inp) as st:
        st.upload_bounce(refl, pvs_off, pvs_list, bounces=MAX_BOUNCES, threshold=BOUNCE_THRESHOLD)
        hit = []
        for _ in range(reps):
            t = {}
            assert C.install(st, idx, packed, timing=t)
            hit.append(t["abi_s"])
        ldr2, hdr2, _, _, bst2 = st.light_pass_ranges()
    raw = 8 * total
    return {"workload": f"{args.side}x{args.side} room grid transfer set ({total} transfers, {len(packed)} chunks "
                        f"of at most {C.DEFAULT_MAX_CHUNK_BYTES} bytes)",
            "transfers": total, "raw_bytes": raw, "packed_bytes": packed_bytes + len(idx),
            "ratio": (packed_bytes + len(idx)) / raw if raw else None,
            "build_ms": build_ms, "store_ms": 1000 * min(store), "hit_ms": 1000 * min(hit),
            "store_gbs": raw / min(store) / 1e9, "hit_gbs": raw / min(hit) / 1e9,
            "host_threads": os.cpu_count(),
            "replay": {"transfers_cached": int(bst2[0].transfers_cached), "transfer_rays": int(bst2[0].transfer_rays),
                       "lumps_equal": bool(np.array_equal(ldr, ldr2) and np.array_equal(hdr, hdr2))}}


def main():
    args = parse()
    if args.workload == "transfer-cache":
        print(json.dumps(transfer_cache_run(args)), flush=True)
        return 0
    if args.workload == "forward":
        print(json.dumps(forward_run()), flush=True)
        return 0
    if args.workload == "ambient":
        # The leaf ambient section alone (also the small case its ncu
        # capture runs): one JSON line of ambient_run's figures.
        print(json.dumps(ambient_run(args, samples=args.ambient_samples)), flush=True)
        return 0
    if args.workload == "seam":
        return run_reference(args) if args.impl == "reference" else main_seam(args)
    return run_reference_stage(args) if args.impl == "reference" else main_stage(args)


if __name__ == "__main__":
    sys.exit(main())
