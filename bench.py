"""Benchmark: vrad's lighting stage on the seeded 8x8 room grid.

One step = one light pass (vrad_light_pass), the whole stage from the
uploaded world to the LIGHTING lump:
  direct  the fused direct gather over every light sample of the map (for
          each of its 5.68 M samples, every light of its cluster's list in
          gather order: shadow segments to 64 point and spot lights, the
          sun's sky test and 162 sky-ambient directions, traced in-kernel);
  bounce  the patches' direct light, the transfer build (every candidate
          patch pair's ray traced, form factors, scales) and the radiosity
          bounces to the stop threshold (0.1, the configuration's);
  final   the luxel radial filters of the direct and the bounced light,
          RGBE encode, medians, into the LIGHTING lump.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --workload seam     # the IRayTracer seam alone, rays in HBM

Prints one JSON line (rank 0).  `value` is rays/s (segments traced per
second, all ranks) with the world resident in HBM; `e2e` is the same
through the C ABI's host-buffer entry points (pinned host samples in,
lighting values out, copies inside the timed region).  `--impl reference`
times the reference's algorithm on the host CPU: the restated KD tracer and
four-sample-group gather, all host threads, on a strided sample of faces.
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

METRIC = "vrad lighting stage rays/s (8x8 room grid, 1 B200)"
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
    ap.add_argument("--workload", default="stage", choices=["stage", "seam"])
    ap.add_argument("--no-e2e", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-cpu", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-learned", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-batch", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--batch-maps", type=int, default=32, help=argparse.SUPPRESS)
    ap.add_argument("--batch-workers", type=int, default=4, help=argparse.SUPPRESS)
    return ap.parse_args()


def world_for(side: int):
    from hl2sdk_tools_sharp_b200 import roomgrid as rg
    cfg = rg.config_8x8(CONFIG_SEED) if side == 8 else rg.config_3x3(CONFIG_SEED)
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
    vals = []
    for i in range(args.warmup + args.steps):
        cb = cpu_reference(w, rays_np, total, budget_s=max(3.0, 60.0 / max(1, args.warmup + args.steps)))
        if i >= args.warmup:
            vals.append(cb["value"])
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / value,
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
                   "roofline": {"bound": "tensor", "kernel": "k_mlp_forward (mma.sync bf16, fp32 accumulate)",
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


def oracle_faces_sample(world, inp, stride: int):
    """Every `stride`-th face with its samples, renumbered, for the CPU leg."""
    sel = np.arange(0, len(inp.faces), stride)
    ff = inp.face_first
    parts = [inp.samples[ff[f]:ff[f + 1]] for f in sel]
    counts = np.array([len(p) for p in parts])
    first = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    samples = np.concatenate(parts).copy()
    samples["face"] = np.repeat(np.arange(len(sel)), counts)
    index = np.concatenate([np.arange(ff[f], ff[f + 1]) for f in sel])
    return sel, samples, first, index


def cpu_stage(world, inp, budget_s: float = 15.0):
    """The reference's direct gather on the host: restated KD build + the
    four-sample-group gather with the KD walk, all host threads, on a
    strided sample of faces sized to about budget_s."""
    from oracle import oracle as O
    threads = O.default_threads()
    tree = O.kd_build(world.tri_verts, world.tri_ids)

    def run(stride):
        sel, samples, first, _ = oracle_faces_sample(world, inp, stride)
        t0 = time.perf_counter()
        _, rays = O.direct(tree, inp.faces[sel], samples, first, inp.lights, inp.cluster_offsets,
                           inp.cluster_lights, inp.sky_directions, inp.sun_jitter, inp.sun_samples,
                           inp.sun_angular_extent, threads=threads, count_rays=True, verts=inp.verts)
        return rays, len(samples), time.perf_counter() - t0, len(sel)
    rays, n, dt, nf = run(max(1, len(inp.faces) // 64))
    stride = max(1, int(len(inp.faces) / max(1.0, nf * budget_s / max(dt, 1e-3))))
    rays, n, dt, nf = run(stride)
    return {"value": rays / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{nf} of {len(inp.faces)} faces (every {stride}th), {n} samples, {rays} segments "
                      f"of the 8x8 direct gather; restated KD build + KD walk + four-sample-group gather",
            "samples_per_s": n / dt}


def batched_run(args, device_index: int) -> dict:
    """The batched workload: `batch_maps` seeded room grids, sides drawn
    from 2..10 rooms, each bounced to the 8x8 map's threshold, lit by the
    native batch runner (host buffers in and out, every map's scene, world
    and bounce uploaded inside the timed run).  The autotuner picks the
    gather's launch shape and the maps in flight on the first eight maps;
    one warm-up run, then the timed run, then the same maps on one worker."""
    from hl2sdk_tools_sharp_b200 import batch as B, roomgrid as rg
    t = time.perf_counter()
    cfgs = [rg.config_batch(i, seed=CONFIG_SEED) for i in range(args.batch_maps)]
    maps = [B.map_inputs(rg.generate(c), bounces=MAX_BOUNCES, threshold=BOUNCE_THRESHOLD) for c in cfgs]
    prep_s = time.perf_counter() - t
    with B.LightingBatch(workers=args.batch_workers, device=device_index) as batch:
        workers, block, tune = batch.autotune(maps[:min(8, len(maps))])
        warm, _ = batch.run(maps)
        results, st = batch.run(maps)
        one, st1 = batch.run(maps, workers=1)
    same = all(np.array_equal(a.lighting, b.lighting) and np.array_equal(a.lighting, c.lighting)
               for a, b, c in zip(results, warm, one))
    return {"maps": len(maps), "sides": [c.side for c in cfgs], "rooms": int(sum(c.side ** 2 for c in cfgs)),
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


def world_and_inputs(side):
    from hl2sdk_tools_sharp_b200 import lighting as L
    w = world_for(side)
    return w, L.prepare(w)


def oracle_bounce(world, inp, tree=None):
    """The oracle's bounce over the world (patches built, nothing traced)."""
    from hl2sdk_tools_sharp_b200 import lighting as L
    from oracle import oracle as O
    tree = tree if tree is not None else O.kd_build(world.tri_verts, world.tri_ids)
    off, lst = L.pvs_lists(world)
    return O.Bounce(tree, inp.faces, inp.verts, inp.samples, inp.face_first, L.face_reflectivity(world), off, lst,
                    bounces=MAX_BOUNCES, threshold=BOUNCE_THRESHOLD)


def cpu_transfers(ob, budget_s: float = 10.0):
    """The transfer build restated (candidate walk, KD-traced rays, form
    factors) on a strided sample of receivers: transfer rays per second."""
    patches, _ = ob.patches()
    leaves = np.flatnonzero(patches["child1"] == -1)

    def run(stride, phase):
        sub = leaves[phase::stride]
        ob.forget_transfers()
        t0 = time.perf_counter()
        _, _, _, rays = ob.transfers(sub)
        return rays, time.perf_counter() - t0, len(sub)
    rays, dt, n = run(max(1, len(leaves) // 400), 1)
    stride = max(1, int(len(leaves) / max(1.0, n * budget_s / max(dt, 1e-3))))
    rays, dt, n = run(stride, 0)
    return rays / dt, f"{n} of {len(leaves)} receivers (every {stride}th), {rays} transfer rays"


WORKLOAD = ("8x8 room grid lighting stage: direct gather (64 point/spot lights, sun, 162-dir sky), "
            "bounce (patch light, transfer build, radiosity to threshold 0.1), final pass")


def run_reference_stage(args):
    """The reference's algorithm on the host cores: the direct gather and
    the transfer build restated (KD build, KD walk, four-sample groups,
    candidate walk, form factors), all host threads, each on a bounded
    sample of the 8x8 stage.  value = the stage's traced rays over the CPU
    seconds those two parts take at the sampled rates; the bounce's
    gathers and the final pass are left out of the CPU time (which only
    flatters the CPU)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O
    w, inp = world_and_inputs(args.side)
    tree = O.kd_build(w.tri_verts, w.tri_ids)
    ob = oracle_bounce(w, inp, tree)
    counts = None
    vals = []
    cb = None
    for i in range(args.warmup + args.steps):
        budget = max(2.0, 40.0 / max(1, args.warmup + args.steps))
        cb = cpu_stage(w, inp, budget_s=budget)
        t_rate, t_sample = cpu_transfers(ob, budget_s=budget)
        if counts is None:
            # Ray counts of one full step: the direct gather's from the
            # sampled rate's own sample scaled to every sample; the transfer
            # build's from the candidate walk (no tracing needed to count).
            direct_rays = cb["value"] * len(inp.samples) / cb["samples_per_s"]
            counts = (direct_rays, ob.count_candidates())
        direct_rays, transfer_rays = counts
        cpu_s = direct_rays / cb["value"] + transfer_rays / t_rate
        if i >= args.warmup:
            vals.append((direct_rays + transfer_rays) / cpu_s)
    value = statistics.median(vals)
    direct_rays, transfer_rays = counts
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * (direct_rays + transfer_rays) / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded room grid)",
        "config": {"workload": WORKLOAD, "side": args.side, "seed": CONFIG_SEED, "samples": int(len(inp.samples)),
                   "bounce_threshold": BOUNCE_THRESHOLD},
        "cpu_baseline": {**cb, "value": value,
                         "sample": cb["sample"] + f"; transfer build: {t_sample}; bounce gathers and final pass not timed"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main_stage(args):
    import torch
    from hl2sdk_tools_sharp_b200 import lighting as L
    rank, world_size, local = dist_setup(args.gpus)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)

    w, inp = world_and_inputs(args.side)
    n = len(inp.samples)
    refl = L.face_reflectivity(w)
    pvs_off, pvs_list = L.pvs_lists(w)
    stage = L.LightingStage(w, inp, device=local)
    stage.upload_bounce(refl, pvs_off, pvs_list, bounces=MAX_BOUNCES, threshold=BOUNCE_THRESHOLD)
    info = stage.tracer.scene_info()
    d_out = torch.empty(n * 4, dtype=torch.float32, device=device)
    block, tune_ms = stage.autotune()                # picks the launch shape (untimed)
    lump_host, lightofs, pstats = stage.light_pass()   # counts the rays of one step
    bst = stage.bounce_stats()
    rays_per_step = int(pstats.visibility_rays + pstats.sky_rays + bst.transfer_rays)
    luxels = int(pstats.luxels)
    d_lump = torch.empty(len(lump_host), dtype=torch.uint8, device=device)
    for _ in range(max(3, args.warmup)):
        stage.light_pass_device(d_lump)
    torch.cuda.synchronize()

    check = None
    ob = None
    cpu_parts = {}
    if rank == 0 and not args.no_cpu:
        # Parity on this run's own output: a strided sample of faces through
        # the oracle's direct gather, a sample of receivers through its
        # transfer build, and the whole lump through its bounce and final
        # pass fed the device's sample light and transfers (each checked
        # here or by the sampled comparisons).
        from oracle import oracle as O
        tree = O.kd_build(w.tri_verts, w.tri_ids)
        sel, samples, first, index = oracle_faces_sample(w, inp, 97)
        want = O.direct(tree, inp.faces[sel], samples, first, inp.lights, inp.cluster_offsets,
                        inp.cluster_lights, inp.sky_directions, inp.sun_jitter, inp.sun_samples,
                        inp.sun_angular_extent, verts=inp.verts)
        stage.direct_device(d_out)
        torch.cuda.synchronize()
        got_all = d_out.view(n, 4).cpu().numpy()
        t_off, t_rec = stage.transfers()
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
        ob.set_transfers(t_off, t_rec["patch"], t_rec["weight"])
        t = time.perf_counter()
        _, _, o_bounces, _ = ob.run(got_all)
        cpu_parts["bounce_s"] = time.perf_counter() - t
        t = time.perf_counter()
        lump_want, _ = ob.final(got_all)
        cpu_parts["final_s"] = time.perf_counter() - t
        lump_got = d_lump.cpu().numpy()
        check = {"samples": int(len(index)),
                 "mismatches": int((got_all[index].view(np.uint32) != want.view(np.uint32)).any(1).sum()),
                 "receivers": int(len(sub)), "receiver_mismatches": tr_bad,
                 "bounces": int(bst.bounces), "oracle_bounces": int(o_bounces),
                 "lump_words": int(len(lump_want) // 4),
                 "lump_mismatches": int((lump_got.view(np.uint32) != lump_want.view(np.uint32)).sum())}
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
            stage.light_pass_device(d_lump)
            ev[2 * s_ + 1].record(stream)
            b = stage.bounce_stats()
            phases.append((b.patch_light_ms, b.transfer_ms, b.bounce_ms, b.bounces))
        t1.record(stream)
        torch.cuda.synchronize()
    barrier(world_size)
    elapsed_ms = max_over_ranks(t0.elapsed_time(t1), world_size)
    per_step = [ev[2 * k].elapsed_time(ev[2 * k + 1]) for k in range(args.steps)]
    ms_per_step = elapsed_ms / args.steps
    value = job_value(rays_per_step, ms_per_step, world_size)
    bst = stage.bounce_stats()

    # End to end through the host-buffer C ABI: the world (samples from
    # pinned memory) and the bounce uploaded, the light pass, the lump read
    # back into pinned memory.
    e2e = None
    if not args.no_e2e:
        pinned = torch.empty(inp.samples.nbytes, dtype=torch.uint8, pin_memory=True)
        pinned.numpy()[:] = inp.samples.view(np.uint8).reshape(-1)
        inp_pinned = L.LightingInputs(**{**inp.__dict__, "samples": pinned.numpy().view(L.SAMPLE_DTYPE)})
        out_pinned = torch.empty(len(lump_host), dtype=torch.uint8, pin_memory=True)
        outv = out_pinned.numpy()

        parts = {"upload_world": [], "upload_bounce": [], "light_pass": []}

        def e2e_step():
            t0 = time.perf_counter()
            stage.upload_world(inp_pinned)
            t1 = time.perf_counter()
            stage.upload_bounce(refl, pvs_off, pvs_list, bounces=MAX_BOUNCES, threshold=BOUNCE_THRESHOLD)
            t2 = time.perf_counter()
            stage.light_pass(outv)
            t3 = time.perf_counter()
            parts["upload_world"].append(t1 - t0)
            parts["upload_bounce"].append(t2 - t1)
            parts["light_pass"].append(t3 - t2)
        e2e_step()
        barrier(world_size)
        t = time.perf_counter()
        e2e_steps = max(1, min(args.steps, 3))
        for _ in range(e2e_steps):
            e2e_step()
        e2e_s = max_over_ranks((time.perf_counter() - t) / e2e_steps, world_size)
        e2e = {"value": world_size * rays_per_step / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(inp.samples.nbytes + inp.faces.nbytes + inp.lights.nbytes
                                         + inp.verts.nbytes + refl.nbytes + pvs_off.nbytes + pvs_list.nbytes),
               "d2h_bytes_per_step": int(len(lump_host)), "stage_s": e2e_s,
               "parts_s": {k: statistics.median(v[1:]) for k, v in parts.items()},
               "step_parts_s": [[round(parts[k][i], 4) for k in parts] for i in range(1, len(parts["light_pass"]))],
               "note": "includes the host-side set-up of the world and the bounce (slot layout, final-pass "
                       "tables, the patch tree) and the device tables' uploads"}
        if not np.array_equal(outv, lump_host):
            e2e["mismatch_vs_device"] = True

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu:
        cpu = cpu_stage(w, inp, budget_s=12.0)
        t_rate, t_sample = cpu_transfers(ob, budget_s=12.0)
        cpu_direct_s = n / cpu["samples_per_s"]
        cpu_transfer_s = bst.transfer_rays / t_rate
        cpu["stage_s"] = cpu_direct_s + cpu_transfer_s + cpu_parts["bounce_s"] + cpu_parts["final_s"]
        cpu["parts_s"] = {"direct": cpu_direct_s, "transfers": cpu_transfer_s, "bounce": cpu_parts["bounce_s"],
                          "final": cpu_parts["final_s"]}
        cpu["value"] = rays_per_step / cpu["stage_s"]
        cpu["sample"] += (f"; transfer build: {t_sample} ({t_rate:.3g} rays/s); bounce (patch light + "
                          f"{bst.bounces} bounces over the device's transfers) and final pass timed whole "
                          f"({cpu_parts['bounce_s']:.2f} s, {cpu_parts['final_s']:.2f} s)")

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
                   "roofline": {"bound": "tensor", "kernel": "k_mlp_forward (mma.sync bf16, fp32 accumulate)",
                                "achieved": flops / (fwd_ms / 1000.0) / 1e12, "peak": tpeak, "unit": "TFLOP/s",
                                "frac": flops / (fwd_ms / 1000.0) / 1e12 / tpeak, "rows": int(len(hx)),
                                "ms": fwd_ms, "flops_per_row": flops / len(hx)}}
        net.close()
    batched = None
    if rank == 0 and world_size == 1 and not args.no_batch:
        try:
            batched = batched_run(args, local)
        except Exception as exc:  # reported in the line; the headline still prints
            batched = {"error": f"{type(exc).__name__}: {exc}"}
    # The dominant phases timed alone on the launching stream: the direct
    # gather kernel, and the transfer build (its phase events).
    a_ev = torch.cuda.Event(enable_timing=True)
    b_ev = torch.cuda.Event(enable_timing=True)
    a_ev.record(stream)
    for _ in range(3):
        stage.direct_device(d_out)
    b_ev.record(stream)
    torch.cuda.synchronize()
    direct_ms = a_ev.elapsed_time(b_ev) / 3.0
    transfer_ms = statistics.median([p[1] for p in phases])
    direct_rays = int(pstats.visibility_rays + pstats.sky_rays)
    if direct_ms >= transfer_ms:
        alg_bytes = 28.0 * direct_rays + 32.0 * n
        kernel, kernel_ms = "k_direct (fused gather + traversal)", direct_ms
        alg_note = "28 B per traced segment + 16 B sample in + 16 B value out"
    else:
        alg_bytes = 28.0 * bst.transfer_rays + 8.0 * bst.transfers
        kernel, kernel_ms = "transfer build (k_candidates + k_transfer + compaction)", transfer_ms
        alg_note = "28 B per candidate ray + 8 B per transfer written"
    achieved = alg_bytes / (kernel_ms / 1000.0) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "kernel": kernel, "kernel_ms": kernel_ms, "algorithmic_bytes": alg_note,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "direct_ms": direct_ms, "transfer_build_ms": transfer_ms}
    nb = int(statistics.median([p[3] for p in phases]))
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded room grid)",
            "config": {"workload": WORKLOAD,
                       "side": args.side, "seed": CONFIG_SEED, "samples": n, "faces": int(len(inp.faces)),
                       "triangles": info.triangles, "lights": int(len(inp.lights)),
                       "rays_per_step": rays_per_step,
                       "visibility_rays": int(pstats.visibility_rays), "sky_rays": int(pstats.sky_rays),
                       "transfer_rays": int(bst.transfer_rays), "transfers": int(bst.transfers),
                       "patches": int(bst.patches), "receivers": int(bst.receivers),
                       "luxels": luxels, "lighting_bytes": int(len(lump_host)),
                       "bounce_threshold": BOUNCE_THRESHOLD, "bounces": nb,
                       "l2": "no L2 flush: the 0.3 GB sample set and 5 GB of candidate pairs exceed L2",
                       "parallelism": f"replicas{world_size}"},
            "samples_per_s": world_size * n / (ms_per_step / 1000.0),
            "luxels_per_s": world_size * luxels / (ms_per_step / 1000.0),
            "stage_s": ms_per_step / 1000.0,
            "phase_ms": {"direct": direct_ms, "patch_light": statistics.median([p[0] for p in phases]),
                         "transfers": transfer_ms, "bounces": statistics.median([p[2] for p in phases])},
            "bounce_iterations": nb,
            "e2e": e2e,
            # Per light pass of this map (the ncu launch list in profiles/):
            # direct 1; supersampling 4 per pass run + 1; patch light 2;
            # transfer build 16 (candidates, rays, count, write, slices,
            # their scans and sort); final 4; per bounce the gather, the 8
            # tree levels of CollectLight and the totals (exact totals add
            # one when needed).
            "gpu_launches": (1 + 4 * int(pstats.extra_passes_run) + 1 + 2 + 16 + 4 + 10 * nb) * args.steps,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "step_ms": per_step,
            "bvh": {"nodes": info.bvh_nodes, "leaves": info.bvh_leaves, "max_leaf": info.max_leaf, "depth": info.bvh_depth,
                    "build_ms": info.build_ms, "pad": info.box_pad},
            "autotune": {"threads_per_cta": block, "ms": tune_ms},
            "check": check,
            "learned": learned,
            "batched": batched,
        }
        print(json.dumps(line), flush=True)
    stage.close()
    if world_size > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.workload == "seam":
        return run_reference(args) if args.impl == "reference" else main_seam(args)
    return run_reference_stage(args) if args.impl == "reference" else main_stage(args)


if __name__ == "__main__":
    sys.exit(main())
