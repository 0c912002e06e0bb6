"""Adversarial rays: hits exactly on triangle edges and vertices, segments
that end exactly on a surface, and rays lying in or leaving the reference KD
tree's split planes, on the room grids and on the reference's own kd-scene
fixture (2,000 triangles in general position).

Three answers are compared per ray:
  device   the CUDA tracer (BVH walk, the reference's FP32 predicate);
  brute    every triangle through the same FP32 predicate (oracle): the
           device's contract, bit for bit;
  kd       the reference's own KD-tree walk (restated, node for node with
           stock on the fixtures).
The KD walk clips each ray to the cells it visits in FP32, so a hit that
lies exactly on a triangle edge in a split plane can fall outside every
cell it is tested in; brute force (and the device) still finds it.  And
where two coplanar triangles overlap (a sky face and an opaque face in one
plane), their crossings tie: the walk keeps the one its traversal meets
first, brute force the lower index, which decides a sky test.  The CPU test
below shows that every ray where the reference's walk and brute force
disagree is one of these two cases: its deciding crossing is, in exact
(FP64) arithmetic, within a relative 1e-6 of a triangle's edge, or the two
answers' first hits are distinct triangles at the same distance.  FP64
cannot settle either (the rays lie on a boundary, or the tie is exact);
the reference's GPU tracer is validated the same way, against an FP64
brute force with margin and tie bands
(Tests/MapTools/Tracing/VulkanRayTracerFacts.cs:1215-1300).  On the
lighting workloads' own rays the device and the reference's walk agree
(tests/test_direct_gpu.py, the bench's parity check).
"""
import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import roomgrid as rg, tracer as T
from tests.golden import fixtures as F

TRACE_ID_SKY = 0x01000000
MARGIN = 1e-6


def _adversarial(verts, tree, rng, n=12000):
    v = verts.reshape(-1, 3, 3).astype(np.float32)
    lo, hi = verts.reshape(-1, 3).min(0), verts.reshape(-1, 3).max(0)
    span = np.float32(np.max(hi - lo))
    out = {}
    t = rng.integers(0, len(v), n)
    e = rng.integers(0, 3, n)
    a, b = v[t, e], v[t, (e + 1) % 3]
    s = rng.uniform(0, 1, n).astype(np.float32)
    s[::5] = 0.0                                            # the vertices themselves
    p = (a + (b - a) * s[:, None]).astype(np.float32)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    r = np.zeros((n, 7), np.float32)
    r[:, :3], r[:, 3:6], r[:, 6] = o, (p - o) * np.float32(2.0), 1.0
    out["edges"] = r
    t = rng.integers(0, len(v), n)
    w = rng.dirichlet([1, 1, 1], n).astype(np.float32)
    p = (v[t, 0] * w[:, :1] + v[t, 1] * w[:, 1:2] + v[t, 2] * w[:, 2:3]).astype(np.float32)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    r = np.zeros((n, 7), np.float32)
    r[:, :3], r[:, 3:6], r[:, 6] = o, p - o, 1.0
    out["end_on_surface"] = r
    nodes = tree["nodes"]
    inner = nodes[(nodes["children"] & 3) != 3]
    k = rng.integers(0, len(inner), n)
    axis, split = inner["children"][k] & 3, inner["split"][k]
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    o[np.arange(n), axis] = split
    d = rng.normal(size=(n, 3)).astype(np.float32) * span
    d2 = d.copy()
    d[np.arange(n), axis] = 0.0
    r = np.zeros((n, 7), np.float32)
    r[:, :3], r[:, 3:6], r[:, 6] = o, d, 1.0
    out["in_split_plane"] = r
    r2 = r.copy()
    r2[:, 3:6] = d2
    out["from_split_plane"] = r2
    return out


def _scenes():
    for name, cfg in (("room3x3", rg.config_3x3(seed=2)), ("room8x8", rg.config_8x8(seed=1))):
        w = rg.generate(cfg)
        yield name, w.tri_verts, w.tri_ids, None
    # The fixture's recorded tree carries stock-normalised triangles; the
    # walk here is over the restated build of the same triangles in Correct
    # mode (the tracer's mode), which is stock's tree node for node.
    fx = F.load("kd-scene")
    yield "kd-scene", fx["verts"], np.zeros(len(fx["verts"]), np.int32), None


def _crossing64(verts, ray, i):
    """(u, v, t) of ray with triangle i in float64 (Moller-Trumbore)."""
    tv = verts[i].astype(np.float64).reshape(3, 3)
    o, d = ray[:3].astype(np.float64), ray[3:6].astype(np.float64)
    e1, e2 = tv[1] - tv[0], tv[2] - tv[0]
    h = np.cross(d, e2)
    a = e1 @ h
    if abs(a) < 1e-300:
        return None
    f = 1.0 / a
    sv = o - tv[0]
    u = f * (sv @ h)
    q = np.cross(sv, e1)
    vv = f * (d @ q)
    return u, vv, f * (e2 @ q)


def _on_edge(verts, ray, i):
    c = _crossing64(verts, ray, i)
    if c is None:
        return False
    u, v, t = c
    return min(abs(u), abs(v), abs(1 - u - v)) < MARGIN or abs(t - ray[6]) < MARGIN * max(1.0, abs(t))


def test_reference_walk_differs_from_brute_force_only_on_edge_hits(oracle_mod):
    O = oracle_mod
    total = 0
    counts = {"edge": 0, "tie": 0, "unexplained": 0}
    for name, verts, ids, tree in _scenes():
        tree = tree if tree is not None else O.kd_build(verts, ids)
        tris = O.prepare_triangles(verts, ids)
        for kind, rays in _adversarial(verts, tree, np.random.default_rng(7)).items():
            for flags in (0, O.SKY_PASS):
                _, _, kb = O.kd_trace(tree, rays, flags=flags, threads=O.default_threads())
                _, _, bb = O.brute_trace(tris, rays, flags=flags)
                diff = np.flatnonzero(O.bits_to_bool(kb, len(rays)) != O.bits_to_bool(bb, len(rays)))
                for i in diff:
                    r = rays[i:i + 1]
                    bt, _, _ = O.brute_trace(tris, r, flags=O.CLOSEST)
                    kt, _, _ = O.kd_trace(tree, r, flags=O.CLOSEST)
                    # The deciding crossing: the brute force's first hit, or the
                    # walk's when only it reports one.
                    cand = [int(x) for x in (bt[0], kt[0]) if x >= 0]
                    edge = any(_on_edge(verts, rays[i], c) for c in cand) or O.fp64_classify(verts, r, MARGIN)[0] == 2
                    tie = False
                    if len(cand) == 2 and cand[0] != cand[1]:
                        c0, c1 = _crossing64(verts, rays[i], cand[0]), _crossing64(verts, rays[i], cand[1])
                        tie = c0 is not None and c1 is not None and abs(c0[2] - c1[2]) <= MARGIN * abs(c0[2])
                    total += 1
                    counts["edge" if edge else "tie" if tie else "unexplained"] += 1
                    assert edge or tie, (name, kind, flags, i, rays[i].tolist(), cand)
    assert total >= 1          # the sets do reach the walk's split-plane cases
    assert counts["unexplained"] == 0, counts


@pytest.mark.gpu
def test_device_equals_brute_force_on_adversarial_rays(oracle_mod):
    O = oracle_mod
    for name, verts, ids, tree in _scenes():
        tree = tree if tree is not None else O.kd_build(verts, ids)
        tris = O.prepare_triangles(verts, ids)
        with T.CudaRayTracer(T.make_triangles(verts, ids)) as tr:
            for kind, rays in _adversarial(verts, tree, np.random.default_rng(7)).items():
                rr = np.ascontiguousarray(rays).view(T.RAY_DTYPE).reshape(-1)
                for flags, opts in ((0, T.RayTraceOptions.stock_exact()),
                                    (O.SKY_PASS, T.RayTraceOptions(0.0, sky_does_not_block=True))):
                    _, _, bb = O.brute_trace(tris, rays, flags=flags)
                    got = tr.visibility(rr, opts)
                    assert np.array_equal(got, O.bits_to_bool(bb, len(rays))), (name, kind, flags)
                bt, bd, _ = O.brute_trace(tris, rays, flags=O.CLOSEST)
                hits = tr.closest(rr)
                assert np.array_equal(hits["surface"], np.where(bt >= 0, ids[np.maximum(bt, 0)], -1)), (name, kind)
                hit = bt >= 0
                assert np.array_equal(hits["fraction"][hit].view(np.uint32), bd[hit].view(np.uint32)), (name, kind)


@pytest.mark.gpu
def test_fp64_recheck_flags_every_questionable_ray(oracle_mod):
    """vrad_trace_visibility_recheck on the adversarial sets: its visibility
    bits are the FP32 trace's; every flagged ray's FP64 class is the oracle's
    (the same FP64 arithmetic); and every ray it does not flag has an FP64
    class that is clear and agrees with its FP32 bit, so the flag misses no
    ray an FP64 test would question."""
    O = oracle_mod
    totals = {"flagged": 0, "fp64_ambiguous": 0, "disagreements": 0, "rays": 0}
    for name, verts, ids, tree in _scenes():
        tree = tree if tree is not None else O.kd_build(verts, ids)
        with T.CudaRayTracer(T.make_triangles(verts, ids)) as tr:
            for kind, rays in _adversarial(verts, tree, np.random.default_rng(7)).items():
                rr = np.ascontiguousarray(rays).view(T.RAY_DTYPE).reshape(-1)
                vis, cls, st = tr.visibility_recheck(rr, T.RayTraceOptions.stock_exact())
                assert np.array_equal(vis, tr.visibility(rr, T.RayTraceOptions.stock_exact())), (name, kind)
                want = O.fp64_classify(verts, rays, MARGIN)
                flagged = cls >= 0
                assert st["flagged"] == int(flagged.sum())
                assert np.array_equal(cls[flagged], want[flagged]), (name, kind)
                quiet = ~flagged
                assert (want[quiet] != 2).all(), (name, kind, int((want[quiet] == 2).sum()))
                assert np.array_equal(want[quiet] == 1, vis[quiet]), (name, kind)
                for k in totals:
                    totals[k] += st[k]
    assert totals["flagged"] > 0 and totals["fp64_ambiguous"] > 0, totals
