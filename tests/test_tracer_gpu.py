"""GPU parity of the CUDA tracer against the CPU oracle, through the C ABI.

The bar is bit-exact: the CUDA tracer's semantic is the oracle's brute
force (every accepted hit with min_distance <= t < max_distance; closest =
smallest (t, triangle index)), with the reference's FP32 predicate.  The
reference's own stock answers (tests/golden) are matched on every ray.
"""
import numpy as np
import pytest

import fixtures
from hl2sdk_tools_sharp_b200 import roomgrid as rg, tracer as T, workload as wl

pytestmark = pytest.mark.gpu


def raw7(rays):
    return np.ascontiguousarray(rays).view(np.float32).reshape(-1, 7)


def as_rays(raw):
    return np.ascontiguousarray(raw, np.float32).view(T.RAY_DTYPE).reshape(-1)


def stock_prepared(scene):
    st = scene["stock_tris"]
    p = np.zeros(len(st), T.KD_TRIANGLE_DTYPE)
    for name in ("n", "d", "id", "e", "cs0", "cs1", "flags"):
        p[name] = st[name]
    return p


@pytest.fixture(scope="module", params=fixtures.SCENES)
def scene(request):
    return fixtures.load(request.param)


def test_stock_fixture_with_stock_coefficients(scene):
    # The stock-normalised coefficients recorded with the fixture: every
    # hit id and distance bit of stock's answers short of the segment end.
    tris = T.make_triangles(scene["verts"])
    rays = as_rays(scene["rays"])
    with T.CudaRayTracer(tris, prepared=stock_prepared(scene)) as tr:
        vis = tr.visibility(rays)
        hits = tr.closest(rays)
    stock = (scene["hit"] >= 0) & (scene["dist"] < 1.0)
    assert np.array_equal(vis, stock)
    assert np.array_equal(hits["surface"], np.where(stock, scene["hit"], -1))
    assert np.array_equal(hits["fraction"].view(np.uint32)[stock], scene["dist"].view(np.uint32)[stock])
    assert np.all(hits["fraction"][~stock] == 1.0)


def test_stock_fixture_with_device_prepared_triangles(oracle_mod, scene):
    # The library computes the Correct-mode intersection form on the GPU;
    # distances must be the oracle's bits (same normalise, same predicate).
    tris = T.make_triangles(scene["verts"])
    rays = as_rays(scene["rays"])
    ref_tris = oracle_mod.prepare_triangles(scene["verts"])
    bt, bd, bb = oracle_mod.brute_trace(ref_tris, scene["rays"], flags=oracle_mod.CLOSEST)
    _, _, vb = oracle_mod.brute_trace(ref_tris, scene["rays"])
    with T.CudaRayTracer(tris) as tr:
        hits = tr.closest(rays)
        vis = tr.visibility(rays)
    n = len(rays)
    assert np.array_equal(vis, oracle_mod.bits_to_bool(vb, n))
    assert np.array_equal(hits["surface"], bt)
    hit = bt >= 0
    assert np.array_equal(hits["fraction"].view(np.uint32)[hit], bd.view(np.uint32)[hit])
    # and the reference's stock answers, on these scenes
    stock = (scene["hit"] >= 0) & (scene["dist"] < 1.0)
    assert np.array_equal(vis, stock)


@pytest.fixture(scope="module")
def grid():
    w = rg.generate(rg.config_3x3(seed=3))
    s = wl.luxel_samples(w, stride=3)
    r = wl.direct_rays(w, s, ambient=True)
    return w, r


@pytest.fixture(scope="module")
def grid_tracer(grid):
    w, _ = grid
    tr = T.CudaRayTracer(T.make_triangles(w.tri_verts, w.tri_ids))
    yield tr
    tr.close()


@pytest.mark.parametrize("which", ["light", "sun", "sky"])
def test_room_grid_visibility_bit_exact(oracle_mod, grid, grid_tracer, which):
    w, r = grid
    rays = getattr(r, which)
    if which == "sky":
        rays = rays[::13]
    rays = np.ascontiguousarray(rays)
    tris = oracle_mod.prepare_triangles(w.tri_verts, w.tri_ids)
    for opts, flags in ((T.RayTraceOptions.stock_exact(), 0),
                        (T.RayTraceOptions(0.0, sky_does_not_block=True), oracle_mod.SKY_PASS)):
        _, _, bb = oracle_mod.brute_trace(tris, raw7(rays), flags=flags)
        got = grid_tracer.visibility(rays, opts)
        want = oracle_mod.bits_to_bool(bb, len(rays))
        assert np.array_equal(got, want), (which, flags, int((got != want).sum()))


@pytest.mark.parametrize("which", ["sun", "sky"])
def test_room_grid_closest_bit_exact(oracle_mod, grid, grid_tracer, which):
    w, r = grid
    rays = np.ascontiguousarray(getattr(r, which)[:: (1 if which == "sun" else 13)])
    tris = oracle_mod.prepare_triangles(w.tri_verts, w.tri_ids)
    bt, bd, _ = oracle_mod.brute_trace(tris, raw7(rays), flags=oracle_mod.CLOSEST)
    hits = grid_tracer.closest(rays)
    want_id = np.where(bt >= 0, w.tri_ids[np.maximum(bt, 0)], -1)
    assert np.array_equal(hits["surface"], want_id)
    hit = bt >= 0
    assert np.array_equal(hits["fraction"].view(np.uint32)[hit], bd.view(np.uint32)[hit])


def test_room_grid_matches_reference_kd_walk(oracle_mod, grid, grid_tracer):
    # The reference's own traversal (restated KD build + packet walk): the
    # same visibility bits on the light rays.
    w, r = grid
    tree = oracle_mod.kd_build(w.tri_verts, w.tri_ids)
    _, _, kb = oracle_mod.kd_trace(tree, raw7(r.light))
    got = grid_tracer.visibility(np.ascontiguousarray(r.light))
    assert np.array_equal(got, oracle_mod.bits_to_bool(kb, len(r.light)))


def test_min_distance_and_skip_id(oracle_mod, grid, grid_tracer):
    w, r = grid
    rays = np.ascontiguousarray(r.sky[::29])
    tris = oracle_mod.prepare_triangles(w.tri_verts, w.tri_ids)
    for tmin in (1e-3, 0.25):
        _, _, bb = oracle_mod.brute_trace(tris, raw7(rays), tmin=tmin)
        got = grid_tracer.visibility(rays, T.RayTraceOptions(tmin))
        assert np.array_equal(got, oracle_mod.bits_to_bool(bb, len(rays)))
        bt, bd, _ = oracle_mod.brute_trace(tris, raw7(rays), tmin=tmin, flags=oracle_mod.CLOSEST)
        hits = grid_tracer.closest(rays, T.RayTraceOptions(tmin))
        assert np.array_equal(hits["surface"], np.where(bt >= 0, w.tri_ids[np.maximum(bt, 0)], -1))
    # Skipping the opaque id leaves only sky triangles.
    _, _, bb = oracle_mod.brute_trace(tris, raw7(rays), skip_id=rg.TRACE_ID_OPAQUE)
    got = grid_tracer.visibility(rays, T.RayTraceOptions(0.0, skip_id=rg.TRACE_ID_OPAQUE))
    assert np.array_equal(got, oracle_mod.bits_to_bool(bb, len(rays)))


def test_edge_cases(oracle_mod, grid_tracer):
    # Empty batch, ragged sizes, NaN and zero directions, zero reach.
    assert grid_tracer.visibility(np.zeros(0, T.RAY_DTYPE)).shape == (0,)
    rng = np.random.default_rng(5)
    for n in (1, 31, 33, 63, 64, 65, 1000):
        raw = np.zeros((n, 7), np.float32)
        raw[:, 0:3] = rng.uniform(0, 3000, (n, 3))
        raw[:, 3:6] = rng.normal(0, 500, (n, 3))
        raw[:, 6] = 1.0
        raw[::7, 3:6] = 0.0            # zero-length segments hit nothing
        raw[::11, 3] = np.nan          # NaN directions hit nothing
        raw[::13, 6] = 0.0             # zero reach: never blocked
        bits = np.full((n + 63) // 64 + 1, 0xAB, np.uint64)  # one spare word must stay untouched
        grid_tracer.trace_visibility(as_rays(raw), bits)
        assert bits[-1] == 0xAB
        got = oracle_mod.bits_to_bool(bits[:-1], n)
        assert not got[::7].any() and not got[::11].any() and not got[::13].any()


def test_argument_errors(grid_tracer):
    rays = np.zeros(100, T.RAY_DTYPE)
    with pytest.raises(ValueError):
        grid_tracer.trace_visibility(rays, np.zeros(1, np.uint64))
    with pytest.raises(ValueError):
        grid_tracer.trace_closest(rays, np.zeros(99, T.HIT_DTYPE))
    with pytest.raises(ValueError):
        grid_tracer.trace_closest(rays, np.zeros(100, T.HIT_DTYPE), T.RayTraceOptions(0.0, sky_does_not_block=True))
    with pytest.raises(NotImplementedError):
        grid_tracer.trace_visibility(rays, np.zeros(2, np.uint64), T.RayTraceOptions(-1.0))
    assert not grid_tracer.supports(T.RayTraceOptions(float("nan")))
    assert grid_tracer.supports(T.RayTraceOptions(0.0, skip_id=5, sky_does_not_block=True))
    assert grid_tracer.tracer_identity.startswith("cuda-bvh-kdexact-1-")


def test_single_triangle_scene(oracle_mod):
    v = np.array([[0, 0, 0, 10, 0, 0, 0, 10, 0]], np.float32)
    raw = np.array([[1, 1, 5, 0, 0, -10, 1], [20, 20, 5, 0, 0, -10, 1], [1, 1, 5, 0, 0, -4, 1]], np.float32)
    with T.CudaRayTracer(v) as tr:
        vis = tr.visibility(as_rays(raw))
        hits = tr.closest(as_rays(raw))
    assert vis.tolist() == [True, False, False]
    assert hits["surface"].tolist() == [0, -1, -1]
    assert hits["fraction"][0] == np.float32(0.5)


def test_device_buffers_on_the_torch_stream(oracle_mod, grid, grid_tracer):
    import torch
    w, r = grid
    rays = np.ascontiguousarray(r.light)
    n = len(rays)
    d_rays = torch.from_numpy(rays.view(np.uint8).copy()).cuda()
    d_bits = torch.zeros((n + 63) // 64, dtype=torch.int64, device="cuda")
    d_hits = torch.zeros(n * 2, dtype=torch.int32, device="cuda")
    grid_tracer.trace_visibility(d_rays, d_bits)
    grid_tracer.trace_closest(d_rays, d_hits)
    torch.cuda.synchronize()
    bits = d_bits.cpu().numpy().view(np.uint64)
    assert np.array_equal(oracle_mod.bits_to_bool(bits, n), grid_tracer.visibility(rays))
    hits = d_hits.cpu().numpy().view(T.HIT_DTYPE)
    assert np.array_equal(hits, grid_tracer.closest(rays))
