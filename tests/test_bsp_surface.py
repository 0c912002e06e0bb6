"""The BSP surface tracer (stock vrad's CLightSurface walk of the map's own
BSP tree, the tracer leaf ambient uses) on the reference's committed real
map, dm_lockdown (BSP v19, 2,682 nodes, 6,536 faces, 2,725 leaves), against
the answers stock's own compiled tracer gave for the reference's recorded
8,100 leaf-ambient rays (Tests/MapTools/Tracing/Fixtures/README-bsp-rays.md,
BspSurfaceStockParityTests.cs): the face hit, the fraction bit for bit, and
m_bHasLuxel (a hit on a face that is not sky).  The oracle's restatement
(oracle/bsp_oracle.cpp) is checked on the CPU; the device's walk
(vrad_bsp_trace_closest) on the GPU, against stock and against the oracle
on a larger seeded set of rays of the same shape."""
import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import bsp as B
from tests.golden import fixtures as F


@pytest.fixture(scope="module")
def lockdown():
    lumps = F.lockdown_lumps()
    return B.trace_geometry(lumps)


def test_lockdown_lumps_read_as_the_reference_counts_them(lockdown):
    g = lockdown
    assert g.nodes.shape[0] == 2682 and g.surfaces.shape[0] == 6536 and len(g.leaf_start) == 2725
    assert g.skipped_displacements > 0 and g.sky.any()


def test_oracle_walk_gives_stocks_answers(oracle_mod, lockdown):
    rays, face, frac, lux = F.lockdown_rays()
    assert len(rays) == 50 * 162
    got_face, got_frac = oracle_mod.bsp_trace(lockdown, rays)
    assert np.array_equal(got_face, face)
    assert np.array_equal(got_frac.view(np.uint32), frac.view(np.uint32))
    derived = (got_face >= 0) & ~lockdown.sky[np.maximum(got_face, 0)]
    assert np.array_equal(derived, lux)
    assert (face >= 0).sum() > len(face) // 2 and ((face >= 0) & ~lux).any()


def _leaf_ambient_rays(n_points=2000, seed=9):
    """Rays of the stock set's shape: points near the recorded set's sample
    points, each with the sampler's 162 directions out to 1.74 x the
    coordinate extent."""
    from hl2sdk_tools_sharp_b200 import workload as wl
    rays, _, _, _ = F.lockdown_rays()
    starts = rays[::162, 0:3]
    rng = np.random.default_rng(seed)
    pts = (starts[rng.integers(0, len(starts), n_points)] + rng.uniform(-48, 48, (n_points, 3))).astype(np.float32)
    dirs = wl.ambient_directions().astype(np.float32) * np.float32(16384 * 2 * 1.74)
    out = np.empty((n_points * 162, 7), np.float32)
    out[:, 0:3] = np.repeat(pts, 162, axis=0)
    out[:, 3:6] = np.tile(dirs, (n_points, 1))
    out[:, 6] = 1.0
    return out


@pytest.mark.gpu
def test_device_walk_gives_stocks_answers_and_the_oracles(oracle_mod, lockdown):
    rays, face, frac, lux = F.lockdown_rays()
    with B.CudaBspTracer(lockdown) as tr:
        hits = tr.trace_closest(rays)
        assert np.array_equal(hits["surface"], face)
        assert np.array_equal(hits["fraction"].view(np.uint32), frac.view(np.uint32))
        assert np.array_equal((hits["surface"] >= 0) & ~lockdown.sky[np.maximum(hits["surface"], 0)], lux)
        big = _leaf_ambient_rays()
        got = tr.trace_closest(big)
        want_face, want_frac = oracle_mod.bsp_trace(lockdown, big)
        assert np.array_equal(got["surface"], want_face)
        assert np.array_equal(got["fraction"].view(np.uint32), want_frac.view(np.uint32))
        assert (want_face >= 0).mean() > 0.5
        # A minimum fraction skips leaf-face hits below it.
        got = tr.trace_closest(big[:16200], min_distance=0.001)
        want_face, want_frac = oracle_mod.bsp_trace(lockdown, big[:16200], min_frac=0.001)
        assert np.array_equal(got["surface"], want_face)
        assert np.array_equal(got["fraction"].view(np.uint32), want_frac.view(np.uint32))


def test_oracle_on_the_seeded_set_stops_within_its_stack(oracle_mod, lockdown):
    face, _ = oracle_mod.bsp_trace(lockdown, _leaf_ambient_rays(200))
    assert (face >= 0).mean() > 0.5
