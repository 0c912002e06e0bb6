"""Host logic: the room-grid generator and its ray workload, against the
oracle (reference KD traversal vs the brute-force semantic)."""
import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import roomgrid as rg, workload as wl


@pytest.fixture(scope="module")
def world3():
    return rg.generate(rg.config_3x3(seed=7))


def test_generator_is_seeded(world3):
    again = rg.generate(rg.config_3x3(seed=7))
    assert np.array_equal(world3.tri_verts, again.tri_verts)
    assert np.array_equal(world3.light_origin, again.light_origin)
    other = rg.generate(rg.config_3x3(seed=8))
    assert not np.array_equal(world3.light_origin, other.light_origin)


def test_shadow_casters_follow_brush_shadow_casters(world3):
    ids = world3.tri_ids
    assert set(np.unique(ids)) == {rg.TRACE_ID_OPAQUE, rg.TRACE_ID_SKY}
    assert (ids == rg.TRACE_ID_SKY).sum() == 2 * 9        # one sky quad per room
    # every brush is a box: 12 triangles, minus each ceiling's sky side
    assert (ids == rg.TRACE_ID_OPAQUE).sum() == 12 * len(world3.brushes) - 2 * 9


def test_lightmaps_respect_the_maximum_dimension(world3):
    assert world3.face_extents.max() <= rg.MAX_LIGHTMAP_DIM
    assert world3.luxel_counts().sum() > 150_000


def test_8x8_counts():
    w = rg.generate(rg.config_8x8(seed=1))
    assert 5_000_000 < w.luxel_counts().sum() < 8_000_000
    assert len(w.light_origin) == 64 and (w.light_type == 2).any()


def test_ambient_directions_are_unit_and_162():
    d = wl.ambient_directions()
    assert d.shape == (162, 3)
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6)


def test_reference_traversal_equals_brute_force_on_room_grid(oracle_mod, world3):
    s = wl.luxel_samples(world3, stride=7)
    r = wl.direct_rays(world3, s, ambient=True)
    tris = oracle_mod.prepare_triangles(world3.tri_verts, world3.tri_ids)
    tree = oracle_mod.kd_build(world3.tri_verts, world3.tri_ids)
    for rays, flags in ((r.light, 0), (r.sun, oracle_mod.SKY_PASS), (r.sky[::40], oracle_mod.SKY_PASS)):
        raw = np.ascontiguousarray(rays).view(np.float32).reshape(-1, 7)
        _, _, kb = oracle_mod.kd_trace(tree, raw, flags=flags)
        _, _, bb = oracle_mod.brute_trace(tris, raw, flags=flags)
        n = len(raw)
        assert n > 1000
        assert np.array_equal(oracle_mod.bits_to_bool(kb, n), oracle_mod.bits_to_bool(bb, n))
