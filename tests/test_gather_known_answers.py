"""The direct gather against the reference's known answers for one sample
and one light (src/SourceSharp.Tests/MapTools/Rad/Light/GatherTests.cs,
Correct compliance), on the oracle (CPU) and through the C ABI on the device
(vrad_world_upload + vrad_direct_lighting), and device against oracle bit
for bit.

The reference's cases gather at a point on a floor whose normal is +z, with
a light of unit intensity, and assert on the gather's dot and falloff; the
lighting value a sample receives is dot x falloff x intensity, so with unit
intensity the expected lighting is the reference's dot x falloff.  The point
here is the illumination point of a one-luxel floor face at z = -1 (the
gather starts one unit off the face, at the origin).  A blocked ray is a
large opaque quad at z = 50; a closed sky is a large opaque quad at z = 10;
an open sky is no geometry above the floor.
"""
import math
import types

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import lighting as L, workload as wl

FLOOR = np.array([[-0.5, -0.5, -1], [0.5, -0.5, -1], [0.5, 0.5, -1], [-0.5, 0.5, -1]], np.float32)


def _quad_tris(z, half, ident):
    a, b, c, d = ([-half, -half, z], [half, -half, z], [half, half, z], [-half, half, z])
    return [np.array(a + b + c, np.float32), np.array(a + c + d, np.float32)], [ident, ident]


def _light(kind, origin, c=1.0, l=0.0, q=0.0, normal=(0, 0, 0), stop=0.0, stop2=0.0, start=0.0, end=-1.0):
    e = np.zeros((), L.LIGHT_DTYPE)
    e["type"] = kind
    e["origin"] = origin
    e["intensity"] = (1, 1, 1)
    e["normal"] = normal
    e["stop_dot"], e["stop_dot2"] = stop, stop2
    e["constant_attn"], e["linear_attn"], e["quadratic_attn"] = c, l, q
    e["start_fade_distance"], e["end_fade_distance"] = start, end
    e["cap_dist"] = 1.0e22
    return e


def _mcos(deg):
    # MathF.Cos(deg * MathF.PI / 180) in float.
    return np.float32(math.cos(float(np.float32(np.float32(deg) * np.float32(math.pi)) / np.float32(180))))


FRINGE_N = (lambda v: (v / np.float32(np.sqrt(np.float32(v @ v)))).astype(np.float32))(
    np.array([0.3, 0, -1], np.float32))


def _fringe_expected():
    dot2 = -np.float32(np.float32(0 * FRINGE_N[0] + 0 * FRINGE_N[1]) + 1 * FRINGE_N[2])
    mult = np.float32((dot2 - np.float32(0.9)) / (np.float32(0.99) - np.float32(0.9)))
    return float(mult * dot2)


# name: (light, blocker z or None, sun samples, expected lighting check, visibility rays, sky rays)
CASES = {
    "point_overhead_unit_dot": (_light(1, (0, 0, 100)), None, 1, lambda v: v == 1.0, 1, 0),
    "inverse_square_falloff": (_light(1, (0, 0, 10), 0, 0, 1), None, 1, lambda v: v == np.float32(0.01), 1, 0),
    "falloff_distance_clamped_to_one": (_light(1, (0, 0, 0.5), 0, 0, 1), None, 1, lambda v: v == 1.0, 1, 0),
    "blocked_ray_zeroes_the_dot": (_light(1, (0, 0, 100)), 50.0, 1, lambda v: v == 0.0, 1, 0),
    "light_behind_asks_no_ray": (_light(1, (0, 0, -100)), None, 1, lambda v: v == 0.0, 0, 0),
    "forty_five_degrees_cosine": (_light(1, (100, 0, 100)), None, 1,
                                  lambda v: abs(v - math.sqrt(0.5)) < 5e-7, 1, 0),
    "spot_outside_outer_cone": (_light(2, (100, 0, 100), normal=(0, 0, -1), stop=_mcos(10), stop2=_mcos(20)),
                                None, 1, lambda v: v == 0.0, 0, 0),
    "spot_inside_inner_cone": (_light(2, (0, 0, 100), normal=(0, 0, -1), stop=_mcos(30), stop2=_mcos(45)),
                               None, 1, lambda v: v == 1.0, 1, 0),
    "spot_fringe_interpolates": (_light(2, (0, 0, 100), normal=tuple(FRINGE_N), stop=0.99, stop2=0.9), None, 1,
                                 lambda v: abs(v - _fringe_expected()) < 5e-6, 1, 0),
    "beyond_hard_falloff_end": (_light(1, (0, 0, 100), start=10, end=50), None, 1, lambda v: v == 0.0, 0, 0),
    "inside_fade_quintic": (_light(1, (0, 0, 30), start=10, end=50), None, 1, lambda v: abs(v - 0.5) < 5e-7, 1, 0),
    "sun_casts_toward_reverse": (_light(3, (0, 0, 0), normal=(0, 0, -1)), None, 1, lambda v: v == 1.0, 0, 1),
    "sun_hitting_geometry_shadowed": (_light(3, (0, 0, 0), normal=(0, 0, -1)), 50.0, 1, lambda v: v == 0.0, 0, 1),
    "soft_sun_thirty_rays": (_light(3, (0, 0, 0), normal=(0, 0, -1)), None, 30, lambda v: v == 1.0, 0, 30),
    "open_sky_ambient_unit_dot": (_light(4, (0, 0, 0)), None, 1, lambda v: abs(v - 1.0) < 5e-7, 0, None),
    # GatherTests.ASurfaceLightFallsOffAsItsNormalDotOverDistanceSquared
    # (GatherTests.cs:197-210): the emitter's cosine over the squared
    # distance; its ray ends DistEpsilon (1/32) short of the emitter: a
    # blocker below that end shadows, one between it and the emitter does not.
    "surface_dot_over_distance_squared": (_light(0, (0, 0, 10), normal=(0, 0, -1)), None, 1,
                                          lambda v: v == np.float32(0.01), 1, 0),
    "surface_blocked_below_the_ray_end": (_light(0, (0, 0, 10), normal=(0, 0, -1)), 9.9, 1,
                                          lambda v: v == 0.0, 1, 0),
    "surface_not_blocked_past_the_ray_end": (_light(0, (0, 0, 10), normal=(0, 0, -1)), 9.99, 1,
                                             lambda v: v == np.float32(0.01), 1, 0),
    "surface_facing_away_lights_nothing": (_light(0, (0, 0, 10), normal=(0, 0, 1)), None, 1,
                                           lambda v: v == 0.0, 0, 0),
    "closed_sky_ambient_nothing": (_light(4, (0, 0, 0)), 10.0, 1, lambda v: v == 0.0, 0, None),
}


def _inputs(name):
    light, blocker, sun_samples, _, _, _ = CASES[name]
    faces = np.zeros(1, L.FACE_DTYPE)
    faces["normal"] = (0, 0, 1)
    faces["dist"] = -1
    faces["lightmap_vecs"][0, 0] = (1, 0, 0, 0.5)
    faces["lightmap_vecs"][0, 1] = (0, 1, 0, 0.5)
    faces["lightmap_size"] = (1, 1)
    faces["num_vertices"] = 4
    samples, first = L.build_samples(faces, FLOOR)
    assert len(samples) == 1 and np.array_equal(samples["position"][0], [0, 0, -1])
    tris, ids = _quad_tris(-1.0, 0.5, 0)                      # the floor itself
    if blocker is not None:
        t2, i2 = _quad_tris(blocker, 1.0e6, 1)
        tris, ids = tris + t2, ids + i2
    world = types.SimpleNamespace(tri_verts=np.stack(tris), tri_ids=np.array(ids, np.int32))
    inp = L.LightingInputs(faces, FLOOR.copy(), samples, first, np.array([light]), np.array([0, 1], np.int32),
                           np.array([0], np.int32), wl.ambient_directions().astype(np.float32),
                           wl.ambient_directions(30).astype(np.float32) if sun_samples > 1 else
                           np.zeros((0, 3), np.float32),
                           sun_samples, np.float32(0.05) if sun_samples > 1 else 0.0)
    return world, inp


def _oracle(O, world, inp):
    tree = O.kd_build(world.tri_verts, world.tri_ids)
    return O.direct(tree, inp.faces, inp.samples, inp.face_first, inp.lights, inp.cluster_offsets,
                    inp.cluster_lights, inp.sky_directions, inp.sun_jitter, inp.sun_samples,
                    inp.sun_angular_extent, verts=inp.verts, extra_passes=0)


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_gather_known_answer(oracle_mod, name):
    world, inp = _inputs(name)
    out = _oracle(oracle_mod, world, inp)
    _, _, _, ok, _, _ = CASES[name]
    assert ok(float(out[0, 0])), (name, out[0])
    assert out[0, 0] == out[0, 1] == out[0, 2]
    if name.startswith("sun_casts"):
        assert out[0, 3] == 10000.0


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_device_gather_known_answer(oracle_mod, name):
    world, inp = _inputs(name)
    _, _, _, ok, vis, sky = CASES[name]
    with L.LightingStage(world, inp) as st:
        st.set_extra_passes(0)
        got, stats = st.direct()
    g = np.concatenate([got["lighting"], got["direct_sun_amount"][:, None]], 1)
    assert ok(float(g[0, 0])), (name, g[0])
    assert stats.visibility_rays == vis
    if sky is not None:
        assert stats.sky_rays == sky
    else:
        assert 1 <= stats.sky_rays <= 161       # the directions in front of the floor
    if name.startswith("sun_casts"):
        assert g[0, 3] == 10000.0
    want = _oracle(oracle_mod, world, inp)
    assert np.array_equal(g.view(np.uint32), want.view(np.uint32))
