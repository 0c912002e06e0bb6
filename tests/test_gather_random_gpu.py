"""The gather's light arithmetic on random lights, device against oracle bit
for bit: the counterpart here of the reference's four-wide-against-scalar
facts (PointLightFourTests.cs:53-114, SurfaceLightFourTests.cs:80-143),
which hold its two code paths to one answer on random lights.

256 one-luxel faces, each facing one of the six axes at a random place and
in a cluster of its own whose list holds one random light: a point, spot or
surface light with random attenuation, cap, hard fade and spot cone, now
and then sitting on the sample's point or in the face's plane.  Each sample
then carries its one light's dot x falloff x intensity (and visibility: the
other faces are the scene), so every bit the gather writes is compared
(two NaNs agree whatever their payloads)."""
import types

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import lighting as L, workload as wl

pytestmark = pytest.mark.gpu

AXES = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.float32)


def _frame(n):
    """Two axes in the face's plane (axis-aligned, so luxel coordinates are exact)."""
    k = int(np.argmax(np.abs(n)))
    s = np.zeros(3, np.float32)
    s[(k + 1) % 3] = 1
    t = np.cross(n, s).astype(np.float32)
    return s, t


def _world(seed, count=256):
    rng = np.random.default_rng(seed)
    faces = np.zeros(count, L.FACE_DTYPE)
    verts, tris = [], []
    lights = np.zeros(count, L.LIGHT_DTYPE)
    for i in range(count):
        n = AXES[rng.integers(6)]
        c = np.round(rng.uniform(-400, 400, 3)).astype(np.float32)
        s, t = _frame(n)
        quad = [c - 0.5 * s - 0.5 * t, c + 0.5 * s - 0.5 * t, c + 0.5 * s + 0.5 * t, c - 0.5 * s + 0.5 * t]
        verts.extend(quad)
        tris += [np.concatenate([quad[0], quad[1], quad[2]]), np.concatenate([quad[0], quad[2], quad[3]])]
        faces[i]["normal"] = n
        faces[i]["dist"] = float(n @ c)
        faces[i]["lightmap_vecs"][0] = (*s, 0.5 - float(s @ c))
        faces[i]["lightmap_vecs"][1] = (*t, 0.5 - float(t @ c))
        faces[i]["lightmap_size"] = (1, 1)
        faces[i]["first_vertex"] = 4 * i
        faces[i]["num_vertices"] = 4
        faces[i]["cluster"] = i
        kind = rng.choice([0, 1, 2])
        L_ = lights[i]
        L_["type"] = kind
        point = c + n                                     # the gather's point, one unit off the face
        r = rng.integers(40)
        if r == 0:
            L_["origin"] = point                          # on the sample's point: a zero distance
        elif r < 4:
            L_["origin"] = point + (s * rng.uniform(-200, 200)).astype(np.float32)   # in the point's plane
        else:
            L_["origin"] = point + rng.uniform(-300, 300, 3).astype(np.float32)
        L_["intensity"] = rng.uniform(10, 400, 3).astype(np.float32)
        d = rng.normal(size=3).astype(np.float32)
        if rng.integers(3) == 0:
            d = AXES[rng.integers(6)].copy()              # axial emitters: exact zero cosines
        L_["normal"] = d / np.float32(np.sqrt(np.float32(d @ d)))
        L_["constant_attn"] = 0 if rng.integers(3) == 0 else rng.uniform()
        L_["linear_attn"] = 0 if rng.integers(2) == 0 else rng.uniform() * 0.1
        L_["quadratic_attn"] = 0 if rng.integers(3) == 0 else rng.uniform() * 0.01
        if L_["constant_attn"] == 0 and L_["linear_attn"] == 0 and L_["quadratic_attn"] == 0:
            L_["constant_attn"] = 1
        L_["cap_dist"] = rng.uniform() * 300 if rng.integers(3) == 0 else 1.0e22
        L_["end_fade_distance"] = -1
        if rng.integers(2) == 0:
            L_["start_fade_distance"] = rng.uniform() * 200
            L_["end_fade_distance"] = L_["start_fade_distance"] + rng.uniform() * 300 - 50
        if kind == 2:
            outer = np.float32(np.cos(np.radians(rng.uniform(10, 80))))
            L_["stop_dot2"] = outer
            L_["stop_dot"] = np.float32(min(0.999, float(outer) + rng.uniform(0.0, 0.3)))
            L_["exponent"] = rng.choice([0.0, 1.0, 2.0, 0.5])
    verts = np.array(verts, np.float32)
    samples, first = L.build_samples(faces, verts)
    assert len(samples) == count
    world = types.SimpleNamespace(tri_verts=np.stack(tris).astype(np.float32),
                                  tri_ids=np.arange(len(tris), dtype=np.int32) // 2)
    inp = L.LightingInputs(faces, verts, samples, first, lights, np.arange(count + 1, dtype=np.int32),
                           np.arange(count, dtype=np.int32), wl.ambient_directions().astype(np.float32),
                           np.zeros((0, 3), np.float32))
    return world, inp


@pytest.mark.parametrize("seed", [4242, 9191])
def test_random_lights_device_equals_oracle(oracle_mod, seed):
    world, inp = _world(seed)
    tree = oracle_mod.kd_build(world.tri_verts, world.tri_ids)
    want = oracle_mod.direct(tree, inp.faces, inp.samples, inp.face_first, inp.lights, inp.cluster_offsets,
                             inp.cluster_lights, inp.sky_directions, inp.sun_jitter, inp.sun_samples,
                             inp.sun_angular_extent, verts=inp.verts, extra_passes=0)
    with L.LightingStage(world, inp) as st:
        st.set_extra_passes(0)
        got, stats = st.direct()
    g = np.concatenate([got["lighting"], got["direct_sun_amount"][:, None]], 1).astype(np.float32)
    # A light on the sample's point gives NaN on both sides; the NaN's
    # payload is the machine's (x86's default NaN is negative), not the
    # arithmetic's, so two NaNs agree and every other value is compared
    # bit for bit.
    same = (g.view(np.uint32) == want.view(np.uint32)) | (np.isnan(g) & np.isnan(want))
    bad = np.flatnonzero(~same.all(1))
    assert len(bad) == 0, f"{len(bad)} of {len(g)} samples differ, first {bad[:5]}"
    # The draw reaches lit samples of every kind, and the ray-tracing branch.
    lit = (want[:, :3] > 0).any(1)
    for kind in (0, 1, 2):
        assert (lit & (inp.lights["type"] == kind)).any()
    assert stats.visibility_rays > 20
