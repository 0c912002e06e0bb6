"""GPU parity of the fused direct gather (vrad_direct_lighting) against the
oracle's restatement of the reference's four-sample-group gather.

The bar is bit-exact per sample: every LightingValue (lighting xyz and the
direct sun amount) equals the oracle's float bits.  The oracle traces with
the reference's own KD walk; the device with its BVH.
"""
import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import lighting as L, roomgrid as rg, workload as wl

pytestmark = pytest.mark.gpu


def oracle_direct(O, world, inp, faces=None):
    tree = O.kd_build(world.tri_verts, world.tri_ids)
    if faces is None:
        return O.direct(tree, inp.faces, inp.samples, inp.face_first, inp.lights, inp.cluster_offsets,
                        inp.cluster_lights, inp.sky_directions, inp.sun_jitter, inp.sun_samples,
                        inp.sun_angular_extent, verts=inp.verts)
    # A subset of faces: their samples, renumbered.
    sel = np.asarray(faces)
    ff = inp.face_first
    parts = [inp.samples[ff[f]:ff[f + 1]] for f in sel]
    counts = np.array([len(p) for p in parts])
    first = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    samples = np.concatenate(parts).copy()
    samples["face"] = np.repeat(np.arange(len(sel)), counts)
    out = O.direct(tree, inp.faces[sel], samples, first, inp.lights, inp.cluster_offsets,
                   inp.cluster_lights, inp.sky_directions, inp.sun_jitter, inp.sun_samples,
                   inp.sun_angular_extent, verts=inp.verts)
    index = np.concatenate([np.arange(ff[f], ff[f + 1]) for f in sel])
    return out, index


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_3x3_direct_bit_exact(oracle_mod):
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    with L.LightingStage(w, inp) as st:
        got, stats = st.direct()
    want = oracle_direct(oracle_mod, w, inp)
    g = np.concatenate([got["lighting"], got["direct_sun_amount"][:, None]], 1)
    assert stats.samples == len(inp.samples)
    assert stats.visibility_rays > 0 and stats.sky_rays > 0
    assert (want[:, :3] > 0).mean() > 0.3              # the map is lit
    diff = (bits(g) != bits(want)).any(1)
    assert not diff.any(), f"{int(diff.sum())} of {len(diff)} samples differ"


def test_3x3_jittered_sun_bit_exact(oracle_mod):
    # A sun with an angular extent: 30 jittered sky tests per sample, the
    # jitter table being the sampler's first 30 directions.
    w = rg.generate(rg.config_3x3(seed=4))
    inp = L.prepare(w)
    inp.sun_samples = 30
    inp.sun_angular_extent = np.float32(np.sin(np.pi / 180.0 * 5.0))
    inp.sun_jitter = wl.ambient_directions(30).astype(np.float32)
    with L.LightingStage(w, inp) as st:
        got, _ = st.direct()
    want = oracle_direct(oracle_mod, w, inp)
    g = np.concatenate([got["lighting"], got["direct_sun_amount"][:, None]], 1)
    sun = g[:, 3]
    assert ((sun > 0) & (sun < 10000)).any()          # partly lit samples exist
    assert np.array_equal(bits(g), bits(want))


def test_8x8_direct_bit_exact_on_sampled_faces(oracle_mod):
    # Spot and point lights, sun and the 162-direction sky: every 40th face.
    w = rg.generate(rg.config_8x8(seed=1))
    inp = L.prepare(w)
    with L.LightingStage(w, inp) as st:
        got, stats = st.direct()
    faces = np.arange(0, len(inp.faces), 40)
    want, index = oracle_direct(oracle_mod, w, inp, faces)
    g = np.concatenate([got["lighting"], got["direct_sun_amount"][:, None]], 1)[index]
    assert len(index) > 50_000
    diff = (bits(g) != bits(want)).any(1)
    assert not diff.any(), f"{int(diff.sum())} of {len(diff)} samples differ"
    assert stats.sky_rays > 50 * stats.samples         # the directions in front of each face


def test_device_output_matches_host_output():
    import torch
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    with L.LightingStage(w, inp) as st:
        host, _ = st.direct()
        d = torch.zeros(len(inp.samples) * 4, dtype=torch.float32, device="cuda")
        st.direct_device(d)
        torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32),
                          np.ascontiguousarray(host).view(np.uint32).reshape(-1))


def test_3x3_supersampling_counts_and_noextra(oracle_mod):
    # The supersampling passes select the same samples as the oracle's
    # (their count), change their light, and -noextra (0 passes) is the
    # plain four-sample-group gather bit for bit.
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    tree = oracle_mod.kd_build(w.tri_verts, w.tri_ids)
    args = (tree, inp.faces, inp.samples, inp.face_first, inp.lights, inp.cluster_offsets, inp.cluster_lights,
            inp.sky_directions, inp.sun_jitter, inp.sun_samples, inp.sun_angular_extent)
    with L.LightingStage(w, inp) as st:
        ss, ss_stats = st.direct()
        st.set_extra_passes(0)
        plain, plain_stats = st.direct()
    o_stats = {}
    want_ss = oracle_mod.direct(*args, verts=inp.verts, extra_passes=4, stats=o_stats)
    want_plain = oracle_mod.direct(*args, verts=inp.verts, extra_passes=0)
    g_ss = np.concatenate([ss["lighting"], ss["direct_sun_amount"][:, None]], 1)
    g_plain = np.concatenate([plain["lighting"], plain["direct_sun_amount"][:, None]], 1)
    assert np.array_equal(bits(g_plain), bits(want_plain))
    assert np.array_equal(bits(g_ss), bits(want_ss))
    assert ss_stats.supersampled == o_stats["supersampled"] > 100
    assert plain_stats.supersampled == 0 and ss_stats.extra_passes_run >= 1
    changed = (bits(g_ss) != bits(g_plain)).any(1)
    assert changed.sum() > 0.5 * ss_stats.supersampled
    assert ss_stats.visibility_rays + ss_stats.sky_rays > plain_stats.visibility_rays + plain_stats.sky_rays


@pytest.mark.parametrize("change", ["area", "coord", "mins", "position", "swap"])
def test_supersampling_refuses_samples_not_the_builders(change):
    # Supersampling needs each partial sample's cell winding, which the
    # library rebuilds from the faces; it accepts the world's samples only
    # when they are the sample builder's own, bit for bit.  One changed
    # field (or two samples of a face swapped) makes the gather refuse the
    # passes; with them off it still runs.
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    s = inp.samples.copy()
    ff = inp.face_first
    face = int(np.argmax(np.diff(ff)))
    k = int(ff[face]) + 1
    if change == "area":
        s["area"][k] = np.nextafter(s["area"][k], np.float32(np.inf))
    elif change == "coord":
        s["coord"][k, 1] = np.nextafter(s["coord"][k, 1], np.float32(-np.inf))
    elif change == "mins":
        s["mins"][k, 0] = np.nextafter(s["mins"][k, 0], np.float32(-np.inf))
    elif change == "position":
        s["position"][k, 2] = np.nextafter(s["position"][k, 2], np.float32(np.inf))
    else:
        s[[k, k + 1]] = s[[k + 1, k]]
    changed = L.LightingInputs(**{**inp.__dict__, "samples": s})
    with L.LightingStage(w, changed) as st:
        with pytest.raises(NotImplementedError, match="builder's own"):
            st.direct()
        st.set_extra_passes(0)
        plain, stats = st.direct()
        assert stats.supersampled == 0 and len(plain) == len(s)
    with L.LightingStage(w, inp) as st:
        st.direct()


def test_a_style_outside_a_byte_is_refused():
    """A face's style slots are bytes and 255 marks an empty one
    (FaceLight.Styles), so a light's style must lie in 0..254."""
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    lights = inp.lights.copy()
    lights["style"][len(lights) // 2] = 255
    with pytest.raises(ValueError, match="style 255"):
        L.LightingStage(w, L.LightingInputs(**{**inp.__dict__, "lights": lights}))
