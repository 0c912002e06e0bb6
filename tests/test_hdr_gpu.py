"""Both ranges of the lighting stage (LDR then HDR, the reference's -both:
MapTools/Rad/Vrad.cs:150-158, 262-285) through vrad_light_pass_ranges,
against the oracle run once per range with that range's light list.

The bar is the same as the LDR pass's: each lump byte for byte, the bounce
counts, and per-sample direct light bit for bit.  The HDR range reuses the
LDR range's transfers (they are geometry), and the first round of the
direct gather lights both ranges from one traversal; the tests check that
neither changes a bit of either range.
"""
import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import lighting as L, roomgrid as rg

pytestmark = pytest.mark.gpu


def _oracle_range(O, tree, w, inp, lights, refl, off, lst, threshold, sample_light=None, transfers=None):
    if sample_light is None:
        sample_light = O.direct(tree, inp.faces, inp.samples, inp.face_first, lights, inp.cluster_offsets,
                                inp.cluster_lights, inp.sky_directions, inp.sun_jitter, inp.sun_samples,
                                inp.sun_angular_extent, verts=inp.verts)
    ob = O.Bounce(tree, inp.faces, inp.verts, inp.samples, inp.face_first, refl, off, lst, bounces=100,
                  threshold=threshold)
    if transfers is not None:
        ob.set_transfers(*transfers)
    _, _, n, _ = ob.run(sample_light)
    lump, ofs = ob.final(sample_light)
    return lump, ofs, n, sample_light


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _values(v):
    return np.concatenate([v["lighting"], v["direct_sun_amount"][:, None]], 1)


@pytest.mark.parametrize("threshold", [1.0, 0.1])
def test_3x3_both_ranges_byte_identical_to_the_oracle(oracle_mod, threshold):
    O = oracle_mod
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w, hdr=True)
    refl = L.face_reflectivity(w)
    off, lst = L.pvs_lists(w)
    assert not np.array_equal(inp.lights["intensity"], inp.lights_hdr["intensity"])
    with L.LightingStage(w, inp) as st:
        st.upload_bounce(refl, off, lst, threshold=threshold)
        ldr, hdr, ofs, stats, bs = st.light_pass_ranges()
        ldr_only, ofs_only, _ = st.light_pass()
    tree = O.kd_build(w.tri_verts, w.tri_ids)
    lo, oo, n_ldr, _ = _oracle_range(O, tree, w, inp, inp.lights, refl, off, lst, threshold)
    ho, _, n_hdr, _ = _oracle_range(O, tree, w, inp, inp.lights_hdr, refl, off, lst, threshold)
    assert np.array_equal(ldr, lo) and np.array_equal(ofs, oo)
    assert np.array_equal(hdr, ho)
    assert not np.array_equal(ldr, hdr)
    assert np.array_equal(ldr, ldr_only) and np.array_equal(ofs, ofs_only)
    assert (bs[0].bounces, bs[1].bounces) == (n_ldr, n_hdr)
    # One transfer build serves both ranges.
    assert bs[0].transfer_rays > 0 and bs[1].transfer_rays == 0
    assert bs[0].transfers == bs[1].transfers > 0
    assert stats.visibility_rays > 0 and stats.sky_rays > 0


def test_8x8_both_ranges_sampled_direct_and_whole_lumps(oracle_mod):
    O = oracle_mod
    w = rg.generate(rg.config_8x8(seed=1))
    inp = L.prepare(w, hdr=True)
    refl = L.face_reflectivity(w)
    off, lst = L.pvs_lists(w)
    with L.LightingStage(w, inp) as st:
        st.upload_bounce(refl, off, lst, threshold=0.1)
        ldr, hdr, ofs, stats, bs = st.light_pass_ranges()
        got_ldr = _values(st.pass_sample_light(L.RANGE_LDR))
        got_hdr = _values(st.pass_sample_light(L.RANGE_HDR))
        t_off, t_rec = st.transfers()
        single, _ = st.direct()                      # the LDR-only gather kernel
    # The two-range gather's LDR values are the one-range kernel's bits.
    assert np.array_equal(bits(got_ldr), bits(_values(single)))
    # Sampled faces of the HDR range against the oracle's gather.
    tree = O.kd_build(w.tri_verts, w.tri_ids)
    sel = np.arange(0, len(inp.faces), 53)
    ff = inp.face_first
    parts = [inp.samples[ff[f]:ff[f + 1]] for f in sel]
    counts = np.array([len(p) for p in parts])
    first = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    samples = np.concatenate(parts).copy()
    samples["face"] = np.repeat(np.arange(len(sel)), counts)
    want = O.direct(tree, inp.faces[sel], samples, first, inp.lights_hdr, inp.cluster_offsets, inp.cluster_lights,
                    inp.sky_directions, inp.sun_jitter, inp.sun_samples, inp.sun_angular_extent, verts=inp.verts)
    index = np.concatenate([np.arange(ff[f], ff[f + 1]) for f in sel])
    assert len(index) > 50_000
    assert np.array_equal(bits(got_hdr[index]), bits(want))
    # The whole HDR lump: the oracle's bounce and final pass fed the
    # device's HDR sample light and transfers (each pinned above and by the
    # LDR tests), byte for byte.
    ho, _, n_hdr, _ = _oracle_range(O, tree, w, inp, inp.lights_hdr, refl, off, lst, 0.1, sample_light=got_hdr,
                                    transfers=(t_off, t_rec["patch"], t_rec["weight"]))
    assert bs[1].bounces == n_hdr
    assert np.array_equal(hdr, ho)
    assert bs[1].transfer_rays == 0 and bs[0].transfer_rays > 0


def test_device_buffers_equal_host_buffers():
    import torch
    w = rg.generate(rg.config_3x3(seed=3))
    inp = L.prepare(w, hdr=True)
    refl = L.face_reflectivity(w)
    off, lst = L.pvs_lists(w)
    with L.LightingStage(w, inp) as st:
        st.upload_bounce(refl, off, lst, threshold=0.1)
        ldr, hdr, _, _, _ = st.light_pass_ranges()
        n = st.lighting_size()
        d_ldr = torch.zeros(n, dtype=torch.uint8, device="cuda")
        d_hdr = torch.zeros(n, dtype=torch.uint8, device="cuda")
        st.light_pass_ranges_device(d_ldr, d_hdr)
        torch.cuda.synchronize()
        # The HDR range alone (its own gather kernel and transfer build).
        none, hdr_only, _, _, bs = st.light_pass_ranges(L.RANGE_HDR)
    assert np.array_equal(d_ldr.cpu().numpy(), ldr) and np.array_equal(d_hdr.cpu().numpy(), hdr)
    assert none is None and np.array_equal(hdr_only, hdr)
    assert bs[0].bounces == 0 and bs[1].transfer_rays > 0


def test_hdr_without_an_hdr_list_is_refused():
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    with L.LightingStage(w, inp) as st:
        with pytest.raises(Exception, match="HDR light list"):
            st.light_pass_ranges()
