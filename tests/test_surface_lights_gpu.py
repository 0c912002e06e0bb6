"""Surface lights on the GPU against the oracle: the 3x3 room grid with one
wall panel made a texlight (its leaf patches, at the bounce's chop sizes,
become 32 surface lights, DirectLightBuilder.AddSurfaceLights), gathered
by GatherSurfaceFour's arithmetic (DirectLightGatherer.cs:1452-1545), with
the panel's patches left unrefined at its edges (PatchSubdivider.cs:
375-380):

  * the LIGHTING lump, supersampling on, byte for byte;
  * with the bounce, LIGHTING and LIGHTING_HDR byte for byte."""
import dataclasses

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import lighting as L, roomgrid as rg

pytestmark = pytest.mark.gpu


def texlit_world():
    w = rg.generate(rg.config_3x3(seed=2))
    emit = np.zeros((w.face_count, 4))
    emit[148] = (220, 230, 255, 300)
    return dataclasses.replace(w, face_emit=emit)


def oracle_gather(O, tree, inp, lights):
    return O.direct(tree, inp.faces, inp.samples, inp.face_first, lights, inp.cluster_offsets, inp.cluster_lights,
                    inp.sky_directions, inp.sun_jitter, inp.sun_samples, inp.sun_angular_extent, verts=inp.verts)


def test_texlit_lump_equals_the_oracle(oracle_mod):
    O = oracle_mod
    w = texlit_world()
    inp = L.prepare(w)
    assert (inp.lights["type"] == 0).sum() == 32
    tree = O.kd_build(w.tri_verts, w.tri_ids)
    want, want_ofs = O.final(inp.faces, inp.verts, inp.samples, inp.face_first, oracle_gather(O, tree, inp, inp.lights))
    with L.LightingStage(w, inp) as st:
        lump, ofs, stats = st.light_pass()
    assert np.array_equal(ofs, want_ofs)
    bad = np.flatnonzero(lump.view(np.uint32) != want.view(np.uint32))
    assert len(bad) == 0, f"{len(bad)} of {len(lump) // 4} words differ"
    # The panel lights its room: the lump differs from the map without it.
    with L.LightingStage(rg.generate(rg.config_3x3(seed=2))) as plain:
        dark, _, _ = plain.light_pass()
    assert len(dark) == len(lump) and not np.array_equal(dark, lump)


def test_texlit_bounce_both_ranges_equal_the_oracle(oracle_mod):
    O = oracle_mod
    w = texlit_world()
    inp = L.prepare(w, hdr=True)
    tree = O.kd_build(w.tri_verts, w.tri_ids)
    off, lst = L.pvs_lists(w)
    refl = L.face_reflectivity(w)
    ob = O.Bounce(tree, inp.faces, inp.verts, inp.samples, inp.face_first, refl, off, lst, bounces=100,
                  threshold=1.0)
    ob.transfers()
    want = {}
    for r, ls in (("ldr", inp.lights), ("hdr", inp.lights_hdr)):
        out = oracle_gather(O, tree, inp, ls)
        ob.run(out)
        want[r] = ob.final(out)
    with L.LightingStage(w, inp) as st:
        st.upload_bounce(refl, off, lst, bounces=100, threshold=1.0)
        ldr, hdr, ofs, _, bst = st.light_pass_ranges()
        patches = st.bounce_stats().patches
    assert patches == len(ob.patches()[0])
    for r, got in (("ldr", ldr), ("hdr", hdr)):
        lump, want_ofs = want[r]
        assert np.array_equal(ofs, want_ofs)
        bad = np.flatnonzero(got.view(np.uint32) != lump.view(np.uint32))
        assert len(bad) == 0, f"{r}: {len(bad)} of {len(lump) // 4} words differ"
    assert bst[0].bounces > 1
