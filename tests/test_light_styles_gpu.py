"""Light styles above 0 on the GPU, against the oracle's restatement of
FaceLightJob's style slots (FaceLightJob.cs:399-455, 465-550, 679-730),
FinalLightFace's per-style loop (FinalLightFace.cs:154-285, 339-380) and
LightmapOffsets (LightmapOffsets.cs:84-123), on the seeded 3x3 room grid
with its lights given styles (one face in some rooms then lit by five
styles, the fifth dropped):

  * each face's style bytes and the faces that dropped one;
  * the LIGHTING lump (every style's luxels and medians, supersampling on)
    and the FACES lightofs, byte for byte;
  * with the bounce, both ranges: the bounced light goes into style 0's
    slot only, LIGHTING and LIGHTING_HDR byte for byte."""
import dataclasses

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import lighting as L, roomgrid as rg
from test_light_styles_cpu import FOUR_AND_SKY, styled

pytestmark = pytest.mark.gpu


def oracle_gather(O, tree, inp, lights):
    return O.direct_styles(tree, inp.faces, inp.samples, inp.face_first, lights, inp.cluster_offsets,
                           inp.cluster_lights, inp.sky_directions, inp.sun_jitter, inp.sun_samples,
                           inp.sun_angular_extent, verts=inp.verts, extra_passes=4)


def test_styled_lump_equals_the_oracle(oracle_mod):
    O = oracle_mod
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    lights = styled(inp, FOUR_AND_SKY)
    tree = O.kd_build(w.tri_verts, w.tri_ids)
    out, slots, want_styles, want_dropped = oracle_gather(O, tree, inp, lights)
    want, want_ofs = O.final_styles(inp.faces, inp.verts, inp.samples, inp.face_first, out, slots, want_styles)
    with L.LightingStage(w, dataclasses.replace(inp, lights=lights)) as st:
        styles, dropped = st.face_styles()
        assert st.lighting_size() == len(want)
        lump, ofs, _ = st.light_pass()
        again, _, _ = st.light_pass()
    assert np.array_equal(styles, want_styles) and dropped == want_dropped > 0
    assert np.array_equal(ofs, want_ofs)
    bad = np.flatnonzero(lump.view(np.uint32) != want.view(np.uint32))
    assert len(bad) == 0, f"{len(bad)} of {len(lump) // 4} words differ"
    assert np.array_equal(again, lump)


def test_styled_bounce_both_ranges_equal_the_oracle(oracle_mod):
    O = oracle_mod
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w, hdr=True)
    marks = {0: 5, 2: 6, 4: 7}
    lights, lights_hdr = styled(inp, marks), inp.lights_hdr.copy()
    for i, s in marks.items():
        lights_hdr["style"][i] = s
    styled_inp = dataclasses.replace(inp, lights=lights, lights_hdr=lights_hdr)
    tree = O.kd_build(w.tri_verts, w.tri_ids)
    off, lst = L.pvs_lists(w)
    ob = O.Bounce(tree, inp.faces, inp.verts, inp.samples, inp.face_first, L.face_reflectivity(w), off, lst,
                  bounces=100, threshold=1.0)
    ob.transfers()
    want = {}
    for r, ls in (("ldr", lights), ("hdr", lights_hdr)):
        out, slots, styles, _ = oracle_gather(O, tree, inp, ls)
        ob.run(out)
        want[r] = ob.final(out, slots, styles)
    with L.LightingStage(w, styled_inp) as st:
        st.upload_bounce(L.face_reflectivity(w), off, lst, bounces=100, threshold=1.0)
        ldr, hdr, ofs, _, bst = st.light_pass_ranges()
        styles, _ = st.face_styles()
    assert (styles[:, 1] != 255).any()
    for r, got in (("ldr", ldr), ("hdr", hdr)):
        lump, want_ofs = want[r]
        assert np.array_equal(ofs, want_ofs)
        bad = np.flatnonzero(got.view(np.uint32) != lump.view(np.uint32))
        assert len(bad) == 0, f"{r}: {len(bad)} of {len(lump) // 4} words differ"
    assert bst[0].bounces > 1


def test_a_map_without_styled_lights_keeps_style_zero_alone():
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    with L.LightingStage(w, inp) as st:
        styles, dropped = st.face_styles()
        size = st.lighting_size()
    assert (styles == [0, 255, 255, 255]).all() and dropped == 0
    assert size == L.lightmap_layout(inp.faces)[1]
