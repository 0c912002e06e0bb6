"""Light styles above 0 on the CPU.

The reference's style cases (RadWorldTests.cs:84-110:
EveryLitFaceHasStyleZeroFirst, AStyledLightTakesTheSecondSlot,
AFifthStyleOnAFaceIsWarnedAndDropped) restated on the oracle's gather
(FaceLightJob's slots: FindOrAllocateStyle at ResolveGroup's skip test,
FaceLightJob.cs:399-455) over the seeded 3x3 room grid, with the grid's
lights given styles; and the library's styled lightmap layout
(vrad_lightmap_layout_styles, LightmapOffsets.cs:84-123) against the
oracle's final pass on the same styles.  The device path is in
test_light_styles_gpu.py."""
import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import lighting as L, roomgrid as rg

# On the 3x3 grid (seed 2) lights 0-3 are point lights, 4 the sky ambient
# and 5 the sun; cluster 6's list holds all six.
FOUR_AND_SKY = {0: 1, 1: 2, 2: 3, 3: 4, 4: 9}


@pytest.fixture(scope="module")
def grid(oracle_mod):
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    return w, inp, oracle_mod.kd_build(w.tri_verts, w.tri_ids)


def styled(inp, styles):
    lights = inp.lights.copy()
    for i, s in styles.items():
        lights["style"][i] = s
    return lights


def gather(O, grid, lights, extra_passes=0):
    w, inp, tree = grid
    return O.direct_styles(tree, inp.faces, inp.samples, inp.face_first, lights, inp.cluster_offsets,
                           inp.cluster_lights, inp.sky_directions, inp.sun_jitter, inp.sun_samples,
                           inp.sun_angular_extent, verts=inp.verts, extra_passes=extra_passes)


def test_every_lit_face_has_style_zero_first(oracle_mod, grid):
    _, _, styles, _ = gather(oracle_mod, grid, styled(grid[1], FOUR_AND_SKY))
    assert (styles[:, 0] == 0).all()


def test_a_styled_light_takes_the_second_slot(oracle_mod, grid):
    w, inp, _ = grid
    out, slots, styles, dropped = gather(oracle_mod, grid, styled(inp, {0: 5}))
    lit = (styles == [0, 5, 255, 255]).all(1)
    plain = (styles == [0, 255, 255, 255]).all(1)
    assert lit.any() and plain.any() and (lit | plain).all() and dropped == 0
    # The style-5 light's light is in slot 1 alone: slot 0 of those faces
    # no longer holds it.
    unstyled, _, _, _ = gather(oracle_mod, grid, inp.lights)
    first = inp.face_first
    f = int(np.flatnonzero(lit)[0])
    a, b = first[f], first[f + 1]
    assert (slots[0, a:b, :3] > 0).any()
    assert (out[a:b, :3] <= unstyled[a:b, :3]).all() and (out[a:b, :3] < unstyled[a:b, :3]).any()
    # Faces without a slot for it have zeros there.
    g = int(np.flatnonzero(plain)[0])
    assert (slots[:, first[g]:first[g + 1]] == 0).all()


def test_a_fifth_style_on_a_face_is_dropped(oracle_mod, grid):
    _, _, styles, dropped = gather(oracle_mod, grid, styled(grid[1], FOUR_AND_SKY))
    assert dropped > 0
    assert ((styles != 255).sum(1) == 4).sum() >= dropped


def test_slot_order_is_the_order_of_first_light(oracle_mod, grid):
    """Two faces can hold the same styles in different slots: the slots
    follow which style's light reaches the face's earliest sample group."""
    _, _, styles, _ = gather(oracle_mod, grid, styled(grid[1], {0: 5, 1: 6, 2: 7, 3: 8}))
    rows = {tuple(r) for r in styles}
    sets = {}
    for r in rows:
        sets.setdefault(frozenset(x for x in r if x != 255), set()).add(r)
    assert any(len(v) > 1 for v in sets.values())


def test_library_layout_equals_the_oracle_with_styles(oracle_mod, grid):
    w, inp, _ = grid
    out, slots, styles, _ = gather(oracle_mod, grid, styled(inp, FOUR_AND_SKY))
    lump, ofs = oracle_mod.final_styles(inp.faces, inp.verts, inp.samples, inp.face_first, out, slots, styles)
    mine, total = L.lightmap_layout(inp.faces, styles)
    assert np.array_equal(mine, ofs) and total == len(lump)
    # Style 0 alone gives the plain layout.
    plain, ptotal = L.lightmap_layout(inp.faces)
    alone = np.zeros_like(styles) + 255
    alone[:, 0] = 0
    assert np.array_equal(L.lightmap_layout(inp.faces, alone)[0], plain)
    assert total > ptotal
