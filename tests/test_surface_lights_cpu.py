"""Surface lights (texlights) on the CPU: the reference's DirectLightTests
cases (DirectLightTests.cs:261-292) restated on the host layer's
AddSurfaceLights (lights.add_surface_lights) and on the room grid's
texlight panels, and the emitting faces' subdivision (no face-edge
refinement, PatchSubdivider.cs:375-380) on the library's patch builder
against the oracle's."""
import dataclasses

import numpy as np

from hl2sdk_tools_sharp_b200 import lighting as L, lights as LT, roomgrid as rg


def _one_patch(base_light, area=256.0 * 256.0, scale=(0.25, 0.25), base_area=64.0 * 64.0, leaf=True):
    f32 = np.float32
    return LT.SurfacePatches(origin=np.array([[0, 0, 100]], f32), normal=np.array([[0, 0, -1]], f32),
                             area=np.array([area], f32), face=np.array([0], np.int32), leaf=np.array([leaf]),
                             base_light=np.array([base_light], f32), base_area=np.array([base_area], f32),
                             scale=np.array([scale], f32))


def test_a_surface_lights_intensity_carries_area_texture_scale_and_direct_scale():
    # ASurfaceLightsIntensityCarriesAreaTextureScaleAndDirectScale: one
    # 256 x 256 patch of a 64 x 64 texel texture at 0.25 world units a texel.
    ls = LT.DirectLightSet()
    LT.add_surface_lights(ls, _one_patch((255, 255, 255)), lambda o: 0)
    (light,) = ls.active
    expected = np.float32(255.0 * 1.0 * (256.0 * 256.0) * 0.25 * 0.25 / (64.0 * 64.0) * 10000.0)
    assert light.type == LT.EMIT_SURFACE and light.intensity[0] == expected
    assert np.array_equal(light.normal, [0, 0, -1]) and np.array_equal(light.origin, [0, 0, 100])


def test_dim_parents_and_textures_without_area_make_no_light():
    for sp in (_one_patch((0.2, 0.05, 0.0)), _one_patch((255, 255, 255), leaf=False),
               _one_patch((255, 255, 255), base_area=0.0)):
        ls = LT.DirectLightSet()
        LT.add_surface_lights(ls, sp, lambda o: 0)
        assert ls.active == []


def _texlit(k=3):
    return rg.generate(dataclasses.replace(rg.config_3x3(seed=2), texlights=k))


def test_an_emissive_texture_makes_one_surface_light_per_leaf_patch():
    w = _texlit()
    sp = L.surface_patches(w)
    emitting = np.flatnonzero(w.face_emit[:, 3] > 0)
    leaves = np.isin(sp.face, emitting) & sp.leaf
    ls = L.light_set(w)
    surface = [l for l in ls.active if l.type == LT.EMIT_SURFACE]
    assert len(surface) == int(leaves.sum()) > len(emitting)
    # Prepended in patch order: the list holds them last, in reverse.
    kinds = [l.type for l in ls.active]
    assert kinds[-len(surface):] == [LT.EMIT_SURFACE] * len(surface)
    origins = np.array([l.origin for l in surface])
    assert np.array_equal(origins, sp.origin[np.flatnonzero(leaves)[::-1]])


def test_an_emissive_texture_sets_surf_light_on_its_faces():
    w = _texlit()
    faces, _ = L.faces_of(w)
    emits = w.face_emit[:, 3] > 0
    assert ((faces["flags"][emits] & (L.SURF_LIGHT | L.FACE_EMITS)) == (L.SURF_LIGHT | L.FACE_EMITS)).all()
    assert (faces["flags"][~emits] == 0).all()


def test_texlights_leave_the_rest_of_the_map_alone():
    w0, w = rg.generate(rg.config_3x3(seed=2)), _texlit()
    assert np.array_equal(w0.tri_verts, w.tri_verts) and np.array_equal(w0.light_origin, w.light_origin)
    assert not (w0.face_emit[:, 3] > 0).any()


def test_emitting_faces_skip_the_edge_refinement_as_the_oracle_does(oracle_mod):
    w = _texlit(6)
    faces, verts = L.faces_of(w)
    refl = L.face_reflectivity(w)
    # (The rule halves a chop above min_chop: chops 16 and 4.)
    mine, _ = L.build_patches(faces, verts, refl, max_chop=16.0, min_chop=4.0)
    inp = L.prepare(w)
    off, lst = L.pvs_lists(w)
    ob = oracle_mod.Bounce(oracle_mod.kd_build(w.tri_verts, w.tri_ids), inp.faces, inp.verts, inp.samples,
                           inp.face_first, refl, off, lst, max_chop=16.0, min_chop=4.0, bounces=1, threshold=1.0)
    theirs, _ = ob.patches()
    assert len(mine) == len(theirs)
    for f in ("origin", "area", "normal", "chop", "parent", "child1", "child2", "face"):
        assert np.array_equal(mine[f], theirs[f]), f
    # Without the bit the same faces refine at their edges: more patches.
    unflagged = faces.copy()
    unflagged["flags"] &= ~L.FACE_EMITS
    more, _ = L.build_patches(unflagged, verts, refl, max_chop=16.0, min_chop=4.0)
    assert len(more) > len(mine)
