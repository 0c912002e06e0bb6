"""The bounce's host-side set-up and its oracle, on the CPU.

The patch tree (PatchBuilder + PatchSubdivider) the library builds natively
must equal the oracle's restatement record for record and bit for bit:
every later stage indexes patches by number.  The oracle's correctly
rounded arcsine (DetMathF.Asin, used by FormFactors.PolyToDiff) is pinned
to the reference's DetMath golden table."""
import numpy as np
import pytest

import fixtures
from hl2sdk_tools_sharp_b200 import lighting as L, roomgrid as rg


def _world(cfg):
    w = rg.generate(cfg)
    return w, L.prepare(w)


@pytest.mark.parametrize("cfg", [rg.config_3x3(seed=2), rg.config_8x8(seed=1)], ids=["3x3", "8x8"])
def test_patches_match_oracle(oracle_mod, cfg):
    w, inp = _world(cfg)
    refl = L.face_reflectivity(w)
    got, pts = L.build_patches(inp.faces, inp.verts, refl)
    off, lst = L.pvs_lists(w)
    tree = oracle_mod.kd_build(w.tri_verts[:1], w.tri_ids[:1])  # patches need no scene
    b = oracle_mod.Bounce(tree, inp.faces, inp.verts, inp.samples, inp.face_first, refl, off, lst)
    want, want_pts = b.patches()
    assert len(got) == len(want)
    for name in got.dtype.names:
        assert np.ascontiguousarray(got[name]).tobytes() == np.ascontiguousarray(want[name]).tobytes(), name
    assert np.array_equal(pts.view(np.uint32), want_pts.view(np.uint32))


def test_patch_tree_shape():
    w, inp = _world(rg.config_3x3(seed=2))
    p, pts = L.build_patches(inp.faces, inp.verts, L.face_reflectivity(w))
    nf = len(inp.faces)
    # One root per face, in face order, then subtrees.
    assert np.array_equal(p["face"][:nf], np.arange(nf))
    assert (p["parent"][:nf] == -1).all() and (p["parent"][nf:] >= 0).all()
    inner = np.flatnonzero(p["child1"] >= 0)
    assert (p["parent"][p["child1"][inner]] == inner).all()
    assert (p["parent"][p["child2"][inner]] == inner).all()
    assert (p["child2"][inner] == p["child1"][inner] + 1).all()
    # Children split the parent's area; leaves are under the chop (4 luxels
    # at 1/16 luxel per unit: 64 units) on every axis.
    a = p["area"]
    assert np.allclose(a[p["child1"][inner]] + a[p["child2"][inner]], a[inner], rtol=1e-5)
    leaves = p["child1"] < 0
    ext = (p["maxs"] - p["mins"])[leaves] * p["lux_scale"][leaves, None]
    assert (ext < 4.0 + 1e-4).all()
    # Reflectivity clamped to 0.99, windings in range.
    assert (p["reflectivity"] <= np.float32(0.99)).all()
    assert p["first_point"][-1] + p["num_points"][-1] == len(pts)


def test_build_patches_rejects_bad_arguments():
    w, inp = _world(rg.config_3x3(seed=2))
    with pytest.raises(ValueError):
        L.build_patches(inp.faces, inp.verts, L.face_reflectivity(w), max_chop=0.0)


def test_oracle_asin_matches_detmath_goldens(oracle_mod):
    a, _, e = fixtures.detmath("Asin")
    assert len(a) > 100
    got = np.array([oracle_mod.asin(x) for x in a.view(np.float32)], np.float32)
    bad = np.flatnonzero(got.view(np.uint32) != e)
    assert len(bad) == 0, [(hex(a[i]), hex(got.view(np.uint32)[i]), hex(e[i])) for i in bad[:5]]


def test_oracle_pow_matches_detmath_goldens(oracle_mod):
    a, b, e = fixtures.detmath("Pow")
    assert len(a) > 100
    got = np.array([oracle_mod.powf(x, y) for x, y in zip(a.view(np.float32), b.view(np.float32))], np.float32)
    bad = np.flatnonzero(got.view(np.uint32) != e)
    assert len(bad) == 0, [(hex(a[i]), hex(b[i]), hex(got.view(np.uint32)[i]), hex(e[i])) for i in bad[:5]]


def test_pvs_lists_are_rows_of_the_pvs():
    w, _ = _world(rg.config_3x3(seed=2))
    off, lst = L.pvs_lists(w)
    for c in range(w.pvs.shape[0]):
        assert np.array_equal(lst[off[c]:off[c + 1]], np.flatnonzero(w.pvs[c]))
