"""Leaf ambient on the CPU: the pieces of stock vrad's per-leaf ambient
cubes that the oracle and the host code restate, pinned to the reference's
own fixtures.

  * the random stream (oracle.Ran1) against the reference's golden vectors
    of stock's stream (StockRandomStreamVectors.cs: eight sets of 512);
  * the 162 sample directions: the frequency-4 geodesic sphere's points;
  * the candidate sample positions, host (vrad_leaf_ambient_positions) and
    oracle alike, against the positions stock's own leaf ambient lumps hold
    in p4g_detail.bsp (the reference's fixture map, compiled by stock vbsp,
    vvis and vrad -both): every stored sample is the 8-bit quantisation of
    one of its leaf's candidates;
  * the oracle's ray cubes (AmbientSampler.ComputeRayCube restated) against
    the cube colours in those lumps: stock's stored cube is the ray cube
    plus the baked surface lights (not restated here), so each stored side
    is at least the RGBE encoding of the ray cube's, and on the sides no
    surface light reaches it is exactly that encoding.
"""
import pathlib

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import ambient as A, bsp as B

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
MAP = GOLDEN / "p4g_detail.bsp"


def _ran1_sets():
    lines = (GOLDEN / "ran1-vectors.txt").read_text().split("\n")
    out, i = [], 0
    while i < len(lines) and lines[i].strip():
        name, seed, lo, hi = lines[i].split()
        vals = [int(x, 16) for k in range(64) for x in lines[i + 1 + k].split()]
        out.append((name, None if seed == "default" else int(seed), float(lo), float(hi), vals))
        i += 65
    return out


@pytest.fixture(scope="module")
def lumps():
    return A.load_lumps(str(MAP))


@pytest.fixture(scope="module")
def sampled(lumps):
    tree = A.ambient_tree(lumps)
    counts, pos = A.candidate_positions(tree)
    return tree, counts, pos


def test_random_stream_matches_the_golden_vectors(oracle_mod):
    sets = _ran1_sets()
    assert len(sets) == 8
    for name, seed, lo, hi, want in sets:
        r = oracle_mod.Ran1(0 if seed is None else seed)
        got = [int(np.float32(r.uniform(lo, hi)).view(np.uint32)) for _ in range(512)]
        assert got == want, name


def test_directions_are_the_geodesic_sphere():
    d = A.anorms().astype(np.float64)
    assert d.shape == (162, 3)
    assert np.abs(np.linalg.norm(d, axis=1) - 1).max() < 2e-6
    phi = (1 + 5 ** 0.5) / 2
    ico = [(s1, 0, s2 * phi) for s1 in (-1, 1) for s2 in (-1, 1)]    # stock's orientation
    pts = np.array([np.roll(v, k) for v in ico for k in range(3)], float)
    pts /= np.linalg.norm(pts, axis=1, keepdims=True)
    tris = [(i, j, k) for i in range(12) for j in range(i + 1, 12) for k in range(j + 1, 12)
            if min(pts[i] @ pts[j], pts[j] @ pts[k], pts[i] @ pts[k]) > 0.4]
    assert len(tris) == 20
    # Each face's frequency-4 grid (barycentric steps of 1/4), projected
    # onto the sphere.
    grid = [(a * pts[i] + b * pts[j] + (4 - a - b) * pts[k]) / 4
            for i, j, k in tris for a in range(5) for b in range(5 - a)]
    grid = np.array(grid)
    pts = np.unique(np.round(grid / np.linalg.norm(grid, axis=1, keepdims=True), 9), axis=0)
    assert len(pts) == 162
    near = np.abs(d[:, None, :] - pts[None, :, :]).max(2).min(1)
    assert near.max() < 1e-6                 # six decimals, then float
    assert len(np.unique(np.round(d, 4), axis=0)) == 162


def _stored(lumps, hdr):
    idx = np.frombuffer(lumps[A.LUMP_LEAF_AMBIENT_INDEX_HDR if hdr else A.LUMP_LEAF_AMBIENT_INDEX][1],
                        A.LEAF_AMBIENT_INDEX)
    lit = np.frombuffer(lumps[A.LUMP_LEAF_AMBIENT_LIGHTING_HDR if hdr else A.LUMP_LEAF_AMBIENT_LIGHTING][1],
                        A.LEAF_AMBIENT_LIGHTING)
    return idx, lit


def _match(tree, counts, pos, idx, lit):
    """For every stored sample, the index of the candidate it quantises."""
    first = np.concatenate([[0], np.cumsum(counts)])
    out = []
    for leaf in range(len(idx)):
        if idx[leaf]["count"] == 0:
            continue
        L = tree.leaves[leaf]
        q = {}
        for k, p in enumerate(pos[first[leaf]:first[leaf + 1]]):
            q.setdefault(tuple(A.fixed8(p[a], L[1 + a], L[4 + a]) for a in range(3)), int(first[leaf]) + k)
        for s in lit[idx[leaf]["first"]:idx[leaf]["first"] + idx[leaf]["count"]]:
            out.append(q.get((int(s["x"]), int(s["y"]), int(s["z"])), -1))
    return np.array(out)


def test_candidate_positions_reproduce_stocks_stored_samples(lumps, sampled):
    tree, counts, pos = sampled
    assert not A.has_displacements(lumps)
    assert counts.sum() == len(pos) > 0
    assert ((tree.leaves[:, 0] & A.CONTENTS_SOLID != 0) == (counts == 0)).all()
    for hdr in (False, True):
        idx, lit = _stored(lumps, hdr)
        m = _match(tree, counts, pos, idx, lit)
        assert len(m) == len(lit) > 100
        assert (m >= 0).all(), f"{int((m < 0).sum())} stored samples match no candidate"


def test_oracle_positions_equal_the_host_sampler(oracle_mod, sampled):
    tree, counts, pos = sampled
    c2, p2 = oracle_mod.leaf_positions(tree.planes, tree.nodes, tree.leaves, tree.leaf_brushes, tree.brushes,
                                       tree.brush_sides)
    assert np.array_equal(counts, c2)
    assert np.array_equal(pos.view(np.uint32), p2.view(np.uint32))


def encode(v):
    """StockLightColor.Encode (StockLightColor.cs:110-150) of one colour."""
    x, y, z = (np.float32(c) for c in v)
    mx = (x if x > z else z) if x > y else (y if y > z else z)
    e = 0 if mx == 0 else int((int(np.float32(mx).view(np.uint32)) & 0x7F800000) >> 23) - (7 + 127)
    sc = np.uint32((127 - e) << 23).view(np.float32)
    return [int(np.float32(c * sc)) & 0xFF for c in (x, y, z)] + [e & 0xFF]


def test_oracle_ray_cubes_against_stocks_stored_cubes(oracle_mod, lumps, sampled):
    tree, counts, pos = sampled
    geom = B.trace_geometry(lumps)
    for hdr in (False, True):
        r = A.ambient_range(lumps, hdr)
        cubes = oracle_mod.ambient_cubes(geom, r.faces, r.lighting, A.anorms(), float(A.cone_tan()),
                                         r.sky_ambient, pos)
        idx, lit = _stored(lumps, hdr)
        m = _match(tree, counts, pos, idx, lit)
        equal = below = 0
        for s, k in zip(lit, m):
            for side in range(6):
                mine = encode(cubes[k, side])
                st = [int(b) for b in s["cube"][side]]
                if mine == st:
                    equal += 1
                    continue
                sv = np.array(st[:3], float) * 2.0 ** int(np.int8(np.uint8(st[3])))
                mv = np.array(mine[:3], float) * 2.0 ** int(np.int8(np.uint8(mine[3])))
                below += int((sv < mv).any())
        assert below == 0, (hdr, below)
        assert equal >= 0.4 * 6 * len(lit), (hdr, equal)


def test_cone_tangent_and_decode_table():
    assert int(A.cone_tan().view(np.uint32)) == 0x3E02B92B        # tan(7.275 deg) rounded once
    p = A.power2n()
    assert p[128] == np.float32(1 / 255.0) and p[0] > 0 and np.isfinite(p).all()
    assert A.decode(np.array([[255, 128, 1, 0]], np.uint8))[0].tolist() == [1.0, np.float32(128 / 255.0), np.float32(1 / 255.0)]


def test_directions_rebuild_stocks_own_rays():
    """The reference's recorded leaf-ambient rays on dm_lockdown (50 sample
    points x 162 directions, stock's own fan) end at start + anorm x
    RayLength, in float, bit for bit: the table's values, its order and
    RayLength (32768 x 1.74) are stock's."""
    rb = (GOLDEN / "rays-lockdown-leafambient.bin").read_bytes()
    n = int(np.frombuffer(rb, "<i4", 1)[0])
    se = np.frombuffer(rb, "<f4", 6 * n, 4).reshape(50, 162, 6)
    start, end = se[..., 0:3], se[..., 3:6]
    assert (start == start[:, :1]).all()
    length = np.float32(np.float32(32768.0) * np.float32(1.74))
    mine = (start + (A.anorms()[None] * length).astype(np.float32)).astype(np.float32)
    assert np.array_equal(mine.view(np.uint32), end.view(np.uint32))


def test_displacement_maps_are_refused(lumps):
    """Stock clips every ambient ray against displacements (DispCollisionSet);
    the device sampler does not, so it refuses such a map before any device
    work."""
    with_disp = dict(lumps)
    with_disp[A.LUMP_DISPINFO] = (0, b"\0" * 176)
    with pytest.raises(NotImplementedError):
        A.CudaAmbientSampler(with_disp)
