"""Leaf ambient's last steps on the CPU: the 16-sample list, its compression
and the two lumps (vrad_leaf_ambient_lumps, host code), against the oracle's
restatement and the reference's own cases.

  * the reference's AmbientSampleListTests (AmbientSampleListTests.cs:36-171),
    restated with the same inputs and answers, on the oracle and through the
    library's entry (a one-leaf map whose box makes each sample's encoded
    position tell which survived);
  * the library's lumps equal the oracle's on p4g_detail, every leaf's
    stock candidates with the oracle's ray cubes, in both tie-break modes;
  * stock's own index lump on p4g_detail: every empty leaf points at the
    neighbour stock chose (that choice depends only on which leaves hold
    samples), and every open leaf keeps at least one sample.
"""
import pathlib

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import ambient as A, bsp as B

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def uniform(v):
    return np.full((6, 3), v, np.float32)


def filled(O, n, position, colour, dead=True):
    s = []
    for i in range(n):
        O.sample_list_add(s, position(i), uniform(colour(i)), dead)
    return s


def tied_pair(O):
    s = []
    O.sample_list_add(s, (0, 0, 0), uniform(0.00005), True)
    O.sample_list_add(s, (1, 0, 0), uniform(0.0), True)
    for i in range(14):
        O.sample_list_add(s, (0, (i + 1) * 1000, 0), uniform(0.0), True)
    return s


def _product(positions, colours, box, correct=False):
    """The library's list for one open leaf with `box` (mins, maxs): the
    surviving records as (fixed8 x, y, z, first colour's RGBE)."""
    mins, maxs = box
    planes = np.array([[1, 0, 0, 1e6]], np.float32)
    nodes = np.array([[0, -2, -1]], np.int32)        # child 0: leaf 1 (solid), child 1: leaf 0
    leaves = np.zeros((2, 9), np.int32)
    leaves[0, 1:4], leaves[0, 4:7] = mins, maxs
    leaves[1, 0] = 1
    leaves[1, 1:4], leaves[1, 4:7] = (2000000, 0, 0), (2000001, 1, 1)
    tree = A.AmbientTree(planes, nodes, leaves, np.zeros(0, np.int32), np.zeros((0, 3), np.int32),
                         np.zeros((0, 2), np.int32))
    pos = np.array(positions, np.float32).reshape(-1, 3)
    cubes = np.stack([uniform(c) for c in colours]).reshape(-1, 6, 3)
    index, light, bad = A.leaf_ambient_lumps(tree, [len(pos), 0], pos, cubes, correct_tiebreak=correct)
    idx = np.frombuffer(index, A.LEAF_AMBIENT_INDEX)
    recs = np.frombuffer(light, A.LEAF_AMBIENT_LIGHTING)
    # Leaf 1 (solid, far away) finds no lit neighbour in its box: itself.
    assert idx[0]["first"] == 0 and idx[0]["count"] == len(recs) and idx[1]["count"] == 0 and idx[1]["first"] == 1
    return [(int(r["x"]), int(r["y"]), int(r["z"]), bytes(r["cube"][0])) for r in recs]


def test_up_to_sixteen_samples_are_kept(oracle_mod):
    assert len(filled(oracle_mod, 16, lambda i: (i * 10, 0, 0), lambda i: 0.5)) == 16
    assert len(filled(oracle_mod, 17, lambda i: (i * 10, 0, 0), lambda i: 0.5)) == 16
    pos = [(i * 10, 0, 0) for i in range(17)]
    # A 17th sample evicts one; a uniform leaf then compresses to one.
    assert len(_product(pos, [0.5] * 17, ((-1, -1, -1), (200, 1, 1)))) == 1


def test_the_earlier_of_the_nearest_pair_goes_and_the_last_fills_its_hole(oracle_mod):
    s = filled(oracle_mod, 16, lambda i: (i * 100, 0, 0), lambda i: 0.5)
    oracle_mod.sample_list_add(s, (501, 0, 0), uniform(0.5), True)
    assert tuple(s[5][0]) == (501, 0, 0)
    # Through the library, before compression would merge the uniform leaf:
    # distinct colours keep every sample, and the box around x 495..505
    # makes sample 5's record tell 500 (byte 128) from 501 (byte 153).
    pos = [(i * 100, 0, 0) for i in range(16)] + [(501, 0, 0)]
    colours = [0.02 * (i + 1) for i in range(16)] + [0.02 * 6]
    recs = _product(pos, colours, ((495, -1, -1), (505, 1, 1)))
    assert recs[5][0] == 153


def test_colour_difference_makes_a_sample_worth_keeping(oracle_mod):
    s = filled(oracle_mod, 16, lambda i: (i * 100, 0, 0), lambda i: 0.5)
    oracle_mod.sample_list_add(s, (550, 0, 0), uniform(5.0), True)
    assert any(tuple(p) == (500, 0, 0) for p, _ in s)


def test_stock_never_uses_the_tie_break_and_correct_does(oracle_mod):
    s = tied_pair(oracle_mod)
    oracle_mod.sample_list_add(s, (10000, 0, 0), uniform(0.0), True)
    assert not any(tuple(p) == (0, 0, 0) for p, _ in s)
    s = tied_pair(oracle_mod)
    oracle_mod.sample_list_add(s, (10000, 0, 0), uniform(0.0), False)
    assert not any(tuple(p) == (1, 0, 0) for p, _ in s)
    # (Through the library the tie-break cannot be seen in the lumps: the
    # leaf's near-black samples then compress to one.  The library's lists
    # equal the oracle's in both modes on the fixture map below.)


def test_compression(oracle_mod):
    table = A.gamma_table()
    s = filled(oracle_mod, 8, lambda i: (i * 50, 0, 0), lambda i: 0.25)
    oracle_mod.sample_list_compress(s, table)
    assert len(s) == 1
    s = filled(oracle_mod, 4, lambda i: (i * 500, 0, 0), lambda i: 0.9 if i == 2 else 0.01)
    oracle_mod.sample_list_compress(s, table)
    assert any(c[0, 0] == np.float32(0.9) for _, c in s)
    # The library: the bright sample survives.
    recs = _product([(i * 500, 0, 0) for i in range(4)], [0.9 if i == 2 else 0.01 for i in range(4)],
                    ((-1, -1, -1), (1600, 1, 1)))
    # (decode divides by 255, as lightmap words are; the cube words are not)
    assert A.decode(np.frombuffer(b"".join(r[3] for r in recs), np.uint8)).max() * 255 > 0.8


def test_reconstruction_and_gamma_delta(oracle_mod):
    s = []
    oracle_mod.sample_list_add(s, (0, 0, 0), uniform(1.0), True)
    oracle_mod.sample_list_add(s, (1, 0, 0), uniform(4.0), True)
    assert abs(float(oracle_mod.color_at_position(s, (0, 0, 0), -1)[0, 0]) - 2.0) < 1e-5
    assert oracle_mod.color_at_position(s, (0, 0, 0), 0)[0, 0] == np.float32(4.0)
    table = A.gamma_table()
    assert oracle_mod.gamma_delta(uniform(0.3), uniform(0.3), table) == 0
    b = uniform(0.0)
    b[3] = (0, 1.0, 0)
    assert oracle_mod.gamma_delta(uniform(0.0), b, table) == 255


@pytest.fixture(scope="module")
def fixture_map(oracle_mod):
    lumps = A.load_lumps(str(GOLDEN / "p4g_detail.bsp"))
    tree = A.ambient_tree(lumps)
    counts, pos = A.candidate_positions(tree)
    r = A.ambient_range(lumps, False)
    cubes = oracle_mod.ambient_cubes(B.trace_geometry(lumps), r.faces, r.lighting, A.anorms(), float(A.cone_tan()),
                                     r.sky_ambient, pos)
    return lumps, tree, counts, pos, cubes


@pytest.mark.parametrize("correct", [False, True])
def test_library_lumps_equal_the_oracle(oracle_mod, fixture_map, correct):
    lumps, tree, counts, pos, cubes = fixture_map
    got = A.leaf_ambient_lumps(tree, counts, pos, cubes, correct_tiebreak=correct)
    want = oracle_mod.leaf_ambient_lumps(tree.planes, tree.nodes, tree.leaves, counts, pos, cubes,
                                         A.gamma_table(), dead_tiebreak=not correct)
    assert got == want


def test_empty_leaves_point_where_stocks_do(fixture_map):
    lumps, tree, counts, pos, cubes = fixture_map
    index, light, bad = A.leaf_ambient_lumps(tree, counts, pos, cubes)
    mine = np.frombuffer(index, A.LEAF_AMBIENT_INDEX)
    assert bad == 0 and len(light) == 28 * int(mine["count"].sum())
    for hdr in (False, True):
        stock = np.frombuffer(lumps[A.LUMP_LEAF_AMBIENT_INDEX_HDR if hdr else A.LUMP_LEAF_AMBIENT_INDEX][1],
                              A.LEAF_AMBIENT_INDEX)
        empty = stock["count"] == 0
        assert np.array_equal(empty, mine["count"] == 0)
        assert np.array_equal(stock["first"][empty], mine["first"][empty])
