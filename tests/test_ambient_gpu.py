"""The leaf ambient ray cubes on the device (vrad_ambient_cubes) against the
oracle's restatement of AmbientSampler.ComputeRayCube, bit for bit:

  * p4g_detail.bsp (the reference's leaf-ambient fixture map), both
    ranges, at every candidate sample position the host sampler draws and
    at random points in the open leaves;
  * dm_lockdown's geometry (2,682 nodes, 6,536 faces) at the 50 sample
    points of the reference's recorded leaf-ambient rays and at random
    points, with a seeded synthetic lighting lump and reflectivities (the
    fixture keeps only the map's geometry lumps);
  * the device form on a torch stream, and the reference's errors: a hit
    on a face whose style averages lie outside the lump fails the call.
The oracle's cubes are themselves pinned to stock's stored cubes on
p4g_detail (tests/test_ambient_cpu.py).
"""
import pathlib

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import ambient as A, bsp as B
from tests.golden import fixtures as F

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def _open_points(tree, rng, n):
    leaves = tree.leaves[(tree.leaves[:, 0] & A.CONTENTS_SOLID) == 0]
    pick = leaves[rng.integers(0, len(leaves), n)]
    u = rng.uniform(0.02, 0.98, (n, 3))
    return (pick[:, 1:4] + u * (pick[:, 4:7] - pick[:, 1:4])).astype(np.float32)


def _oracle(O, lumps, rng_or_r, pos):
    r = rng_or_r
    return O.ambient_cubes(B.trace_geometry(lumps), r.faces, r.lighting, A.anorms(), float(A.cone_tan()),
                           r.sky_ambient, pos)


def _same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


def test_fixture_map_cubes_equal_the_oracle(oracle_mod):
    lumps = A.load_lumps(str(GOLDEN / "p4g_detail.bsp"))
    tree = A.ambient_tree(lumps)
    _, cand = A.candidate_positions(tree)
    pos = np.concatenate([cand, _open_points(tree, np.random.default_rng(5), 20000)])
    for hdr in (False, True):
        with A.CudaAmbientSampler(lumps, hdr=hdr) as s:
            got = s.cubes(pos)
        want = _oracle(oracle_mod, lumps, A.ambient_range(lumps, hdr), pos)
        assert np.isfinite(got).all() and (got > 0).any()
        assert _same(got, want), (hdr, int((got != want).any(axis=(1, 2)).sum()))


def _lockdown_lumps(seed=3):
    """dm_lockdown's geometry with a seeded synthetic lighting lump, texture
    reflectivities and a sky ambient light; no displacement info (the walk
    skips displacement faces either way)."""
    lumps = dict(F.lockdown_lumps())
    rng = np.random.default_rng(seed)
    faces = np.frombuffer(lumps[B.LUMP_FACES][1], B.FACE)
    texinfo = np.frombuffer(lumps[B.LUMP_TEXINFO][1], B.TEXINFO)
    ntex = int(texinfo["texdata"].max()) + 1
    td = np.zeros(ntex, A.TEXDATA)
    td["reflectivity"] = rng.uniform(0.05, 0.9, (ntex, 3)).astype(np.float32)
    styles = (faces["styles"] != 255).sum(1)
    size = (faces["lm_size"][:, 0].astype(np.int64) + 1) * (faces["lm_size"][:, 1] + 1) * 4 * np.maximum(styles, 1)
    end = int(np.max(np.where(faces["lightofs"] >= 0, faces["lightofs"] + 4 * size, 0)))
    light = rng.integers(0, 256, end + 64, dtype=np.uint8)
    light[3::4] = rng.integers(-9, 3, len(light[3::4])).astype(np.int8).view(np.uint8)
    wl = np.zeros(2, A.WORLDLIGHT)
    wl["type"] = (1, A.EMIT_SKYAMBIENT)
    wl["intensity"][1] = (0.25, 0.5, 0.75)
    lumps[B.LUMP_TEXDATA] = (0, td.tobytes())
    lumps[B.LUMP_LIGHTING] = (1, light.tobytes())
    lumps[A.LUMP_WORLDLIGHTS] = (0, wl.tobytes())
    return lumps


def test_lockdown_cubes_equal_the_oracle(oracle_mod):
    lumps = _lockdown_lumps()
    rays, _, _, _ = F.lockdown_rays()
    starts = rays[::162, :3].copy()
    leaves = np.frombuffer(lumps[B.LUMP_LEAFS][1], B.LEAF_V0 if lumps[B.LUMP_LEAFS][0] == 0 else B.LEAF_V1)
    L = np.zeros((len(leaves), 9), np.int32)
    L[:, 0], L[:, 1:4], L[:, 4:7] = leaves["contents"], leaves["mins"], leaves["maxs"]
    tree = A.AmbientTree(None, None, L, None, None, None)
    pos = np.concatenate([starts, _open_points(tree, np.random.default_rng(9), 30000)])
    r = A.ambient_range(lumps, False)
    with A.CudaAmbientSampler(lumps) as s:
        got = s.cubes(pos)
    want = _oracle(oracle_mod, lumps, r, pos)
    assert (got[:50] > 0).any()
    assert _same(got, want), int((got != want).any(axis=(1, 2)).sum())


def test_device_form_and_errors(oracle_mod):
    import torch
    lumps = A.load_lumps(str(GOLDEN / "p4g_detail.bsp"))
    tree = A.ambient_tree(lumps)
    _, pos = A.candidate_positions(tree)
    with A.CudaAmbientSampler(lumps) as s:
        host = s.cubes(pos)
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            d = torch.from_numpy(pos).cuda()
            out = s.cubes_device(d, stream=stream.cuda_stream)
        stream.synchronize()
        s.status()
        assert _same(out.cpu().numpy(), host)
        assert s.cubes(np.zeros((0, 3), np.float32)).shape == (0, 6, 3)
    # Every lit face's averages outside the lump: the first hit on one fails.
    bad = dict(lumps)
    faces = np.frombuffer(lumps[B.LUMP_FACES][1], B.FACE).copy()
    texinfo = np.frombuffer(lumps[B.LUMP_TEXINFO][1], B.TEXINFO)
    lit = (texinfo["flags"][faces["texinfo"]] & B.SURF_SKY) == 0
    faces["lightofs"][lit & (faces["lightofs"] >= 0)] = 0      # the averages would sit before the lump
    bad[B.LUMP_FACES] = (lumps[B.LUMP_FACES][0], faces.tobytes())
    r = A.ambient_range(bad, False)
    assert (r.faces["flags"] & A.VRAD_AMBIENT_BAD_AVERAGE).any()
    with A.CudaAmbientSampler(bad) as s:
        with pytest.raises(ValueError, match="averages"):      # VRAD_ERR_ARG
            s.cubes(pos)
        # The context stays usable, and the oracle agrees it is the
        # reference's error.
        with pytest.raises(ValueError, match="averages"):
            s.cubes(pos)
    with pytest.raises(RuntimeError):
        _oracle(oracle_mod, bad, r, pos)

