"""The transfer cache on the GPU: ReadPacked decoded on the device
(vrad_transfer_read_packed) against the oracle on the reference's
TransferSetCodecTests cases, and the store and the hit of
TransferCacheBounceTests (src/SourceSharp.Tests/MapTools/Rad/Bounce/
TransferCacheBounceTests.cs:70-117) on the 3x3 room grid: a light pass's
transfers exported (the index and planes the oracle writes for the same
lists), installed on a stage whose lights changed, and that stage's pass
lighting the same lump as one that built its own transfers."""
import dataclasses

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import lighting as L, roomgrid as rg, tracer as T, transfer_cache as C
from oracle import transfer_codec_oracle as O
from test_transfer_codec_cpu import packed_refusals, sample, same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tracer():
    tri = T.make_triangles(np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], np.float32), np.array([1], np.int32))
    t = T.CudaRayTracer(tri)
    yield t
    t.close()


def lists_from(got):
    return None if got is None else [got[1][got[0][p]:got[0][p + 1]] for p in range(len(got[0]) - 1)]


@pytest.mark.parametrize("chunk_bytes", [24, 8, 1 << 20])
def test_device_read_packed_equals_the_oracle(tracer, chunk_bytes):
    s = sample()
    packed = [O.pack(c) for c in O.chunks(s, chunk_bytes)]
    got = lists_from(C.read_packed(tracer, O.index(s), packed, 4))
    assert same(got, O.read_packed(O.index(s), packed, 4))
    # The library's own packing reads the same.
    mine = [C.pack(c) for c in O.chunks(s, chunk_bytes)]
    assert same(lists_from(C.read_packed(tracer, O.index(s), mine, 4)), s)


def test_device_read_packed_refuses_what_the_reference_refuses(tracer):
    packed_refusals(lambda idx, packed, n: lists_from(C.read_packed(tracer, idx, packed, n)))


def test_device_read_packed_on_a_large_random_set(tracer):
    # 300,000 transfers over 5,000 patches in 37 chunks (one list straddles
    # many chunk edges); wrapping deltas both ways.
    rng = np.random.default_rng(11)
    counts = rng.integers(0, 120, 5000)
    counts[17] = 4000
    lists = []
    for c in counts:
        tr = np.zeros(c, O.TRANSFER_DTYPE)
        tr["patch"] = rng.integers(0, 5000, c)
        tr["weight"] = rng.random(c, np.float32)
        lists.append(tr)
    total = int(counts.sum())
    b = 8 * (total // 37 + 1)
    packed = [C.pack(c) for c in O.chunks(lists, b)]
    got = lists_from(C.read_packed(tracer, O.index(lists), packed, 5000))
    assert same(got, lists)


def _stage(w, inp, max_chop=4.0):
    st = L.LightingStage(w, inp)
    off, lst = L.pvs_lists(w)
    st.upload_bounce(L.face_reflectivity(w), off, lst, max_chop=max_chop, threshold=0.1)
    return st


def _edited(inp):
    """The same map with its lights changed (RadWorld.TransferKey reads no
    light, so a light edit keeps the key)."""
    lights = inp.lights.copy()
    lights["intensity"] *= np.float32(0.5)
    lights["intensity"][0] *= np.float32(3.0)
    return dataclasses.replace(inp, lights=lights)


def test_a_replay_bounces_the_same_light_as_a_fresh_build():
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    with _stage(w, inp) as first:
        with pytest.raises(ValueError):
            C.export(first)                      # no pass has bounced yet
        first.light_pass()
        off, tr = first.transfers()
        idx, packed = C.export(first, 1 << 12)
    lists = [tr[off[p]:off[p + 1]] for p in range(len(off) - 1)]
    # The store's bytes: the oracle's index and, inside every packed chunk,
    # the oracle's planes of the oracle's chunk.
    assert idx == O.index(lists)
    assert len(packed) > 3
    assert [O.unpack(p) for p in packed] == O.chunks(lists, 1 << 12)

    edited = _edited(inp)
    with _stage(w, edited) as fresh:
        want_lump, want_ofs, _ = fresh.light_pass()
        want_total, _ = fresh.patch_light()
        want_stats = fresh.bounce_stats()
    with _stage(w, edited) as replay:
        assert C.install(replay, idx, packed)
        lump, ofs, _ = replay.light_pass()
        stats = replay.bounce_stats()
        total, _ = replay.patch_light()
        r_off, r_tr = replay.transfers()
        # A second pass replays them again.
        lump2, _, _ = replay.light_pass()
        again_idx, again = C.export(replay, 1 << 20)
    assert stats.transfers_cached == 1 and want_stats.transfers_cached == 0
    assert stats.transfer_rays == 0 and stats.transfers == want_stats.transfers == len(tr)
    assert stats.bounces == want_stats.bounces
    assert np.array_equal(r_off, off) and np.array_equal(r_tr.view(np.uint64), tr.view(np.uint64))
    assert np.array_equal(total.view(np.uint32), want_total.view(np.uint32))
    assert np.array_equal(ofs, want_ofs)
    assert np.array_equal(lump, want_lump) and np.array_equal(lump2, want_lump)
    assert again_idx == idx and O.read_packed(again_idx, again, len(off) - 1) is not None
    assert b"".join(O.unpack(p) for p in again) == b"".join(O.chunks(lists, 1 << 12))


def test_a_set_of_another_patch_tree_is_refused_and_changes_nothing():
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    with _stage(w, inp, max_chop=16.0) as coarse:
        coarse.light_pass()
        idx, packed = C.export(coarse)
    with _stage(w, inp) as st:
        want, _, _ = st.light_pass()
        n = st.bounce_stats().patches
        assert len(idx) != 20 + 4 * n
        assert not C.install(st, idx, packed)    # another patch count
        # A set with a list on a patch that receives nothing here: a parent
        # patch (only leaves receive).
        patches, _ = L.build_patches(inp.faces, inp.verts, L.face_reflectivity(w))
        assert len(patches) == n
        off, tr = st.transfers()
        idle = int(np.flatnonzero(patches["child1"] >= 0)[0])
        assert off[idle + 1] == off[idle]
        lists = [tr[off[p]:off[p + 1]] for p in range(n)]
        lists[idle] = tr[:1].copy()
        bad = [C.pack(c) for c in O.chunks(lists, 1 << 20)]
        assert not C.install(st, O.index(lists), bad)
        lump, _, _ = st.light_pass()
        assert st.bounce_stats().transfers_cached == 0
    assert np.array_equal(lump, want)
