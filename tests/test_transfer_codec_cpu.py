"""The transfer cache's byte format on the CPU: the reference's
TransferSetCodecTests (src/SourceSharp.Tests/MapTools/Rad/Bounce/
TransferSetCodecTests.cs:22-210), restated on the oracle
(oracle/transfer_codec_oracle.py), and the library's host codec
(vrad_transfer_index, vrad_transfer_pack, vrad_transfer_unpack; the
package's raw-chunk reader) against the oracle on the same sets.

The device half (ReadPacked decoded on the GPU, export and install) is in
test_transfer_cache_gpu.py."""
import zlib

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import transfer_cache as C
from oracle import transfer_codec_oracle as O

EPSILON = float(np.frombuffer(np.uint32(1).tobytes(), np.float32)[0])   # float.Epsilon


def sample():
    """TransferSetCodecTests.Sample (:22-34): four patches of 3, 0, 5 and 2
    transfers, as TransferSet.For reads them out of the two segments."""
    return [
        [(1, 0.5), (2, 0.25), (3, 1e-7)],
        [],
        [(0, 0.1), (3, 0.2), (1, 0.3), (2, EPSILON), (0, 0.9)],
        [(0, 0.75), (2, 0.125)],
    ]


def lists_of(lists):
    return [[(int(p), np.float32(w).tobytes()) for p, w in zip(l["patch"], l["weight"])] for l in O.as_lists(lists)]


def same(a, b):
    return a is not None and b is not None and lists_of(a) == lists_of(b)


def flat(lists):
    """(offsets, transfers) of the package's API."""
    ls = O.as_lists(lists)
    off = np.concatenate([[0], np.cumsum([len(l) for l in ls])]).astype(np.int64)
    tr = np.concatenate(ls) if ls else np.zeros(0, O.TRANSFER_DTYPE)
    return off, tr


def from_flat(off, tr):
    return [tr[off[p]:off[p + 1]] for p in range(len(off) - 1)]


# ---- the reference's cases, on the oracle ----------------------------------

def test_a_set_round_trips_through_index_and_chunks():
    s = sample()
    back = O.read(O.index(s), O.chunks(s, 1 << 20), 4)
    assert same(back, s)
    assert max(len(l) for l in back) == 5 and sum(len(l) for l in back) == 10


def test_chunks_split_across_patch_lists():
    c = O.chunks(sample(), 24)
    assert [len(x) for x in c] == [24, 24, 24, 8]
    assert same(O.read(O.index(sample()), c, 4), sample())


def test_packed_chunks_unpack_to_the_same_bytes():
    for chunk in O.chunks(sample(), 24):
        assert O.unpack(O.pack(chunk)) == chunk


def test_an_empty_set_round_trips():
    empty = [[], []]
    assert O.chunks(empty, 64) == []
    back = O.read(O.index(empty), O.chunks(empty, 64), 2)
    assert back is not None and sum(len(l) for l in back) == 0


def test_refusals():
    s = sample()
    assert O.read(O.index(s), O.chunks(s, 1 << 20), 5) is None            # another patch count
    assert O.read(O.index(s), O.chunks(s, 24)[:-1], 4) is None            # a missing chunk
    chunk = bytearray(O.chunks(s, 1 << 20)[0])
    chunk[0] = 9
    assert O.read(O.index(s), [bytes(chunk)], 4) is None                  # a patch out of range


@pytest.mark.parametrize("chunk_bytes", [24, 8, 1 << 20])
def test_a_packed_set_reads_as_the_unpacked_reader_reads_it(chunk_bytes):
    s = sample()
    raw = O.read(O.index(s), O.chunks(s, chunk_bytes), 4)
    packed = O.read_packed(O.index(s), [O.pack(c) for c in O.chunks(s, chunk_bytes)], 4)
    assert same(raw, packed)


def packed_refusals(read_packed):
    """The reference's ReadPacked refusals (:145-201) through `read_packed`."""
    s = sample()
    idx = O.index(s)
    packed = [O.pack(c) for c in O.chunks(s, 24)]
    assert read_packed(idx, packed, 5) is None                            # another patch count
    assert read_packed(idx, packed[:-1], 4) is None                       # a missing chunk
    wrong = [bytearray(p) for p in packed]
    wrong[0][0] += 1                                                      # counts that still add up,
    wrong[1][0] -= 1                                                      # but not the streams'
    assert read_packed(idx, [bytes(p) for p in wrong], 4) is None
    chunk = bytearray(O.chunks(s, 1 << 20)[0])
    chunk[0] = 9
    assert read_packed(idx, [O.pack(bytes(chunk))], 4) is None            # a patch out of range
    for junk in (bytes([1, 2]), bytes([0xFF] * 4), bytes([10, 0, 0, 0, 0xDE, 0xAD, 0xBE, 0xEF])):
        assert read_packed(idx, [junk], 4) is None
    empty = read_packed(O.index([[], []]), [O.pack(c) for c in O.chunks([[], []], 64)], 2)
    assert empty is not None and sum(len(l) for l in empty) == 0            # an empty set reads


def test_packed_refusals_on_the_oracle():
    packed_refusals(O.read_packed)


def test_junk_does_not_unpack():
    assert O.unpack(bytes([1, 0, 0, 0, 0xDE, 0xAD, 0xBE, 0xEF])) is None
    assert O.unpack(bytes([1, 2])) is None


def test_oracle_planes_follow_the_reference_layout():
    # Two transfers (patch 5, weight bits 0x04030201), (patch 3, 0x08070605):
    # deltas 5 and 0xFFFFFFFE; plane b holds byte b of both deltas, then
    # plane 4 + b byte b of both weights.
    chunk = np.array([(5, 0), (3, 0)], O.TRANSFER_DTYPE)
    chunk["weight"] = np.array([0x04030201, 0x08070605], np.uint32).view(np.float32)
    p = O.planes(chunk.tobytes())
    assert p == bytes([5, 0xFE, 0, 0xFF, 0, 0xFF, 0, 0xFF, 1, 5, 2, 6, 3, 7, 4, 8])


# ---- the library's host codec, against the oracle ---------------------------

def test_library_index_equals_the_oracle():
    for lists in (sample(), [[], []], [[(0, 1.0)] * 7, [], [(1, 2.0)]]):
        off, _ = flat(lists)
        assert C.index(off) == O.index(lists)


def test_library_chunks_equal_the_oracle():
    off, tr = flat(sample())
    for b in (8, 16, 24, 25, 1 << 20, 0, -5):
        assert C.chunks(off, tr, b) == O.chunks(sample(), b)


def test_library_pack_holds_the_reference_planes_and_unpacks():
    rng = np.random.default_rng(7)
    chunks = O.chunks(sample(), 24) + O.chunks(sample(), 1 << 20)
    big = np.zeros(5000, O.TRANSFER_DTYPE)
    big["patch"] = rng.integers(0, 1 << 20, 5000)
    big["weight"] = rng.random(5000, np.float32)
    chunks.append(big.tobytes())
    chunks.append(b"")
    for chunk in chunks:
        mine = C.pack(chunk)
        n = len(chunk) // 8
        assert int.from_bytes(mine[:4], "little") == n
        assert zlib.decompress(mine[4:]) == O.planes(chunk)
        assert C.unpack(mine) == chunk
        assert C.unpack(O.pack(chunk)) == chunk
        assert O.unpack(mine) == chunk


def test_library_unpack_refuses_what_the_oracle_refuses():
    good = O.pack(O.chunks(sample(), 1 << 20)[0])
    cases = [bytes([1, 0, 0, 0, 0xDE, 0xAD, 0xBE, 0xEF]), bytes([1, 2]), bytes([0xFF] * 4),
             good[:-6],                                       # cut inside the data
             good + b"\x00\x01",                             # bytes after the stream: ignored
             (int.from_bytes(good[:4], "little") - 1).to_bytes(4, "little") + good[4:],   # one too many
             (int.from_bytes(good[:4], "little") + 1).to_bytes(4, "little") + good[4:]]   # one too few
    for c in cases:
        assert C.unpack(c) == O.unpack(c), c[:8]


def test_library_read_equals_the_oracle():
    s = sample()
    off, tr = flat(s)
    for b in (24, 8, 1 << 20):
        got = C.read(C.index(off), C.chunks(off, tr, b), 4)
        assert got is not None and same(from_flat(*got), O.read(O.index(s), O.chunks(s, b), 4))
    assert C.read(C.index(off), C.chunks(off, tr, 24), 5) is None
    assert C.read(C.index(off), C.chunks(off, tr, 24)[:-1], 4) is None
    bad = bytearray(C.chunks(off, tr, 1 << 20)[0])
    bad[0] = 9
    assert C.read(C.index(off), [bytes(bad)], 4) is None
