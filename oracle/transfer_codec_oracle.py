"""CPU restatement of the reference's transfer-set codec
(src/SourceSharp.MapTools/Rad/Bounce/TransferSetCodec.cs), in numpy and
Python's zlib.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the
library's codec, never by the product.

A set is a list of per-patch lists of (patch, weight) pairs, weights as
float32 (TransferSet.For(p)).  Every function cites the lines it follows.
"""
from __future__ import annotations

import zlib

import numpy as np

MAGIC = 0x31465254          # TransferSetCodec.cs:26
TRANSFER_BYTES = 8          # :25
ARRAY_MAX_LENGTH = 0x7FFFFFC7
INT_MAX = 0x7FFFFFFF
TRANSFER_DTYPE = np.dtype([("patch", "<i4"), ("weight", "<f4")])


def as_lists(lists):
    return [np.array([(int(p), np.float32(w)) for p, w in l], TRANSFER_DTYPE) for l in lists]


def index(lists) -> bytes:
    """Index (:31-45): magic, patch count, max, total, every count."""
    counts = [len(l) for l in lists]
    out = bytearray(20 + 4 * len(lists))
    out[0:4] = MAGIC.to_bytes(4, "little")
    out[4:8] = len(lists).to_bytes(4, "little", signed=True)
    out[8:12] = max(counts, default=0).to_bytes(4, "little", signed=True)
    out[12:20] = sum(counts).to_bytes(8, "little", signed=True)
    for p, c in enumerate(counts):
        out[20 + 4 * p:24 + 4 * p] = c.to_bytes(4, "little", signed=True)
    return bytes(out)


def chunks(lists, max_chunk_bytes: int) -> list[bytes]:
    """Chunks / ChunksIterator / Copy (:51-96): patch after patch, whole
    transfers, each chunk min(remaining, per) transfers long; C#'s division
    truncates toward zero, so any max below 8 gives one transfer a chunk."""
    q = abs(int(max_chunk_bytes)) // TRANSFER_BYTES
    per = min(max(q if max_chunk_bytes >= 0 else -q, 1), INT_MAX // TRANSFER_BYTES)
    flat = b"".join(np.asarray(l, TRANSFER_DTYPE).tobytes() for l in as_lists(lists))
    step = per * TRANSFER_BYTES
    return [flat[s:s + step] for s in range(0, len(flat), step)]


def planes(chunk: bytes) -> bytes:
    """Pack's shuffle (:107-122): patch deltas (wrapping) and weights, byte b
    of each at plane b and 4 + b."""
    n = len(chunk) // TRANSFER_BYTES
    rec = np.frombuffer(chunk, "<u4").reshape(n, 2) if n else np.zeros((0, 2), "<u4")
    patch = rec[:, 0].astype(np.uint32)
    delta = patch - np.concatenate([[np.uint32(0)], patch[:-1]]).astype(np.uint32)
    words = np.stack([delta.astype("<u4"), rec[:, 1].astype("<u4")])       # (2, n)
    by = words.view(np.uint8).reshape(2, n, 4)                             # (word, k, b)
    return by.transpose(0, 2, 1).reshape(8 * n).tobytes()                 # plane (word*4 + b), then k


def pack(chunk: bytes) -> bytes:
    """Pack (:103-133): count, then the zlib stream of the planes at the
    fastest level (the deflated bytes are Python's zlib's)."""
    n = len(chunk) // TRANSFER_BYTES
    return n.to_bytes(4, "little", signed=True) + zlib.compress(planes(chunk), 1)


def _inflate_exact(stream: bytes, want: int):
    """ReadExactly(want) then ReadByte() == -1 (:155-166): the bytes, or
    None when the stream holds fewer, more, or is not a zlib stream."""
    d = zlib.decompressobj()
    try:
        out = d.decompress(stream, want + 1)
        if len(out) < want and not d.eof:
            out += d.flush()
    except zlib.error:
        return None
    return out if len(out) == want else None


def unplanes(data: bytes, n: int) -> bytes:
    """Unpack's inverse shuffle and the deltas' running sum (:170-185)."""
    by = np.frombuffer(data, np.uint8).reshape(2, 4, n).transpose(0, 2, 1).copy()
    words = by.view("<u4").reshape(2, n)
    patch = np.cumsum(words[0].astype(np.uint64)).astype(np.uint64) & 0xFFFFFFFF
    out = np.stack([patch.astype("<u4"), words[1]], axis=1)
    return out.tobytes()


def unpack(packed: bytes):
    """Unpack (:140-188): the raw chunk, or None."""
    if len(packed) < 4:
        return None
    n = int.from_bytes(packed[:4], "little", signed=True)
    if n < 0 or n > ARRAY_MAX_LENGTH // TRANSFER_BYTES:
        return None
    data = _inflate_exact(packed[4:], n * TRANSFER_BYTES)
    return None if data is None else unplanes(data, n)


def _try_read_index(idx: bytes, patch_count: int):
    """TryReadIndex (:329-372): the counts, or None."""
    if (len(idx) < 20 or int.from_bytes(idx[0:4], "little") != MAGIC
            or int.from_bytes(idx[4:8], "little", signed=True) != patch_count
            or len(idx) != 20 + 4 * patch_count):
        return None
    mx = int.from_bytes(idx[8:12], "little", signed=True)
    total = int.from_bytes(idx[12:20], "little", signed=True)
    if total < 0 or total > ARRAY_MAX_LENGTH:
        return None
    counts = [int.from_bytes(idx[20 + 4 * p:24 + 4 * p], "little", signed=True) for p in range(patch_count)]
    if any(c < 0 for c in counts) or sum(counts) != total or max(counts, default=0) != mx:
        return None
    return counts


def _lists(counts, flat: bytes):
    rec = np.frombuffer(flat, TRANSFER_DTYPE)
    out, at = [], 0
    for c in counts:
        out.append(rec[at:at + c].copy())
        at += c
    return out


def read(idx: bytes, raw_chunks, patch_count: int):
    """Read (:374-446): the lists, or None."""
    counts = _try_read_index(idx, patch_count)
    if counts is None or any(len(c) % TRANSFER_BYTES for c in raw_chunks):
        return None
    if sum(len(c) for c in raw_chunks) != sum(counts) * TRANSFER_BYTES:
        return None
    flat = b"".join(raw_chunks)
    rec = np.frombuffer(flat, TRANSFER_DTYPE)
    if ((rec["patch"] < 0) | (rec["patch"] >= patch_count)).any():
        return None
    return _lists(counts, flat)


def read_packed(idx: bytes, packed, patch_count: int):
    """ReadPacked (:215-297) and UnpackInto (:301-326): the lists, or None."""
    counts = _try_read_index(idx, patch_count)
    if counts is None:
        return None
    ns = []
    for chunk in packed:
        if chunk is None or len(chunk) < 4:
            return None
        n = int.from_bytes(chunk[:4], "little", signed=True)
        if n < 0 or n > ARRAY_MAX_LENGTH // TRANSFER_BYTES:
            return None
        ns.append(n)
    if sum(ns) != sum(counts):
        return None
    parts = []
    for chunk, n in zip(packed, ns):
        data = _inflate_exact(chunk[4:], n * TRANSFER_BYTES)
        if data is None:
            return None
        raw = unplanes(data, n)
        rec = np.frombuffer(raw, TRANSFER_DTYPE)
        if ((rec["patch"] < 0) | (rec["patch"] >= patch_count)).any():
            return None
        parts.append(raw)
    return _lists(counts, b"".join(parts))
