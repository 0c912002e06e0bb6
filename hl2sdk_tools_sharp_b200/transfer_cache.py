"""The transfer cache's byte format and the cache hit, over libvrad_cuda.so.

The reference stores a compile's transfers so that a later compile of the
same geometry replays them (TransferSetCodec,
MapTools/Rad/Bounce/TransferSetCodec.cs:23-447; the store,
Compile/Cache/StoreTransferCache.cs:241-262 and 360-378; the cache branch of
RadWorld.BounceAsync, MapTools/Rad/Light/RadWorld.Bounce.cs:364-386).  A set
here is (offsets, transfers): patch p's list is
transfers[offsets[p]:offsets[p + 1]], TRANSFER_DTYPE records (the source
patch, the weight), as LightingStage.transfers() returns it.

    index(offsets)                         TransferSetCodec.Index
    chunks(offsets, transfers, max_bytes)  TransferSetCodec.Chunks
    pack(chunk), unpack(packed)            Pack, Unpack (None: not a packed chunk)
    read(index, chunks, patch_count)       Read (None: they do not fit together)
    read_packed(owner, index, packed, n)   ReadPacked, the planes decoded on the device
    export(stage, max_bytes)               the stage's transfers as (index, packed chunks)
    install(stage, index, packed)          a cache hit: later light passes bounce with
                                           them instead of building (False: refused)

`owner` is anything holding a context (a CudaRayTracer or a LightingStage).
The deflate is zlib's level 1: the planes inside are the reference's byte
for byte, the deflated bytes are zlib's.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import tracer as T

MAGIC = 0x31465254            # "TRF1"
TRANSFER_BYTES = 8
ARRAY_MAX_LENGTH = 0x7FFFFFC7  # .NET Array.MaxLength, the reference's bound on a count
DEFAULT_MAX_CHUNK_BYTES = 16 * 1024 * 1024  # CachePolicy.DefaultMaxBlobBytes
TRANSFER_DTYPE = np.dtype([("patch", "<i4"), ("weight", "<f4")])
ERR_FORMAT = -8


def _lib():
    lib = T.load_library()
    if not getattr(lib, "_transfer_cache_bound", False):
        P, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
        pi64 = ctypes.POINTER(i64)
        lib.vrad_transfer_index.argtypes = [P, i32, P, i64]
        lib.vrad_transfer_index.restype = i32
        lib.vrad_transfer_pack_bound.argtypes = [i64]
        lib.vrad_transfer_pack_bound.restype = i64
        lib.vrad_transfer_pack.argtypes = [P, i64, P, i64, pi64]
        lib.vrad_transfer_pack.restype = i32
        lib.vrad_transfer_unpack.argtypes = [P, i64, P, i64, pi64]
        lib.vrad_transfer_unpack.restype = i32
        lib.vrad_transfer_export_size.argtypes = [P, i64, pi64, pi64, pi64]
        lib.vrad_transfer_export_size.restype = i32
        lib.vrad_transfer_export.argtypes = [P, i64, P, i64, P, i64, P, i64, pi64]
        lib.vrad_transfer_export.restype = i32
        lib.vrad_transfer_read_packed.argtypes = [P, P, i64, P, P, i64, i32, P, P, i64, pi64]
        lib.vrad_transfer_read_packed.restype = i32
        lib.vrad_transfer_install.argtypes = [P, P, i64, P, P, i64]
        lib.vrad_transfer_install.restype = i32
        lib._transfer_cache_bound = True
    return lib


def _buf(data):
    """A ctypes view of bytes the library only reads."""
    a = np.frombuffer(data, np.uint8) if memoryview(data).nbytes else np.zeros(1, np.uint8)
    return a, a.ctypes.data


def _joined(packed):
    """Packed chunks back to back, and their sizes (no copy when they are
    already consecutive views of one buffer, as export returns them)."""
    sizes = np.array([memoryview(p).nbytes for p in packed], np.int64)
    views = [np.frombuffer(p, np.uint8) for p in packed]
    if views and all(isinstance(p, memoryview) for p in packed):
        base = views[0].__array_interface__["data"][0]
        at = base
        for v in views:
            if v.__array_interface__["data"][0] != at:
                break
            at += len(v)
        else:
            return np.frombuffer((ctypes.c_uint8 * int(sizes.sum())).from_address(base), np.uint8), sizes
    return (np.concatenate(views) if views else np.zeros(0, np.uint8)), sizes


# ---------------------------------------------------------------- host codec

def index(offsets) -> bytes:
    """TransferSetCodec.Index: magic, patch count, longest list, total, counts."""
    off = np.ascontiguousarray(offsets, np.int64)
    n = len(off) - 1
    out = np.zeros(20 + 4 * n, np.uint8)
    T._check(_lib().vrad_transfer_index(off.ctypes.data, n, out.ctypes.data, len(out)), None)
    return out.tobytes()


def chunks(offsets, transfers, max_chunk_bytes: int = DEFAULT_MAX_CHUNK_BYTES) -> list[bytes]:
    """TransferSetCodec.Chunks: the transfers patch after patch, a new chunk
    every clamp(max_chunk_bytes // 8, 1, int.MaxValue // 8) transfers."""
    off = np.asarray(offsets, np.int64)
    tr = np.ascontiguousarray(transfers, TRANSFER_DTYPE)
    # The lists are already patch after patch when offsets start at 0 and rise.
    flat = np.concatenate([tr[off[p]:off[p + 1]] for p in range(len(off) - 1)]) if len(off) > 1 else tr[:0]
    per = min(max(int(max_chunk_bytes) // TRANSFER_BYTES, 1), 0x7FFFFFFF // TRANSFER_BYTES)
    return [flat[s:s + per].tobytes() for s in range(0, len(flat), per)]


def pack(chunk: bytes) -> bytes:
    """TransferSetCodec.Pack: the count, then the deflated planes."""
    lib = _lib()
    keep, src = _buf(chunk)
    out = np.zeros(lib.vrad_transfer_pack_bound(len(chunk)), np.uint8)
    written = ctypes.c_int64()
    T._check(lib.vrad_transfer_pack(src, len(chunk), out.ctypes.data, len(out), ctypes.byref(written)), None)
    return out[:written.value].tobytes()


def unpack(packed: bytes) -> bytes | None:
    """TransferSetCodec.Unpack; None when the bytes are not a packed chunk."""
    lib = _lib()
    keep, src = _buf(packed)
    n = int.from_bytes(bytes(packed[:4]), "little", signed=True) if len(packed) >= 4 else 0
    out = np.zeros(max(1, TRANSFER_BYTES * max(n, 0)) if 0 <= n <= ARRAY_MAX_LENGTH // 8 else 1, np.uint8)
    written = ctypes.c_int64()
    rc = lib.vrad_transfer_unpack(src, len(packed), out.ctypes.data, len(out), ctypes.byref(written))
    if rc == ERR_FORMAT:
        return None
    T._check(rc, None)
    return out[:written.value].tobytes()


def _read_index(idx: bytes, patch_count: int):
    """TransferSetCodec.TryReadIndex: (counts, max, total), or None."""
    idx = bytes(idx)
    if (len(idx) < 20 or int.from_bytes(idx[0:4], "little") != MAGIC
            or int.from_bytes(idx[4:8], "little", signed=True) != patch_count
            or len(idx) != 20 + 4 * patch_count):
        return None
    longest = int.from_bytes(idx[8:12], "little", signed=True)
    total = int.from_bytes(idx[12:20], "little", signed=True)
    counts = np.frombuffer(idx, "<i4", patch_count, 20).astype(np.int64)
    if total < 0 or total > ARRAY_MAX_LENGTH or (counts < 0).any():
        return None
    if int(counts.sum()) != total or int(counts.max(initial=0)) != longest:
        return None
    return counts, longest, total


def read(idx: bytes, raw_chunks, patch_count: int):
    """TransferSetCodec.Read from raw chunks: (offsets, transfers), or None
    when they do not fit together (the index, the chunks' bytes against its
    total, a patch out of range)."""
    head = _read_index(idx, patch_count)
    if head is None:
        return None
    counts, _, total = head
    if any(len(c) % TRANSFER_BYTES for c in raw_chunks) or sum(len(c) for c in raw_chunks) != total * TRANSFER_BYTES:
        return None
    tr = np.frombuffer(b"".join(bytes(c) for c in raw_chunks), TRANSFER_DTYPE).copy()
    if ((tr["patch"] < 0) | (tr["patch"] >= patch_count)).any():
        return None
    off = np.zeros(patch_count + 1, np.int64)
    np.cumsum(counts, out=off[1:])
    return off, tr


# ---------------------------------------------------------------- on the device

def read_packed(owner, idx: bytes, packed, patch_count: int):
    """TransferSetCodec.ReadPacked: (offsets, transfers) from the index and
    the packed chunks, inflated on the host's threads and decoded on the
    owner's device; None when they do not fit together."""
    lib = _lib()
    ctx = owner._ctx
    data, sizes = _joined(packed)
    ik, ip = _buf(idx)
    dk, dp = _buf(data)
    off = np.zeros(patch_count + 1, np.int64)
    total = ctypes.c_int64()
    args = (ctx, ip, len(idx), dp, sizes.ctypes.data if len(sizes) else None, len(sizes), patch_count, off.ctypes.data)
    rc = lib.vrad_transfer_read_packed(*args, None, 0, ctypes.byref(total))
    if rc == ERR_FORMAT:
        return None
    T._check(rc, ctx)
    tr = np.zeros(max(1, total.value), TRANSFER_DTYPE)
    T._check(lib.vrad_transfer_read_packed(*args, tr.ctypes.data, len(tr), ctypes.byref(total)), ctx)
    return off, tr[:total.value]


def export(stage, max_chunk_bytes: int = DEFAULT_MAX_CHUNK_BYTES, timing: dict | None = None):
    """The stage's transfers (after a light pass that bounced, or an
    install) as the store writes them: (index bytes, [packed chunks], each a
    read-only view of one buffer).  timing, when given, receives the
    library call's own seconds ("abi_s")."""
    lib = _lib()
    ctx = stage._ctx
    ilen, nchunks, bound = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    T._check(lib.vrad_transfer_export_size(ctx, max_chunk_bytes, ctypes.byref(ilen), ctypes.byref(nchunks),
                                           ctypes.byref(bound)), ctx)
    idx = np.zeros(ilen.value, np.uint8)
    out = np.empty(max(1, bound.value), np.uint8)
    sizes = np.zeros(max(1, nchunks.value), np.int64)
    used = ctypes.c_int64()
    t0 = time.perf_counter()
    T._check(lib.vrad_transfer_export(ctx, max_chunk_bytes, idx.ctypes.data, len(idx), out.ctypes.data, len(out),
                                      sizes.ctypes.data, len(sizes), ctypes.byref(used)), ctx)
    if timing is not None:
        timing["abi_s"] = time.perf_counter() - t0
    at = np.concatenate([[0], np.cumsum(sizes[:nchunks.value])])
    out.flags.writeable = False
    return idx.tobytes(), [memoryview(out[at[k]:at[k + 1]]) for k in range(nchunks.value)]


def install(stage, idx: bytes, packed, timing: dict | None = None) -> bool:
    """A cache hit: the set becomes the stage's transfers and every later
    light pass bounces with them (BounceStats.transfers_cached) until the
    bounce is uploaded again.  False when the set is refused (it does not
    decode, or it cannot be this bounce's); the stage's transfers are then
    as they were.  timing, when given, receives the library call's own
    seconds ("abi_s")."""
    lib = _lib()
    ctx = stage._ctx
    data, sizes = _joined(packed)
    ik, ip = _buf(idx)
    dk, dp = _buf(data)
    t0 = time.perf_counter()
    rc = lib.vrad_transfer_install(ctx, ip, len(idx), dp, sizes.ctypes.data if len(sizes) else None, len(sizes))
    if timing is not None:
        timing["abi_s"] = time.perf_counter() - t0
    if rc == ERR_FORMAT:
        return False
    T._check(rc, ctx)
    return True
