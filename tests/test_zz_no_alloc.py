"""vrad_trace_visibility_static: the visibility trace that allocates nothing.

It serves callers that must not allocate device memory during a run
(processes that reserve all device memory at start-up, hosts that must not
stall on the synchronisation freeing memory can bring), staging rays and
bits through a fixed array inside the library.
Its answers must be exactly those of vrad_trace_visibility, on two calls in
a row (the array keeps the previous call's contents), and a batch above its
stated maximum must be refused.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import roomgrid as rg, tracer as T, workload as wl

pytestmark = pytest.mark.gpu

MAX_RAYS = 65536  # VRAD_STATIC_MAX_RAYS in include/vrad_cuda.h


def _static_fn():
    lib = T.load_library()
    fn = lib.vrad_trace_visibility_static
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                   ctypes.POINTER(T._Options), ctypes.c_void_p]
    fn.restype = ctypes.c_int32
    return fn


def _static_bits(tr, rays, opts):
    fn = _static_fn()
    n = len(rays)
    bits = np.full((n + 63) // 64, 0xA5A5A5A5A5A5A5A5, np.uint64)  # stale garbage must be overwritten
    o = opts._c()
    rc = fn(tr._ctx, rays.ctypes.data, n, ctypes.byref(o), bits.ctypes.data)
    assert rc == 0, T._message(tr._ctx)
    return bits


def _free_device_bytes():
    # The runtime library the vrad library itself loaded (same soname).
    rt = ctypes.CDLL("libcudart.so.12")
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    assert rt.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    return free.value


def test_static_entry_takes_no_device_memory():
    """On a fresh context, calls of the static entry (a full batch among
    them) leave the device's free memory exactly where it was: nothing is
    allocated, and no kernel code is placed on the device, after set-up.
    The allocating entry is not called before the check, so a static call
    that fell back to the context's own buffers would show here."""
    w = rg.generate(rg.config_3x3(seed=7))
    r = wl.direct_rays(w, wl.luxel_samples(w, stride=3), ambient=True)
    full = np.ascontiguousarray(r.sky[:MAX_RAYS])
    part = np.ascontiguousarray(r.light[:777])
    assert len(full) == MAX_RAYS
    sky = T.RayTraceOptions(0.0, sky_does_not_block=True)
    with T.CudaRayTracer(T.make_triangles(w.tri_verts, w.tri_ids)) as tr:
        _static_bits(tr, part, T.RayTraceOptions.stock_exact())
        before = _free_device_bytes()
        a = _static_bits(tr, full, sky)
        b = _static_bits(tr, part, T.RayTraceOptions.stock_exact())
        c = _static_bits(tr, full, sky)
        after = _free_device_bytes()
        assert after == before, f"{before - after} bytes of device memory taken by static calls"
        assert np.array_equal(a, c)
        want = np.zeros_like(b)
        tr.trace_visibility(part, want, T.RayTraceOptions.stock_exact())
        assert np.array_equal(b, want)


def test_static_entry_matches_the_allocating_one_on_two_calls():
    w = rg.generate(rg.config_3x3(seed=5))
    r = wl.direct_rays(w, wl.luxel_samples(w, stride=3), ambient=True)
    first = np.ascontiguousarray(r.sky[:MAX_RAYS])        # a full batch
    second = np.ascontiguousarray(r.light[:12345])          # a smaller, ragged one after it
    assert len(first) == MAX_RAYS
    with T.CudaRayTracer(T.make_triangles(w.tri_verts, w.tri_ids)) as tr:
        for rays, opts in ((first, T.RayTraceOptions(0.0, sky_does_not_block=True)),
                           (second, T.RayTraceOptions.stock_exact())):
            want = np.zeros((len(rays) + 63) // 64, np.uint64)
            tr.trace_visibility(rays, want, opts)
            got = _static_bits(tr, rays, opts)
            assert np.array_equal(got, want)
            assert 0 < np.unpackbits(got.view(np.uint8)).sum() < len(rays)


def test_static_entry_refuses_more_than_its_maximum():
    w = rg.generate(rg.config_3x3(seed=5))
    fn = _static_fn()
    with T.CudaRayTracer(T.make_triangles(w.tri_verts, w.tri_ids)) as tr:
        rays = np.zeros(MAX_RAYS + 1, T.RAY_DTYPE)
        bits = np.zeros((len(rays) + 63) // 64, np.uint64)
        o = T.RayTraceOptions()._c()
        assert fn(tr._ctx, rays.ctypes.data, len(rays), ctypes.byref(o), bits.ctypes.data) == -1
        assert "exceed" in T._message(tr._ctx)
