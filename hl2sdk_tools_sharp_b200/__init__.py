"""hl2sdk_tools_sharp_b200: vrad's lighting-stage ray tracing on B200 (sm_100a).

The compute lives in libvrad_cuda.so (hand-written CUDA behind the C ABI in
include/vrad_cuda.h).  This package is the host layer over it, mirroring the
reference's IRayTracer seam (tracer.py), plus the seeded room-grid scene
generator used for benchmarks and parity tests (roomgrid.py).
"""
from .tracer import (  # noqa: F401
    CudaRayTracer, RayTraceOptions, VradError, RAY_DTYPE, HIT_DTYPE, TRIANGLE_DTYPE,
    KD_TRIANGLE_DTYPE, TRACE_ID_SKY, load_library, make_rays, make_triangles, segment_rays,
)

__all__ = [
    "CudaRayTracer", "RayTraceOptions", "VradError", "RAY_DTYPE", "HIT_DTYPE", "TRIANGLE_DTYPE",
    "KD_TRIANGLE_DTYPE", "TRACE_ID_SKY", "load_library", "make_rays", "make_triangles",
    "segment_rays",
]
