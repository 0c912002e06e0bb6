"""CPU-side checks of the C ABI: the library loads, exports every entry point
include/vrad_cuda.h declares, and refuses cleanly without a device."""
import ctypes
import pathlib
import re

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "vrad_cuda.h").read_text()
    return sorted(set(re.findall(r"^\w[\w\s\*]*?\b(vrad_\w+)\s*\(", text, re.M)))


def test_header_declares_the_seam():
    names = declared_symbols()
    for must in ("vrad_create", "vrad_scene_upload", "vrad_trace_visibility", "vrad_trace_closest",
                 "vrad_trace_visibility_device", "vrad_trace_closest_device", "vrad_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from hl2sdk_tools_sharp_b200 import tracer
    lib = tracer.load_library()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert set(tracer.EXPORTS) <= set(declared_symbols())


def test_record_sizes_match_the_wire_format():
    from hl2sdk_tools_sharp_b200 import tracer
    assert tracer.RAY_DTYPE.itemsize == 28        # Ray: seven floats
    assert tracer.HIT_DTYPE.itemsize == 8         # HitId: eight bytes
    assert tracer.KD_TRIANGLE_DTYPE.itemsize == 48  # KdTriangle: 48, not 64


def test_supports_rule():
    from hl2sdk_tools_sharp_b200 import tracer
    lib = tracer.load_library()
    for md, ok in ((0.0, 1), (1e-3, 1), (-1.0, 0), (float("nan"), 0)):
        o = tracer.RayTraceOptions(md)._c()
        assert lib.vrad_supports(ctypes.byref(o)) == ok


def test_create_without_a_device_fails_with_a_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from hl2sdk_tools_sharp_b200 import tracer
    lib = tracer.load_library()
    ctx = ctypes.c_void_p()
    rc = lib.vrad_create(0, ctypes.byref(ctx))
    assert rc == -7 and not ctx.value
    buf = ctypes.create_string_buffer(256)
    assert lib.vrad_last_error(None, buf, 256) > 0
    with pytest.raises(tracer.VradError):
        tracer.CudaRayTracer(np.zeros((1, 9), np.float32))


def test_null_context_calls_are_argument_errors():
    from hl2sdk_tools_sharp_b200 import tracer
    lib = tracer.load_library()
    assert lib.vrad_scene_upload(None, None, 0) == -1
    assert lib.vrad_trace_visibility(None, None, 0, None, None) == -1
    assert lib.vrad_destroy(None) == 0
