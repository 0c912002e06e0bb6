"""Host-side mirror of the reference's ray-tracing seam over libvrad_cuda.

Names and argument meanings follow the reference's C# interface
(muflub/hl2sdk_tools_sharp, src/SourceSharp.MapTools/Tracing):

  Ray              IRayTracer.cs:32-42    seven float32: origin, direction, reach
  HitId            HitId.cs:70            (surface, fraction), miss = (-1, 1.0)
  RayTraceOptions  RayTraceOptions.cs:65  min_distance, skip_id, sky_does_not_block,
                                          isolated_rays; StockExact / SelfIntersectionSafe
  TracedTriangle   KdTree.cs:30-38        id, three vertices, FCACHETRI flags
  IRayTracer       IRayTracer.cs:128-230  trace_visibility / trace_closest / supports /
                                          tracer_identity

Error behaviour follows the reference: a short output buffer raises
ValueError (ArgumentException), an option the tracer cannot honour raises
NotImplementedError (NotSupportedException), a sky-passing closest-hit
query raises ValueError.  There is no CPU fallback: if libvrad_cuda.so is
missing or no sm_100 device is present, construction raises.

Buffers may be numpy arrays (host: the call copies in and out and blocks)
or CUDA torch tensors (device: the call enqueues on the current torch
stream and returns at once).
"""
from __future__ import annotations

import ctypes
import dataclasses
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libvrad_cuda.so"

VRAD_OK = 0
ERRORS = {
    -1: "VRAD_ERR_ARG", -2: "VRAD_ERR_CUDA", -3: "VRAD_ERR_OOM", -4: "VRAD_ERR_TIMEOUT",
    -5: "VRAD_ERR_NO_SCENE", -6: "VRAD_ERR_UNSUPPORTED", -7: "VRAD_ERR_NO_DEVICE", -8: "VRAD_ERR_FORMAT",
}

TRACE_ID_SKY = 0x01000000   # TraceId.Sky (MapTools/Rad/TraceId.cs)
TRANSPARENT = 0x01          # TracedTriangle.Transparent
NEGATIVE_NORMAL = 0x02      # TracedTriangle.NegativeNormal

RAY_DTYPE = np.dtype([("origin", "<f4", (3,)), ("direction", "<f4", (3,)), ("max_distance", "<f4")])
HIT_DTYPE = np.dtype([("surface", "<i4"), ("fraction", "<f4")])
TRIANGLE_DTYPE = np.dtype([("id", "<i4"), ("v0", "<f4", (3,)), ("v1", "<f4", (3,)),
                           ("v2", "<f4", (3,)), ("flags", "u1"), ("pad", "u1", (3,))])
KD_TRIANGLE_DTYPE = np.dtype([("n", "<f4", (3,)), ("d", "<f4"), ("id", "<i4"), ("e", "<f4", (6,)),
                              ("cs0", "u1"), ("cs1", "u1"), ("flags", "u1"), ("unused", "u1")])
assert RAY_DTYPE.itemsize == 28 and HIT_DTYPE.itemsize == 8
assert TRIANGLE_DTYPE.itemsize == 44 and KD_TRIANGLE_DTYPE.itemsize == 48

EXPORTS = (
    "vrad_abi_version", "vrad_create", "vrad_destroy", "vrad_scene_upload",
    "vrad_scene_upload_prepared", "vrad_scene_get_info", "vrad_supports",
    "vrad_trace_visibility", "vrad_trace_closest", "vrad_trace_visibility_device",
    "vrad_trace_closest_device", "vrad_tracer_identity", "vrad_last_error",
)


class VradError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


class _Options(ctypes.Structure):
    _fields_ = [("min_distance", ctypes.c_float), ("skip_id", ctypes.c_int32),
                ("sky_does_not_block", ctypes.c_int32), ("isolated_rays", ctypes.c_int32)]


class SceneInfo(ctypes.Structure):
    _fields_ = [("triangles", ctypes.c_int32), ("bvh_nodes", ctypes.c_int32),
                ("bvh_leaves", ctypes.c_int32), ("max_leaf", ctypes.c_int32),
                ("bounds_min", ctypes.c_float * 3), ("bounds_max", ctypes.c_float * 3),
                ("box_pad", ctypes.c_float), ("build_ms", ctypes.c_float),
                ("device_bytes", ctypes.c_int64), ("bvh_depth", ctypes.c_int32)]


@dataclasses.dataclass(frozen=True)
class RayTraceOptions:
    """RayTraceOptions (RayTraceOptions.cs:65-145)."""
    min_distance: float = 0.0
    skip_id: int | None = None
    sky_does_not_block: bool = False
    isolated_rays: bool = False

    @property
    def is_plain(self) -> bool:
        return self.skip_id is None and not self.sky_does_not_block

    @staticmethod
    def stock_exact() -> "RayTraceOptions":
        return RayTraceOptions(0.0)

    @staticmethod
    def self_intersection_safe() -> "RayTraceOptions":
        return RayTraceOptions(1.0e-3)

    @staticmethod
    def test_line(skip_id: int = -1, sky_does_not_block: bool = False) -> "RayTraceOptions":
        return RayTraceOptions(0.0, None if skip_id < 0 else skip_id, sky_does_not_block, True)

    def _c(self) -> _Options:
        return _Options(self.min_distance, -1 if self.skip_id is None else int(self.skip_id),
                        int(bool(self.sky_does_not_block)), int(bool(self.isolated_rays)))


class RecheckStats(ctypes.Structure):
    _fields_ = [("rays", ctypes.c_int64), ("flagged", ctypes.c_int64), ("fp64_hit", ctypes.c_int64),
                ("fp64_miss", ctypes.c_int64), ("fp64_ambiguous", ctypes.c_int64),
                ("disagreements", ctypes.c_int64)]


_lib = None


def load_library() -> ctypes.CDLL:
    """Loads libvrad_cuda.so; raises if it is missing (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with python -m hl2sdk_tools_sharp_b200.build")
    lib = ctypes.CDLL(str(LIB_PATH))
    P, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    sig = {
        "vrad_abi_version": ([], i32),
        "vrad_create": ([i32, ctypes.POINTER(P)], i32),
        "vrad_destroy": ([P], i32),
        "vrad_scene_upload": ([P, P, i32], i32),
        "vrad_scene_upload_prepared": ([P, P, P, i32], i32),
        "vrad_scene_get_info": ([P, ctypes.POINTER(SceneInfo)], i32),
        "vrad_supports": ([ctypes.POINTER(_Options)], i32),
        "vrad_trace_visibility": ([P, P, i64, ctypes.POINTER(_Options), P], i32),
        "vrad_trace_closest": ([P, P, i64, ctypes.POINTER(_Options), P], i32),
        "vrad_trace_visibility_device": ([P, P, i64, ctypes.POINTER(_Options), P, P], i32),
        "vrad_trace_closest_device": ([P, P, i64, ctypes.POINTER(_Options), P, P], i32),
        "vrad_trace_visibility_recheck": ([P, P, i64, ctypes.POINTER(_Options), P, i32, ctypes.c_float,
                                           ctypes.c_double, P, P, ctypes.POINTER(RecheckStats)], i32),
        "vrad_tracer_identity": ([P, ctypes.c_char_p, i32], i32),
        "vrad_last_error": ([P, ctypes.c_char_p, i32], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _message(ctx) -> str:
    buf = ctypes.create_string_buffer(1024)
    load_library().vrad_last_error(ctx, buf, len(buf))
    return buf.value.decode(errors="replace")


def _check(rc: int, ctx) -> None:
    if rc == VRAD_OK:
        return
    msg = _message(ctx)
    if rc == -6:
        raise NotImplementedError(msg)
    if rc == -1:
        raise ValueError(msg)
    raise VradError(rc, msg)


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def make_triangles(verts: np.ndarray, ids: np.ndarray | None = None,
                   flags: np.ndarray | None = None) -> np.ndarray:
    """TracedTriangle records from (n, 9) vertices."""
    verts = np.asarray(verts, np.float32).reshape(-1, 9)
    t = np.zeros(len(verts), TRIANGLE_DTYPE)
    t["id"] = np.arange(len(verts)) if ids is None else ids
    t["v0"], t["v1"], t["v2"] = verts[:, 0:3], verts[:, 3:6], verts[:, 6:9]
    if flags is not None:
        t["flags"] = flags
    return t


def make_rays(origins: np.ndarray, directions: np.ndarray, reach) -> np.ndarray:
    r = np.zeros(len(origins), RAY_DTYPE)
    r["origin"] = origins
    r["direction"] = directions
    r["max_distance"] = reach
    return r


def segment_rays(starts: np.ndarray, ends: np.ndarray) -> np.ndarray:
    """LightRayLog.MakeRay (MapTools/Rad/Light/LightRayLog.cs:686): the whole
    segment as the direction, reach 1."""
    starts = np.asarray(starts, np.float32)
    ends = np.asarray(ends, np.float32)
    return make_rays(starts, ends - starts, 1.0)


class CudaRayTracer:
    """IRayTracer over libvrad_cuda on one CUDA device.

    Construct with the scene's triangles (TracedTriangle records, or (n, 9)
    vertices).  `prepared` optionally supplies the 48-byte intersection
    form (e.g. stock-normalised coefficients) for the same triangles.
    """

    def __init__(self, triangles, device: int = 0, prepared: np.ndarray | None = None):
        lib = load_library()
        self._lib = lib
        ctx = ctypes.c_void_p()
        rc = lib.vrad_create(device, ctypes.byref(ctx))
        if rc != VRAD_OK:
            raise VradError(rc, _message(None))
        self._ctx = ctx
        tris = triangles
        if not (isinstance(tris, np.ndarray) and tris.dtype == TRIANGLE_DTYPE):
            tris = make_triangles(tris)
        tris = np.ascontiguousarray(tris)
        self.triangle_count = len(tris)
        self._tris = tris
        if prepared is not None:
            prepared = np.ascontiguousarray(prepared, KD_TRIANGLE_DTYPE)
            if len(prepared) != len(tris):
                raise ValueError("one prepared triangle per triangle")
            rc = lib.vrad_scene_upload_prepared(ctx, tris.ctypes.data, prepared.ctypes.data, len(tris))
        else:
            rc = lib.vrad_scene_upload(ctx, tris.ctypes.data, len(tris))
        _check(rc, ctx)

    def upload_scene(self, triangles) -> None:
        """vrad_scene_upload again: a new scene (intersection form and BVH)
        for this context's later traces and light passes."""
        tris = triangles
        if not (isinstance(tris, np.ndarray) and tris.dtype == TRIANGLE_DTYPE):
            tris = make_triangles(tris)
        tris = np.ascontiguousarray(tris)
        self.triangle_count = len(tris)
        self._tris = tris
        _check(self._lib.vrad_scene_upload(self._ctx, tris.ctypes.data, len(tris)), self._ctx)

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_ctx", None):
            self._lib.vrad_destroy(self._ctx)
            self._ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- IRayTracer ---------------------------------------------------------
    @property
    def tracer_identity(self) -> str:
        buf = ctypes.create_string_buffer(256)
        self._lib.vrad_tracer_identity(self._ctx, buf, len(buf))
        return buf.value.decode()

    def supports(self, options: RayTraceOptions) -> bool:
        o = options._c()
        return bool(self._lib.vrad_supports(ctypes.byref(o)))

    def scene_info(self) -> SceneInfo:
        info = SceneInfo()
        _check(self._lib.vrad_scene_get_info(self._ctx, ctypes.byref(info)), self._ctx)
        return info

    def trace_visibility(self, rays, hit_bits, options: RayTraceOptions = RayTraceOptions()):
        """TraceVisibilityAsync: one bit per ray, LSB first, set when an
        accepted hit lies in [min_distance, max_distance)."""
        o = options._c()
        if _is_torch(rays):
            n = rays.numel() * rays.element_size() // 28
            need = (n + 63) // 64
            if hit_bits.numel() * hit_bits.element_size() < 8 * need:
                raise ValueError(f"{n} rays need {need} words of hit bits")
            import torch
            stream = torch.cuda.current_stream(rays.device).cuda_stream
            _check(self._lib.vrad_trace_visibility_device(
                self._ctx, rays.data_ptr(), n, ctypes.byref(o), hit_bits.data_ptr(),
                ctypes.c_void_p(stream)), self._ctx)
            return hit_bits
        rays = np.ascontiguousarray(rays)
        n = rays.nbytes // 28
        need = (n + 63) // 64
        if hit_bits.dtype != np.uint64 or len(hit_bits) < need or not hit_bits.flags.c_contiguous:
            raise ValueError(f"{n} rays need {need} contiguous uint64 words of hit bits, got {len(hit_bits)}")
        _check(self._lib.vrad_trace_visibility(self._ctx, rays.ctypes.data, n, ctypes.byref(o),
                                               hit_bits.ctypes.data), self._ctx)
        return hit_bits

    def trace_closest(self, rays, hits, options: RayTraceOptions = RayTraceOptions()):
        """TraceClosestAsync: the nearest accepted hit in
        [min_distance, max_distance); a miss is (-1, 1.0)."""
        if options.sky_does_not_block:
            raise ValueError("sky pass-through is a visibility option; a closest-hit trace "
                             "reports the sky hit itself")
        o = options._c()
        if _is_torch(rays):
            n = rays.numel() * rays.element_size() // 28
            if hits.numel() * hits.element_size() < 8 * n:
                raise ValueError(f"{n} rays need {n} hit slots")
            import torch
            stream = torch.cuda.current_stream(rays.device).cuda_stream
            _check(self._lib.vrad_trace_closest_device(
                self._ctx, rays.data_ptr(), n, ctypes.byref(o), hits.data_ptr(),
                ctypes.c_void_p(stream)), self._ctx)
            return hits
        rays = np.ascontiguousarray(rays)
        n = rays.nbytes // 28
        if hits.dtype != HIT_DTYPE or len(hits) < n or not hits.flags.c_contiguous:
            raise ValueError(f"{n} rays need {n} hit slots, got {len(hits)}")
        _check(self._lib.vrad_trace_closest(self._ctx, rays.ctypes.data, n, ctypes.byref(o),
                                            hits.ctypes.data), self._ctx)
        return hits

    # -- conveniences -----------------------------------------------------
    def visibility(self, rays, options: RayTraceOptions = RayTraceOptions()) -> np.ndarray:
        rays = np.ascontiguousarray(rays)
        n = rays.nbytes // 28
        bits = np.zeros((n + 63) // 64, np.uint64)
        self.trace_visibility(rays, bits, options)
        return np.unpackbits(bits.view(np.uint8), bitorder="little")[:n].astype(bool)

    def visibility_recheck(self, rays, options: RayTraceOptions = RayTraceOptions(), flag_margin: float = 1e-3,
                           fp64_margin: float = 1e-6):
        """vrad_trace_visibility_recheck: (the FP32 visibility, as visibility
        gives it; per ray the FP64 class of a flagged ray, 0 miss, 1 hit,
        2 ambiguous, -1 not flagged; the counts as a dict)."""
        rays = np.ascontiguousarray(rays)
        n = rays.nbytes // 28
        bits = np.zeros((n + 63) // 64 or 1, np.uint64)
        cls = np.zeros(n or 1, np.int8)
        st = RecheckStats()
        o = options._c()
        _check(self._lib.vrad_trace_visibility_recheck(self._ctx, rays.ctypes.data, n, ctypes.byref(o),
                                                       self._tris.ctypes.data, len(self._tris), flag_margin,
                                                       fp64_margin, bits.ctypes.data, cls.ctypes.data,
                                                       ctypes.byref(st)), self._ctx)
        vis = np.unpackbits(bits.view(np.uint8), bitorder="little")[:n].astype(bool)
        return vis, cls[:n], {k: int(getattr(st, k)) for k, _ in RecheckStats._fields_}

    def closest(self, rays, options: RayTraceOptions = RayTraceOptions()) -> np.ndarray:
        rays = np.ascontiguousarray(rays)
        n = rays.nbytes // 28
        hits = np.zeros(n, HIT_DTYPE)
        self.trace_closest(rays, hits, options)
        return hits
