"""Many maps lit on one device through the native batch runner (vrad_batch_*).

The reference lights one map per call (Vrad.RunAsync,
MapTools/Rad/Vrad.cs:160-390); a batch has no counterpart there.  The
runner is C++ inside libvrad_cuda.so. Its persistent worker threads each
own a context and take maps from one shared queue, largest first.  Each map
runs the whole lighting stage through the single-map entry points (scene,
world and bounce uploads, the light pass), so every lump equals the
single-map lump byte for byte.  This module only lays out the maps' input
descriptors and owns their arrays while a run reads them.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import lighting as L
from . import tracer as T
from .roomgrid import World

MAX_WORKERS = 8


class _BatchMap(ctypes.Structure):
    _fields_ = [("triangles", ctypes.c_void_p), ("world", ctypes.c_void_p), ("bounce", ctypes.c_void_p),
                ("lighting", ctypes.c_void_p), ("lightofs", ctypes.c_void_p), ("capacity", ctypes.c_int64),
                ("ntriangles", ctypes.c_int32), ("extra_passes", ctypes.c_int32),
                ("status", ctypes.c_int32), ("worker", ctypes.c_int32), ("lighting_bytes", ctypes.c_int64),
                ("seconds", ctypes.c_double), ("scene_s", ctypes.c_double), ("world_s", ctypes.c_double),
                ("bounce_s", ctypes.c_double), ("pass_s", ctypes.c_double),
                ("pass_stats", L.PassStats), ("bounce_stats", L.BounceStats),
                ("error", ctypes.c_char * 256)]


class BatchStats(ctypes.Structure):
    _fields_ = [("workers", ctypes.c_int32), ("maps", ctypes.c_int32), ("failed", ctypes.c_int32),
                ("block", ctypes.c_int32), ("seconds", ctypes.c_double), ("busy_seconds", ctypes.c_double),
                ("rays", ctypes.c_int64), ("luxels", ctypes.c_int64), ("lighting_bytes", ctypes.c_int64),
                ("device_mallocs", ctypes.c_int64), ("device_malloc_bytes", ctypes.c_int64),
                ("device_trims", ctypes.c_int64)]


def _lib():
    lib = L._lib()
    if not getattr(lib, "_batch_bound", False):
        P, i32 = ctypes.c_void_p, ctypes.c_int32
        lib.vrad_batch_create.argtypes = [i32, i32, ctypes.POINTER(P)]
        lib.vrad_batch_create.restype = i32
        lib.vrad_batch_destroy.argtypes = [P]
        lib.vrad_batch_destroy.restype = i32
        lib.vrad_batch_run.argtypes = [P, P, i32, i32, ctypes.POINTER(BatchStats)]
        lib.vrad_batch_run.restype = i32
        lib.vrad_batch_autotune.argtypes = [P, P, i32, ctypes.POINTER(i32), ctypes.POINTER(i32), P]
        lib.vrad_batch_autotune.restype = i32
        lib._batch_bound = True
    return lib


@dataclasses.dataclass
class MapInputs:
    """One map of a batch: its shadow casters, lighting world and bounce."""
    triangles: np.ndarray
    inputs: L.LightingInputs
    lighting_bytes: int
    reflectivity: np.ndarray | None = None
    pvs_offsets: np.ndarray | None = None
    pvs_clusters: np.ndarray | None = None
    bounces: int = 100
    threshold: float = 1.0
    max_chop: float = 4.0
    min_chop: float = 4.0
    extra_passes: int = -1

    @property
    def bounced(self) -> bool:
        return self.reflectivity is not None


def map_inputs(world: World, inputs: L.LightingInputs | None = None, bounce: bool = True, bounces: int = 100,
               threshold: float = 1.0, extra_passes: int = -1) -> MapInputs:
    """The batch inputs of a room-grid world (host set-up only)."""
    inp = inputs if inputs is not None else L.prepare(world)
    tris = T.make_triangles(world.tri_verts, world.tri_ids)
    _, size = L.lightmap_layout(inp.faces)
    m = MapInputs(tris, inp, size, bounces=bounces, threshold=threshold, extra_passes=extra_passes)
    if bounce:
        m.reflectivity = L.face_reflectivity(world)
        m.pvs_offsets, m.pvs_clusters = L.pvs_lists(world)
    return m


@dataclasses.dataclass
class MapResult:
    lighting: np.ndarray
    lightofs: np.ndarray
    worker: int
    seconds: float
    pass_stats: L.PassStats
    bounce_stats: L.BounceStats
    status: int = 0
    error: str = ""
    phases_s: dict = dataclasses.field(default_factory=dict)


class LightingBatch:
    """A persistent batch runner on one device: `workers` host threads,
    each with its own context, lighting whole maps from one queue."""

    def __init__(self, workers: int = 2, device: int = 0):
        self._b = ctypes.c_void_p()
        T._check(_lib().vrad_batch_create(device, workers, ctypes.byref(self._b)), None)
        self.workers = workers

    def close(self):
        if self._b:
            _lib().vrad_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _descriptors(self, maps: list[MapInputs], outputs=None):
        keep = []
        arr = (_BatchMap * max(1, len(maps)))()
        for k, m in enumerate(maps):
            i = m.inputs
            a = [np.ascontiguousarray(x) for x in (i.faces, i.samples, i.lights, i.cluster_offsets,
                                                    i.cluster_lights, i.sky_directions, i.sun_jitter, i.verts)]
            f, s, l, off, cl, dirs, jit, vv = a
            wd = L._WorldDesc(f.ctypes.data, len(f), s.ctypes.data, len(s), l.ctypes.data, len(l),
                              off.ctypes.data, cl.ctypes.data, len(off) - 1, dirs.ctypes.data, len(dirs),
                              jit.ctypes.data if len(jit) else None, len(jit), i.sun_angular_extent, i.sun_samples,
                              vv.ctypes.data, len(vv))
            keep += a + [wd]
            bd = None
            if m.bounced:
                refl = np.ascontiguousarray(m.reflectivity, np.float32).reshape(-1, 3)
                po = np.ascontiguousarray(m.pvs_offsets, np.int32)
                pl = np.ascontiguousarray(m.pvs_clusters, np.int32)
                bd = L._BounceDesc(refl.ctypes.data, po.ctypes.data, pl.ctypes.data if len(pl) else None,
                                   len(po) - 1, m.max_chop, m.min_chop, m.bounces, m.threshold)
                keep += [refl, po, pl, bd]
            tris = np.ascontiguousarray(m.triangles)
            if outputs is not None:
                lump, ofs = outputs[k]
            else:
                lump = np.zeros(max(1, m.lighting_bytes), np.uint8)
                ofs = np.zeros(len(f), np.int32)
            keep += [tris, lump, ofs]
            d = arr[k]
            d.triangles = tris.ctypes.data
            d.ntriangles = len(tris)
            d.world = ctypes.addressof(wd)
            d.bounce = ctypes.addressof(bd) if bd is not None else None
            d.lighting = lump.ctypes.data
            d.capacity = m.lighting_bytes
            d.lightofs = ofs.ctypes.data
            d.extra_passes = m.extra_passes
        return arr, keep

    @staticmethod
    def _results(arr, keep_outputs, n) -> list[MapResult]:
        out = []
        for k in range(n):
            d = arr[k]
            lump, ofs = keep_outputs[k]
            ps = L.PassStats.from_buffer_copy(d.pass_stats)
            bs = L.BounceStats.from_buffer_copy(d.bounce_stats)
            out.append(MapResult(lump[:d.lighting_bytes], ofs, d.worker, d.seconds, ps, bs, d.status,
                                 d.error.decode(errors="replace"),
                                 {"scene": d.scene_s, "world": d.world_s, "bounce": d.bounce_s, "pass": d.pass_s}))
        return out

    def _check_maps(self, rc, arr, n):
        if rc == 0:
            return
        for k in range(n):
            if arr[k].status != 0:
                err = arr[k].error.decode(errors="replace")
                if arr[k].status == -6:
                    raise NotImplementedError(f"map {k}: {err}")
                if arr[k].status == -1:
                    raise ValueError(f"map {k}: {err}")
                raise T.VradError(arr[k].status, f"map {k}: {err}")
        T._check(rc, None)

    def run(self, maps: list[MapInputs], workers: int = 0, raise_on_error: bool = True):
        """Lights every map; returns ([MapResult], BatchStats).  workers: how
        many of the batch's workers take maps (0: the tuned count, else all).
        A map that fails does not stop the others; with raise_on_error the
        first failure is raised after the run, else each result carries its
        status and message."""
        outs = [(np.zeros(max(1, m.lighting_bytes), np.uint8), np.zeros(len(m.inputs.faces), np.int32))
                for m in maps]
        arr, keep = self._descriptors(maps, outs)
        st = BatchStats()
        rc = _lib().vrad_batch_run(self._b, ctypes.cast(arr, ctypes.c_void_p), len(maps), workers, ctypes.byref(st))
        if raise_on_error or not any(arr[k].status for k in range(len(maps))):
            self._check_maps(rc, arr, len(maps))
        del keep
        return self._results(arr, outs, len(maps)), st

    def autotune(self, maps: list[MapInputs]):
        """vrad_batch_autotune: the gather's launch shape on the largest map,
        then the batch timed at 1..workers maps in flight.  Returns
        (workers, threads per CTA, {workers: seconds})."""
        outs = [(np.zeros(max(1, m.lighting_bytes), np.uint8), np.zeros(len(m.inputs.faces), np.int32))
                for m in maps]
        arr, keep = self._descriptors(maps, outs)
        w, blk = ctypes.c_int32(), ctypes.c_int32()
        secs = np.zeros(self.workers, np.float64)
        rc = _lib().vrad_batch_autotune(self._b, ctypes.cast(arr, ctypes.c_void_p), len(maps), ctypes.byref(w),
                                        ctypes.byref(blk), secs.ctypes.data)
        self._check_maps(rc, arr, len(maps))
        del keep
        return w.value, blk.value, {k + 1: float(secs[k]) for k in range(self.workers)}
