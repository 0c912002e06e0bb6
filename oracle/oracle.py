"""ctypes binding for the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline leg, always as the checker, never as the thing
measured for the GPU path.  The product (hl2sdk_tools_sharp_b200) never
imports this module.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

CLOSEST = 1
ISOLATED = 2
SKY_PASS = 4
FULL_WALK = 8
TRACE_ID_SKY = 0x01000000

# KdTriangle, 48 bytes (MapTools/Tracing/KdTree.cs:120-167).
TRI_DTYPE = np.dtype([
    ("n", "<f4", (3,)), ("d", "<f4"), ("id", "<i4"), ("e", "<f4", (6,)),
    ("cs0", "u1"), ("cs1", "u1"), ("flags", "u1"), ("unused", "u1"),
])
assert TRI_DTYPE.itemsize == 48
NODE_DTYPE = np.dtype([("children", "<i4"), ("split", "<f4")])


def build(force: bool = False) -> None:
    """Compile liboracle.so with the committed Makefile."""
    if force or not LIB_PATH.exists() or any(
            p.stat().st_mtime > LIB_PATH.stat().st_mtime
            for p in HERE.glob("*.[ch]*") if p.suffix in (".cpp", ".h")):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.c_void_p
        i32 = ctypes.c_int32
        f32 = ctypes.c_float
        _lib.orc_tri_prepare.argtypes = [P, P, P, i32, P]
        _lib.orc_kd_trace.argtypes = [P, i32, P, i32, P, i32, P, P, i32, f32, i32, i32, P, P, P, i32]
        _lib.orc_brute_trace.argtypes = [P, i32, P, i32, f32, i32, i32, P, P, P, i32]
        _lib.orc_fp64_classify.argtypes = [P, i32, P, i32, ctypes.c_double, P, i32]
        for name in ("orc_tri_prepare", "orc_kd_trace", "orc_brute_trace", "orc_fp64_classify"):
            getattr(_lib, name).restype = ctypes.c_int
        _lib.orc_build_samples.argtypes = [P, i32, P, P, ctypes.c_int64, P, P]
        _lib.orc_build_samples.restype = ctypes.c_int
        _lib.orc_direct.argtypes = [P, P, P, P, P, i32, P, P, P, P, P, P, P, i32, P, i32, f32, i32, P, i32, P, P]
        _lib.orc_direct.restype = ctypes.c_int
        _lib.orc_neighbours.argtypes = [P, i32, P, f32, P, P, ctypes.c_int64, P]
        _lib.orc_neighbours.restype = ctypes.c_int
        _lib.orc_final.argtypes = [P, i32, P, P, P, P, P, ctypes.c_int64, P, P]
        _lib.orc_final.restype = ctypes.c_int
        _lib.orc_direct_styles.argtypes = [P, P, P, P, P, i32, P, P, P, P, P, P, P, i32, P, i32, f32, i32, P, P, P,
                                           P, i32, P, P]
        _lib.orc_direct_styles.restype = ctypes.c_int
        _lib.orc_final_styles.argtypes = [P, i32, P, P, P, P, P, P, P, ctypes.c_int64, P, P]
        _lib.orc_final_styles.restype = ctypes.c_int
        if hasattr(_lib, "orc_kd_build"):
            _lib.orc_kd_build.argtypes = [P, P, P, i32, P]
            _lib.orc_kd_build.restype = ctypes.c_int
            _lib.orc_kd_free.argtypes = [P]
            _lib.orc_kd_free.restype = None
    return _lib


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def default_threads() -> int:
    return max(1, os.cpu_count() or 1)


def prepare_triangles(verts: np.ndarray, ids: np.ndarray | None = None,
                      flags: np.ndarray | None = None) -> np.ndarray:
    """Correct-mode intersection format for (n, 9) float32 vertices."""
    verts = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 9)
    n = verts.shape[0]
    ids = None if ids is None else np.ascontiguousarray(ids, dtype=np.int32)
    flags = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint8)
    out = np.zeros(n, dtype=TRI_DTYPE)
    rc = lib().orc_tri_prepare(_p(verts), _p(ids), _p(flags), n, _p(out))
    if rc != 0:
        raise RuntimeError(f"orc_tri_prepare failed: {rc}")
    return out


def kd_trace(tree: dict, rays: np.ndarray, tmin: float = 0.0, skip_id: int = -1,
             flags: int = 0, threads: int = 1):
    """Restated KdRayTracer over a tree dict (nodes, indices, tris, bounds)."""
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 7)
    n = rays.shape[0]
    tri = np.empty(n, dtype=np.int32)
    dist = np.empty(n, dtype=np.float32)
    bits = np.zeros((n + 63) // 64, dtype=np.uint64)
    nodes = np.ascontiguousarray(tree["nodes"], dtype=NODE_DTYPE)
    idx = np.ascontiguousarray(tree["indices"], dtype=np.int32)
    tris = np.ascontiguousarray(tree["tris"], dtype=TRI_DTYPE)
    bounds = np.ascontiguousarray(tree["bounds"], dtype=np.float32)
    rc = lib().orc_kd_trace(_p(nodes), len(nodes), _p(idx), len(idx), _p(tris), len(tris),
                            _p(bounds), _p(rays), n, tmin, skip_id, flags, _p(tri), _p(dist),
                            _p(bits), threads)
    if rc != 0:
        raise RuntimeError(f"orc_kd_trace failed: {rc}")
    return tri, dist, bits


def brute_trace(tris: np.ndarray, rays: np.ndarray, tmin: float = 0.0, skip_id: int = -1,
                flags: int = 0, threads: int | None = None):
    """The CUDA tracer's exact semantic, by brute force (see vrad_oracle.h)."""
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 7)
    tris = np.ascontiguousarray(tris, dtype=TRI_DTYPE)
    n = rays.shape[0]
    tri = np.empty(n, dtype=np.int32)
    dist = np.empty(n, dtype=np.float32)
    bits = np.zeros((n + 63) // 64, dtype=np.uint64)
    rc = lib().orc_brute_trace(_p(tris), len(tris), _p(rays), n, tmin, skip_id, flags,
                               _p(tri), _p(dist), _p(bits),
                               threads if threads is not None else default_threads())
    if rc != 0:
        raise RuntimeError(f"orc_brute_trace failed: {rc}")
    return tri, dist, bits


def kd_build(verts: np.ndarray, ids: np.ndarray | None = None,
             flags: np.ndarray | None = None) -> dict:
    """Restated KdTreeBuilder (SAH); returns a tree dict for kd_trace."""
    L = lib()
    if not hasattr(L, "orc_kd_build"):
        raise NotImplementedError("orc_kd_build is not in this oracle build")

    class _Tree(ctypes.Structure):
        _fields_ = [("nodes", ctypes.c_void_p), ("nnodes", ctypes.c_int32),
                    ("indices", ctypes.c_void_p), ("nindices", ctypes.c_int32),
                    ("tris", ctypes.c_void_p), ("ntris", ctypes.c_int32),
                    ("bounds", ctypes.c_float * 6)]

    verts = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 9)
    ids = None if ids is None else np.ascontiguousarray(ids, dtype=np.int32)
    flags = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint8)
    t = _Tree()
    rc = L.orc_kd_build(_p(verts), _p(ids), _p(flags), verts.shape[0], ctypes.byref(t))
    if rc != 0:
        raise RuntimeError(f"orc_kd_build failed: {rc}")
    try:
        def arr(ptr, count, dtype):
            nbytes = count * np.dtype(dtype).itemsize
            buf = (ctypes.c_char * nbytes).from_address(ptr) if count else b""
            return np.frombuffer(bytes(buf), dtype=dtype).copy()
        tree = {
            "nodes": arr(t.nodes, t.nnodes, NODE_DTYPE),
            "indices": arr(t.indices, t.nindices, np.int32),
            "tris": arr(t.tris, t.ntris, TRI_DTYPE),
            "bounds": np.array(list(t.bounds), dtype=np.float32),
        }
    finally:
        L.orc_kd_free(ctypes.byref(t))
    return tree


def fp64_classify(verts: np.ndarray, rays: np.ndarray, rel_margin: float = 1e-6,
                  threads: int | None = None) -> np.ndarray:
    """1 blocked, 0 clear, 2 within the margin of a boundary."""
    verts = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 9)
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 7)
    out = np.empty(rays.shape[0], dtype=np.int8)
    rc = lib().orc_fp64_classify(_p(verts), verts.shape[0], _p(rays), rays.shape[0],
                                 rel_margin, _p(out),
                                 threads if threads is not None else default_threads())
    if rc != 0:
        raise RuntimeError(f"orc_fp64_classify failed: {rc}")
    return out


def bsp_trace(geom, rays: np.ndarray, min_frac: float = 0.0, threads: int | None = None):
    """The reference's BSP surface tracer (bsp_oracle.cpp) over a
    hl2sdk_tools_sharp_b200.bsp.TraceGeometry: (face per ray, -1 for none;
    fraction along the ray's delta, 1 for none)."""
    L = lib()
    if not getattr(L, "_bsp_typed", False):
        P = ctypes.c_void_p
        L.orc_bsp_trace.argtypes = [P, P, P, P, P, P, ctypes.c_int32, P, P, P, P, ctypes.c_int64, ctypes.c_float,
                                    P, P, ctypes.c_int32]
        L.orc_bsp_trace.restype = ctypes.c_int
        L._bsp_typed = True
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 7)
    keep = [np.ascontiguousarray(a) for a in (geom.nodes, geom.surfaces, geom.node_faces, geom.leaf_faces,
                                               geom.leaf_start, geom.leaf_count, geom.sky_points, geom.sky_start,
                                               geom.sky_count)]
    face = np.empty(len(rays), np.int32)
    frac = np.empty(len(rays), np.float32)
    rc = L.orc_bsp_trace(_p(keep[0]), _p(keep[1]), _p(keep[2]), _p(keep[3]), _p(keep[4]), _p(keep[5]),
                         len(geom.leaf_start), _p(keep[6]), _p(keep[7]), _p(keep[8]), _p(rays), len(rays), min_frac,
                         _p(face), _p(frac), threads if threads is not None else default_threads())
    if rc != 0:
        raise RuntimeError("orc_bsp_trace: the walk outgrew its stack")
    return face, frac


def ambient_cubes(geom, faces: np.ndarray, light: np.ndarray, dirs: np.ndarray, tan_theta: float, sky,
                  positions: np.ndarray, threads: int | None = None) -> np.ndarray:
    """AmbientSampler.ComputeRayCube restated (bsp_oracle.cpp) at each
    position: (n, 6, 3) float32.  faces is the product's 88-byte face record
    array; sky the sky ambient (3 floats) or None."""
    L = lib()
    if not getattr(L, "_ambient_typed", False):
        P, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
        L.orc_ambient_cubes.argtypes = [P, P, P, P, P, P, i32, P, P, P, P, P, i64, P, f32, i32, P, P, i64, P, i32]
        L.orc_ambient_cubes.restype = ctypes.c_int
        L._ambient_typed = True
    keep = [np.ascontiguousarray(a) for a in (geom.nodes, geom.surfaces, geom.node_faces, geom.leaf_faces,
                                               geom.leaf_start, geom.leaf_count, geom.sky_points, geom.sky_start,
                                               geom.sky_count)]
    faces = np.ascontiguousarray(faces)
    assert faces.dtype.itemsize == 88
    light = np.ascontiguousarray(light, np.uint8)
    dirs = np.ascontiguousarray(dirs, np.float32)
    pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    skyv = np.zeros(3, np.float32) if sky is None else np.asarray(sky, np.float32)
    out = np.zeros((len(pos), 6, 3), np.float32)
    rc = L.orc_ambient_cubes(_p(keep[0]), _p(keep[1]), _p(keep[2]), _p(keep[3]), _p(keep[4]), _p(keep[5]),
                             len(geom.leaf_start), _p(keep[6]), _p(keep[7]), _p(keep[8]), _p(faces),
                             _p(light) if len(light) else None, len(light), _p(dirs), tan_theta,
                             int(sky is not None), _p(skyv), _p(pos), len(pos), _p(out),
                             threads if threads is not None else default_threads())
    if rc != 0:
        raise RuntimeError(f"orc_ambient_cubes failed: {rc}")
    return out


class Ran1:
    """Stock's uniform random stream (MapTools/Rad/Ambient/StockRandomStream.cs:
    13-234): Park-Miller minimal standard draws through a 32-entry
    Bays-Durham shuffle; RandomFloat = (float)(AM * draw), capped at
    RNMX, scaled into [lo, hi] in float."""
    NTAB, IA, IM, IQ, IR = 32, 16807, 2147483647, 127773, 2836
    NDIV = 1 + (IM - 1) // NTAB
    AM = 1.0 / IM
    RNMX = 1.0 - 1.2e-7

    def __init__(self, seed: int = 0):
        self.idum = seed if seed < 0 else -seed
        self.iy = 0
        self.iv = [0] * self.NTAB

    def _step(self):
        k = int(self.idum / self.IQ)          # C# int division truncates toward zero
        self.idum = self.IA * (self.idum - k * self.IQ) - self.IR * k
        if self.idum < 0:
            self.idum += self.IM

    def draw(self) -> int:
        if self.idum <= 0 or self.iy == 0:
            self.idum = 1 if -self.idum < 1 else -self.idum
            for j in range(self.NTAB + 7, -1, -1):
                self._step()
                if j < self.NTAB:
                    self.iv[j] = self.idum
            self.iy = self.iv[0]
        self._step()
        slot = self.iy // self.NDIV
        self.iy = self.iv[slot]
        self.iv[slot] = self.idum
        return self.iy

    def uniform(self, lo=0.0, hi=1.0) -> np.float32:
        fl = np.float32(self.AM * self.draw())
        if float(fl) > self.RNMX:
            fl = np.float32(self.RNMX)
        lo, hi = np.float32(lo), np.float32(hi)
        return np.float32(np.float32(fl * np.float32(hi - lo)) + lo)


def leaf_positions(planes, nodes, leaves, leaf_brushes, brushes, brush_sides):
    """Every leaf's candidate ambient sample positions, restated in Python
    (MapTools/Rad/Ambient: LeafAmbientBuilder.CandidateSampleCount :420-454
    with stock's all-axes-by-x quirk, BspParents :31-96,
    LeafBoundaryPlanes.Gather :32-70, LeafBrushTrace :43-265,
    LeafSampler.Generate :38-148); the arrays are the product's
    vrad_ambient_tree layout.  Returns (counts, (n, 3) float32)."""
    f32 = np.float32

    def dot(a, b):
        return f32(f32(f32(a[0] * b[0]) + f32(a[1] * b[1])) + f32(a[2] * b[2]))

    node_parent = [0] * len(nodes)
    leaf_parent = [0] * len(leaves)
    if len(nodes):
        node_parent[0] = -1
        stack = [0]
        while stack:
            n = stack.pop()
            for ch in (int(nodes[n][1]), int(nodes[n][2])):
                if ch < 0:
                    leaf_parent[-ch - 1] = n
                else:
                    node_parent[ch] = n
                    stack.append(ch)

    def clip(brush, p1, p2):
        first, count = int(brushes[brush][0]), int(brushes[brush][1])
        if count == 0:
            return f32(1), None, False
        enter, leave, clip_plane, start_out = f32(-9999.0), f32(1.0), -1, False
        for i in range(count):
            pnum, bevel = int(brush_sides[first + i][0]), int(brush_sides[first + i][1])
            if bevel == 1:
                continue
            nrm, dist = planes[pnum][:3], planes[pnum][3]
            d1 = f32(dot(p1, nrm) - dist)
            d2 = f32(dot(p2, nrm) - dist)
            if d1 > 0 and d2 > 0:
                return f32(1), None, False
            if d1 > 0:
                start_out = True
            if d1 <= 0 and d2 <= 0:
                continue
            if d1 > d2:
                f = f32((float(d1) - 0.03125) / float(f32(d1 - d2)))
                if f > enter:
                    enter, clip_plane = f, pnum
            else:
                f = f32((float(d1) + 0.03125) / float(f32(d1 - d2)))
                if f < leave:
                    leave = f
        if not start_out:
            return f32(1), None, True
        if enter < leave and enter > f32(-9999.0) and enter < f32(1.0):
            return max(enter, f32(0)), planes[clip_plane][:3], False
        return f32(1), None, False

    def brush_trace(leaf, start, end):
        L = leaves[leaf]
        for i in range(int(L[8])):
            b = int(leaf_brushes[int(L[7]) + i])
            if (int(brushes[b][2]) & (0x1 | 0x4000 | 0x80)) == 0:
                continue
            frac, nrm, solid = clip(b, start, end)
            if frac != 1 or solid:
                return (f32(0) if solid else frac), nrm, solid
        return f32(1), None, False

    counts = np.zeros(len(leaves), np.int32)
    out = []
    for l, L in enumerate(leaves):
        if int(L[0]) & 1:
            continue
        x = max((int(L[4]) - int(L[1])) // 32 if int(L[4]) >= int(L[1]) else -((int(L[1]) - int(L[4])) // 32), 1)
        v = (x * x * x) & 0xFFFFFFFF
        v = v - (1 << 32) if v >= 1 << 31 else v
        counts[l] = min(max(v, 1), 128)
        bound_planes = []
        node, child = leaf_parent[l], -(l + 1)
        while node >= 0:
            p = planes[int(nodes[node][0])]
            if int(nodes[node][1]) == child:
                bound_planes.append((p[:3].astype(f32), f32(p[3])))
            else:
                bound_planes.append(((-p[:3]).astype(f32), f32(-p[3])))
            child, node = node, node_parent[node]
        mn = [f32(L[1]), f32(L[2]), f32(L[3])]
        mx = [f32(L[4]), f32(L[5]), f32(L[6])]
        ext = [f32(int(L[4]) - int(L[1])), f32(int(L[5]) - int(L[2])), f32(int(L[6]) - int(L[3]))]
        rng = Ran1()
        for _ in range(int(counts[l])):
            pos, valid = None, False
            for _try in range(1000):
                a, b, c = rng.uniform(0, ext[0]), rng.uniform(0, ext[1]), rng.uniform(0, ext[2])
                pos = [f32(mn[0] + a), f32(mn[1] + b), f32(mn[2] + c)]
                valid = all(f32(dot(n, pos) - d) >= f32(0.03125) for n, d in bound_planes)
                if not valid:
                    continue
                for j in range(6):
                    axis = j % 3
                    end = list(pos)
                    end[axis] = mn[axis] if j < 3 else mx[axis]
                    t, nrm, _solid = brush_trace(l, pos, end)
                    if t == 0:
                        valid = False
                        break
                    if t != 1:
                        delta = [f32(end[k] - pos[k]) for k in range(3)]
                        if dot(delta, nrm) > 0:
                            valid = False
                            break
                if valid:
                    break
            if not valid:
                pos = [f32(f32(mn[k] + mx[k]) * f32(0.5)) for k in range(3)]
            out.append(pos)
    return counts, np.array(out, np.float32).reshape(-1, 3)


def bits_to_bool(bits: np.ndarray, n: int) -> np.ndarray:
    """Unpack LSB-first u64 words into n booleans."""
    b = np.ascontiguousarray(bits, dtype="<u8").view(np.uint8)
    return np.unpackbits(b, bitorder="little")[:n].astype(bool)


def build_samples(faces: np.ndarray, verts: np.ndarray):
    """FaceSampleBuilder restated: (samples as a 56-byte record array viewed
    through the caller's dtype, face_first)."""
    faces = np.ascontiguousarray(faces)
    verts = np.ascontiguousarray(verts, np.float32)
    count = ctypes.c_int64()
    rc = lib().orc_build_samples(_p(faces), len(faces), _p(verts), None, 0, ctypes.byref(count), None)
    if rc != 0:
        raise RuntimeError(f"orc_build_samples failed: {rc}")
    out = np.zeros(count.value * 56, np.uint8)
    first = np.zeros(len(faces) + 1, np.int64)
    rc = lib().orc_build_samples(_p(faces), len(faces), _p(verts), _p(out), count.value,
                                 ctypes.byref(count), _p(first))
    if rc != 0:
        raise RuntimeError(f"orc_build_samples failed: {rc}")
    return out, first


def direct(tree: dict, faces, samples, face_first, lights, cl_off, cl_list, dirs,
           jitter=None, sun_samples: int = 1, sun_extent: float = 0.0,
           threads: int | None = None, count_rays: bool = False, verts=None, extra_passes: int = 4,
           stats: dict | None = None):
    """The direct gather restated; (nsamples, 4) float32: lighting xyz, sun
    (and the number of segments traced, with count_rays).  With verts, up to
    extra_passes supersampling passes follow (the reference's default is 4);
    without verts, none."""
    nodes = np.ascontiguousarray(tree["nodes"], dtype=NODE_DTYPE)
    idx = np.ascontiguousarray(tree["indices"], dtype=np.int32)
    tris = np.ascontiguousarray(tree["tris"], dtype=TRI_DTYPE)
    bounds = np.ascontiguousarray(tree["bounds"], dtype=np.float32)
    faces = np.ascontiguousarray(faces)
    samples = np.ascontiguousarray(samples)
    face_first = np.ascontiguousarray(face_first, np.int64)
    lights = np.ascontiguousarray(lights)
    cl_off = np.ascontiguousarray(cl_off, np.int32)
    cl_list = np.ascontiguousarray(cl_list, np.int32)
    dirs = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
    jit = np.ascontiguousarray(jitter if jitter is not None and len(jitter) else np.zeros((1, 3)), np.float32)
    vv = None if verts is None else np.ascontiguousarray(verts, np.float32)
    n = int(face_first[-1])
    out = np.zeros((n, 4), np.float32)
    rays = ctypes.c_int64()
    ss = ctypes.c_int64()
    rc = lib().orc_direct(_p(nodes), _p(idx), _p(tris), _p(bounds), _p(faces), len(faces), _p(vv), _p(samples),
                          _p(face_first), _p(lights), _p(cl_off), _p(cl_list), _p(dirs), len(dirs),
                          _p(jit), sun_samples, sun_extent, extra_passes if vv is not None else 0, _p(out),
                          threads if threads is not None else default_threads(), ctypes.byref(rays),
                          ctypes.byref(ss))
    if rc != 0:
        raise RuntimeError(f"orc_direct failed: {rc}")
    if stats is not None:
        stats["rays"] = rays.value
        stats["supersampled"] = ss.value
    return (out, rays.value) if count_rays else out


def direct_styles(tree, faces, samples, face_first, lights, cl_off, cl_list, dirs, jitter=None, sun_samples: int = 1,
                  sun_extent: float = 0.0, threads: int | None = None, verts=None, extra_passes: int = 4):
    """The direct gather with light styles (FaceLightJob's slots): (slot 0
    (nsamples, 4), slots 1..3 (3, nsamples, 4), face styles (nfaces, 4)
    uint8 with 255 for an empty slot, faces warned of a fifth style)."""
    nodes = np.ascontiguousarray(tree["nodes"], dtype=NODE_DTYPE)
    idx = np.ascontiguousarray(tree["indices"], dtype=np.int32)
    tris = np.ascontiguousarray(tree["tris"], dtype=TRI_DTYPE)
    bounds = np.ascontiguousarray(tree["bounds"], dtype=np.float32)
    faces = np.ascontiguousarray(faces)
    samples = np.ascontiguousarray(samples)
    face_first = np.ascontiguousarray(face_first, np.int64)
    lights = np.ascontiguousarray(lights)
    cl_off = np.ascontiguousarray(cl_off, np.int32)
    cl_list = np.ascontiguousarray(cl_list, np.int32)
    dirs = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
    jit = np.ascontiguousarray(jitter if jitter is not None and len(jitter) else np.zeros((1, 3)), np.float32)
    vv = None if verts is None else np.ascontiguousarray(verts, np.float32)
    n = int(face_first[-1])
    out = np.zeros((n, 4), np.float32)
    slots = np.zeros((3, n, 4), np.float32)
    styles = np.zeros((len(faces), 4), np.uint8)
    dropped, rays, ss = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    rc = lib().orc_direct_styles(_p(nodes), _p(idx), _p(tris), _p(bounds), _p(faces), len(faces), _p(vv),
                                 _p(samples), _p(face_first), _p(lights), _p(cl_off), _p(cl_list), _p(dirs), len(dirs),
                                 _p(jit), sun_samples, sun_extent, extra_passes if vv is not None else 0, _p(out),
                                 _p(slots), _p(styles), ctypes.byref(dropped),
                                 threads if threads is not None else default_threads(), ctypes.byref(rays),
                                 ctypes.byref(ss))
    if rc != 0:
        raise RuntimeError(f"orc_direct_styles failed: {rc}")
    return out, slots, styles, dropped.value


def final_styles(faces, verts, samples, face_first, sample_light, slots_light, face_styles):
    """FinalLightFace restated with light styles: (LIGHTING bytes, lightofs)."""
    faces = np.ascontiguousarray(faces)
    verts = np.ascontiguousarray(verts, np.float32)
    samples = np.ascontiguousarray(samples)
    face_first = np.ascontiguousarray(face_first, np.int64)
    light = np.ascontiguousarray(sample_light, np.float32).reshape(-1, 4)
    slots = np.ascontiguousarray(slots_light, np.float32).reshape(3, -1, 4)
    styles = np.ascontiguousarray(face_styles, np.uint8).reshape(-1, 4)
    total = ctypes.c_int64()
    ofs = np.zeros(len(faces), np.int32)
    args = (_p(faces), len(faces), _p(verts), _p(samples), _p(face_first), _p(light), _p(slots), _p(styles))
    lib().orc_final_styles(*args, None, 0, _p(ofs), ctypes.byref(total))
    out = np.zeros(total.value, np.uint8)
    rc = lib().orc_final_styles(*args, _p(out), len(out), _p(ofs), ctypes.byref(total))
    if rc != 0:
        raise RuntimeError(f"orc_final_styles failed: {rc}")
    return out, ofs


def neighbours(faces, verts, threshold: float = 0.7071067):
    faces = np.ascontiguousarray(faces)
    verts = np.ascontiguousarray(verts, np.float32)
    off = np.zeros(len(faces) + 1, np.int32)
    count = ctypes.c_int64()
    lib().orc_neighbours(_p(faces), len(faces), _p(verts), threshold, _p(off), None, 0, ctypes.byref(count))
    lst = np.zeros(max(1, count.value), np.int32)
    lib().orc_neighbours(_p(faces), len(faces), _p(verts), threshold, _p(off), _p(lst), count.value,
                         ctypes.byref(count))
    return off, lst[:count.value]


def final(faces, verts, samples, face_first, sample_light):
    """FinalLightFace restated: (LIGHTING bytes, lightofs)."""
    faces = np.ascontiguousarray(faces)
    verts = np.ascontiguousarray(verts, np.float32)
    samples = np.ascontiguousarray(samples)
    face_first = np.ascontiguousarray(face_first, np.int64)
    light = np.ascontiguousarray(sample_light, np.float32).reshape(-1, 4)
    total = ctypes.c_int64()
    ofs = np.zeros(len(faces), np.int32)
    lib().orc_final(_p(faces), len(faces), _p(verts), _p(samples), _p(face_first), _p(light), None, 0,
                    _p(ofs), ctypes.byref(total))
    out = np.zeros(total.value, np.uint8)
    rc = lib().orc_final(_p(faces), len(faces), _p(verts), _p(samples), _p(face_first), _p(light), _p(out),
                         len(out), _p(ofs), ctypes.byref(total))
    if rc != 0:
        raise RuntimeError(f"orc_final failed: {rc}")
    return out, ofs


# Patch, 144 bytes (the library's vrad_patch layout).
PATCH_DTYPE = np.dtype([
    ("origin", "<f4", (3,)), ("area", "<f4"), ("normal", "<f4", (3,)), ("plane_dist", "<f4"),
    ("mins", "<f4", (3,)), ("chop", "<f4"), ("maxs", "<f4", (3,)), ("lux_scale", "<f4"),
    ("face_mins", "<f4", (3,)), ("face", "<i4"), ("face_maxs", "<f4", (3,)), ("cluster", "<i4"),
    ("reflectivity", "<f4", (3,)), ("sky", "<i4"), ("parent", "<i4"), ("child1", "<i4"),
    ("child2", "<i4"), ("first_point", "<i4"), ("num_points", "<i4"), ("pad", "<i4", (3,)),
])
assert PATCH_DTYPE.itemsize == 144


class _BounceIn(ctypes.Structure):
    _fields_ = [
        ("faces", ctypes.c_void_p), ("nfaces", ctypes.c_int32), ("verts", ctypes.c_void_p),
        ("samples", ctypes.c_void_p), ("face_first", ctypes.c_void_p), ("reflectivity", ctypes.c_void_p),
        ("pvs_off", ctypes.c_void_p), ("pvs_list", ctypes.c_void_p), ("nclusters", ctypes.c_int32),
        ("max_chop", ctypes.c_float), ("min_chop", ctypes.c_float), ("bounces", ctypes.c_int32),
        ("threshold", ctypes.c_float), ("nodes", ctypes.c_void_p), ("indices", ctypes.c_void_p),
        ("tris", ctypes.c_void_p), ("bounds6", ctypes.c_void_p), ("threads", ctypes.c_int32),
    ]


def _bounce_lib():
    L = lib()
    if not getattr(L, "_bounce_typed", False):
        P = ctypes.c_void_p
        i32, i64, f32 = ctypes.c_int32, ctypes.c_int64, ctypes.c_float
        L.orc_bounce_new.argtypes = [P]
        L.orc_bounce_new.restype = P
        L.orc_bounce_free.argtypes = [P]
        L.orc_bounce_free.restype = None
        L.orc_bounce_patches.argtypes = [P, P, i64, P, P, i64, P]
        L.orc_bounce_transfers.argtypes = [P, P, i32, P, P, P, i64, P, P]
        L.orc_bounce_set_transfers.argtypes = [P, P, P, P]
        L.orc_bounce_run.argtypes = [P, P, P, P, P, P]
        L.orc_bounce_final.argtypes = [P, P, P, i64, P, P]
        L.orc_bounce_final_styles.argtypes = [P, P, P, P, P, i64, P, P]
        L.orc_bounce_stats.argtypes = [P, P]
        L.orc_bounce_stats.restype = i64
        L.orc_bounce_forget_transfers.argtypes = [P]
        L.orc_bounce_forget_transfers.restype = None
        L.orc_bounce_count_candidates.argtypes = [P]
        L.orc_bounce_count_candidates.restype = i64
        L.orc_asin.argtypes = [f32]
        L.orc_asin.restype = f32
        L.orc_diff_to_diff.argtypes = [P]
        L.orc_diff_to_diff.restype = f32
        L.orc_poly_to_diff.argtypes = [P, i32, f32, P, P]
        L.orc_poly_to_diff.restype = f32
        L._bounce_typed = True
    return L


def powf(x: float, y: float) -> float:
    """DetMathF.Pow as the oracle computes it."""
    L = lib()
    L.orc_powf.argtypes = [ctypes.c_float, ctypes.c_float]
    L.orc_powf.restype = ctypes.c_float
    return L.orc_powf(float(x), float(y))


def asin(x: float) -> float:
    """DetMathF.Asin as the oracle computes it."""
    return _bounce_lib().orc_asin(float(x))


def diff_to_diff(o1, n1, o2, n2) -> np.float32:
    """FormFactors.DiffToDiff as the oracle computes it."""
    q = np.ascontiguousarray(np.concatenate([o1, n1, o2, n2]), np.float32)
    return np.float32(_bounce_lib().orc_diff_to_diff(_p(q)))


def poly_to_diff(points, area, origin, normal) -> np.float32:
    """FormFactors.PolyToDiff as the oracle computes it."""
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    o = np.ascontiguousarray(origin, np.float32)
    n = np.ascontiguousarray(normal, np.float32)
    return np.float32(_bounce_lib().orc_poly_to_diff(_p(pts), len(pts), float(area), _p(o), _p(n)))


class Bounce:
    """The bounce restated (patches, patch light, transfers, radiosity and
    the final pass with the bounced light) over one world."""

    def __init__(self, tree: dict, faces, verts, samples, face_first, reflectivity, pvs_off, pvs_list,
                 max_chop: float = 4.0, min_chop: float = 4.0, bounces: int = 100, threshold: float = 1.0,
                 threads: int | None = None):
        self._keep = dict(
            faces=np.ascontiguousarray(faces), verts=np.ascontiguousarray(verts, np.float32),
            samples=np.ascontiguousarray(samples), face_first=np.ascontiguousarray(face_first, np.int64),
            refl=np.ascontiguousarray(reflectivity, np.float32).reshape(-1, 3),
            pvs_off=np.ascontiguousarray(pvs_off, np.int32), pvs_list=np.ascontiguousarray(pvs_list, np.int32),
            nodes=np.ascontiguousarray(tree["nodes"], dtype=NODE_DTYPE),
            idx=np.ascontiguousarray(tree["indices"], dtype=np.int32),
            tris=np.ascontiguousarray(tree["tris"], dtype=TRI_DTYPE),
            bounds=np.ascontiguousarray(tree["bounds"], dtype=np.float32))
        k = self._keep
        self._in = _BounceIn(_p(k["faces"]), len(k["faces"]), _p(k["verts"]), _p(k["samples"]),
                             _p(k["face_first"]), _p(k["refl"]), _p(k["pvs_off"]), _p(k["pvs_list"]),
                             len(k["pvs_off"]) - 1, max_chop, min_chop, bounces, threshold, _p(k["nodes"]),
                             _p(k["idx"]), _p(k["tris"]), _p(k["bounds"]),
                             threads if threads is not None else default_threads())
        self._h = _bounce_lib().orc_bounce_new(ctypes.byref(self._in))
        self.npatches = len(self.patches()[0])

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _bounce_lib().orc_bounce_free(h)
            self._h = None

    def patches(self):
        """(patch records, winding points (n, 3))."""
        L = _bounce_lib()
        n, m = ctypes.c_int64(), ctypes.c_int64()
        L.orc_bounce_patches(self._h, None, 0, ctypes.byref(n), None, 0, ctypes.byref(m))
        out = np.zeros(n.value, PATCH_DTYPE)
        pts = np.zeros((max(1, m.value), 3), np.float32)
        L.orc_bounce_patches(self._h, _p(out), n.value, ctypes.byref(n), _p(pts), m.value, ctypes.byref(m))
        return out, pts[:m.value]

    def transfers(self, receivers=None):
        """VisMatrix for the receivers (patch indices; None = all): (offsets by
        patch, sources, weights, rays traced)."""
        L = _bounce_lib()
        recv = None if receivers is None else np.ascontiguousarray(receivers, np.int32)
        off = np.zeros(self.npatches + 1, np.int64)
        count, rays = ctypes.c_int64(), ctypes.c_int64()
        rc = L.orc_bounce_transfers(self._h, _p(recv), 0 if recv is None else len(recv), _p(off), None, None, 0,
                                    ctypes.byref(count), ctypes.byref(rays))
        if rc != 0:
            raise RuntimeError(f"orc_bounce_transfers failed: {rc}")
        src = np.zeros(max(1, count.value), np.int32)
        w = np.zeros(max(1, count.value), np.float32)
        # The lists are kept from the first call; this one only copies them.
        rc = L.orc_bounce_transfers(self._h, _p(recv), 0 if recv is None else len(recv), _p(off), _p(src), _p(w),
                                    count.value, ctypes.byref(count), None)
        if rc != 0:
            raise RuntimeError(f"orc_bounce_transfers failed: {rc}")
        return off, src[:count.value], w[:count.value], rays.value

    def forget_transfers(self) -> None:
        """Drop the built lists: the next transfers() call traces again."""
        _bounce_lib().orc_bounce_forget_transfers(self._h)

    def count_candidates(self) -> int:
        """Every receiver's candidate pairs (one full build's transfer rays)."""
        return int(_bounce_lib().orc_bounce_count_candidates(self._h))

    def set_transfers(self, offsets, src, weight):
        self._tr = (np.ascontiguousarray(offsets, np.int64), np.ascontiguousarray(src, np.int32),
                    np.ascontiguousarray(weight, np.float32))
        _bounce_lib().orc_bounce_set_transfers(self._h, *(_p(a) for a in self._tr))

    def run(self, sample_light):
        """(TotalLight (P, 3), DirectLight (P, 3), bounces run, last total)."""
        light = np.ascontiguousarray(sample_light, np.float32).reshape(-1, 4)
        total = np.zeros((self.npatches, 3), np.float32)
        direct = np.zeros((self.npatches, 3), np.float32)
        n = ctypes.c_int32()
        added = np.zeros(3, np.float32)
        rc = _bounce_lib().orc_bounce_run(self._h, _p(light), _p(total), _p(direct), ctypes.byref(n), _p(added))
        if rc != 0:
            raise RuntimeError(f"orc_bounce_run failed: {rc}")
        return total, direct, n.value, added

    def final(self, sample_light, slots_light=None, face_styles=None):
        """FinalLightFace with the last run's bounced light: (LIGHTING, lightofs).
        With light styles, slots 1..3 and the faces' style bytes as
        direct_styles returns them (the bounce goes into slot 0)."""
        L = _bounce_lib()
        light = np.ascontiguousarray(sample_light, np.float32).reshape(-1, 4)
        slots = None if slots_light is None else np.ascontiguousarray(slots_light, np.float32).reshape(3, -1, 4)
        styles = None if face_styles is None else np.ascontiguousarray(face_styles, np.uint8).reshape(-1, 4)
        total = ctypes.c_int64()
        nf = len(self._keep["faces"])
        ofs = np.zeros(nf, np.int32)
        L.orc_bounce_final_styles(self._h, _p(light), _p(slots), _p(styles), None, 0, _p(ofs), ctypes.byref(total))
        out = np.zeros(total.value, np.uint8)
        rc = L.orc_bounce_final_styles(self._h, _p(light), _p(slots), _p(styles), _p(out), len(out), _p(ofs),
                                       ctypes.byref(total))
        if rc != 0:
            raise RuntimeError(f"orc_bounce_final failed: {rc}")
        return out, ofs


# ---- Leaf ambient: the 16-sample list and the lumps (restated in Python) ----
#
# Follows MapTools/Rad/Ambient: AmbientSampleList.cs:40-222 (Add, Compress,
# ColorAtPosition, CubeDeltaGammaSpace), LeafAmbientBuilder.cs:503-670
# (Encode, NearestNeighborWithLight, AabbDistance, Fixed8Fraction),
# ToolBspTree.cs:20-90 (EnumerateLeavesInBox), StockLightColor.cs:110-150
# (Encode).  A sample is (position, cube): three float32 and 6 x 3 float32.

def _f32(x):
    return np.float32(x)


def _len(v):
    return _f32(np.sqrt(_f32(_f32(_f32(v[0] * v[0]) + _f32(v[1] * v[1])) + _f32(v[2] * v[2]))))


def _len_sq(v):
    return _f32(_f32(_f32(v[0] * v[0]) + _f32(v[1] * v[1])) + _f32(v[2] * v[2]))


def sample_list_add(samples: list, pos, cube, dead_tiebreak: bool = True) -> None:
    """AmbientSampleList.Add; samples is a list of (pos (3,), cube (6, 3))
    float32 arrays, changed in place."""
    samples.append((np.asarray(pos, np.float32), np.asarray(cube, np.float32).reshape(6, 3)))
    if len(samples) <= 16:
        return
    nearest, nearest_dist, nearest_total = 0, _f32(3.4028234663852886e38), _f32(0)
    for i, (pa, ca) in enumerate(samples):
        closest, total = _f32(3.4028234663852886e38), _f32(0)
        for j, (pb, cb) in enumerate(samples):
            if j == i:
                continue
            dist = _len((pa - pb).astype(np.float32))
            max_dc = _f32(0)
            for k in range(6):
                for c in range(3):
                    d = _f32(abs(_f32(ca[k, c] - cb[k, c])))
                    max_dc = max_dc if max_dc > d else d
                total = _f32(total + max_dc)
            if max_dc < _f32(1e-4):
                max_dc = _f32(0)
            elif max_dc > _f32(1):
                max_dc = _f32(1)
            dist = _f32(dist * _f32(_f32(0.1) + _f32(max_dc * _f32(0.9))))
            if dist < closest:
                closest = dist
        if closest < nearest_dist or (not dead_tiebreak and closest == nearest_dist and total < nearest_total):
            nearest_dist, nearest = closest, i
            if not dead_tiebreak:
                nearest_total = total
    samples[nearest] = samples[-1]
    samples.pop()


def color_at_position(samples: list, pos, skip: int) -> np.ndarray:
    """AmbientSampleList.ColorAtPosition: (6, 3) float32."""
    into = np.zeros((6, 3), np.float32)
    total = _f32(0)
    for i, (p, c) in enumerate(samples):
        if i == skip:
            continue
        factor = _f32(_f32(1) / _f32(_len_sq((p - np.asarray(pos, np.float32)).astype(np.float32)) + _f32(1)))
        total = _f32(total + factor)
        into = (into + (c * factor).astype(np.float32)).astype(np.float32)
    return (into * _f32(_f32(1) / total)).astype(np.float32)


def gamma_delta(a, b, table) -> int:
    """AmbientSampleList.CubeDeltaGammaSpace over the 1,024-entry table."""
    def g(f):
        i = int(np.trunc(np.float32(np.float32(f) * np.float32(1023)))) if np.isfinite(f) else 0
        return int(table[min(max(i, 0), 1023)])
    return max(abs(g(x) - g(y)) for x, y in zip(np.asarray(a).ravel(), np.asarray(b).ravel()))


def sample_list_compress(samples: list, table) -> None:
    """AmbientSampleList.Compress, in place."""
    i = 0
    while i < len(samples):
        if len(samples) > 1:
            test = color_at_position(samples, samples[i][0], i)
            if gamma_delta(test, samples[i][1], table) < 3:
                samples[i] = samples[-1]
                samples.pop()
                i -= 1
        i += 1


def encode_rgbe(v) -> bytes:
    """StockLightColor.Encode of one colour."""
    x, y, z = (np.float32(c) for c in v)
    mx = (x if x > z else z) if x > y else (y if y > z else z)
    e = 0 if mx == 0 else int((int(np.float32(mx).view(np.uint32)) & 0x7F800000) >> 23) - (7 + 127)
    sc = np.uint32(((127 - e) << 23) & 0xFFFFFFFF).view(np.float32)
    return bytes([int(np.float32(c * sc)) & 0xFF for c in (x, y, z)] + [e & 0xFF])


def fixed8(t, lo, hi) -> int:
    t, lo, hi = np.float32(t), np.float32(lo), np.float32(hi)
    if hi <= lo:
        return 0
    cv = np.float32(np.float32(t - lo) / np.float32(hi - lo))
    cv = np.float32(min(max(cv, np.float32(0)), np.float32(1)))
    return int(np.float32(np.float32(np.float32(0) + np.float32(np.float32(255) * cv)) + np.float32(0.5))) & 0xFF


def leaves_in_box(planes, nodes, mins, maxs) -> list:
    out, pending = [], [0]
    while pending:
        node = pending.pop()
        while node >= 0:
            p = planes[int(nodes[node][0])]
            cmin = [mins[i] if p[i] >= 0 else maxs[i] for i in range(3)]
            cmax = [maxs[i] if p[i] >= 0 else mins[i] for i in range(3)]
            dmax = _f32(_f32(_f32(p[0] * cmax[0]) + _f32(p[1] * cmax[1])) + _f32(p[2] * cmax[2]))
            dmin = _f32(_f32(_f32(p[0] * cmin[0]) + _f32(p[1] * cmin[1])) + _f32(p[2] * cmin[2]))
            if _f32(dmax - p[3]) <= _f32(-0.03125):
                node = int(nodes[node][2])
            elif _f32(dmin - p[3]) >= _f32(0.03125):
                node = int(nodes[node][1])
            else:
                pending.append(int(nodes[node][2]))
                node = int(nodes[node][1])
        out.append(-node - 1)
    return out


def leaf_ambient_lumps(planes, nodes, leaves, counts, positions, cubes, table, dead_tiebreak: bool = True):
    """The leaf ambient lumps from every leaf's samples: (index bytes,
    lighting bytes, bad leaves)."""
    first = np.concatenate([[0], np.cumsum(counts)])
    lists = []
    for l in range(len(leaves)):
        s = []
        for k in range(int(first[l]), int(first[l + 1])):
            sample_list_add(s, positions[k], cubes[k], dead_tiebreak)
        sample_list_compress(s, table)
        lists.append(s)
    count = [len(s) for s in lists]
    firstrec, lighting, at = [0] * len(leaves), bytearray(), 0
    for l, s in enumerate(lists):
        L = leaves[l]
        mn, mx = [np.float32(L[1 + a]) for a in range(3)], [np.float32(L[4 + a]) for a in range(3)]
        firstrec[l] = at if s else 0
        for p, c in s:
            lighting += b"".join(encode_rgbe(c[j]) for j in range(6))
            lighting += bytes([fixed8(p[a], mn[a], mx[a]) for a in range(3)] + [0])
            at += 1
    bad = 0
    for l in range(len(leaves)):
        if count[l]:
            continue
        L = leaves[l]
        if (int(L[0]) & 1) == 0:
            bad += 1
        mn = [np.float32(L[1 + a]) for a in range(3)]
        mx = [np.float32(L[4 + a]) for a in range(3)]
        size = [_f32(mx[a] - mn[a]) for a in range(3)]
        near = leaves_in_box(planes, nodes, [_f32(mn[a] - size[a]) for a in range(3)],
                             [_f32(mx[a] + size[a]) for a in range(3)])
        best, best_leaf = _f32(3.4028234663852886e38), l
        for o in near:
            if count[o] == 0:
                continue
            M = leaves[o]
            d = []
            for a in range(3):
                g = max(mn[a], np.float32(M[1 + a]))
                s_ = min(mx[a], np.float32(M[4 + a]))
                d.append(_f32(0) if g < s_ else _f32(s_ - g))
            dist = _len(np.array(d, np.float32))
            if dist < best:
                best, best_leaf = dist, o
        firstrec[l] = best_leaf
    index = b"".join(int(c).to_bytes(2, "little") + int(f & 0xFFFF).to_bytes(2, "little")
                     for c, f in zip(count, firstrec))
    return index, bytes(lighting), bad
