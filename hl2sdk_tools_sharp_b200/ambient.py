"""The leaf ambient sample over libvrad_cuda: candidate sample positions per
leaf (host) and their ray cubes (device).

Stock vrad's ComputePerLeafAmbientLighting (the reference's
MapTools/Rad/Ambient/LeafAmbientBuilder.cs:22-688) spends most of its time
in the 162 rays each candidate sample fires into the map
(AmbientSampler.ComputeRayCube, AmbientSampler.cs:211-227).  This module
builds the reference's AmbientScene inputs from a BSP's lumps
(AmbientScene.cs:40-318: the faces' lightmap records, the tinted style
averages, the sky ambient), draws each leaf's candidate positions
(LeafAmbientBuilder.PlanSamples, :252-276, through
vrad_leaf_ambient_positions) and computes their ray cubes on the device
(vrad_ambient_cubes).  The baked surface lights, the 16-sample list and the
lump encoding are not here, nor are displacements: a map with displacement
faces raises NotImplementedError, because stock clips every ray against
them.
"""
from __future__ import annotations

import ctypes
import dataclasses
import hashlib
import pathlib

import numpy as np

from . import bsp as B
from . import detmath as DM

LUMP_WORLDLIGHTS, LUMP_LEAFBRUSHES, LUMP_BRUSHES, LUMP_BRUSHSIDES = 15, 17, 18, 19
LUMP_DISPINFO, LUMP_LEAF_AMBIENT_INDEX_HDR, LUMP_LEAF_AMBIENT_INDEX = 26, 51, 52
LUMP_LIGHTING_HDR, LUMP_WORLDLIGHTS_HDR = 53, 54
LUMP_LEAF_AMBIENT_LIGHTING_HDR, LUMP_LEAF_AMBIENT_LIGHTING, LUMP_FACES_HDR = 55, 56, 58
AMBIENT_LUMPS = tuple(sorted(set(B.TRACE_LUMPS) | {B.LUMP_TEXDATA, B.LUMP_LIGHTING, LUMP_WORLDLIGHTS,
                                                   LUMP_LEAFBRUSHES, LUMP_BRUSHES, LUMP_BRUSHSIDES,
                                                   LUMP_DISPINFO, LUMP_LEAF_AMBIENT_INDEX_HDR,
                                                   LUMP_LEAF_AMBIENT_INDEX, LUMP_LIGHTING_HDR,
                                                   LUMP_WORLDLIGHTS_HDR, LUMP_LEAF_AMBIENT_LIGHTING_HDR,
                                                   LUMP_LEAF_AMBIENT_LIGHTING, LUMP_FACES_HDR}))

SIDES = 6
DIRECTIONS = 162
CONTENTS_SOLID = 0x1
SURF_BUMPLIGHT = 0x0800
EMIT_SKYAMBIENT = 5
VRAD_AMBIENT_SKY, VRAD_AMBIENT_BAD_AVERAGE = 1, 2

TEXDATA = np.dtype([("reflectivity", "<f4", (3,)), ("name", "<i4"), ("width", "<i4"), ("height", "<i4"),
                    ("view_width", "<i4"), ("view_height", "<i4")])
BRUSH = np.dtype([("firstside", "<i4"), ("numsides", "<i4"), ("contents", "<i4")])
BRUSHSIDE = np.dtype([("planenum", "<u2"), ("texinfo", "<i2"), ("dispinfo", "<i2"), ("bevel", "<i2")])
WORLDLIGHT = np.dtype([("origin", "<f4", (3,)), ("intensity", "<f4", (3,)), ("normal", "<f4", (3,)),
                       ("cluster", "<i4"), ("type", "<i4"), ("style", "<i4"), ("stopdot", "<f4"),
                       ("stopdot2", "<f4"), ("exponent", "<f4"), ("radius", "<f4"), ("constant_attn", "<f4"),
                       ("linear_attn", "<f4"), ("quadratic_attn", "<f4"), ("flags", "<i4"), ("texinfo", "<i4"),
                       ("owner", "<i4")])
LEAF_AMBIENT_INDEX = np.dtype([("count", "<u2"), ("first", "<u2")])
LEAF_AMBIENT_LIGHTING = np.dtype([("cube", "u1", (6, 4)), ("x", "u1"), ("y", "u1"), ("z", "u1"), ("pad", "u1")])
# vrad_ambient_face (include/vrad_cuda.h).
AMBIENT_FACE = np.dtype([("lightofs", "<i4"), ("smax", "<i4"), ("tmax", "<i4"), ("stride", "<i4"),
                         ("nstyles", "<i4"), ("styles", "<u4"), ("flags", "<i4"), ("reflectivity", "<f4", (3,)),
                         ("averages", "<f4", (4, 3))])
assert (TEXDATA.itemsize, BRUSH.itemsize, BRUSHSIDE.itemsize, WORLDLIGHT.itemsize) == (32, 12, 8, 88)
assert (LEAF_AMBIENT_LIGHTING.itemsize, AMBIENT_FACE.itemsize) == (28, 88)

# The 162 sample directions, stock's g_anorms in stock's order
# (make_anorms.py beside this file wrote them).
ANORMS_SHA256 = "db1cf609aca1c6ea814184177998a887768136e9f082406f11aeec61e08efe9c"


def anorms() -> np.ndarray:
    """(162, 3) float32: VertexNormals.Directions (VertexNormals.cs:37-228)."""
    raw = (pathlib.Path(__file__).resolve().parent / "anorms.bin").read_bytes()
    if hashlib.sha256(raw).hexdigest() != ANORMS_SHA256:
        raise RuntimeError("anorms.bin is not the 162-direction table this module was written against")
    return np.frombuffer(raw, "<f4").reshape(DIRECTIONS, 3).copy()


def cone_tan() -> np.float32:
    """tan of the cone's inner half-angle: DetMathF.Tan(7.275f x (MathF.PI /
    180f)), all float (AmbientSampler.cs:142, VertexNormals.cs:35)."""
    angle = np.float32(np.float32(7.275) * np.float32(np.float32(np.pi) / np.float32(180.0)))
    return DM.tan_f(angle)


def power2n() -> np.ndarray:
    """StockLightColor's decode table: (float)(2^(k - 128) / 255) in double,
    rounded once (StockLightColor.cs:262-271)."""
    return (np.ldexp(1.0, np.arange(256) - 128) / 255.0).astype(np.float32)


def decode(rgbe: np.ndarray) -> np.ndarray:
    """TexLightToLinear of (n, 4) RGBE bytes: (n, 3) float32."""
    rgbe = np.asarray(rgbe, np.uint8).reshape(-1, 4)
    e = power2n()[rgbe[:, 3].view(np.int8).astype(np.int64) + 128]
    return (rgbe[:, :3].astype(np.float32) * e[:, None]).astype(np.float32)


def load_lumps(path: str) -> dict:
    return B.lumps_of(path, AMBIENT_LUMPS)


@dataclasses.dataclass
class AmbientRange:
    """One lighting range's lookups (AmbientScene for LightingMode.Ldr or
    Hdr): the lighting lump, the face records, the sky ambient."""
    hdr: bool
    lighting: np.ndarray
    faces: np.ndarray
    sky_ambient: np.ndarray | None


def _faces_for(lumps: dict, hdr: bool) -> np.ndarray:
    # The HDR range reads the HDR face lump when the map has one (stock
    # copies the LDR faces into it otherwise): AmbientScene.cs:52-58.
    if hdr and len(lumps.get(LUMP_FACES_HDR, (0, b""))[1]):
        return np.frombuffer(lumps[LUMP_FACES_HDR][1], B.FACE)
    return np.frombuffer(lumps[B.LUMP_FACES][1], B.FACE)


def ambient_range(lumps: dict, hdr: bool) -> AmbientRange:
    """AmbientScene.BuildShades (AmbientScene.cs:247-300) for one range."""
    light = np.frombuffer(lumps[LUMP_LIGHTING_HDR if hdr else B.LUMP_LIGHTING][1], np.uint8)
    faces = _faces_for(lumps, hdr)
    texinfo = np.frombuffer(lumps[B.LUMP_TEXINFO][1], B.TEXINFO)
    texdata = np.frombuffer(lumps[B.LUMP_TEXDATA][1], TEXDATA)
    rec = np.zeros(len(faces), AMBIENT_FACE)
    for f, face in enumerate(faces):
        tex = texinfo[int(face["texinfo"])]
        flags = int(tex["flags"])
        r = rec[f]
        r["lightofs"] = int(face["lightofs"])
        r["smax"] = int(face["lm_size"][0]) + 1
        r["tmax"] = int(face["lm_size"][1]) + 1
        sky = bool(flags & B.SURF_SKY)
        bumped = bool(flags & SURF_BUMPLIGHT) and not (flags & B.SURF_NOLIGHT)
        r["stride"] = int(r["smax"]) * int(r["tmax"]) * (4 if bumped else 1)
        refl = texdata[int(tex["texdata"])]["reflectivity"].astype(np.float32)
        r["reflectivity"] = refl
        styles = [int(x) for x in face["styles"]]
        count = 0
        while count < 4 and styles[count] != 255:
            count += 1
        r["nstyles"] = count
        r["styles"] = styles[0] | styles[1] << 8 | styles[2] << 16 | styles[3] << 24
        fl = VRAD_AMBIENT_SKY if sky else 0
        if not sky:
            for m in range(count):
                ofs = int(face["lightofs"]) - (m + 1) * 4
                if ofs < 0 or ofs + 4 > len(light):
                    fl |= VRAD_AMBIENT_BAD_AVERAGE
                    continue
                c = decode(light[ofs:ofs + 4])[0]
                r["averages"][m] = (c * refl).astype(np.float32)
        r["flags"] = fl
    wl = np.frombuffer(lumps[LUMP_WORLDLIGHTS_HDR if hdr else LUMP_WORLDLIGHTS][1], WORLDLIGHT)
    sky_amb = next((w["intensity"].astype(np.float32) for w in wl if int(w["type"]) == EMIT_SKYAMBIENT), None)
    return AmbientRange(hdr, light.copy(), rec, sky_amb)


@dataclasses.dataclass
class AmbientTree:
    """vrad_ambient_tree's arrays (include/vrad_cuda.h)."""
    planes: np.ndarray        # (P, 4) float32
    nodes: np.ndarray         # (N, 3) int32
    leaves: np.ndarray        # (L, 9) int32
    leaf_brushes: np.ndarray  # int32
    brushes: np.ndarray       # (B, 3) int32
    brush_sides: np.ndarray   # (S, 2) int32


def ambient_tree(lumps: dict) -> AmbientTree:
    planes = np.frombuffer(lumps[B.LUMP_PLANES][1], B.PLANE)
    nodes = np.frombuffer(lumps[B.LUMP_NODES][1], B.NODE)
    ver, leaf_bytes = lumps[B.LUMP_LEAFS]
    leaves = np.frombuffer(leaf_bytes, B.LEAF_V0 if ver == 0 else B.LEAF_V1)
    brushes = np.frombuffer(lumps[LUMP_BRUSHES][1], BRUSH)
    sides = np.frombuffer(lumps[LUMP_BRUSHSIDES][1], BRUSHSIDE)
    P = np.zeros((len(planes), 4), np.float32)
    P[:, :3], P[:, 3] = planes["normal"], planes["dist"]
    N = np.zeros((len(nodes), 3), np.int32)
    N[:, 0], N[:, 1:] = nodes["planenum"], nodes["children"]
    L = np.zeros((len(leaves), 9), np.int32)
    L[:, 0] = leaves["contents"]
    L[:, 1:4], L[:, 4:7] = leaves["mins"], leaves["maxs"]
    L[:, 7], L[:, 8] = leaves["firstleafbrush"], leaves["numleafbrushes"]
    Bt = np.zeros((len(brushes), 3), np.int32)
    Bt[:, 0], Bt[:, 1], Bt[:, 2] = brushes["firstside"], brushes["numsides"], brushes["contents"]
    S = np.zeros((len(sides), 2), np.int32)
    S[:, 0], S[:, 1] = sides["planenum"], sides["bevel"]
    lb = np.frombuffer(lumps[LUMP_LEAFBRUSHES][1], "<u2").astype(np.int32)
    return AmbientTree(P, N, L, lb, Bt, S)


def has_displacements(lumps: dict) -> bool:
    return len(lumps.get(LUMP_DISPINFO, (0, b""))[1]) > 0


def _lib():
    from . import tracer as T
    lib = T.load_library()
    if not getattr(lib, "_ambient_bound", False):
        P, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64

        class Tree(ctypes.Structure):
            _fields_ = [("planes", P), ("nplanes", i32), ("nodes", P), ("nnodes", i32), ("leaves", P),
                        ("nleaves", i32), ("leaf_brushes", P), ("nleaf_brushes", i32), ("brushes", P),
                        ("nbrushes", i32), ("brush_sides", P), ("nbrush_sides", i32)]

        class Lighting(ctypes.Structure):
            _fields_ = [("lighting", P), ("lighting_bytes", i64), ("faces", P), ("nfaces", i32),
                        ("directions", P), ("ndirections", i32), ("tan_theta", ctypes.c_float),
                        ("has_sky_ambient", i32), ("sky_ambient", ctypes.c_float * 3)]
        lib._AmbientTree, lib._AmbientLighting = Tree, Lighting
        lib.vrad_leaf_ambient_positions.argtypes = [ctypes.POINTER(Tree), P, P, i64, ctypes.POINTER(i64), i32]
        lib.vrad_ambient_upload.argtypes = [P, ctypes.POINTER(Lighting)]
        lib.vrad_ambient_cubes.argtypes = [P, P, i64, P]
        lib.vrad_ambient_cubes_device.argtypes = [P, P, i64, P, P]
        lib.vrad_ambient_status.argtypes = [P]
        for n in ("vrad_leaf_ambient_positions", "vrad_ambient_upload", "vrad_ambient_cubes",
                  "vrad_ambient_cubes_device", "vrad_ambient_status"):
            getattr(lib, n).restype = i32
        lib._ambient_bound = True
    return lib


def candidate_positions(tree: AmbientTree, threads: int = 0):
    """(counts per leaf, (n, 3) float32 positions leaf after leaf): every
    leaf's candidate samples, LeafSampler.Generate over each leaf's own
    stream (vrad_leaf_ambient_positions)."""
    from . import tracer as T
    lib = _lib()
    keep = [np.ascontiguousarray(a) for a in (tree.planes, tree.nodes, tree.leaves, tree.leaf_brushes,
                                               tree.brushes, tree.brush_sides)]
    pl, nd, lv, lb, br, bs = keep
    ptr = lambda a: a.ctypes.data if a.size else None  # noqa: E731
    t = lib._AmbientTree(ptr(pl), len(pl), ptr(nd), len(nd), ptr(lv), len(lv), ptr(lb), len(lb), ptr(br), len(br),
                         ptr(bs), len(bs))
    counts = np.zeros(len(lv), np.int32)
    total = ctypes.c_int64()
    T._check(lib.vrad_leaf_ambient_positions(ctypes.byref(t), counts.ctypes.data, None, 0, ctypes.byref(total),
                                             threads), None)
    pos = np.zeros((total.value, 3), np.float32)
    if total.value:
        T._check(lib.vrad_leaf_ambient_positions(ctypes.byref(t), counts.ctypes.data, pos.ctypes.data, total.value,
                                                 ctypes.byref(total), threads), None)
    return counts, pos


class CudaAmbientSampler:
    """AmbientSampler.ComputeRayCube on one device: the map's BSP tree and
    one range's lighting resident; cubes(positions) -> (n, 6, 3) float32,
    sides +x, -x, +y, -y, +z, -z."""

    def __init__(self, lumps: dict, hdr: bool = False, device: int = 0):
        if has_displacements(lumps):
            raise NotImplementedError("leaf ambient on a map with displacements: stock clips every ray against "
                                      "them (DispCollisionSet), which this sampler does not")
        from . import tracer as T
        self._bsp = B.CudaBspTracer(B.trace_geometry(lumps), device=device)
        self._ctx = self._bsp._ctx
        self.range = ambient_range(lumps, hdr)
        lib = _lib()
        self._lib = lib
        r = self.range
        self._dirs = anorms()
        sky = r.sky_ambient if r.sky_ambient is not None else np.zeros(3, np.float32)
        desc = lib._AmbientLighting(r.lighting.ctypes.data if len(r.lighting) else None, len(r.lighting),
                                    r.faces.ctypes.data if len(r.faces) else None, len(r.faces),
                                    self._dirs.ctypes.data, DIRECTIONS, float(cone_tan()),
                                    int(r.sky_ambient is not None), (ctypes.c_float * 3)(*[float(x) for x in sky]))
        T._check(lib.vrad_ambient_upload(self._ctx, ctypes.byref(desc)), self._ctx)

    def cubes(self, positions) -> np.ndarray:
        from . import tracer as T
        p = np.ascontiguousarray(np.asarray(positions, np.float32).reshape(-1, 3))
        out = np.zeros((len(p), SIDES, 3), np.float32)
        if len(p):
            T._check(self._lib.vrad_ambient_cubes(self._ctx, p.ctypes.data, len(p), out.ctypes.data), self._ctx)
        return out

    def cubes_device(self, positions, out=None, stream=None):
        """Device form: positions (n, 3) float32 CUDA tensor; returns (n, 6, 3)."""
        import torch
        from . import tracer as T
        assert positions.dtype == torch.float32 and positions.is_contiguous()
        n = positions.shape[0]
        y = out if out is not None else torch.empty((n, SIDES, 3), dtype=torch.float32, device=positions.device)
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        T._check(self._lib.vrad_ambient_cubes_device(self._ctx, positions.data_ptr(), n, y.data_ptr(),
                                                     ctypes.c_void_p(s)), self._ctx)
        return y

    def status(self) -> None:
        from . import tracer as T
        T._check(self._lib.vrad_ambient_status(self._ctx), self._ctx)

    def close(self) -> None:
        if getattr(self, "_bsp", None) is not None:
            self._bsp.close()
            self._bsp = None
            self._ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def fixed8(t, lo, hi) -> int:
    """LeafAmbientBuilder.Fixed8Fraction (LeafAmbientBuilder.cs:660-670): a
    coordinate as a byte fraction of the leaf's extent."""
    t, lo, hi = np.float32(t), np.float32(lo), np.float32(hi)
    if hi <= lo:
        return 0
    cv = np.float32(np.float32(t - lo) / np.float32(hi - lo))
    cv = np.float32(min(max(cv, np.float32(0.0)), np.float32(1.0)))
    frac = np.float32(np.float32(0.0) + np.float32(np.float32(255.0) * cv))
    return int(np.float32(frac + np.float32(0.5)))


def gamma_table() -> np.ndarray:
    """StockLightColor's linear-to-screen table (StockLightColor.cs:186-250):
    1,024 ints, entry i = (int)(255 x DetMath.Pow(f, 1 / 2.2)) of the
    piecewise-remapped (float)(i / 1023)."""
    g = np.float32(1.0 / float(np.float32(2.2)))
    g3 = np.float32(0.125)
    out = np.zeros(1024, np.int32)
    for i in range(1024):
        f = np.float32(i / 1023.0)
        if f <= g3:
            f = np.float32(float(np.float32(f / g3)) * 0.125)
        else:
            f = np.float32(0.125 + ((float(np.float32(f - g3)) / (1.0 - float(g3))) * 0.875))
        v = int(255 * DM.pow_d(float(f), float(g)))
        out[i] = min(max(v, 0), 255)
    return out


def leaf_ambient_lumps(tree: AmbientTree, counts, positions, cubes, correct_tiebreak: bool = False):
    """vrad_leaf_ambient_lumps: every leaf's samples (counts and positions
    as candidate_positions gives them, cubes (n, 6, 3)) through the 16-sample
    list and its compression into (LEAF_AMBIENT_INDEX bytes,
    LEAF_AMBIENT_LIGHTING bytes, bad leaf count)."""
    from . import tracer as T
    lib = _lib()
    if not getattr(lib, "_lumps_bound", False):
        P, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
        lib.vrad_leaf_ambient_lumps.argtypes = [ctypes.POINTER(lib._AmbientTree), P, P, P, P, i32, P, P, i64,
                                                ctypes.POINTER(i64), ctypes.POINTER(i32)]
        lib.vrad_leaf_ambient_lumps.restype = i32
        lib._lumps_bound = True
    keep = [np.ascontiguousarray(a) for a in (tree.planes, tree.nodes, tree.leaves, tree.leaf_brushes,
                                               tree.brushes, tree.brush_sides)]
    pl, nd, lv, lb, br, bs = keep
    ptr = lambda a: a.ctypes.data if a is not None and a.size else None  # noqa: E731
    t = lib._AmbientTree(ptr(pl), len(pl), ptr(nd), len(nd), ptr(lv), len(lv), ptr(lb), len(lb), ptr(br), len(br),
                         ptr(bs), len(bs))
    c = np.ascontiguousarray(counts, np.int32)
    p = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    q = np.ascontiguousarray(cubes, np.float32).reshape(-1, 18)
    table = gamma_table()
    index = np.zeros(4 * len(lv), np.uint8)
    recs, bad = ctypes.c_int64(), ctypes.c_int32()
    T._check(lib.vrad_leaf_ambient_lumps(ctypes.byref(t), c.ctypes.data, ptr(p), ptr(q), table.ctypes.data,
                                         int(correct_tiebreak), index.ctypes.data, None, 0, ctypes.byref(recs),
                                         ctypes.byref(bad)), None)
    light = np.zeros(max(1, 28 * recs.value), np.uint8)
    T._check(lib.vrad_leaf_ambient_lumps(ctypes.byref(t), c.ctypes.data, ptr(p), ptr(q), table.ctypes.data,
                                         int(correct_tiebreak), index.ctypes.data, light.ctypes.data, recs.value,
                                         ctypes.byref(recs), ctypes.byref(bad)), None)
    return index.tobytes(), light[:28 * recs.value].tobytes(), int(bad.value)
