"""Reading Source BSP files (versions 19 and 20) for the lighting tracer.

The layouts follow the public BSP format that the reference reads in
MapFormats/Bsp (BspFile, BspLump ids in BspLump.cs, the structs in
Bsp/Structs: DPlane, DNode, DFace, TexInfo, DLeaf / DLeafVersion0, DEdge):
a 1036-byte header of 64 lump records (offset, length, version, fourCC),
each lump an array of little-endian records.  Only uncompressed lumps are
read (a lump stored LZMA-compressed raises).

`lumps_of(path)` returns the raw bytes and versions of the lumps the BSP
surface tracer needs; `trace_geometry(lumps)` flattens them into the arrays
that tracer walks, as the reference's BspTraceGeometry.Build does
(MapTools/Tracing/BspTraceGeometry.cs:291-899).
"""
from __future__ import annotations

import dataclasses
import struct

import numpy as np

# Lump ids (MapFormats/Bsp/BspLump.cs).
LUMP_ENTITIES, LUMP_PLANES, LUMP_TEXDATA, LUMP_VERTEXES = 0, 1, 2, 3
LUMP_NODES, LUMP_TEXINFO, LUMP_FACES, LUMP_LIGHTING = 5, 6, 7, 8
LUMP_LEAFS, LUMP_EDGES, LUMP_SURFEDGES, LUMP_LEAFFACES = 10, 12, 13, 16
TRACE_LUMPS = (LUMP_PLANES, LUMP_VERTEXES, LUMP_NODES, LUMP_TEXINFO, LUMP_FACES, LUMP_LEAFS, LUMP_EDGES,
               LUMP_SURFEDGES, LUMP_LEAFFACES)

SURF_SKY = 0x0004
SURF_NOLIGHT = 0x0400

PLANE = np.dtype([("normal", "<f4", (3,)), ("dist", "<f4"), ("type", "<i4")])
NODE = np.dtype([("planenum", "<i4"), ("children", "<i4", (2,)), ("mins", "<i2", (3,)), ("maxs", "<i2", (3,)),
                 ("firstface", "<u2"), ("numfaces", "<u2"), ("area", "<i2"), ("pad", "<i2")])
FACE = np.dtype([("planenum", "<u2"), ("side", "u1"), ("on_node", "u1"), ("firstedge", "<i4"),
                 ("numedges", "<i2"), ("texinfo", "<i2"), ("dispinfo", "<i2"), ("fog", "<i2"),
                 ("styles", "u1", (4,)), ("lightofs", "<i4"), ("area", "<f4"), ("lm_mins", "<i4", (2,)),
                 ("lm_size", "<i4", (2,)), ("orig_face", "<i4"), ("num_prims", "<u2"), ("first_prim", "<u2"),
                 ("smoothing", "<u4")])
TEXINFO = np.dtype([("texture_vecs", "<f4", (2, 4)), ("lightmap_vecs", "<f4", (2, 4)), ("flags", "<i4"),
                    ("texdata", "<i4")])
LEAF_V0 = np.dtype([("contents", "<i4"), ("cluster", "<i2"), ("area_flags", "<i2"), ("mins", "<i2", (3,)),
                    ("maxs", "<i2", (3,)), ("firstleafface", "<u2"), ("numleaffaces", "<u2"),
                    ("firstleafbrush", "<u2"), ("numleafbrushes", "<u2"), ("water", "<i2"),
                    ("ambient", "u1", (24,)), ("pad", "<i2")])
LEAF_V1 = np.dtype([("contents", "<i4"), ("cluster", "<i2"), ("area_flags", "<i2"), ("mins", "<i2", (3,)),
                    ("maxs", "<i2", (3,)), ("firstleafface", "<u2"), ("numleaffaces", "<u2"),
                    ("firstleafbrush", "<u2"), ("numleafbrushes", "<u2"), ("water", "<i2"), ("pad", "<i2")])
EDGE = np.dtype([("v", "<u2", (2,))])
assert (PLANE.itemsize, NODE.itemsize, FACE.itemsize, TEXINFO.itemsize) == (20, 32, 56, 72)
assert (LEAF_V0.itemsize, LEAF_V1.itemsize, EDGE.itemsize) == (56, 32, 4)


def lumps_of(path: str, ids=TRACE_LUMPS) -> dict:
    """{lump id: (version, bytes)} of a BSP file (versions 19 and 20)."""
    with open(path, "rb") as f:
        head = f.read(1036)
        ident, version = struct.unpack_from("<4si", head, 0)
        if ident != b"VBSP" or version not in (19, 20):
            raise ValueError(f"{path}: not a version 19/20 BSP ({ident!r} {version})")
        out = {}
        for i in ids:
            ofs, length, ver, fourcc = struct.unpack_from("<iii4s", head, 8 + 16 * i)
            if fourcc != b"\0\0\0\0":
                raise ValueError(f"{path}: lump {i} is compressed")
            f.seek(ofs)
            out[i] = (ver, f.read(length))
    return out


@dataclasses.dataclass
class TraceGeometry:
    """BspTraceGeometry's flattened arrays.

    nodes      (N, 8) float32 words: plane normal xyz, dist, child0, child1
               (int bits), first node face (int bits), packed (int bits:
               solid count | sky count << 15 | axis << 30, axis 3 = not axial)
    surfaces   (F, 16) float32: plane normal xyz, dist, lightmap s (xyz,
               offset), t (xyz, offset), mins s, t, sizes s, t (-1 for a
               face with no lightmap)
    node_faces candidate faces of each node (its lit faces, then its sky faces)
    leaf_faces candidate faces of each leaf; leaf_start, leaf_count per leaf
    sky_points the sky faces' windings with colinear points removed;
               sky_start, sky_count per face
    sky        per face: the face is a sky face
    """
    nodes: np.ndarray
    surfaces: np.ndarray
    node_faces: np.ndarray
    leaf_faces: np.ndarray
    leaf_start: np.ndarray
    leaf_count: np.ndarray
    sky_points: np.ndarray
    sky_start: np.ndarray
    sky_count: np.ndarray
    sky: np.ndarray
    skipped_displacements: int


def _normalise(v):
    """Vec3.Normalise: float length sqrt((x*x + y*y) + z*z), three divides."""
    v = np.asarray(v, np.float32)
    sq = np.float32(np.float32(v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])
    ln = np.float32(np.sqrt(sq))
    if ln == 0:
        return np.zeros(3, np.float32)
    return np.array([v[0] / ln, v[1] / ln, v[2] / ln], np.float32)


def trace_geometry(lumps: dict) -> TraceGeometry:
    """BspTraceGeometry.Build (Correct mode) over the lumps lumps_of read."""
    planes = np.frombuffer(lumps[LUMP_PLANES][1], PLANE)
    nodes = np.frombuffer(lumps[LUMP_NODES][1], NODE)
    faces = np.frombuffer(lumps[LUMP_FACES][1], FACE)
    texinfo = np.frombuffer(lumps[LUMP_TEXINFO][1], TEXINFO)
    leafface = np.frombuffer(lumps[LUMP_LEAFFACES][1], "<u2")
    ver, leaf_bytes = lumps[LUMP_LEAFS]
    leaves = np.frombuffer(leaf_bytes, LEAF_V0 if ver == 0 else LEAF_V1)
    verts = np.frombuffer(lumps[LUMP_VERTEXES][1], "<f4").reshape(-1, 3)
    edges = np.frombuffer(lumps[LUMP_EDGES][1], EDGE)
    surfedges = np.frombuffer(lumps[LUMP_SURFEDGES][1], "<i4")
    F = len(faces)

    ti = faces["texinfo"].astype(np.int64)
    valid = (ti >= 0) & (ti < len(texinfo))
    flags = np.where(valid, texinfo["flags"][np.clip(ti, 0, len(texinfo) - 1)], SURF_NOLIGHT).astype(np.int32)
    if (faces["planenum"] >= len(planes)).any():
        raise ValueError("a face names a plane the map does not have")

    # Surfaces (BuildSurfaces).
    surf = np.zeros((F, 16), np.float32)
    pl = planes[faces["planenum"]]
    surf[:, 0:3] = pl["normal"]
    surf[:, 3] = pl["dist"]
    lit = valid & ((flags & SURF_NOLIGHT) == 0)
    tx = texinfo[np.clip(ti, 0, len(texinfo) - 1)]
    surf[lit, 4:8] = tx["lightmap_vecs"][lit, 0]
    surf[lit, 8:12] = tx["lightmap_vecs"][lit, 1]
    surf[lit, 12:14] = faces["lm_mins"][lit]
    surf[lit, 14:16] = faces["lm_size"][lit]
    surf[~lit, 14:16] = -1.0

    # Nodes (BuildNodes): each node's on-node faces, lit first then sky.
    N = len(nodes)
    if ((nodes["planenum"] < 0) | (nodes["planenum"] >= len(planes))).any():
        raise ValueError("a node names a plane the map does not have")
    words = np.zeros((N, 8), np.float32)
    npl = planes[nodes["planenum"]]
    words[:, 0:3] = npl["normal"]
    words[:, 3] = npl["dist"]
    iw = words.view(np.int32)
    iw[:, 4] = nodes["children"][:, 0]
    iw[:, 5] = nodes["children"][:, 1]
    node_faces = []
    for n in range(N):
        solid, sky = [], []
        for f in range(int(nodes["firstface"][n]), int(nodes["firstface"][n]) + int(nodes["numfaces"][n])):
            if f >= F:
                raise ValueError(f"node {n} names face {f}")
            if faces["on_node"][f] == 0 or faces["dispinfo"][f] != -1:
                continue
            (sky if flags[f] & SURF_SKY else solid).append(f)
        iw[n, 6] = len(node_faces)
        node_faces.extend(solid)
        node_faces.extend(sky)
        nx, ny, nz = (float(x) for x in npl["normal"][n])
        ax = 3
        if (nx, ny, nz) == (1.0, 0.0, 0.0):
            ax = 0
        elif (nx, ny, nz) == (0.0, 1.0, 0.0):
            ax = 1
        elif (nx, ny, nz) == (0.0, 0.0, 1.0):
            ax = 2
        if len(solid) > 0x7FFF or len(sky) > 0x7FFF:
            raise ValueError(f"node {n} has too many candidate faces")
        iw[n, 7] = np.int32(np.uint32(len(solid) | (len(sky) << 15) | (ax << 30)).view(np.int32))

    # Leaves (BuildLeaves): each leaf's faces that are neither on a node nor
    # displacements, in leaf-face order.
    L = len(leaves)
    leaf_start = np.zeros(L, np.int32)
    leaf_count = np.zeros(L, np.int32)
    leaf_faces = []
    for l in range(L):
        leaf_start[l] = len(leaf_faces)
        for slot in range(int(leaves["firstleafface"][l]), int(leaves["firstleafface"][l]) + int(leaves["numleaffaces"][l])):
            if slot >= len(leafface):
                raise ValueError(f"leaf {l} names leafface {slot}")
            f = int(leafface[slot])
            if f >= F:
                raise ValueError(f"leaf {l} names face {f}")
            if faces["dispinfo"][f] != -1 or faces["on_node"][f] != 0:
                continue
            leaf_faces.append(f)
        leaf_count[l] = len(leaf_faces) - leaf_start[l]

    # Sky windings (BuildSkyWindings, WindingFromFace then
    # RemoveColinearPoints, Correct normalise).
    sky = (flags & SURF_SKY) != 0
    sky_start = np.zeros(F, np.int32)
    sky_count = np.zeros(F, np.int32)
    pts = []
    for f in np.flatnonzero(sky & (faces["dispinfo"] == -1)):
        raw = []
        for i in range(int(faces["numedges"][f])):
            se = int(surfedges[int(faces["firstedge"][f]) + i])
            v = int(edges["v"][-se][1]) if se < 0 else int(edges["v"][se][0])
            raw.append(verts[v].astype(np.float32))
        sky_start[f] = len(pts)
        m = len(raw)
        for i in range(m):
            j, k = (i + 1) % m, (i + m - 1) % m
            v1 = _normalise(raw[j] - raw[i])
            v2 = _normalise(raw[i] - raw[k])
            d = np.float32(np.float32(v1[0] * v2[0] + v1[1] * v2[1]) + v1[2] * v2[2])
            if d < np.float32(0.999):
                pts.append(raw[i])
        sky_count[f] = len(pts) - sky_start[f]
    return TraceGeometry(words, surf, np.array(node_faces, np.int32), np.array(leaf_faces, np.int32), leaf_start,
                         leaf_count, np.array(pts, np.float32).reshape(-1, 3), sky_start, sky_count, sky,
                         int((faces["dispinfo"] != -1).sum()))


def _bsp_lib():
    import ctypes
    from . import tracer as T
    lib = T.load_library()
    if not getattr(lib, "_bsp_bound", False):
        P, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64

        class Desc(ctypes.Structure):
            _fields_ = [("nodes", P), ("nnodes", i32), ("surfaces", P), ("nsurfaces", i32), ("node_faces", P),
                        ("nnode_faces", i32), ("leaf_faces", P), ("nleaf_faces", i32), ("leaf_start", P),
                        ("leaf_count", P), ("nleaves", i32), ("sky_points", P), ("nsky_points", i32),
                        ("sky_start", P), ("sky_count", P)]
        lib._BspDesc = Desc
        lib.vrad_bsp_upload.argtypes = [P, ctypes.POINTER(Desc)]
        lib.vrad_bsp_upload.restype = i32
        lib.vrad_bsp_trace_closest.argtypes = [P, P, i64, ctypes.POINTER(T._Options), P]
        lib.vrad_bsp_trace_closest.restype = i32
        lib.vrad_bsp_trace_closest_device.argtypes = [P, P, i64, ctypes.c_float, P, P]
        lib.vrad_bsp_trace_closest_device.restype = i32
        lib._bsp_bound = True
    return lib


class CudaBspTracer:
    """The BSP surface walk over libvrad_cuda on one device: BspSurfaceTracer
    (MapTools/Tracing/BspSurfaceTracer.cs) with the map's tree resident."""

    def __init__(self, geom: TraceGeometry, device: int = 0):
        import ctypes
        from . import tracer as T
        lib = _bsp_lib()
        self._lib = lib
        ctx = ctypes.c_void_p()
        rc = lib.vrad_create(device, ctypes.byref(ctx))
        if rc != 0:
            raise T.VradError(rc, T._message(None))
        self._ctx = ctx
        keep = [np.ascontiguousarray(a) for a in (geom.nodes, geom.surfaces, geom.node_faces, geom.leaf_faces,
                                                   geom.leaf_start, geom.leaf_count, geom.sky_points,
                                                   geom.sky_start, geom.sky_count)]
        nd, sf, nf, lf, ls, lc, sp, ss, sc = keep
        d = lib._BspDesc(nd.ctypes.data, len(nd), sf.ctypes.data, len(sf), nf.ctypes.data, len(nf),
                         lf.ctypes.data, len(lf), ls.ctypes.data, lc.ctypes.data, len(ls),
                         sp.ctypes.data if len(sp) else None, len(sp), ss.ctypes.data, sc.ctypes.data)
        T._check(lib.vrad_bsp_upload(ctx, ctypes.byref(d)), ctx)

    def trace_closest(self, rays, min_distance: float = 0.0) -> np.ndarray:
        """Per ray (RAY_DTYPE or (n, 7) floats) the face hit (-1: none) and
        the fraction along direction x reach (1: none), as HIT_DTYPE."""
        import ctypes
        from . import tracer as T
        r = np.ascontiguousarray(np.asarray(rays, np.float32).reshape(-1, 7) if not (
            isinstance(rays, np.ndarray) and rays.dtype == T.RAY_DTYPE) else rays)
        hits = np.zeros(len(r), T.HIT_DTYPE)
        o = T.RayTraceOptions(min_distance)._c()
        T._check(self._lib.vrad_bsp_trace_closest(self._ctx, r.ctypes.data, len(r), ctypes.byref(o),
                                                 hits.ctypes.data), self._ctx)
        return hits

    def close(self) -> None:
        if getattr(self, "_ctx", None):
            self._lib.vrad_destroy(self._ctx)
            self._ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
