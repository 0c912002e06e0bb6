"""Host side of vrad's lighting stage over libvrad_cuda.

Builds what the reference's RadWorld set-up builds before any ray is traced
(muflub/hl2sdk_tools_sharp, src/SourceSharp.MapTools/Rad/Light), from a
room-grid World:

  faces      vrad_face records (plane, texinfo lightmap vectors, lightmap
             extents, winding, cluster); the inputs of FaceLightInfo.Build
  samples    vrad_build_samples (native): FaceSampleBuilder.CalcPoints
  lights     the DirectLight list in gather order (DirectLightBuilder.Build,
             DirectLightBuilder.cs:43-505): ParseIntensity's gamma and
             brightness (MapFormats/Text/RadLightFile.cs:344-410), literal
             attenuation and its normalisation (LightFalloff.cs:40-90), spot
             cones as cosines, the light_environment's sun and its ambient
             partner; the active list is built by prepending, so it holds the
             entities in reverse order
  clusters   per cluster, the lights whose PVS reaches it, in list order
             (DirectLightGatherer's per-cluster lists)

and runs the fused direct gather on the device (vrad_direct_lighting).
"""
from __future__ import annotations

import ctypes
import dataclasses
import math

import numpy as np

from . import lights as LT, roomgrid as rg, tracer as T
from .roomgrid import World
from .workload import ambient_directions

FACE_DTYPE = np.dtype([
    ("normal", "<f4", (3,)), ("dist", "<f4"), ("lightmap_vecs", "<f4", (2, 4)),
    ("lightmap_mins", "<i4", (2,)), ("lightmap_size", "<i4", (2,)), ("first_vertex", "<i4"),
    ("num_vertices", "<i4"), ("cluster", "<i4"), ("flags", "<i4"),
])
SAMPLE_DTYPE = np.dtype([
    ("position", "<f4", (3,)), ("area", "<f4"), ("coord", "<f4", (2,)), ("mins", "<f4", (2,)),
    ("maxs", "<f4", (2,)), ("s", "<i4"), ("t", "<i4"), ("face", "<i4"), ("cluster", "<i4"),
])
LIGHT_DTYPE = np.dtype([
    ("type", "<i4"), ("style", "<i4"), ("origin", "<f4", (3,)), ("intensity", "<f4", (3,)),
    ("normal", "<f4", (3,)), ("stop_dot", "<f4"), ("stop_dot2", "<f4"), ("exponent", "<f4"),
    ("constant_attn", "<f4"), ("linear_attn", "<f4"), ("quadratic_attn", "<f4"),
    ("start_fade_distance", "<f4"), ("end_fade_distance", "<f4"), ("cap_dist", "<f4"),
])
LIGHTING_DTYPE = np.dtype([("lighting", "<f4", (3,)), ("direct_sun_amount", "<f4")])
PATCH_DTYPE = np.dtype([
    ("origin", "<f4", (3,)), ("area", "<f4"), ("normal", "<f4", (3,)), ("plane_dist", "<f4"),
    ("mins", "<f4", (3,)), ("chop", "<f4"), ("maxs", "<f4", (3,)), ("lux_scale", "<f4"),
    ("face_mins", "<f4", (3,)), ("face", "<i4"), ("face_maxs", "<f4", (3,)), ("cluster", "<i4"),
    ("reflectivity", "<f4", (3,)), ("sky", "<i4"), ("parent", "<i4"), ("child1", "<i4"),
    ("child2", "<i4"), ("first_point", "<i4"), ("num_points", "<i4"), ("pad", "<i4", (3,)),
])
TRANSFER_DTYPE = np.dtype([("patch", "<i4"), ("weight", "<f4")])
assert FACE_DTYPE.itemsize == 80 and SAMPLE_DTYPE.itemsize == 56 and LIGHT_DTYPE.itemsize == 80
assert PATCH_DTYPE.itemsize == 144 and TRANSFER_DTYPE.itemsize == 8

EMIT_POINT, EMIT_SPOT, EMIT_SKY, EMIT_AMBIENT = 1, 2, 3, 4
SURF_LIGHT, FACE_EMITS = 0x0001, 0x40000000     # VRAD_SURF_LIGHT, VRAD_FACE_EMITS
EQUAL_EPSILON = np.float32(0.001)


class _WorldDesc(ctypes.Structure):
    _fields_ = [("faces", ctypes.c_void_p), ("nfaces", ctypes.c_int32),
                ("samples", ctypes.c_void_p), ("nsamples", ctypes.c_int64),
                ("lights", ctypes.c_void_p), ("nlights", ctypes.c_int32),
                ("cluster_light_offsets", ctypes.c_void_p), ("cluster_lights", ctypes.c_void_p),
                ("nclusters", ctypes.c_int32), ("sky_directions", ctypes.c_void_p),
                ("nsky_directions", ctypes.c_int32), ("sun_jitter", ctypes.c_void_p),
                ("nsun_jitter", ctypes.c_int32), ("sun_angular_extent", ctypes.c_float),
                ("sun_samples", ctypes.c_int32), ("vertices", ctypes.c_void_p), ("nvertices", ctypes.c_int64),
                ("lights_hdr", ctypes.c_void_p)]


class PassStats(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_int64), ("luxels", ctypes.c_int64), ("visibility_rays", ctypes.c_int64),
                ("sky_rays", ctypes.c_int64), ("lighting_bytes", ctypes.c_int64), ("direct_ms", ctypes.c_float),
                ("final_ms", ctypes.c_float), ("extra_passes_run", ctypes.c_int32), ("supersampled", ctypes.c_int64),
                ("supersample_ms", ctypes.c_float)]


class _BounceDesc(ctypes.Structure):
    _fields_ = [("reflectivity", ctypes.c_void_p), ("pvs_offsets", ctypes.c_void_p),
                ("pvs_clusters", ctypes.c_void_p), ("nclusters", ctypes.c_int32), ("max_chop", ctypes.c_float),
                ("min_chop", ctypes.c_float), ("bounces", ctypes.c_int32), ("threshold", ctypes.c_float)]


class BounceStats(ctypes.Structure):
    _fields_ = [("patches", ctypes.c_int64), ("receivers", ctypes.c_int64), ("transfer_rays", ctypes.c_int64),
                ("blocked", ctypes.c_int64), ("transfers", ctypes.c_int64), ("bounces", ctypes.c_int32),
                ("exact_totals", ctypes.c_int32), ("added", ctypes.c_double * 3),
                ("patch_light_ms", ctypes.c_float), ("transfer_ms", ctypes.c_float),
                ("bounce_ms", ctypes.c_float), ("final_ms", ctypes.c_float), ("unsettled_asin", ctypes.c_int64),
                ("transfers_cached", ctypes.c_int32)]


class DirectStats(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_int64), ("visibility_rays", ctypes.c_int64),
                ("sky_rays", ctypes.c_int64), ("kernel_ms", ctypes.c_float), ("extra_passes_run", ctypes.c_int32),
                ("supersampled", ctypes.c_int64)]


def _lib():
    lib = T.load_library()
    if not getattr(lib, "_lighting_bound", False):
        P, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
        lib.vrad_build_samples.argtypes = [P, i32, P, i64, P, i64, ctypes.POINTER(i64), P]
        lib.vrad_build_samples.restype = i32
        lib.vrad_world_upload.argtypes = [P, ctypes.POINTER(_WorldDesc)]
        lib.vrad_world_upload.restype = i32
        lib.vrad_direct_lighting.argtypes = [P, P, ctypes.POINTER(DirectStats)]
        lib.vrad_direct_lighting.restype = i32
        lib.vrad_direct_lighting_device.argtypes = [P, P, P]
        lib.vrad_direct_lighting_device.restype = i32
        lib.vrad_direct_autotune.argtypes = [P, ctypes.POINTER(i32), P]
        lib.vrad_direct_autotune.restype = i32
        lib.vrad_build_neighbours.argtypes = [P, i32, P, i64, ctypes.c_float, P, P, i64, ctypes.POINTER(i64)]
        lib.vrad_build_neighbours.restype = i32
        lib.vrad_lightmap_layout.argtypes = [P, i32, P, ctypes.POINTER(i64)]
        lib.vrad_lightmap_layout.restype = i32
        lib.vrad_lighting_size.argtypes = [P, ctypes.POINTER(i64)]
        lib.vrad_lighting_size.restype = i32
        lib.vrad_lightmap_layout_styles.argtypes = [P, i32, P, P, ctypes.POINTER(i64)]
        lib.vrad_lightmap_layout_styles.restype = i32
        lib.vrad_face_styles.argtypes = [P, P, i32, ctypes.POINTER(i64)]
        lib.vrad_face_styles.restype = i32
        lib.vrad_light_pass.argtypes = [P, P, i64, P, ctypes.POINTER(PassStats)]
        lib.vrad_light_pass.restype = i32
        lib.vrad_light_pass_device.argtypes = [P, P, P]
        lib.vrad_light_pass_device.restype = i32
        lib.vrad_light_pass_ranges.argtypes = [P, i32, P, i64, P, i64, P, ctypes.POINTER(PassStats),
                                               ctypes.POINTER(BounceStats)]
        lib.vrad_light_pass_ranges.restype = i32
        lib.vrad_light_pass_ranges_device.argtypes = [P, i32, P, P, P]
        lib.vrad_light_pass_ranges_device.restype = i32
        lib.vrad_pass_sample_light.argtypes = [P, i32, P, i64]
        lib.vrad_pass_sample_light.restype = i32
        lib.vrad_bounce_stats_ranges.argtypes = [P, ctypes.POINTER(BounceStats)]
        lib.vrad_bounce_stats_ranges.restype = i32
        lib.vrad_set_extra_passes.argtypes = [P, i32]
        lib.vrad_set_extra_passes.restype = i32
        lib.vrad_build_patches.argtypes = [P, i32, P, i64, P, ctypes.c_float, ctypes.c_float, P, i64,
                                           ctypes.POINTER(i64), P, i64, ctypes.POINTER(i64)]
        lib.vrad_build_patches.restype = i32
        lib.vrad_bounce_upload.argtypes = [P, ctypes.POINTER(_BounceDesc)]
        lib.vrad_bounce_upload.restype = i32
        lib.vrad_bounce_stats_get.argtypes = [P, ctypes.POINTER(BounceStats)]
        lib.vrad_bounce_stats_get.restype = i32
        lib.vrad_bounce_patch_light.argtypes = [P, P, P, i64]
        lib.vrad_bounce_patch_light.restype = i32
        lib.vrad_bounce_set_model.argtypes = [P, P]
        lib.vrad_bounce_set_model.restype = i32
        lib.vrad_bounce_features_device.argtypes = [P, P, P, i64, ctypes.POINTER(i64), P]
        lib.vrad_bounce_features_device.restype = i32
        lib.vrad_bounce_last_total.argtypes = [P, P]
        lib.vrad_bounce_last_total.restype = i32
        lib.vrad_bounce_transfers.argtypes = [P, P, i64, P, i64, ctypes.POINTER(i64)]
        lib.vrad_bounce_transfers.restype = i32
        lib.vrad_form_factor_diff.argtypes = [P, P, i64, P]
        lib.vrad_form_factor_diff.restype = i32
        lib.vrad_form_factor_poly.argtypes = [P, P, P, P, i64, P]
        lib.vrad_form_factor_poly.restype = i32
        lib._lighting_bound = True
    return lib


# ---------------------------------------------------------------- faces

def faces_of(world: World):
    """vrad_face records and the shared vertex array."""
    nf = world.face_count
    faces = np.zeros(nf, FACE_DTYPE)
    counts = np.array([len(v) for v in world.face_verts], np.int32)
    first = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int32)
    faces["normal"] = world.face_normal
    faces["dist"] = world.face_dist
    faces["lightmap_vecs"][:, 0] = world.face_s
    faces["lightmap_vecs"][:, 1] = world.face_t
    faces["lightmap_mins"] = world.face_mins
    faces["lightmap_size"] = world.face_extents
    faces["first_vertex"] = first
    faces["num_vertices"] = counts
    faces["cluster"] = world.face_cluster
    if world.face_emit is not None:
        # An emitting texture: SURF_LIGHT (PatchBuilder.MakePatchForFace)
        # and the library's emitting-face bit.
        emits = world.face_emit[:, 3] > 0
        faces["flags"][emits] |= SURF_LIGHT | FACE_EMITS
    verts = np.concatenate(world.face_verts).astype(np.float32)
    return faces, verts


def build_samples(faces: np.ndarray, verts: np.ndarray, out: np.ndarray | None = None):
    """FaceSampleBuilder.CalcPoints for every face (native); returns the
    samples and face_first (index of each face's first sample).  A face has
    at most one sample per lightmap cell, so one call into a buffer of that
    many records builds them all; `out` (SAMPLE_DTYPE, at least that long)
    lets a caller reuse one buffer across maps."""
    lib = _lib()
    faces = np.ascontiguousarray(faces, FACE_DTYPE)
    verts = np.ascontiguousarray(verts, np.float32)
    cap = int((faces["lightmap_size"][:, 0].astype(np.int64) * faces["lightmap_size"][:, 1]).sum())
    if out is None or len(out) < cap:
        out = np.empty(max(1, cap), SAMPLE_DTYPE)
    count = ctypes.c_int64()
    first = np.zeros(len(faces) + 1, np.int64)
    rc = lib.vrad_build_samples(faces.ctypes.data, len(faces), verts.ctypes.data, len(verts),
                                out.ctypes.data, len(out), ctypes.byref(count), first.ctypes.data)
    if rc != 0:
        raise ValueError(f"vrad_build_samples failed ({rc})")
    return out[:count.value], first


def build_patches(faces: np.ndarray, verts: np.ndarray, reflectivity: np.ndarray, max_chop: float = 4.0,
                  min_chop: float = 4.0):
    """PatchBuilder + PatchSubdivider (native): the patch records in the
    reference's index order and the winding points (n, 3)."""
    lib = _lib()
    faces = np.ascontiguousarray(faces, FACE_DTYPE)
    verts = np.ascontiguousarray(verts, np.float32)
    refl = np.ascontiguousarray(reflectivity, np.float32).reshape(-1, 3)
    n, m = ctypes.c_int64(), ctypes.c_int64()
    rc = lib.vrad_build_patches(faces.ctypes.data, len(faces), verts.ctypes.data, len(verts), refl.ctypes.data,
                                max_chop, min_chop, None, 0, ctypes.byref(n), None, 0, ctypes.byref(m))
    if rc != 0:
        raise ValueError(f"vrad_build_patches failed ({rc})")
    out = np.zeros(n.value, PATCH_DTYPE)
    pts = np.zeros((max(1, m.value), 3), np.float32)
    rc = lib.vrad_build_patches(faces.ctypes.data, len(faces), verts.ctypes.data, len(verts), refl.ctypes.data,
                                max_chop, min_chop, out.ctypes.data, len(out), ctypes.byref(n), pts.ctypes.data,
                                m.value, ctypes.byref(m))
    if rc != 0:
        raise ValueError(f"vrad_build_patches failed ({rc})")
    return out, pts[:m.value]


def face_reflectivity(world: World) -> np.ndarray:
    """Each lit face's material reflectivity (F, 3)."""
    return np.ascontiguousarray(world.reflectivity[world.face_material], np.float32)


def form_factors_diff(ctx_owner, cases) -> np.ndarray:
    """vrad_form_factor_diff on the device of ctx_owner (a tracer or a
    stage): cases (n, 12) = o1, n1, o2, n2."""
    c = np.ascontiguousarray(cases, np.float32).reshape(-1, 12)
    out = np.zeros(len(c), np.float32)
    T._check(_lib().vrad_form_factor_diff(ctx_owner._ctx, c.ctypes.data, len(c), out.ctypes.data), ctx_owner._ctx)
    return out


def form_factors_poly(ctx_owner, windings, cases) -> np.ndarray:
    """vrad_form_factor_poly: windings a list of (k, 3) point arrays, cases
    (n, 7) = area, receiving point, normal."""
    pts = np.ascontiguousarray(np.concatenate([np.asarray(w, np.float32).reshape(-1, 3) for w in windings]))
    first = np.zeros(len(windings) + 1, np.int32)
    first[1:] = np.cumsum([len(w) for w in windings])
    c = np.ascontiguousarray(cases, np.float32).reshape(-1, 7)
    out = np.zeros(len(c), np.float32)
    T._check(_lib().vrad_form_factor_poly(ctx_owner._ctx, pts.ctypes.data, first.ctypes.data, c.ctypes.data, len(c),
                                          out.ctypes.data), ctx_owner._ctx)
    return out


def pvs_lists(world: World):
    """The PVS as CSR: per cluster, the clusters its row sets, ascending."""
    C = world.pvs.shape[0]
    rows = [np.flatnonzero(world.pvs[c]).astype(np.int32) for c in range(C)]
    off = np.zeros(C + 1, np.int32)
    off[1:] = np.cumsum([len(r) for r in rows])
    return off, (np.concatenate(rows) if rows else np.zeros(0, np.int32)).astype(np.int32)


def build_neighbours(faces: np.ndarray, verts: np.ndarray, threshold: float = 0.7071067):
    """vrad_build_neighbours (native): CSR offsets and lists."""
    lib = _lib()
    faces = np.ascontiguousarray(faces, FACE_DTYPE)
    verts = np.ascontiguousarray(verts, np.float32)
    off = np.zeros(len(faces) + 1, np.int32)
    count = ctypes.c_int64()
    rc = lib.vrad_build_neighbours(faces.ctypes.data, len(faces), verts.ctypes.data, len(verts), threshold,
                                   off.ctypes.data, None, 0, ctypes.byref(count))
    if rc != 0:
        raise ValueError(f"vrad_build_neighbours failed ({rc})")
    lst = np.zeros(max(1, count.value), np.int32)
    rc = lib.vrad_build_neighbours(faces.ctypes.data, len(faces), verts.ctypes.data, len(verts), threshold,
                                   off.ctypes.data, lst.ctypes.data, count.value, ctypes.byref(count))
    if rc != 0:
        raise ValueError(f"vrad_build_neighbours failed ({rc})")
    return off, lst[:count.value]


def lightmap_layout(faces: np.ndarray, styles: np.ndarray | None = None):
    """vrad_lightmap_layout: (lightofs per face, LIGHTING size); with styles
    ((nfaces, 4) style bytes, 255 an empty slot), vrad_lightmap_layout_styles."""
    faces = np.ascontiguousarray(faces, FACE_DTYPE)
    ofs = np.zeros(len(faces), np.int32)
    total = ctypes.c_int64()
    if styles is None:
        rc = _lib().vrad_lightmap_layout(faces.ctypes.data, len(faces), ofs.ctypes.data, ctypes.byref(total))
    else:
        st = np.ascontiguousarray(styles, np.uint8).reshape(len(faces), 4)
        rc = _lib().vrad_lightmap_layout_styles(faces.ctypes.data, len(faces), st.ctypes.data, ofs.ctypes.data,
                                                ctypes.byref(total))
    if rc != 0:
        raise ValueError(f"vrad_lightmap_layout failed ({rc})")
    return ofs, total.value


# ---------------------------------------------------------------- lights

def parse_intensity(color, light_scale: float = 1.0, hdr: bool = False) -> np.ndarray:
    """RadLightFile.ParseIntensity of a "_light" value given as its fields
    (r g b brightness): gamma 2.2 by DetMath.Pow in double, narrowed to
    float, times (float)(brightness / 255) (lights.parse_intensity)."""
    text = " ".join(repr(float(c)) for c in color)
    return LT.parse_intensity(text, hdr=hdr, light_scale=light_scale)[0]


def surface_patches(world: World, hdr: bool = False, max_chop: float = 4.0, min_chop: float = 4.0):
    """The patch set's part that AddSurfaceLights reads, for a map with
    texlights (None without): the patches at the bounce's chop sizes
    (vrad_build_patches) and each face's emission, parsed from its
    texlight value as the lights file's are (ParseIntensity, HDR keys for
    the HDR range)."""
    if world.face_emit is None or not (world.face_emit[:, 3] > 0).any():
        return None
    faces, verts = faces_of(world)
    patches, _ = build_patches(faces, verts, face_reflectivity(world), max_chop, min_chop)
    base = np.zeros((world.face_count, 3), np.float32)
    for f in np.flatnonzero(world.face_emit[:, 3] > 0):
        base[f] = parse_intensity(world.face_emit[f], hdr=hdr)
    F = world.face_count
    return LT.SurfacePatches(origin=patches["origin"], normal=patches["normal"], area=patches["area"],
                             face=patches["face"], leaf=patches["child1"] == -1, base_light=base,
                             base_area=np.full(F, world.texel_area, np.float32),
                             scale=np.tile(np.array(world.texel_scale, np.float32), (F, 1)))


def light_set(world: World, hdr: bool = False, max_chop: float = 4.0, min_chop: float = 4.0) -> LT.DirectLightSet:
    """The map's lights through the restated DirectLightBuilder: its
    texlights' surface lights (from the patches at the bounce's chop sizes),
    then its light entities."""
    return LT.build(rg.entities(world), lambda o: rg.cluster_of_point(world, o), hdr=hdr,
                    surface=surface_patches(world, hdr, max_chop, min_chop))


def build_lights(world: World, hdr: bool = False, max_chop: float = 4.0, min_chop: float = 4.0):
    """The active DirectLight list and the per-cluster light lists, for the
    LDR pass or (hdr) the HDR pass: the map's light entities
    (roomgrid.entities) through the restated DirectLightBuilder
    (lights.build).  Returns (lights, cluster_offsets, cluster_lights)."""
    ls = light_set(world, hdr, max_chop, min_chop)
    if ls.unsupported_class_names:
        raise ValueError(f"unsupported light entities: {ls.unsupported_class_names}")
    lights = LT.to_records(ls.active, LIGHT_DTYPE)
    home = [l.cluster if l.type not in (EMIT_SKY, EMIT_AMBIENT) else -1 for l in ls.active]
    C = world.pvs.shape[0]
    lists = []
    for c in range(C):
        # Sun and ambient reach every cluster that sees sky: every room here.
        lists.append([k for k, h in enumerate(home) if h < 0 or world.pvs[h, c]])
    offsets = np.zeros(C + 1, np.int32)
    offsets[1:] = np.cumsum([len(x) for x in lists])
    flat = np.array([k for x in lists for k in x], np.int32)
    return lights, offsets, flat


# ---------------------------------------------------------------- stage

@dataclasses.dataclass
class LightingInputs:
    faces: np.ndarray
    verts: np.ndarray
    samples: np.ndarray
    face_first: np.ndarray
    lights: np.ndarray
    cluster_offsets: np.ndarray
    cluster_lights: np.ndarray
    sky_directions: np.ndarray
    sun_jitter: np.ndarray
    sun_samples: int = 1
    sun_angular_extent: float = 0.0
    lights_hdr: np.ndarray | None = None    # the HDR range's list (intensities differ), or none


RANGE_LDR, RANGE_HDR = 1, 2      # VRAD_RANGE_*


def prepare(world: World, hdr: bool = False, sample_out: np.ndarray | None = None, max_chop: float = 4.0,
            min_chop: float = 4.0) -> LightingInputs:
    """The lighting stage's inputs; with hdr, also the HDR range's light
    list.  sample_out: a caller's buffer for the samples (build_samples).
    A map with texlights takes its surface lights from the patch tree at
    max_chop / min_chop: the chop sizes its bounce is uploaded with."""
    faces, verts = faces_of(world)
    samples, first = build_samples(faces, verts, out=sample_out)
    lights, off, flat = build_lights(world, max_chop=max_chop, min_chop=min_chop)
    inp = LightingInputs(faces, verts, samples, first, lights, off, flat,
                         ambient_directions().astype(np.float32), np.zeros((0, 3), np.float32))
    extent = LT.build(rg.entities(world)).sun_angular_extent   # the light_environment's alone
    if extent > 0:
        # A sun with a spread: the configured count of jittered rays, ray d
        # jittered by the sampler's direction d - 1 (DirectLightGatherer's
        # SamplerPrefix).
        inp.sun_angular_extent = np.float32(extent)
        inp.sun_samples = int(world.config.sun_samples)
        inp.sun_jitter = ambient_directions(max(1, inp.sun_samples - 1)).astype(np.float32)
    if hdr:
        inp.lights_hdr, off_h, flat_h = build_lights(world, hdr=True, max_chop=max_chop, min_chop=min_chop)
        assert np.array_equal(off, off_h) and np.array_equal(flat, flat_h)
    return inp


class LightingStage:
    """The lighting stage of one map on one device: the shadow casters and
    the lighting world resident, the direct gather on demand."""

    def __init__(self, world: World, inputs: LightingInputs | None = None, device: int = 0):
        self.inputs = inputs if inputs is not None else prepare(world)
        self.tracer = T.CudaRayTracer(T.make_triangles(world.tri_verts, world.tri_ids), device=device)
        self._ctx = self.tracer._ctx
        self.upload_world(self.inputs)

    def upload_world(self, i: LightingInputs) -> None:
        """vrad_world_upload: faces, samples, lights, cluster lists, tables."""
        keep = [np.ascontiguousarray(a) for a in (i.faces, i.samples, i.lights, i.cluster_offsets,
                                                  i.cluster_lights, i.sky_directions, i.sun_jitter, i.verts)]
        f, s, l, off, cl, dirs, jit, vv = keep
        lh = None if i.lights_hdr is None else np.ascontiguousarray(i.lights_hdr, LIGHT_DTYPE)
        keep.append(lh)
        d = _WorldDesc(f.ctypes.data, len(f), s.ctypes.data, len(s), l.ctypes.data, len(l),
                       off.ctypes.data, cl.ctypes.data, len(off) - 1, dirs.ctypes.data, len(dirs),
                       jit.ctypes.data if len(jit) else None, len(jit), i.sun_angular_extent, i.sun_samples,
                       vv.ctypes.data, len(vv), None if lh is None else lh.ctypes.data)
        T._check(_lib().vrad_world_upload(self._ctx, ctypes.byref(d)), self._ctx)
        self.inputs = i

    def set_extra_passes(self, passes: int) -> None:
        """vrad_set_extra_passes: supersampling passes (4 default, 0 off)."""
        T._check(_lib().vrad_set_extra_passes(self._ctx, passes), self._ctx)

    def upload_bounce(self, reflectivity: np.ndarray, pvs_offsets: np.ndarray, pvs_clusters: np.ndarray,
                      bounces: int = 100, threshold: float = 1.0, max_chop: float = 4.0,
                      min_chop: float = 4.0) -> None:
        """vrad_bounce_upload: the patch tree and the transfer tables; every
        later light pass bounces (Radiosity.BounceAsync's stop rule: at most
        `bounces` bounces, or until one adds less than `threshold`)."""
        refl = np.ascontiguousarray(reflectivity, np.float32).reshape(-1, 3)
        off = np.ascontiguousarray(pvs_offsets, np.int32)
        lst = np.ascontiguousarray(pvs_clusters, np.int32)
        self._bounce_keep = (refl, off, lst)
        d = _BounceDesc(refl.ctypes.data, off.ctypes.data, lst.ctypes.data if len(lst) else None, len(off) - 1,
                        max_chop, min_chop, bounces, threshold)
        T._check(_lib().vrad_bounce_upload(self._ctx, ctypes.byref(d)), self._ctx)

    def bounce_stats(self) -> BounceStats:
        st = BounceStats()
        T._check(_lib().vrad_bounce_stats_get(self._ctx, ctypes.byref(st)), self._ctx)
        return st

    def patch_light(self):
        """After a light pass: (TotalLight (P, 3), DirectLight (P, 3))."""
        n = self.bounce_stats().patches
        total = np.zeros((n, 3), np.float32)
        direct = np.zeros((n, 3), np.float32)
        T._check(_lib().vrad_bounce_patch_light(self._ctx, total.ctypes.data, direct.ctypes.data, n), self._ctx)
        return total, direct

    def set_bounce_model(self, net) -> None:
        """vrad_bounce_set_model: later light passes start their bounce from
        the network's guess (None: the plain bounce)."""
        self._model = net
        T._check(_lib().vrad_bounce_set_model(self._ctx, net.handle if net is not None else None), self._ctx)

    def bounce_features(self):
        """After a light pass: (x (R, 32) bfloat16, log1p of the converged
        bounced light (R, 3) float32), CUDA tensors, per receiver."""
        import torch
        n = ctypes.c_int64()
        T._check(_lib().vrad_bounce_features_device(self._ctx, None, None, 0, ctypes.byref(n), None), self._ctx)
        x = torch.empty((n.value, 32), dtype=torch.bfloat16, device="cuda")
        t = torch.empty((n.value, 3), dtype=torch.float32, device="cuda")
        s = torch.cuda.current_stream().cuda_stream
        T._check(_lib().vrad_bounce_features_device(self._ctx, x.data_ptr(), t.data_ptr(), n.value, ctypes.byref(n),
                                                    ctypes.c_void_p(s)), self._ctx)
        return x, t

    def last_total(self) -> np.ndarray:
        """After a light pass: CollectLight's float total of the last bounce."""
        out = np.zeros(3, np.float32)
        T._check(_lib().vrad_bounce_last_total(self._ctx, out.ctypes.data), self._ctx)
        return out

    def transfers(self):
        """After a light pass: (offsets by patch (P + 1), TRANSFER_DTYPE records)."""
        n = self.bounce_stats().patches
        off = np.zeros(n + 1, np.int64)
        count = ctypes.c_int64()
        T._check(_lib().vrad_bounce_transfers(self._ctx, off.ctypes.data, n, None, 0, ctypes.byref(count)),
                 self._ctx)
        tr = np.zeros(max(1, count.value), TRANSFER_DTYPE)
        T._check(_lib().vrad_bounce_transfers(self._ctx, off.ctypes.data, n, tr.ctypes.data, len(tr),
                                              ctypes.byref(count)), self._ctx)
        return off, tr[:count.value]

    def face_styles(self):
        """vrad_face_styles: each face's four style bytes ((nfaces, 4) uint8,
        255 an empty slot) and the number of faces that dropped a fifth style."""
        n = len(self.inputs.faces)
        out = np.zeros((n, 4), np.uint8)
        dropped = ctypes.c_int64()
        T._check(_lib().vrad_face_styles(self._ctx, out.ctypes.data, n, ctypes.byref(dropped)), self._ctx)
        return out, dropped.value

    def close(self):
        self.tracer.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def direct(self):
        """Every sample's LightingValue (style 0), and the kernel's stats."""
        out = np.zeros(len(self.inputs.samples), LIGHTING_DTYPE)
        st = DirectStats()
        T._check(_lib().vrad_direct_lighting(self._ctx, out.ctypes.data, ctypes.byref(st)), self._ctx)
        return out, st

    def autotune(self):
        """vrad_direct_autotune: times each launch shape once on this world
        and keeps the fastest.  Returns (threads per CTA, {shape: ms})."""
        chosen = ctypes.c_int32()
        times = np.zeros(3, np.float32)
        T._check(_lib().vrad_direct_autotune(self._ctx, ctypes.byref(chosen), times.ctypes.data), self._ctx)
        return chosen.value, {32: float(times[0]), 64: float(times[1]), 128: float(times[2])}

    def lighting_size(self) -> int:
        n = ctypes.c_int64()
        T._check(_lib().vrad_lighting_size(self._ctx, ctypes.byref(n)), self._ctx)
        return n.value

    def light_pass(self, lighting: np.ndarray | None = None):
        """vrad_light_pass: the LIGHTING lump bytes, each face's lightofs, and
        the stats (with the bounce when upload_bounce ran)."""
        if lighting is None:
            lighting = np.zeros(self.lighting_size(), np.uint8)
        ofs = np.zeros(len(self.inputs.faces), np.int32)
        st = PassStats()
        T._check(_lib().vrad_light_pass(self._ctx, lighting.ctypes.data, len(lighting), ofs.ctypes.data,
                                        ctypes.byref(st)), self._ctx)
        return lighting, ofs, st

    def light_pass_ranges(self, ranges: int = RANGE_LDR | RANGE_HDR, ldr: np.ndarray | None = None,
                          hdr: np.ndarray | None = None):
        """vrad_light_pass_ranges: (LIGHTING bytes or None, LIGHTING_HDR bytes
        or None, lightofs, PassStats, [BounceStats LDR, BounceStats HDR])."""
        n = self.lighting_size()
        if ranges & RANGE_LDR and ldr is None:
            ldr = np.zeros(n, np.uint8)
        if ranges & RANGE_HDR and hdr is None:
            hdr = np.zeros(n, np.uint8)
        ofs = np.zeros(len(self.inputs.faces), np.int32)
        st = PassStats()
        bs = (BounceStats * 2)()
        T._check(_lib().vrad_light_pass_ranges(
            self._ctx, ranges, ldr.ctypes.data if ranges & RANGE_LDR else None, len(ldr) if ranges & RANGE_LDR else 0,
            hdr.ctypes.data if ranges & RANGE_HDR else None, len(hdr) if ranges & RANGE_HDR else 0,
            ofs.ctypes.data, ctypes.byref(st), bs), self._ctx)
        return (ldr if ranges & RANGE_LDR else None, hdr if ranges & RANGE_HDR else None, ofs, st, [bs[0], bs[1]])

    def bounce_stats_ranges(self):
        """vrad_bounce_stats_ranges: [LDR, HDR] BounceStats of the last pass."""
        bs = (BounceStats * 2)()
        T._check(_lib().vrad_bounce_stats_ranges(self._ctx, bs), self._ctx)
        return [bs[0], bs[1]]

    def pass_sample_light(self, rng: int) -> np.ndarray:
        """vrad_pass_sample_light: the last pass's direct light of one range
        (LIGHTING_DTYPE per sample)."""
        out = np.zeros(len(self.inputs.samples), LIGHTING_DTYPE)
        T._check(_lib().vrad_pass_sample_light(self._ctx, rng, out.ctypes.data, len(out)), self._ctx)
        return out

    def light_pass_ranges_device(self, d_ldr, d_hdr, ranges: int = RANGE_LDR | RANGE_HDR, stream=None):
        """vrad_light_pass_ranges_device into CUDA tensors (uint8)."""
        import torch
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        T._check(_lib().vrad_light_pass_ranges_device(
            self._ctx, ranges, d_ldr.data_ptr() if d_ldr is not None else None,
            d_hdr.data_ptr() if d_hdr is not None else None, ctypes.c_void_p(s)), self._ctx)

    def light_pass_device(self, d_lighting, stream=None):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        T._check(_lib().vrad_light_pass_device(self._ctx, d_lighting.data_ptr(), ctypes.c_void_p(s)), self._ctx)
        return d_lighting

    def direct_into(self, out: np.ndarray):
        """vrad_direct_lighting into a caller's host buffer (LIGHTING_DTYPE)."""
        st = DirectStats()
        T._check(_lib().vrad_direct_lighting(self._ctx, out.ctypes.data, ctypes.byref(st)), self._ctx)
        return st

    def direct_device(self, d_out, stream=None):
        """Into a CUDA tensor of nsamples * 16 bytes, on `stream` (default:
        torch's current stream)."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        T._check(_lib().vrad_direct_lighting_device(self._ctx, d_out.data_ptr(), ctypes.c_void_p(s)),
                 self._ctx)
        return d_out
