"""Seeded room-grid maps: the synthetic input of the lighting-stage benchmarks.

A map is an R x R grid of 1024-unit cube rooms with 16-unit walls shared
between neighbours, a 128 x 192 doorway in every interior wall, optional
pillars, a floor slab, and a ceiling slab whose underside is sky.  What the
generator returns is what vrad's lighting stage reads from a compiled BSP:

* the shadow casters, built as the reference's BrushShadowCasters.AddWorld
  does (MapTools/Rad/BrushShadowCasters.cs:183-214, 360-535): every side of
  every opaque brush, fan-triangulated, id TraceId.Opaque (0x02000000),
  except sky sides; then each visible sky face, id TraceId.Sky (0x01000000);
* the lit faces: convex polygons with a plane, lightmap axes (texinfo
  lightmapVecs at the map's luxel scale) and lightmap extents, split so no
  face's lightmap exceeds 32 luxels per axis (vbsp's maximum lightmap
  dimension), a material reflectivity, and the room (cluster) it lies in;
* lights as the entity keys vrad reads (light / light_spot with "_light",
  attenuation, cone and target; a light_environment with "_light" and
  "_ambient" aimed by a target), placed inside rooms;
* a PVS with one cluster per room: a room sees itself and the rooms up to
  two steps away along its row or column (straight lines through doors).

Every room has its own floor and ceiling brush, as an authored map would.

There is no BSP tree, no vbsp CSG and no visibility compile: those are
outside the lighting stage.  Floor faces are not split around pillars; the
luxels under a pillar are simply in its shadow.
"""
from __future__ import annotations

import dataclasses

import numpy as np

TRACE_ID_SKY = 0x01000000
TRACE_ID_OPAQUE = 0x02000000

ROOM = 1024.0
WALL = 16.0
PITCH = ROOM + WALL
DOOR_W = 128.0
DOOR_H = 192.0
MAX_LIGHTMAP_DIM = 32


@dataclasses.dataclass
class Config:
    side: int = 3
    seed: int = 1
    luxel_scale: float = 16.0
    pillars: tuple[int, int] = (0, 0)          # per room, inclusive range
    pillar_size: tuple[float, float] = (32.0, 96.0)
    lights: int = 4
    spot_fraction: float = 0.0
    intensity: tuple[float, float] = (50.0, 300.0)
    reflectivity: tuple[float, float] = (0.1, 0.7)
    materials: int = 8
    sky_ambient: bool = False
    sun_spread: float = 0.0          # the light_environment's SunSpreadAngle (degrees); 0: one sun ray
    sun_samples: int = 30            # jittered sun rays with a spread (the reference fixes 30)
    texlights: int = 0               # faces whose texture emits (surface lights)


def config_3x3(seed: int = 1) -> Config:
    """Plain vrad, CPU-runnable: 3 x 3 rooms, scale 16, 4 point lights + sun."""
    return Config(side=3, seed=seed, luxel_scale=16.0, pillars=(0, 0), lights=4, spot_fraction=0.0,
                  sky_ambient=False)


def config_large(seed: int = 1) -> Config:
    """The Large configuration without its displaced floors and AO (neither
    is built): 16 x 16 rooms + 0-6 pillars each, scale 8, 256 point and spot
    lights, a sun of 256 jittered rays (spread 2 degrees) + sky, HDR."""
    return Config(side=16, seed=seed, luxel_scale=8.0, pillars=(0, 6), lights=256, spot_fraction=0.5,
                  sky_ambient=True, sun_spread=2.0, sun_samples=256)


def config_8x8(seed: int = 1) -> Config:
    """Plain GPU vrad: 8 x 8 rooms + 0-6 pillars each, scale 8, 64 point and
    spot lights, sun + sky, reflectivity U[0.1, 0.7]."""
    return Config(side=8, seed=seed, luxel_scale=8.0, pillars=(0, 6), lights=64, spot_fraction=0.5,
                  sky_ambient=True)


BATCH_SIDES = (2, 10)


def config_batch(index: int, seed: int = 1) -> Config:
    """Map `index` of the batched workload: a side drawn uniformly from 2..10
    rooms by (seed, index); otherwise the 8 x 8 map's settings (scale 8, 0-6
    pillars per room, spot fraction 0.5, sun + sky), with one light per room
    as the 8 x 8 map has."""
    rng = np.random.default_rng([seed, index])
    side = int(rng.integers(BATCH_SIDES[0], BATCH_SIDES[1] + 1))
    return Config(side=side, seed=seed * 1000 + index, luxel_scale=8.0, pillars=(0, 6), lights=side * side,
                  spot_fraction=0.5, sky_ambient=True)


@dataclasses.dataclass
class World:
    config: Config
    tri_verts: np.ndarray        # (T, 9) float32
    tri_ids: np.ndarray          # (T,) int32
    brushes: np.ndarray          # (B, 6) float32 min xyz, max xyz
    face_verts: list             # F arrays (k, 3) float32, counter-clockwise from the front
    face_normal: np.ndarray      # (F, 3) float32
    face_dist: np.ndarray        # (F,) float32
    face_s: np.ndarray           # (F, 4) float32 lightmap s axis (xyz per unit, offset)
    face_t: np.ndarray           # (F, 4) float32
    face_mins: np.ndarray        # (F, 2) int32 lightmap mins in luxels
    face_extents: np.ndarray     # (F, 2) int32 lightmap size - 1 in luxels
    face_cluster: np.ndarray     # (F,) int32
    face_material: np.ndarray    # (F,) int32
    reflectivity: np.ndarray     # (M, 3) float32
    light_type: np.ndarray       # (L,) int32: 1 point (light), 2 spot (light_spot)
    light_origin: np.ndarray     # (L, 3) float32
    light_color: np.ndarray      # (L, 4) float64 "_light" r g b brightness
    light_attn: np.ndarray       # (L, 3) float64 _constant_attn, _linear_attn, _quadratic_attn
    light_target: np.ndarray     # (L, 3) float32 origin of the spot's target entity
    light_normal: np.ndarray     # (L, 3) float32 unit spot direction (for workload culling)
    light_cone: np.ndarray       # (L, 3) float32 _inner_cone, _cone (degrees), _exponent
    light_cluster: np.ndarray    # (L,) int32
    sun_direction: np.ndarray    # (3,) float32, from the sun towards the world
    sun_target: np.ndarray       # (3,) float32 target point of the light_environment (origin 0)
    sun_color: np.ndarray        # (4,) float64 "_light" of the light_environment
    ambient_color: np.ndarray    # (4,) float64 "_ambient" of the light_environment
    sky_intensity: np.ndarray    # (3,) float32 nonzero when the sky ambient is on
    pvs: np.ndarray              # (C, C) bool
    # The HDR pass's keys (drawn from a stream of their own, so the LDR map
    # is the same with or without them): "_lightHDR" per light (a row of -1
    # is Hammer's "-1 -1 -1 1", which falls back to "_light"),
    # "_lightscaleHDR", and the light_environment's "_lightHDR",
    # "_ambientHDR" and "_AmbientScaleHDR".
    light_color_hdr: np.ndarray = None   # (L, 4) float64
    light_scale_hdr: np.ndarray = None   # (L,) float64
    sun_color_hdr: np.ndarray = None     # (4,) float64
    ambient_color_hdr: np.ndarray = None  # (4,) float64
    ambient_scale_hdr: float = 1.0
    # Texlights (the level's lights file, TextureLightTable): per face the
    # emitting texture's "r g b brightness" (a zero row: the face does not
    # emit), and every face's texture: its texel area (texdata width x
    # height) and texels per world unit along s and t.
    face_emit: np.ndarray = None         # (F, 4) float64
    texel_area: float = 256.0 * 256.0
    texel_scale: tuple = (4.0, 4.0)

    @property
    def face_count(self) -> int:
        return len(self.face_verts)

    def luxel_counts(self) -> np.ndarray:
        return (self.face_extents[:, 0] + 1) * (self.face_extents[:, 1] + 1)


def _box_sides(mn, mx):
    """Six quads of an axis-aligned box, each counter-clockwise seen from
    outside, with the axis and sign of its outward normal."""
    x0, y0, z0 = mn
    x1, y1, z1 = mx
    return [
        (2, -1, [(x0, y0, z0), (x0, y1, z0), (x1, y1, z0), (x1, y0, z0)]),  # bottom
        (2, +1, [(x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)]),  # top
        (0, -1, [(x0, y0, z0), (x0, y0, z1), (x0, y1, z1), (x0, y1, z0)]),
        (0, +1, [(x1, y0, z0), (x1, y1, z0), (x1, y1, z1), (x1, y0, z1)]),
        (1, -1, [(x0, y0, z0), (x1, y0, z0), (x1, y0, z1), (x0, y0, z1)]),
        (1, +1, [(x0, y1, z0), (x0, y1, z1), (x1, y1, z1), (x1, y1, z0)]),
    ]


def _room_origin(i: int, j: int) -> tuple[float, float]:
    return WALL + i * PITCH, WALL + j * PITCH


def _door_span(i: int) -> tuple[float, float]:
    """Doorway interval along a wall belonging to room index i."""
    c = WALL + i * PITCH + ROOM / 2
    return c - DOOR_W / 2, c + DOOR_W / 2


def _brushes(cfg: Config, rng: np.random.Generator):
    R = cfg.side
    boxes = []     # (min, max)
    sky = []       # index of the brush side (in _box_sides order) that is sky, or -1
    # A floor slab and a ceiling slab per room, each overlapping the wall
    # footprints around the room; the ceiling's underside is sky.
    for i in range(R):
        for j in range(R):
            x0, y0 = i * PITCH, j * PITCH
            boxes.append(((x0, y0, -WALL), (x0 + PITCH + WALL, y0 + PITCH + WALL, 0.0)))
            sky.append(-1)
            boxes.append(((x0, y0, ROOM), (x0 + PITCH + WALL, y0 + PITCH + WALL, ROOM + WALL)))
            sky.append(0)
    # Corner posts.
    for i in range(R + 1):
        for j in range(R + 1):
            boxes.append(((i * PITCH, j * PITCH, 0.0), (i * PITCH + WALL, j * PITCH + WALL, ROOM)))
            sky.append(-1)
    # Walls; interior ones carry a doorway (left, right, lintel).
    for axis in (0, 1):
        for i in range(R + 1):
            w0 = i * PITCH
            for j in range(R):
                a0 = WALL + j * PITCH
                a1 = a0 + ROOM
                interior = 0 < i < R
                spans = [(a0, a1, 0.0, ROOM)]
                if interior:
                    d0, d1 = _door_span(j)
                    spans = [(a0, d0, 0.0, ROOM), (d1, a1, 0.0, ROOM), (d0, d1, DOOR_H, ROOM)]
                for s0, s1, z0, z1 in spans:
                    if axis == 0:
                        boxes.append(((w0, s0, z0), (w0 + WALL, s1, z1)))
                    else:
                        boxes.append(((s0, w0, z0), (s1, w0 + WALL, z1)))
                    sky.append(-1)
    # Pillars.
    pillars = []
    lo, hi = cfg.pillars
    for i in range(R):
        for j in range(R):
            ox, oy = _room_origin(i, j)
            for _ in range(int(rng.integers(lo, hi + 1)) if hi > 0 else 0):
                w = float(np.round(rng.uniform(*cfg.pillar_size)))
                h = float(rng.choice([256.0, 512.0, 768.0, ROOM]))
                x = float(np.round(rng.uniform(ox + 96, ox + ROOM - 96 - w)))
                y = float(np.round(rng.uniform(oy + 96, oy + ROOM - 96 - w)))
                boxes.append(((x, y, 0.0), (x + w, y + w, h)))
                sky.append(-1)
                pillars.append((i, j, x, y, w, h))
    return boxes, sky, pillars


def _triangulate(poly):
    """Fan triangulation, as the reference's (points[0], points[j-1], points[j])."""
    return [(poly[0], poly[j - 1], poly[j]) for j in range(2, len(poly))]


def _split_rect(u0, u1, v0, v1, max_len):
    nu = max(1, int(np.ceil((u1 - u0) / max_len - 1e-9)))
    nv = max(1, int(np.ceil((v1 - v0) / max_len - 1e-9)))
    us = np.linspace(u0, u1, nu + 1)
    vs = np.linspace(v0, v1, nv + 1)
    for a in range(nu):
        for b in range(nv):
            yield float(us[a]), float(us[a + 1]), float(vs[b]), float(vs[b + 1])


# Texture axes of an axis-aligned face, as vbsp's world-aligned default:
# (s axis, t axis) per normal axis.
_TEX_AXES = {
    0: (np.array([0, 1, 0], np.float32), np.array([0, 0, -1], np.float32)),
    1: (np.array([1, 0, 0], np.float32), np.array([0, 0, -1], np.float32)),
    2: (np.array([1, 0, 0], np.float32), np.array([0, -1, 0], np.float32)),
}


def _faces(cfg: Config, pillars, rng: np.random.Generator):
    """Visible lit faces: (normal axis, sign, plane coord, u-range, v-range,
    cluster, z-range kind)."""
    R = cfg.side
    out = []  # (axis, sign, d, (a0,a1), (b0,b1), cluster) ; rect in the two other axes (sorted order)

    def add(axis, sign, d, r0, r1, cluster):
        out.append((axis, sign, d, r0, r1, cluster))

    for i in range(R):
        for j in range(R):
            cl = i * R + j
            ox, oy = _room_origin(i, j)
            # floor (normal +z); other axes x, y
            add(2, +1, 0.0, (ox, ox + ROOM), (oy, oy + ROOM), cl)
            # walls: -x side of room faces +x, etc.  other axes: (y, z) for x walls, (x, z) for y walls
            for axis, sign, d, lo, has_door in (
                (0, +1, ox, oy, i > 0), (0, -1, ox + ROOM, oy, i < R - 1),
                (1, +1, oy, ox, j > 0), (1, -1, oy + ROOM, ox, j < R - 1),
            ):
                a0, a1 = lo, lo + ROOM
                if has_door:
                    d0, d1 = _door_span(j if axis == 0 else i)
                    add(axis, sign, d, (a0, d0), (0.0, ROOM), cl)
                    add(axis, sign, d, (d1, a1), (0.0, ROOM), cl)
                    add(axis, sign, d, (d0, d1), (DOOR_H, ROOM), cl)
                else:
                    add(axis, sign, d, (a0, a1), (0.0, ROOM), cl)
            # doorway passages to the +x and +y neighbours (owned by this room)
            if i < R - 1:
                w0 = (i + 1) * PITCH
                d0, d1 = _door_span(j)
                add(2, +1, 0.0, (w0, w0 + WALL), (d0, d1), cl)               # passage floor
                add(2, -1, DOOR_H, (w0, w0 + WALL), (d0, d1), cl)            # lintel underside
                add(1, +1, d0, (w0, w0 + WALL), (0.0, DOOR_H), cl)           # jambs
                add(1, -1, d1, (w0, w0 + WALL), (0.0, DOOR_H), cl)
            if j < R - 1:
                w0 = (j + 1) * PITCH
                d0, d1 = _door_span(i)
                add(2, +1, 0.0, (d0, d1), (w0, w0 + WALL), cl)
                add(2, -1, DOOR_H, (d0, d1), (w0, w0 + WALL), cl)
                add(0, +1, d0, (w0, w0 + WALL), (0.0, DOOR_H), cl)
                add(0, -1, d1, (w0, w0 + WALL), (0.0, DOOR_H), cl)
    for (i, j, x, y, w, h) in pillars:
        cl = i * R + j
        add(0, -1, x, (y, y + w), (0.0, h), cl)
        add(0, +1, x + w, (y, y + w), (0.0, h), cl)
        add(1, -1, y, (x, x + w), (0.0, h), cl)
        add(1, +1, y + w, (x, x + w), (0.0, h), cl)
        if h < ROOM:
            add(2, +1, h, (x, x + w), (y, y + w), cl)
    return out


def _rect_poly(axis, sign, d, r0, r1):
    """Counter-clockwise polygon (seen from the normal side) of an
    axis-aligned rectangle."""
    others = [a for a in range(3) if a != axis]
    u, v = others
    pts = []
    for (a, b) in ((r0[0], r1[0]), (r0[1], r1[0]), (r0[1], r1[1]), (r0[0], r1[1])):
        p = [0.0, 0.0, 0.0]
        p[axis] = d
        p[u] = a
        p[v] = b
        pts.append(p)
    pts = np.array(pts, np.float32)
    n = np.zeros(3, np.float32)
    n[axis] = sign
    e = np.cross(pts[1] - pts[0], pts[2] - pts[0])
    if np.dot(e, n) < 0:
        pts = pts[::-1].copy()
    return pts


def generate(cfg: Config) -> World:
    rng = np.random.default_rng(cfg.seed)
    R = cfg.side
    boxes, sky_side, pillars = _brushes(cfg, rng)

    # Shadow casters: opaque brush sides, then visible sky faces.
    tris, ids = [], []
    for (mn, mx), sky in zip(boxes, sky_side):
        for k, (_, _, quad) in enumerate(_box_sides(mn, mx)):
            if k == sky:
                continue
            for t in _triangulate(quad):
                tris.append(np.array(t, np.float32).reshape(9))
                ids.append(TRACE_ID_OPAQUE)
    for i in range(R):
        for j in range(R):
            ox, oy = _room_origin(i, j)
            quad = _rect_poly(2, -1, ROOM, (ox, ox + ROOM), (oy, oy + ROOM))
            for t in _triangulate(quad):
                tris.append(np.array(t, np.float32).reshape(9))
                ids.append(TRACE_ID_SKY)

    # Lit faces, split to the maximum lightmap dimension.
    scale = cfg.luxel_scale
    max_len = MAX_LIGHTMAP_DIM * scale
    refl = rng.uniform(cfg.reflectivity[0], cfg.reflectivity[1], size=(cfg.materials, 3)).astype(np.float32)
    fv, fn, fd, fs, ft, fmin, fext, fcl, fmat = [], [], [], [], [], [], [], [], []
    for (axis, sign, d, r0, r1, cl) in _faces(cfg, pillars, rng):
        mat = int(rng.integers(0, cfg.materials))
        for a0, a1, b0, b1 in _split_rect(r0[0], r0[1], r1[0], r1[1], max_len):
            poly = _rect_poly(axis, sign, d, (a0, a1), (b0, b1))
            n = np.zeros(3, np.float32)
            n[axis] = sign
            sa, ta = _TEX_AXES[axis]
            s = np.concatenate([sa / scale, [0.0]]).astype(np.float32)
            t = np.concatenate([ta / scale, [0.0]]).astype(np.float32)
            sv = poly @ s[:3] + s[3]
            tv = poly @ t[:3] + t[3]
            mins = np.floor(np.array([sv.min(), tv.min()]))
            maxs = np.ceil(np.array([sv.max(), tv.max()]))
            fv.append(poly)
            fn.append(n)
            fd.append(np.float32(sign * d))
            fs.append(s)
            ft.append(t)
            fmin.append(mins.astype(np.int32))
            fext.append((maxs - mins).astype(np.int32))
            fcl.append(cl)
            fmat.append(mat)

    # Lights, uniformly over rooms, inside the room away from the walls.
    L = cfg.lights
    room_of = rng.integers(0, R * R, size=L)
    lo = np.stack([_room_origin(c // R, c % R) for c in room_of]) if L else np.zeros((0, 2))
    pos = np.zeros((L, 3), np.float32)
    pos[:, 0:2] = lo + rng.uniform(64.0, ROOM - 64.0, size=(L, 2))
    pos[:, 2] = rng.uniform(128.0, ROOM - 128.0, size=L)
    # "_light" r g b brightness: a warm-to-white colour, brightness in the
    # configured range; Hammer's default falloff (_quadratic_attn 1).
    color = np.zeros((L, 4))
    color[:, 0:3] = np.round(rng.uniform(180.0, 255.0, size=(L, 3)))
    color[:, 3] = np.round(rng.uniform(cfg.intensity[0], cfg.intensity[1], size=L))
    attn = np.zeros((L, 3))
    attn[:, 2] = 1.0
    ltype = np.where(rng.uniform(size=L) < cfg.spot_fraction, 2, 1).astype(np.int32)
    ldir = rng.normal(size=(L, 3))
    ldir[:, 2] = -np.abs(ldir[:, 2]) - 0.5
    ldir /= np.linalg.norm(ldir, axis=1, keepdims=True)
    target = (pos + 256.0 * ldir).astype(np.float32)
    ldir = (target - pos) / np.linalg.norm(target - pos, axis=1, keepdims=True)
    inner = np.round(rng.uniform(20.0, 45.0, size=L))
    outer = inner + np.round(rng.uniform(5.0, 30.0, size=L))
    expo = rng.choice([0.0, 1.0, 2.0, 5.0], size=L)

    # Sun: from high above at a seeded azimuth and 35-70 degrees elevation,
    # aimed by a target entity (light_environment at the origin).
    az = rng.uniform(0, 2 * np.pi)
    el = np.radians(rng.uniform(35.0, 70.0))
    sun_dir = -np.array([np.cos(el) * np.cos(az), np.cos(el) * np.sin(az), np.sin(el)])
    sun_target = (sun_dir * 1000.0).astype(np.float32)
    sun_dir = (sun_target / np.linalg.norm(sun_target)).astype(np.float32)

    # PVS: self, and two steps along the row or the column.
    C = R * R
    pvs = np.zeros((C, C), bool)
    for a in range(C):
        ai, aj = divmod(a, R)
        for b in range(C):
            bi, bj = divmod(b, R)
            pvs[a, b] = (ai == bi and abs(aj - bj) <= 2) or (aj == bj and abs(ai - bi) <= 2)

    return World(
        config=cfg,
        tri_verts=np.stack(tris).astype(np.float32),
        tri_ids=np.array(ids, np.int32),
        brushes=np.array([list(a) + list(b) for a, b in boxes], np.float32),
        face_verts=fv,
        face_normal=np.stack(fn),
        face_dist=np.array(fd, np.float32),
        face_s=np.stack(fs),
        face_t=np.stack(ft),
        face_mins=np.stack(fmin),
        face_extents=np.stack(fext),
        face_cluster=np.array(fcl, np.int32),
        face_material=np.array(fmat, np.int32),
        reflectivity=refl,
        light_type=ltype,
        light_origin=pos,
        light_color=color,
        light_attn=attn,
        light_target=target,
        light_normal=ldir.astype(np.float32),
        light_cone=np.stack([inner, outer, expo], 1).astype(np.float32),
        light_cluster=room_of.astype(np.int32),
        sun_direction=sun_dir,
        sun_target=sun_target,
        sun_color=np.array([255.0, 240.0, 200.0, 220.0]),
        ambient_color=np.array([120.0, 150.0, 210.0, 60.0]) if cfg.sky_ambient else np.zeros(4),
        sky_intensity=np.array([1.0, 1.0, 1.0], np.float32) if cfg.sky_ambient else np.zeros(3, np.float32),
        pvs=pvs,
        face_emit=_texlights(cfg, np.stack(fext)),
        **_hdr_keys(cfg, L),
    )


def _texlights(cfg: Config, extents: np.ndarray) -> np.ndarray:
    """cfg.texlights panels: faces of at least 8 x 8 luxels (the rooms are
    open to the sky, so these are walls and pillar sides) drawn from a
    stream of their own, each with a texlight value "r g b brightness"."""
    emit = np.zeros((len(extents), 4))
    if cfg.texlights <= 0:
        return emit
    rng = np.random.default_rng([cfg.seed, 0x544C])
    large = np.flatnonzero((extents[:, 0] >= 7) & (extents[:, 1] >= 7))
    pick = rng.choice(large, size=min(cfg.texlights, len(large)), replace=False)
    emit[pick, 0:3] = np.round(rng.uniform(180.0, 255.0, size=(len(pick), 3)))
    emit[pick, 3] = np.round(rng.uniform(100.0, 400.0, size=len(pick)))
    return emit


def _hdr_keys(cfg: Config, L: int) -> dict:
    """Seeded HDR keys: half the lights fall back to "_light" ("-1 -1 -1 1"),
    the others get an HDR colour and brightness of their own; every light a
    "_lightscaleHDR" of 0.5 to 3; the sun and sky brighter than in LDR."""
    rng = np.random.default_rng([cfg.seed, 0x4844])
    color = np.full((L, 4), -1.0)
    color[:, 3] = 1.0
    own = rng.uniform(size=L) < 0.5
    n = int(own.sum())
    color[own, 0:3] = np.round(rng.uniform(160.0, 255.0, size=(n, 3)))
    color[own, 3] = np.round(rng.uniform(cfg.intensity[0], 2.0 * cfg.intensity[1], size=n))
    scale = rng.choice([0.5, 1.0, 1.5, 2.0, 3.0], size=L)
    return dict(light_color_hdr=color, light_scale_hdr=scale,
                sun_color_hdr=np.array([255.0, 235.0, 190.0, 600.0]),
                ambient_color_hdr=np.array([110.0, 145.0, 215.0, 150.0]) if cfg.sky_ambient else np.zeros(4),
                ambient_scale_hdr=1.5 if cfg.sky_ambient else 1.0)


def _num(x) -> str:
    """A key value that parses back to exactly x (a float32 or a double)."""
    return repr(float(x))


def entities(world: World) -> list:
    """The map's light entities in file order, as (key, value) records the
    reference's DirectLightBuilder reads: the light_environment at the origin
    aimed by a target, then each light or light_spot (spots aimed by a
    target), with "_light", the literal attenuation keys, cones, and the
    HDR keys."""
    def col(c):
        return " ".join(_num(v) for v in c)

    out = [[("classname", "worldspawn")]]
    env = [("classname", "light_environment"), ("origin", "0 0 0"), ("target", "sun_target"),
           ("_light", col(world.sun_color)), ("_ambient", col(world.ambient_color))]
    if world.config.sun_spread > 0:
        env.append(("SunSpreadAngle", _num(world.config.sun_spread)))
    if world.sun_color_hdr is not None:
        env += [("_lightHDR", col(world.sun_color_hdr)), ("_ambientHDR", col(world.ambient_color_hdr)),
                ("_AmbientScaleHDR", _num(world.ambient_scale_hdr))]
    out.append(env)
    out.append([("classname", "info_target"), ("targetname", "sun_target"), ("origin", col(world.sun_target))])
    for l in range(len(world.light_origin)):
        spot = int(world.light_type[l]) == 2
        e = [("classname", "light_spot" if spot else "light"), ("origin", col(world.light_origin[l])),
             ("_light", col(world.light_color[l]))]
        if world.light_color_hdr is not None:
            e += [("_lightHDR", col(world.light_color_hdr[l])), ("_lightscaleHDR", _num(world.light_scale_hdr[l]))]
        a = world.light_attn[l]
        e += [("_constant_attn", _num(a[0])), ("_linear_attn", _num(a[1])), ("_quadratic_attn", _num(a[2]))]
        if spot:
            inner, outer, expo = world.light_cone[l]
            e += [("target", f"spot_{l}"), ("_inner_cone", _num(inner)), ("_cone", _num(outer)),
                  ("_exponent", _num(expo))]
        out.append(e)
        if spot:
            out.append([("classname", "info_target"), ("targetname", f"spot_{l}"),
                        ("origin", col(world.light_target[l]))])
    return out


def cluster_of_point(world: World, p) -> int:
    """The cluster (room) holding point p, or -1 outside every room."""
    R = world.config.side
    i = int(np.floor((float(p[0]) - WALL) / PITCH))
    j = int(np.floor((float(p[1]) - WALL) / PITCH))
    if not (0 <= i < R and 0 <= j < R):
        return -1
    x0, y0 = _room_origin(i, j)
    if not (x0 <= p[0] <= x0 + ROOM and y0 <= p[1] <= y0 + ROOM):
        return -1
    return i * R + j
