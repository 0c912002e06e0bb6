"""The DirectLight list from light entities: the reference's DirectLightBuilder.

Restates, for the entity keys this build's maps carry, the reference's
(muflub/hl2sdk_tools_sharp, src/SourceSharp.MapTools/Rad/Light)
  DirectLightBuilder.Build           DirectLightBuilder.cs:84-133: the
                                     classname dispatch ("light" prefix,
                                     light_dynamic skipped, unknown kinds
                                     recorded)
  DirectLightBuilder.ParseGeneric    :198-278: style (float, truncated),
                                     _lightHDR before _light in an HDR pass,
                                     the target's direction or the angle keys,
                                     _lightscaleHDR
  ParseLightPoint / ParseLightSpot   :305-397: cones as angles, defaults,
                                     the fully open spot, the 90-degree clamp,
                                     DetMath.CosToSingle of the radians
  ParseLightEnvironment              :399-505: the sun and its ambient
                                     partner, _ambient(HDR), half the sun
                                     when absent, _AmbientScaleHDR,
                                     SunSpreadAngle, a second environment
                                     orphaned
  LightFalloff.Apply                 LightFalloff.cs:71-142, the literal
                                     coefficients and their normalisation
                                     at 100 units
  LightNormals.FromProps             LightNormals.cs:66-131
  EntityKeys                         EntityKeys.cs (last duplicate key wins,
                                     strtod prefix scans)
  RadLightFile.ParseIntensity        MapFormats/Text/RadLightFile.cs:344-420
in the reference's Correct compliance mode (its default).  The active list
is built by prepending, as DirectLightSet.AddToActiveList does, so it holds
the entities in reverse creation order, the environment's ambient ahead of
its sun.

Surface lights come from the emitting textures' leaf patches
(add_surface_lights); the _fifty_percent_distance falloff is the fitted
quadratic of LightFalloff.ApplySolvedCurve (solve_inverse_quadratic*).
"""
from __future__ import annotations

import dataclasses
import math
import re

import numpy as np

from . import detmath as DM

EMIT_SURFACE, EMIT_POINT, EMIT_SPOT, EMIT_SKY, EMIT_AMBIENT = 0, 1, 2, 3, 4
EQUAL_EPSILON = np.float32(0.001)         # LightConstants.EqualEpsilon
DEFAULT_INNER_CONE = np.float32(10.0)     # DirectLightBuilder.DefaultInnerCone
MAX_CONE_ANGLE = np.float32(90.0)         # DirectLightBuilder.MaxConeAngle
NORMALISATION_DISTANCE = np.float32(100.0)

_NUM = re.compile(r"\s*([+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?)")

Entity = list  # [(key, value), ...] in file order


def entity(*pairs) -> Entity:
    return [(str(k), str(v)) for k, v in pairs]


# ---------------------------------------------------------------- keys

def value_for_key(e: Entity, key: str) -> str:
    """EntityKeys.ValueForKey: the LAST pair with the key wins; '' if none."""
    v = value_for_key_with_default(e, key)
    return "" if v is None else v


def value_for_key_with_default(e: Entity, key: str):
    for k, v in reversed(e):
        if k == key:
            return v
    return None


def _scan(text: str, pos: int):
    """strtod's prefix scan from pos: (value, new pos) or (None, pos)."""
    m = _NUM.match(text, pos)
    if not m:
        return None, pos
    return float(m.group(1)), m.end()


def atof(text: str) -> float:
    v, _ = _scan(text, 0)
    return 0.0 if v is None else v


def float_for_key(e: Entity, key: str) -> np.float32:
    """VmfValue.ParseFloat: atof in double, narrowed to float."""
    return np.float32(atof(value_for_key(e, key)))


def float_for_key_with_default(e: Entity, key: str, default: float) -> np.float32:
    v = value_for_key_with_default(e, key)
    return np.float32(default) if v is None else np.float32(atof(v))


def int_for_key(e: Entity, key: str) -> int:
    m = re.match(r"\s*([+-]?\d+)", value_for_key(e, key))
    return int(m.group(1)) if m else 0


def vector_for_key(e: Entity, key: str) -> np.ndarray:
    """EntityKeys.GetVectorForKey: up to three doubles, stopping at the
    first field that does not scan; each narrowed to float."""
    text = value_for_key(e, key)
    parts = [0.0, 0.0, 0.0]
    pos = 0
    for i in range(3):
        v, pos = _scan(text, pos)
        if v is None:
            break
        parts[i] = v
    return np.array(parts, np.float32)


def scan_doubles(text: str, maximum: int) -> list:
    out, pos = [], 0
    while len(out) < maximum:
        v, pos = _scan(text, pos)
        if v is None:
            break
        out.append(v)
    return out


# ---------------------------------------------------------------- values

def parse_intensity(text: str, hdr: bool = False, light_scale: float = 1.0):
    """RadLightFile.ParseIntensity: (intensity float32[3], parsed)."""
    f = scan_doubles(text, 8)
    count = len(f)
    r = f[0] if count > 0 else 0.0
    g = f[1] if count > 1 else 0.0
    b = f[2] if count > 2 else 0.0
    scaler = f[3] if count > 3 else 0.0
    if count == 8:
        if hdr:
            r, g, b, scaler = f[4], f[5], f[6], f[7]
        count = 4
    if r < 0.0 or g < 0.0 or b < 0.0 or scaler < 0.0:
        return np.zeros(3, np.float32), False
    ls = np.float32(light_scale)
    x = np.float32(DM.pow_d(r / 255.0, 2.2) * 255)
    if count == 1:
        return np.array([x, x, x], np.float32) * ls, True
    if count in (3, 4):
        y = np.float32(DM.pow_d(g / 255.0, 2.2) * 255)
        z = np.float32(DM.pow_d(b / 255.0, 2.2) * 255)
        v = np.array([x, y, z], np.float32)
        if count == 4:
            v = v * np.float32(scaler / 255.0)
        return (v * ls).astype(np.float32), True
    return np.array([x, 0, 0], np.float32) * ls, False


def radians(degrees) -> float:
    """LightNormals.Radians, Correct mode: a float divide by 180, then a
    double multiply by pi."""
    return float(np.float32(np.float32(degrees) / np.float32(180))) * math.pi


def normalise(v) -> np.ndarray:
    """Vec3.Normalise (MapFormats/Geometry/Vec3.cs:178-189): the float length
    sqrt((x*x + y*y) + z*z), then three divides; zero stays zero."""
    v = np.asarray(v, np.float32)
    sq = np.float32(np.float32(v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])
    ln = np.float32(math.sqrt(float(sq)))
    if ln == 0:
        return np.zeros(3, np.float32)
    return np.array([v[0] / ln, v[1] / ln, v[2] / ln], np.float32)


def from_props(angles, angle, pitch) -> np.ndarray:
    """LightNormals.FromProps (Correct mode)."""
    angle, pitch = np.float32(angle), np.float32(pitch)
    if angle == -1 or angle == -2:        # ANGLE_UP, ANGLE_DOWN
        x = y = np.float32(0)
    else:
        if angle == 0:
            angle = np.float32(angles[1])
        x = np.float32(DM.cos_d(radians(angle)))
        y = DM.sin_to_single(radians(angle))
    if pitch == 0:
        pitch = np.float32(angles[0])
    z = DM.sin_to_single(radians(pitch))
    cp = np.float32(DM.cos_d(radians(pitch)))
    return np.array([x * cp, y * cp, z], np.float32)


# ---------------------------------------------------------------- the list

LIGHT_FIELDS = ("type", "style", "origin", "intensity", "normal", "stop_dot", "stop_dot2", "exponent",
                "constant_attn", "linear_attn", "quadratic_attn", "start_fade_distance",
                "end_fade_distance", "cap_dist")


@dataclasses.dataclass
class DirectLight:
    index: int
    origin: np.ndarray
    cluster: int
    type: int = EMIT_SURFACE
    style: int = 0
    intensity: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(3, np.float32))
    normal: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(3, np.float32))
    stop_dot: np.float32 = np.float32(0)
    stop_dot2: np.float32 = np.float32(0)
    exponent: np.float32 = np.float32(0)
    constant_attn: np.float32 = np.float32(0)
    linear_attn: np.float32 = np.float32(0)
    quadratic_attn: np.float32 = np.float32(0)
    start_fade_distance: np.float32 = np.float32(0)
    end_fade_distance: np.float32 = np.float32(-1)      # DirectLight.cs:129
    cap_dist: np.float32 = np.float32(1.0e22)           # DirectLight.cs:141


@dataclasses.dataclass
class DirectLightSet:
    active: list = dataclasses.field(default_factory=list)
    count: int = 0
    sky_light: DirectLight | None = None
    ambient: DirectLight | None = None
    sun_angular_extent: np.float32 = np.float32(0)
    orphaned_sky_lights: int = 0
    unsupported_class_names: list = dataclasses.field(default_factory=list)
    warnings: list = dataclasses.field(default_factory=list)

    def alloc(self, origin, cluster: int, add: bool) -> DirectLight:
        light = DirectLight(index=self.count, origin=np.asarray(origin, np.float32), cluster=cluster)
        self.count += 1
        if add:
            self.active.insert(0, light)
        return light


def _find_target(entities, name: str):
    for e in entities:
        if value_for_key(e, "targetname") == name:
            return e
    return None


def _parse_generic(entities, e, light: DirectLight, lights: DirectLightSet, hdr: bool) -> None:
    light.style = int(float_for_key(e, "style"))
    have = False
    if hdr:
        v, ok = parse_intensity(value_for_key(e, "_lightHDR"), hdr=True)
        if ok:
            light.intensity, have = v, True
    if not have:
        light.intensity, _ = parse_intensity(value_for_key(e, "_light"), hdr=hdr)
    target = value_for_key(e, "target")
    if target:
        t = _find_target(entities, target)
        if t is None:
            o = light.origin
            lights.warnings.append(f"WARNING: light at ({int(o[0])} {int(o[1])} {int(o[2])}) has missing target")
        else:
            light.normal = normalise(vector_for_key(t, "origin") - light.origin)
    else:
        light.normal = from_props(vector_for_key(e, "angles"), float_for_key(e, "angle"), float_for_key(e, "pitch"))
    if hdr:
        light.intensity = (light.intensity * float_for_key_with_default(e, "_lightscaleHDR", 1.0)).astype(np.float32)


def solve_inverse_quadratic(x1, y1, x2, y2, x3, y3):
    """MathSolvers.SolveInverseQuadratic (MathSolvers.cs): the quadratic
    a x^2 + b x + c through three points, float by float in the reference's
    order; None when two x coincide."""
    f = np.float32
    x1, y1, x2, y2, x3, y3 = (f(v) for v in (x1, y1, x2, y2, x3, y3))
    det = f(f(x1 - x2) * f(x1 - x3)) * f(x2 - x3)
    if det == f(0):
        return None
    na = f(f(x3 * f(-y1 + y2)) + f(x2 * f(y1 - y3))) + f(x1 * f(-y2 + y3))
    nb = f(f(f(x3 * x3) * f(y1 - y2)) + f(f(x1 * x1) * f(y2 - y3))) + f(f(x2 * x2) * f(-y1 + y3))
    nc = f(f(f(f(x1 * x3) * f(-x1 + x3)) * y2) + f(f(x2 * x2) * f(f(x3 * y1) - f(x1 * y3)))) + \
        f(x2 * f(-f(f(x3 * x3) * y1) + f(f(x1 * x1) * y3)))
    return f(na / det), f(nb / det), f(nc / det)


def solve_inverse_quadratic_monotonic(x1, y1, x2, y2, x3, y3, a, b, c):
    """MathSolvers.SolveInverseQuadraticMonotonic: the points sorted by x,
    then the middle point blended toward the straight line in float steps
    of (double) 0.05 until the slope at the first point agrees with the
    data's direction.  (ok, a, b, c); a failed solve keeps a, b, c."""
    f = np.float32
    x1, y1, x2, y2, x3, y3 = (f(v) for v in (x1, y1, x2, y2, x3, y3))
    if x1 > x2:
        x1, x2, y1, y2 = x2, x1, y2, y1
    if x2 > x3:
        x2, x3, y2, y3 = x3, x2, y3, y2
    if x1 > x2:
        x1, x2, y1, y2 = x2, x1, y2, y1
    blend = f(0)
    while blend <= f(1):
        linear = f(y1 + f(f(f(y3 - y1) * f(x2 - x1)) / f(x3 - x1)))       # FLerp
        temp_y2 = f(f(f(1) - blend) * y2) + f(blend * linear)
        sol = solve_inverse_quadratic(x1, y1, x2, temp_y2, x3, y3)
        if sol is None:
            return False, a, b, c
        a, b, c = sol
        derivative = f((2.0 * float(a) * float(x1)) + float(b))
        if y1 < y2 < y3:
            if derivative >= f(0):
                return True, a, b, c
        elif y1 > y2 > y3:
            if derivative <= f(0):
                return True, a, b, c
        else:
            return True, a, b, c
        blend = f(float(blend) + 0.05)
    return True, a, b, c


def _solved_falloff(e, light: DirectLight, d50, warnings) -> None:
    """LightFalloff.ApplySolvedCurve (LightFalloff.cs:116-200): a falloff
    whose reciprocal brightness is 1 at the light, 2 at
    _fifty_percent_distance and 256 at _zero_percent_distance; the
    constants are double literals, so their expressions narrow from double."""
    f = np.float32
    d0 = float_for_key(e, "_zero_percent_distance")
    if d0 < d50:
        warnings.append(f"light has _fifty_percent_distance of {d50} but _zero_percent_distance of {d0}")
        d0 = f(2.0 * float(d50))
    ok, a, b, c = solve_inverse_quadratic_monotonic(f(0), f(1), d50, f(2), d0, f(256), f(0), f(1), f(0))
    if not ok:
        warnings.append(f"can't solve quadratic for light {d50} {d0}")
    v50 = f(c + f(d50 * f(b + f(d50 * a))))
    scale = f(2.0 / float(v50))
    a, b, c = f(a * scale), f(b * scale), f(c * scale)
    light.quadratic_attn, light.linear_attn, light.constant_attn = a, b, c
    if int_for_key(e, "_hardfalloff") != 0:
        light.end_fade_distance = f(d0)
        light.start_fade_distance = f((0.75 * float(d0)) + (0.25 * float(d50)))
        return
    if abs(float(a)) > 0.0:
        top = f(float(b) / (-2.0 * float(a)))
        if top > f(0):
            light.cap_dist = top
            light.start_fade_distance = top
            light.end_fade_distance = f(10.0 * float(top))


def _falloff(e, light: DirectLight, warnings=None) -> None:
    light.start_fade_distance = np.float32(0)
    light.end_fade_distance = np.float32(-1)
    light.cap_dist = np.float32(1.0e22)
    d50 = float_for_key(e, "_fifty_percent_distance")
    if d50 != 0:
        _solved_falloff(e, light, d50, warnings if warnings is not None else [])
        return
    c, l, q = (float_for_key(e, k) for k in ("_constant_attn", "_linear_attn", "_quadratic_attn"))
    c = np.float32(0) if c < EQUAL_EPSILON else c
    l = np.float32(0) if l < EQUAL_EPSILON else l
    q = np.float32(0) if q < EQUAL_EPSILON else q
    if c < EQUAL_EPSILON and l < EQUAL_EPSILON and q < EQUAL_EPSILON:
        c = np.float32(1)
    light.constant_attn, light.linear_attn, light.quadratic_attn = c, l, q
    d = NORMALISATION_DISTANCE
    ratio = np.float32(np.float32(c + d * l) + np.float32(d * d) * q)
    if ratio > 0:
        light.intensity = (light.intensity * ratio).astype(np.float32)


def _parse_point(entities, e, cluster_of, lights, hdr):
    o = vector_for_key(e, "origin")
    light = lights.alloc(o, cluster_of(o), True)
    _parse_generic(entities, e, light, lights, hdr)
    light.type = EMIT_POINT
    _falloff(e, light, lights.warnings)


def _parse_spot(entities, e, cluster_of, lights, hdr):
    o = vector_for_key(e, "origin")
    light = lights.alloc(o, cluster_of(o), True)
    _parse_generic(entities, e, light, lights, hdr)
    light.type = EMIT_SPOT
    inner = float_for_key(e, "_inner_cone")
    if inner == 0:
        inner = DEFAULT_INNER_CONE
    outer = float_for_key(e, "_cone")
    if outer == 0:
        outer = inner
    if outer < inner:
        outer = inner
    if inner == 180 and outer == 180:
        light.stop_dot = light.stop_dot2 = np.float32(0)
        light.type = EMIT_POINT
        light.exponent = np.float32(0)
    else:
        where = f"({int(o[0])} {int(o[1])} {int(o[2])})"
        if inner > MAX_CONE_ANGLE:
            lights.warnings.append(f"WARNING: light_spot at {where} has inner angle larger than 90 degrees! "
                                   "Clamping to 90...")
            inner = MAX_CONE_ANGLE
        if outer > MAX_CONE_ANGLE:
            lights.warnings.append(f"WARNING: light_spot at {where} has outer angle larger than 90 degrees! "
                                   "Clamping to 90...")
            outer = MAX_CONE_ANGLE
        light.stop_dot2 = DM.cos_to_single(radians(outer))
        light.stop_dot = DM.cos_to_single(radians(inner))
        light.exponent = float_for_key(e, "_exponent")
    _falloff(e, light, lights.warnings)


def _parse_environment(entities, e, cluster_of, lights, hdr):
    o = vector_for_key(e, "origin")
    light = lights.alloc(o, cluster_of(o), False)
    _parse_generic(entities, e, light, lights, hdr)
    spread = value_for_key_with_default(e, "SunSpreadAngle")
    if spread is not None and lights.sky_light is None:
        lights.sun_angular_extent = DM.sin_to_single(math.pi / 180.0 * float(np.float32(atof(spread))))
    if lights.sky_light is not None:
        lights.orphaned_sky_lights += 1
        return
    lights.sky_light = light
    light.type = EMIT_SKY
    ambient = lights.alloc(light.origin, cluster_of(light.origin), False)
    ambient.type = EMIT_AMBIENT
    lights.ambient = ambient
    have = False
    if hdr:
        v, ok = parse_intensity(value_for_key(e, "_ambientHDR"), hdr=True)
        if ok:
            ambient.intensity, have = v, True
    if not have:
        v, ok = parse_intensity(value_for_key(e, "_ambient"), hdr=hdr)
        ambient.intensity = v if ok else (light.intensity * np.float32(0.5)).astype(np.float32)
    if hdr:
        ambient.intensity = (ambient.intensity * float_for_key_with_default(e, "_AmbientScaleHDR", 1.0)).astype(
            np.float32)
    # Sun, then ambient, each prepended: the ambient heads the list.
    lights.active.insert(0, light)
    lights.active.insert(0, ambient)


# LightConstants.DirectScale and DirectLightingSettings.DLightThreshold.
DIRECT_SCALE = np.float32(100.0 * 100.0)
DLIGHT_THRESHOLD = np.float32(0.1)


@dataclasses.dataclass
class SurfacePatches:
    """What AddSurfaceLights reads of the patch set: per patch its origin,
    shading normal, area, face and whether it has children (patch index
    order), and per face its texture's emission (BaseLight), texel area
    (BaseArea) and texels per world unit (ScaleS, ScaleT)."""
    origin: np.ndarray       # (P, 3) float32
    normal: np.ndarray       # (P, 3) float32
    area: np.ndarray         # (P,) float32
    face: np.ndarray         # (P,) int32
    leaf: np.ndarray         # (P,) bool
    base_light: np.ndarray   # (F, 3) float32
    base_area: np.ndarray    # (F,) float32
    scale: np.ndarray        # (F, 2) float32


def add_surface_lights(lights: DirectLightSet, sp: SurfacePatches, cluster_of, light_scale: float = 1.0,
                       threshold=DLIGHT_THRESHOLD) -> None:
    """DirectLightBuilder.AddSurfaceLights (DirectLightBuilder.cs:145-189):
    every leaf patch of an emitting texture, in patch index order (each
    prepended, so the list ends in reverse patch order), whose emission
    averages at least the threshold, becomes a surface light at the
    patch's origin with its normal and intensity BaseLight * (LightScale *
    Area * ScaleS * ScaleT / BaseArea) * DirectScale, float by float."""
    f32 = np.float32
    for i in range(len(sp.area)):
        f = int(sp.face[i])
        if not sp.leaf[i] or float(sp.base_area[f]) < 1e-6:
            continue
        bl = sp.base_light[f].astype(f32)
        average = f32(f32(bl[0] + bl[1]) + bl[2]) / f32(3.0)
        if average < threshold:
            continue
        light = lights.alloc(sp.origin[i], cluster_of(sp.origin[i]), True)
        light.type = EMIT_SURFACE
        light.normal = sp.normal[i].astype(f32)
        scale = f32(f32(f32(f32(light_scale) * sp.area[i]) * sp.scale[f, 0]) * sp.scale[f, 1]) / sp.base_area[f]
        light.intensity = (bl * f32(scale)).astype(f32) * DIRECT_SCALE


def build(entities, cluster_of=lambda origin: 0, hdr: bool = False, surface: SurfacePatches | None = None) -> DirectLightSet:
    """DirectLightBuilder.Build (DirectLightBuilder.cs:88-140): the surface
    lights (with surface given), then the light entities.  cluster_of(origin)
    gives the cluster of a point (the tree's leaf)."""
    lights = DirectLightSet()
    if surface is not None:
        add_surface_lights(lights, surface, cluster_of)
    for e in entities:
        name = value_for_key(e, "classname")
        if not name.startswith("light") or name == "light_dynamic":
            continue
        if name == "light_spot":
            _parse_spot(entities, e, cluster_of, lights, hdr)
        elif name == "light_environment":
            _parse_environment(entities, e, cluster_of, lights, hdr)
        elif name == "light":
            _parse_point(entities, e, cluster_of, lights, hdr)
        else:
            lights.unsupported_class_names.append(name)
    return lights


def to_records(active, dtype) -> np.ndarray:
    """The active list as the C ABI's vrad_light records."""
    out = np.zeros(len(active), dtype)
    for i, l in enumerate(active):
        for f in LIGHT_FIELDS:
            out[i][f] = getattr(l, f)
    return out
