"""The direct-lighting ray workload of a room-grid map.

For every luxel sample of every lit face this emits the rays vrad's direct
gather traces (MapTools/Rad/Light/DirectLightGatherer.cs):

* one visibility segment from the sample to each point or spot light whose
  cluster is in the sample's PVS, that the sample faces (dot > 0) and, for
  a spot, whose cone reaches it (EmitStandardLight / GatherStandardLane,
  :1074-1300);
* one sun segment, from the sample towards the sun over MaxTraceLength, when
  the face faces the sun (EmitSkyLight, :536-600): a closest-hit sky test;
* one sky segment per ambient direction in front of the face, 162 Halton
  directions (AmbientSky, :847-1011; DirectionalSampler.cs:96-111): a
  closest-hit sky test.

Rays are built as LightRayLog.MakeRay does (whole segment, reach 1).  The
sample point is the luxel centre on the face plane moved one unit along the
face normal (FaceLightJob.ComputeIlluminationPointAndNormals).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .roomgrid import World
from .tracer import RAY_DTYPE

MAX_TRACE_LENGTH = np.float32(1.732050807569 * (2 * 16384))   # LightConstants.MaxTraceLength
EQUAL_EPSILON = np.float32(0.001)                              # LightConstants.EqualEpsilon
AMBIENT_DIRECTIONS = 162                                       # LightConstants.VertexNormalCount


def halton(base: int, count: int) -> np.ndarray:
    """HaltonSequence.NextValue, seeds 2..count+1 (DirectionalSampler.cs:14-40),
    in float32 arithmetic."""
    out = np.empty(count, np.float32)
    fbase = np.float32(base)
    for k in range(count):
        seed = k + 2
        ret = np.float32(0.0)
        inv = np.float32(1.0 / float(fbase))
        while seed:
            dig = seed % base
            ret = np.float32(ret + np.float32(dig) * inv)
            inv = np.float32(inv / fbase)
            seed //= base
        out[k] = ret
    return out


def ambient_directions(count: int = AMBIENT_DIRECTIONS) -> np.ndarray:
    """DirectionalSampler.NextValue x count: z from Halton(2), azimuth from
    Halton(3); trigonometry in double, rounded once to float."""
    z = halton(2, count)
    v = halton(3, count)
    out = np.empty((count, 3), np.float32)
    for k in range(count):
        zv = np.float32(2.0 * float(z[k]) - 1.0)
        phi = np.float32(math.acos(float(zv)))
        theta = np.float32(2.0 * math.pi * float(v[k]))
        sp = np.float32(math.sin(float(phi)))
        out[k] = (np.float32(math.cos(float(theta))) * sp, np.float32(math.sin(float(theta))) * sp, zv)
    return out


@dataclasses.dataclass
class Samples:
    points: np.ndarray    # (N, 3) float32 illumination points
    normals: np.ndarray   # (N, 3) float32
    face: np.ndarray      # (N,) int32
    cluster: np.ndarray   # (N,) int32


def luxel_samples(world: World, stride: int = 1) -> Samples:
    """One sample per luxel (every `stride`-th luxel of the map)."""
    pts, nrm, fid = [], [], []
    for f in range(world.face_count):
        S, T = world.face_s[f], world.face_t[f]
        n = world.face_normal[f]
        d = world.face_dist[f]
        # Rows solve (S.xyz, T.xyz, n) . p = (s - S.w, t - T.w, d).
        M = np.stack([S[:3], T[:3], n]).astype(np.float64)
        Minv = np.linalg.inv(M)
        w, h = world.face_extents[f] + 1
        s = world.face_mins[f, 0] + np.arange(w) + 0.5
        t = world.face_mins[f, 1] + np.arange(h) + 0.5
        ss, tt = np.meshgrid(s, t, indexing="xy")
        rhs = np.stack([ss.ravel() - S[3], tt.ravel() - T[3], np.full(ss.size, d)], 0)
        p = (Minv @ rhs).T
        # Clamp luxel centres that fall outside the face onto it.
        poly = world.face_verts[f].astype(np.float64)
        lo, hi = poly.min(0), poly.max(0)
        p = np.clip(p, lo, hi)
        pts.append((p + n).astype(np.float32))
        nrm.append(np.broadcast_to(n, p.shape).astype(np.float32))
        fid.append(np.full(len(p), f, np.int32))
    points = np.concatenate(pts)
    normals = np.concatenate(nrm)
    face = np.concatenate(fid)
    sel = slice(None, None, stride)
    return Samples(points[sel].copy(), normals[sel].copy(), face[sel].copy(),
                   world.face_cluster[face[sel]].copy())


@dataclasses.dataclass
class DirectRays:
    light: np.ndarray     # visibility rays (any-hit), RAY_DTYPE
    sun: np.ndarray       # sky tests (closest hit / sky pass-through)
    sky: np.ndarray       # sky tests, ambient directions
    light_sample: np.ndarray
    light_index: np.ndarray

    @property
    def total(self) -> int:
        return len(self.light) + len(self.sun) + len(self.sky)


def _segments(starts: np.ndarray, ends: np.ndarray) -> np.ndarray:
    r = np.empty(len(starts), RAY_DTYPE)
    r["origin"] = starts
    r["direction"] = (ends.astype(np.float32) - starts.astype(np.float32)).astype(np.float32)
    r["max_distance"] = 1.0
    return r


def direct_rays(world: World, samples: Samples, ambient: bool | None = None,
                directions: np.ndarray | None = None) -> DirectRays:
    P, N, C = samples.points, samples.normals, samples.cluster
    # Lights in the PVS that the sample faces.
    li_s, li_l = [], []
    for l in range(len(world.light_origin)):
        vis = world.pvs[C, world.light_cluster[l]]
        delta = world.light_origin[l][None, :] - P
        dot = np.einsum("ij,ij->i", delta, N)
        ok = vis & (dot > 0)
        if world.light_type[l] == 2:
            dist = np.linalg.norm(delta, axis=1)
            cos_to = -np.einsum("ij,j->i", delta, world.light_normal[l]) / np.maximum(dist, 1e-6)
            ok &= cos_to > np.cos(np.radians(world.light_cone[l, 1]))
        idx = np.nonzero(ok)[0]
        li_s.append(idx)
        li_l.append(np.full(len(idx), l, np.int32))
    li_s = np.concatenate(li_s) if li_s else np.zeros(0, np.int64)
    li_l = np.concatenate(li_l) if li_l else np.zeros(0, np.int32)
    order = np.lexsort((li_l, li_s))     # sample-major, light order within a sample
    li_s, li_l = li_s[order], li_l[order]
    light = _segments(P[li_s], world.light_origin[li_l])

    # Sun.
    sun_dir = world.sun_direction
    faces_sun = -(N @ sun_dir) > 0
    sp = P[faces_sun]
    sun = _segments(sp, sp + (sun_dir * -MAX_TRACE_LENGTH)[None, :])

    # Sky ambient.
    if ambient is None:
        ambient = bool(np.any(world.sky_intensity > 0))
    if ambient:
        dirs = ambient_directions() if directions is None else directions
        dots = -(N @ dirs.T)                           # (N, D)
        si, di = np.nonzero(dots > EQUAL_EPSILON)
        starts = P[si]
        ends = starts + (dirs[di] * -MAX_TRACE_LENGTH)
        sky = _segments(starts, ends)
    else:
        sky = np.zeros(0, RAY_DTYPE)
    return DirectRays(light, sun, sky, li_s.astype(np.int64), li_l)
