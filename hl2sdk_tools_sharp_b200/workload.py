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
import functools
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
    return _ambient_directions(count).copy()


@functools.lru_cache(maxsize=8)
def _ambient_directions(count: int) -> np.ndarray:
    """DirectionalSampler.NextValue x count (DirectionalSampler.cs:96-121): z
    from Halton(2), azimuth from Halton(3); 2z - 1 and 2 pi v in double,
    narrowed; DetMathF.Acos, Sin and Cos (correctly rounded float functions,
    detmath.py); the products in float."""
    from . import detmath as DM
    z = halton(2, count)
    v = halton(3, count)
    out = np.empty((count, 3), np.float32)
    for k in range(count):
        zv = np.float32(2.0 * float(z[k]) - 1.0)
        phi = DM.acos_f(zv)
        theta = np.float32(2.0 * math.pi * float(v[k]))
        sp = DM.sin_f(phi)
        out[k] = (DM.cos_f(theta) * sp, DM.sin_f(theta) * sp, zv)
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


def _face_runs(face: np.ndarray):
    """Start and length of each face's run of consecutive samples."""
    change = np.flatnonzero(np.diff(face)) + 1
    starts = np.concatenate([[0], change])
    counts = np.diff(np.concatenate([starts, [len(face)]]))
    return starts, counts, face[starts]


def direct_rays(world: World, samples: Samples, ambient: bool | None = None,
                directions: np.ndarray | None = None) -> DirectRays:
    """Rays in the order a warp-per-32-luxels emitter produces them: face by
    face, and within a face light by light (or direction by direction),
    sample by sample, so neighbouring rays share a target and a direction."""
    P, N, C = samples.points, samples.normals, samples.cluster
    starts, counts, fids = _face_runs(samples.face)
    run_of = np.repeat(np.arange(len(starts)), counts)

    # Lights in the PVS that the sample faces; a spot's cone must reach it.
    ok = np.zeros((len(P), len(world.light_origin)), bool)
    for l in range(len(world.light_origin)):
        delta = world.light_origin[l][None, :] - P
        m = world.pvs[C, world.light_cluster[l]] & (np.einsum("ij,ij->i", delta, N) > 0)
        if world.light_type[l] == 2:
            dist = np.maximum(np.linalg.norm(delta, axis=1), 1e-6)
            cos_to = -np.einsum("ij,j->i", delta, world.light_normal[l]) / dist
            m &= cos_to > np.cos(np.radians(world.light_cone[l, 1]))
        ok[:, l] = m
    si, li = np.nonzero(ok)
    order = np.lexsort((si, li, run_of[si]))        # face, then light, then sample
    li_s, li_l = si[order], li[order].astype(np.int32)
    light = _segments(P[li_s], world.light_origin[li_l])

    # Sun: every sample of a face that faces it.
    sun_dir = world.sun_direction
    faces_sun = -(N @ sun_dir) > 0
    sp = P[faces_sun]
    sun = _segments(sp, sp + (sun_dir * -MAX_TRACE_LENGTH)[None, :])

    # Sky ambient: per face, per direction in front of it, every sample.
    if ambient is None:
        ambient = bool(np.any(world.sky_intensity > 0))
    if ambient:
        dirs = ambient_directions() if directions is None else directions
        valid = -(world.face_normal[fids] @ dirs.T) > EQUAL_EPSILON      # (runs, D)
        pr, pd = np.nonzero(valid)
        reps = counts[pr]
        pair = np.repeat(np.arange(len(pr)), reps)
        first = np.concatenate([[0], np.cumsum(reps)[:-1]])
        sample = starts[pr][pair] + (np.arange(len(pair)) - first[pair])
        st = P[sample]
        sky = _segments(st, st + dirs[pd][pair] * -MAX_TRACE_LENGTH)
    else:
        sky = np.zeros(0, RAY_DTYPE)
    return DirectRays(light, sun, sky, li_s.astype(np.int64), li_l)


def direct_rays_device(world: World, samples: Samples, device) -> dict:
    """direct_rays built on a CUDA device with torch, same rays in the same
    order, as (n, 7) float32 tensors."""
    import torch
    P = torch.from_numpy(samples.points).to(device)
    N = torch.from_numpy(samples.normals).to(device)
    C = torch.from_numpy(samples.cluster.astype(np.int64)).to(device)
    starts, counts, fids = _face_runs(samples.face)
    run_of = torch.from_numpy(np.repeat(np.arange(len(starts)), counts)).to(device)
    pvs = torch.from_numpy(world.pvs).to(device)
    Lo = torch.from_numpy(world.light_origin).to(device)
    LC = torch.from_numpy(world.light_cluster.astype(np.int64)).to(device)
    Ln = torch.from_numpy(world.light_normal).to(device)
    cos_outer = torch.from_numpy(np.cos(np.radians(world.light_cone[:, 1])).astype(np.float32)).to(device)
    spot = torch.from_numpy(world.light_type == 2).to(device)
    nl = len(world.light_origin)

    def seg(a, b):
        r = torch.empty((a.shape[0], 7), dtype=torch.float32, device=device)
        r[:, 0:3] = a
        r[:, 3:6] = b - a
        r[:, 6] = 1.0
        return r

    keys = []
    chunk = 1 << 20
    for b in range(0, P.shape[0], chunk):
        p, n, c = P[b:b + chunk], N[b:b + chunk], C[b:b + chunk]
        delta = Lo[None, :, :] - p[:, None, :]
        ok = pvs[c][:, LC] & ((delta * n[:, None, :]).sum(-1) > 0)
        dist = delta.norm(dim=-1).clamp_min(1e-6)
        cos_to = -(delta * Ln[None]).sum(-1) / dist
        ok &= ~spot[None, :] | (cos_to > cos_outer[None, :])
        si, li = torch.nonzero(ok, as_tuple=True)
        si = si + b
        keys.append((run_of[si] * nl + li) * P.shape[0] + si)
    key = torch.sort(torch.cat(keys)).values
    si = key % P.shape[0]
    li = (key // P.shape[0]) % nl
    light = seg(P[si], Lo[li])
    del keys, key

    sun_dir = torch.from_numpy(world.sun_direction).to(device)
    sp = P[-(N @ sun_dir) > 0]
    sun = seg(sp, sp + sun_dir * -float(MAX_TRACE_LENGTH))

    dirs = torch.from_numpy(ambient_directions()).to(device)
    fn = torch.from_numpy(world.face_normal[fids]).to(device)
    pr, pd = torch.nonzero(-(fn @ dirs.T) > float(EQUAL_EPSILON), as_tuple=True)
    cnt = torch.from_numpy(counts).to(device)
    st0 = torch.from_numpy(starts).to(device)
    reps = cnt[pr]
    sky_parts = []
    pair_chunk = 1 << 16
    for b in range(0, pr.shape[0], pair_chunk):
        r = reps[b:b + pair_chunk]
        pair = torch.repeat_interleave(torch.arange(r.shape[0], device=device), r)
        first = torch.cumsum(r, 0) - r
        sample = st0[pr[b:b + pair_chunk]][pair] + (torch.arange(pair.shape[0], device=device) - first[pair])
        st = P[sample]
        sky_parts.append(seg(st, st + dirs[pd[b:b + pair_chunk]][pair] * -float(MAX_TRACE_LENGTH)))
    sky = torch.cat(sky_parts)
    del sky_parts
    return {"light": light.contiguous(), "sun": sun.contiguous(), "sky": sky.contiguous(),
            "luxels": int(P.shape[0])}
