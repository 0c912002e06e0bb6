"""Loader for the reference's stock KD-tracer fixtures (see make_golden.py).

Layouts follow the reference's Tracing/Fixtures/README-kd-scene.md and its
loader (Tests/MapTools/Tracing/StockKdScene.cs:72-200):

  tris     int32 count, then count x 9 float32 (three vertices)
  rays     int32 count, then count x 6 float32 (start xyz, end xyz)
  tree     int32 nodes, (children, split) pairs; int32 n, index list;
           6 float32 bounds; int32 n, per triangle n(3) d id e(6) cs0 cs1
  answers  int32 count, count int32 hit triangle index, count float32 distance

Rays are the whole segment as direction with a reach of 1, as the reference
builds them (StockKdScene.cs:107-120).
"""
from __future__ import annotations

import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
SCENES = ("kd-scene", "kd-boxes")

STOCK_TRI = np.dtype([("n", "<f4", (3,)), ("d", "<f4"), ("id", "<i4"), ("e", "<f4", (6,)),
                      ("cs", "u1", (2,))])
assert STOCK_TRI.itemsize == 46


def load(prefix: str) -> dict:
    tris = (HERE / f"{prefix}.tris.bin").read_bytes()
    rays = (HERE / f"{prefix}.rays.bin").read_bytes()
    tree = (HERE / f"{prefix}.tree.bin").read_bytes()
    ans = (HERE / f"{prefix}.answers.bin").read_bytes()

    nt = int(np.frombuffer(tris, "<i4", 1)[0])
    verts = np.frombuffer(tris, "<f4", nt * 9, 4).reshape(nt, 9).copy()

    nr = int(np.frombuffer(rays, "<i4", 1)[0])
    se = np.frombuffer(rays, "<f4", nr * 6, 4).reshape(nr, 6)
    r = np.empty((nr, 7), np.float32)
    r[:, 0:3] = se[:, 0:3]
    r[:, 3:6] = se[:, 3:6] - se[:, 0:3]
    r[:, 6] = 1.0

    p = 0
    nn = int(np.frombuffer(tree, "<i4", 1, p)[0]); p += 4
    nodes_raw = np.frombuffer(tree, "<i4", nn * 2, p).reshape(nn, 2); p += 8 * nn
    ni = int(np.frombuffer(tree, "<i4", 1, p)[0]); p += 4
    indices = np.frombuffer(tree, "<i4", ni, p).copy(); p += 4 * ni
    bounds = np.frombuffer(tree, "<f4", 6, p).copy(); p += 24
    nt2 = int(np.frombuffer(tree, "<i4", 1, p)[0]); p += 4
    st = np.frombuffer(tree, STOCK_TRI, nt2, p)
    p += nt2 * STOCK_TRI.itemsize
    assert p == len(tree), (p, len(tree))

    na = int(np.frombuffer(ans, "<i4", 1)[0])
    assert na == nr
    hit = np.frombuffer(ans, "<i4", na, 4).copy()
    dist = np.frombuffer(ans, "<f4", na, 4 + 4 * na).copy()

    nodes = np.zeros(nn, dtype=[("children", "<i4"), ("split", "<f4")])
    nodes["children"] = nodes_raw[:, 0]
    nodes["split"] = nodes_raw[:, 1].view("<f4")

    tri48 = np.zeros(nt2, dtype=[
        ("n", "<f4", (3,)), ("d", "<f4"), ("id", "<i4"), ("e", "<f4", (6,)),
        ("cs0", "u1"), ("cs1", "u1"), ("flags", "u1"), ("unused", "u1")])
    tri48["n"] = st["n"]
    tri48["d"] = st["d"]
    tri48["id"] = st["id"]
    tri48["e"] = st["e"]
    tri48["cs0"] = st["cs"][:, 0]
    tri48["cs1"] = st["cs"][:, 1]

    return {
        "verts": verts, "rays": r, "starts": se[:, 0:3].copy(), "ends": se[:, 3:6].copy(),
        "tree": {"nodes": nodes, "indices": indices, "tris": tri48, "bounds": bounds},
        "stock_tris": tri48, "hit": hit, "dist": dist,
    }


def detmath(function: str):
    """Rows of the reference's DetMath golden table for one function
    ("Asin" or "Pow"): (a, b, expected) as uint32 bit patterns."""
    rows = [line.split() for line in (HERE / "detmath-goldens.txt").read_text().splitlines() if line.strip()]
    sel = [r for r in rows if r[0] == function]
    a = np.array([int(r[1], 16) for r in sel], np.uint32)
    b = np.array([int(r[2], 16) for r in sel], np.uint32)
    e = np.array([int(r[3], 16) for r in sel], np.uint32)
    return a, b, e


def lockdown_lumps() -> dict:
    """dm_lockdown's geometry lumps as {id: (version, bytes)} (the layout
    make_golden.py writes: "VLMP", count, then id, version, length, bytes)."""
    blob = (HERE / "dm_lockdown.lumps.bin").read_bytes()
    assert blob[:4] == b"VLMP"
    n = int(np.frombuffer(blob, "<i4", 1, 4)[0])
    p, out = 8, {}
    for _ in range(n):
        i, ver, ln = (int(x) for x in np.frombuffer(blob, "<i4", 3, p))
        p += 12
        out[i] = (ver, blob[p:p + ln])
        p += ln
    assert p == len(blob)
    return out


def lockdown_rays():
    """The reference's recorded BSP surface tracer set: (rays (n, 7) as
    start + (end - start) x 1, stock's face per ray (-1 none), its fraction,
    its m_bHasLuxel)."""
    rb = (HERE / "rays-lockdown-leafambient.bin").read_bytes()
    ab = (HERE / "stock-lockdown-leafambient.bin").read_bytes()
    n = int(np.frombuffer(rb, "<i4", 1)[0])
    se = np.frombuffer(rb, "<f4", 6 * n, 4).reshape(n, 6)
    rays = np.empty((n, 7), np.float32)
    rays[:, 0:3] = se[:, 0:3]
    rays[:, 3:6] = se[:, 3:6] - se[:, 0:3]
    rays[:, 6] = 1.0
    assert int(np.frombuffer(ab, "<i4", 1)[0]) == n and len(ab) == 4 + 9 * n
    face = np.frombuffer(ab, "<i4", n, 4).copy()
    frac = np.frombuffer(ab, "<f4", n, 4 + 4 * n).copy()
    lux = np.frombuffer(ab, "u1", n, 4 + 8 * n) != 0
    return rays, face, frac, lux
