"""Copy the reference's stock-tracer fixtures into tests/golden/.

The reference ships, under src/SourceSharp.Tests/MapTools/Tracing/Fixtures/,
two scenes recorded by compiling stock vrad's KD tracer unchanged
(README-kd-scene.md there):

  kd-scene  2,000 triangles in general position, 8,000 rays, seed 31337
  kd-boxes  1,800 triangles of axis-aligned boxes, 6,000 rays, seed 90210

Each scene is four little-endian binary files (tris, rays, tree, answers).
They are data, not source, and the GPU test machine has no copy of the
reference, so the bytes are committed here unchanged.

It also copies the reference's BSP surface tracer fixtures
(rays-lockdown-leafambient.bin: 8,100 rays; stock-lockdown-leafambient.bin:
stock's CLightSurface answers for them; README-bsp-rays.md there) and, from
game/mod_sharp/maps/dm_lockdown.bsp, the geometry lumps that tracer reads
(planes, vertexes, nodes, texinfo, faces, leafs, edges, surfedges,
leaffaces), unchanged, into dm_lockdown.lumps.bin.

It also extracts, as text, rows of the reference's DetMath golden table
(src/SourceSharp.Tests/MapFormats/Numerics/DetMathGoldens.cs, computed by
the reference's tools/detmath_goldens.py with mpmath at 3000 bits):
  detmath-goldens.txt       the single-precision arcsine and power rows
                            (the device's asin and pow), "function a b
                            expected" as 32-bit hex patterns;
  detmath-goldens-host.txt  the rows of the functions the host-side tables
                            use: single-precision Acos, Sin and Cos, double
                            Sin, Cos and Pow, "kind function a b expected"
                            as hex patterns of the kind's width.
It also copies the reference's leaf-ambient fixture map
src/SourceSharp.Tests/MapTools/Rad/Ambient/Fixtures/p4g_detail.bsp
(gen_ambient_fixture.py --detail there: one sealed room, a func_detail
pillar, a sky section, a point and a spot light, no displacements; run
through stock vbsp, vvis and vrad -both, so it holds stock's own leaf
ambient lumps), unchanged, and extracts as text the reference's golden
vectors of stock's random stream (StockRandomStreamVectors.cs there, made
by gen_stock_random_vectors.py from the stock stream): ran1-vectors.txt,
one "name low high" header line per set and then its 512 float results as
32-bit hex patterns.

Run from anywhere, naming the reference's root (or set VRAD_REFERENCE_ROOT):

    python tests/golden/make_golden.py <reference-root>
"""
import hashlib
import os
import pathlib
import re
import shutil
import struct
import sys

SRC_REL = "src/SourceSharp.Tests/MapTools/Tracing/Fixtures"
DETMATH_REL = "src/SourceSharp.Tests/MapFormats/Numerics/DetMathGoldens.cs"
DETMATH_ROWS = {("F1", "Asin"), ("F2", "Pow")}
HOST_ROWS = {("F1", "Acos"), ("F1", "Sin"), ("F1", "Cos"), ("F1", "Tan"), ("D1", "Sin"), ("D1", "Cos"),
             ("D2", "Pow")}
AMBIENT_REL = "src/SourceSharp.Tests/MapTools/Rad/Ambient"
AMBIENT_NAMES = ["p4g_detail.bsp"]
# StockRandomStreamVectors' sets: (seed, low, high); seed None is the stream
# as constructed (SetSeed(0) in its constructor).
RAN1_SETS = {"DefaultUnit": (None, 0.0, 1.0), "DefaultRanged1024": (None, 0.0, 1024.0),
             "Seed0": (0, 0.0, 1.0), "Seed1": (1, 0.0, 1.0), "Seed7": (7, 0.0, 1.0),
             "Seed12345": (12345, 0.0, 1.0), "SeedMinus3": (-3, 0.0, 1.0),
             "Seed2147483647": (2147483647, 0.0, 1.0)}
NAMES = [f"{scene}.{part}.bin" for scene in ("kd-scene", "kd-boxes")
         for part in ("tris", "rays", "tree", "answers")] + ["rays-lockdown-leafambient.bin",
                                                             "stock-lockdown-leafambient.bin"]
BSP_REL = "game/mod_sharp/maps/dm_lockdown.bsp"


def main() -> None:
    arg = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("VRAD_REFERENCE_ROOT")
    if not arg:
        sys.exit("usage: make_golden.py <reference-root> (or set VRAD_REFERENCE_ROOT)")
    root = pathlib.Path(arg)
    src = root / SRC_REL
    dst = pathlib.Path(__file__).resolve().parent
    lines = []
    for name in NAMES:
        shutil.copyfile(src / name, dst / name)
        digest = hashlib.sha256((dst / name).read_bytes()).hexdigest()
        lines.append(f"{digest}  {name}")
    for name in AMBIENT_NAMES:
        shutil.copyfile(root / AMBIENT_REL / "Fixtures" / name, dst / name)
        lines.append(f"{hashlib.sha256((dst / name).read_bytes()).hexdigest()}  {name}")
    text = (root / AMBIENT_REL / "StockRandomStreamVectors.cs").read_text()
    body = []
    for set_name, (seed, lo, hi) in RAN1_SETS.items():
        m = re.search(rf"ReadOnlySpan<uint> {set_name} =>\s*\[(.*?)\]", text, re.S)
        vals = re.findall(r"0x([0-9A-Fa-f]{8})", m.group(1))
        assert len(vals) == 512, (set_name, len(vals))
        body.append(f"{set_name} {'default' if seed is None else seed} {lo!r} {hi!r}")
        body += [" ".join(v.lower() for v in vals[k:k + 8]) for k in range(0, 512, 8)]
    (dst / "ran1-vectors.txt").write_text("\n".join(body) + "\n")
    lines.append(f"{hashlib.sha256((dst / 'ran1-vectors.txt').read_bytes()).hexdigest()}  ran1-vectors.txt")
    # dm_lockdown's geometry lumps (the BSP surface tracer's inputs), each
    # copied unchanged: "VLMP", lump count, then per lump its id, version,
    # length and bytes.
    sys.path.insert(0, str(dst.parent.parent))
    from hl2sdk_tools_sharp_b200 import bsp as B
    lumps = B.lumps_of(str(root / BSP_REL))
    blob = [b"VLMP", struct.pack("<i", len(lumps))]
    for i in sorted(lumps):
        ver, data = lumps[i]
        blob += [struct.pack("<iii", i, ver, len(data)), data]
    (dst / "dm_lockdown.lumps.bin").write_bytes(b"".join(blob))
    lines.append(f"{hashlib.sha256((dst / 'dm_lockdown.lumps.bin').read_bytes()).hexdigest()}  dm_lockdown.lumps.bin")
    lines.append(f"# the lumps' source, {BSP_REL}: {hashlib.sha256((root / BSP_REL).read_bytes()).hexdigest()}")
    rows, host = [], []
    pat = re.compile(r'\("(\w+)", "(\w+)", 0x([0-9A-Fa-f]+)UL, 0x([0-9A-Fa-f]+)UL, 0x([0-9A-Fa-f]+)UL\)')
    for m in pat.finditer((root / DETMATH_REL).read_text()):
        kind, fn, a, b, e = m.groups()
        if (kind, fn) in DETMATH_ROWS:
            rows.append(f"{fn} {int(a, 16):08x} {int(b, 16):08x} {int(e, 16):08x}")
        if (kind, fn) in HOST_ROWS:
            w = 8 if kind.startswith("F") else 16
            host.append(f"{kind} {fn} {int(a, 16):0{w}x} {int(b, 16):0{w}x} {int(e, 16):0{w}x}")
    for name, body in (("detmath-goldens.txt", rows), ("detmath-goldens-host.txt", host)):
        (dst / name).write_text("\n".join(body) + "\n")
        digest = hashlib.sha256((dst / name).read_bytes()).hexdigest()
        lines.append(f"{digest}  {name}")
    (dst / "SHA256SUMS").write_text("\n".join(lines) + "\n")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
