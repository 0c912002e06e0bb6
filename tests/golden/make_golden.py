"""Copy the reference's stock-tracer fixtures into tests/golden/.

The reference ships, under src/SourceSharp.Tests/MapTools/Tracing/Fixtures/,
two scenes recorded by compiling stock vrad's KD tracer unchanged
(README-kd-scene.md there):

  kd-scene  2,000 triangles in general position, 8,000 rays, seed 31337
  kd-boxes  1,800 triangles of axis-aligned boxes, 6,000 rays, seed 90210

Each scene is four little-endian binary files (tris, rays, tree, answers).
They are data, not source, and the GPU test machine has no copy of the
reference, so the bytes are committed here unchanged.

It also extracts, as text, the correctly rounded single-precision arcsine
and power rows of the reference's DetMath golden table
(src/SourceSharp.Tests/MapFormats/Numerics/DetMathGoldens.cs, computed by
the reference's tools/detmath_goldens.py with mpmath at 3000 bits) into
detmath-goldens.txt: one row per line, "function a b expected" as hex bit
patterns.  Run from anywhere:

    python tests/golden/make_golden.py [reference-root]
"""
import hashlib
import pathlib
import re
import shutil
import sys

SRC_REL = "src/SourceSharp.Tests/MapTools/Tracing/Fixtures"
DETMATH_REL = "src/SourceSharp.Tests/MapFormats/Numerics/DetMathGoldens.cs"
DETMATH_ROWS = {("F1", "Asin"), ("F2", "Pow")}
NAMES = [f"{scene}.{part}.bin" for scene in ("kd-scene", "kd-boxes")
         for part in ("tris", "rays", "tree", "answers")]


def main() -> None:
    root = pathlib.Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    src = root / SRC_REL
    dst = pathlib.Path(__file__).resolve().parent
    lines = []
    for name in NAMES:
        shutil.copyfile(src / name, dst / name)
        digest = hashlib.sha256((dst / name).read_bytes()).hexdigest()
        lines.append(f"{digest}  {name}")
    rows = []
    pat = re.compile(r'\("(\w+)", "(\w+)", 0x([0-9A-Fa-f]+)UL, 0x([0-9A-Fa-f]+)UL, 0x([0-9A-Fa-f]+)UL\)')
    for m in pat.finditer((root / DETMATH_REL).read_text()):
        kind, fn, a, b, e = m.groups()
        if (kind, fn) in DETMATH_ROWS:
            rows.append(f"{fn} {int(a, 16):08x} {int(b, 16):08x} {int(e, 16):08x}")
    (dst / "detmath-goldens.txt").write_text("\n".join(rows) + "\n")
    digest = hashlib.sha256((dst / "detmath-goldens.txt").read_bytes()).hexdigest()
    lines.append(f"{digest}  detmath-goldens.txt")
    (dst / "SHA256SUMS").write_text("\n".join(lines) + "\n")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
