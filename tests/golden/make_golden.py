"""Copy the reference's stock-tracer fixtures into tests/golden/.

The reference ships, under src/SourceSharp.Tests/MapTools/Tracing/Fixtures/,
two scenes recorded by compiling stock vrad's KD tracer unchanged
(README-kd-scene.md there):

  kd-scene  2,000 triangles in general position, 8,000 rays, seed 31337
  kd-boxes  1,800 triangles of axis-aligned boxes, 6,000 rays, seed 90210

Each scene is four little-endian binary files (tris, rays, tree, answers).
They are data, not source, and the GPU test machine has no copy of the
reference, so the bytes are committed here unchanged.  Run from anywhere:

    python tests/golden/make_golden.py [reference-root]
"""
import hashlib
import pathlib
import shutil
import sys

SRC_REL = "src/SourceSharp.Tests/MapTools/Tracing/Fixtures"
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
    (dst / "SHA256SUMS").write_text("\n".join(lines) + "\n")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
