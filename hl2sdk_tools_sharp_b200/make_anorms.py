"""Write anorms.bin, the 162 ray directions of the leaf ambient sample.

Stock vrad samples the light arriving at a point along the fixed table
g_anorms[162] (the points of a frequency-4 geodesic icosahedron, each
component rounded to six decimals); the reference carries the same table
as VertexNormals.Directions (MapTools/Rad/Ambient/VertexNormals.cs:37-228).
The table's values AND its order are part of the result: each ray's light
is summed onto the ambient cube in table order, in single precision, so the
sum's rounding depends on the order.  The directions are therefore read
from the reference's table, not regenerated, and written as 162 x 3
little-endian float32 (1,944 bytes) beside this script;
tests/test_ambient_cpu.py checks that they are the 162 points of the
frequency-4 geodesic sphere.

    python hl2sdk_tools_sharp_b200/make_anorms.py <reference-root>
"""
import hashlib
import os
import pathlib
import re
import sys

import numpy as np

TABLE_REL = "src/SourceSharp.MapTools/Rad/Ambient/VertexNormals.cs"


def main() -> None:
    arg = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("VRAD_REFERENCE_ROOT")
    if not arg:
        sys.exit("usage: make_anorms.py <reference-root> (or set VRAD_REFERENCE_ROOT)")
    text = (pathlib.Path(arg) / TABLE_REL).read_text()
    num = r"(-?\d+\.\d+)f"
    rows = re.findall(rf"new\({num},\s*{num},\s*{num}\)", text)
    if len(rows) != 162:
        sys.exit(f"expected 162 directions, found {len(rows)}")
    table = np.array([[np.float32(v) for v in r] for r in rows], "<f4")
    out = pathlib.Path(__file__).resolve().parent / "anorms.bin"
    out.write_bytes(table.tobytes())
    print(hashlib.sha256(out.read_bytes()).hexdigest(), out.name)


if __name__ == "__main__":
    main()
