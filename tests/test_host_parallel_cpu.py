"""The host set-up's thread pool and block cache under concurrent callers
(no device needed): several threads building patch trees, samples and
neighbour lists at once through the C ABI (ctypes releases the GIL) must
get exactly what one caller alone gets, call after call (the second and
later calls reuse the cached host blocks)."""
import concurrent.futures as cf

import numpy as np

from hl2sdk_tools_sharp_b200 import lighting as L, roomgrid as rg


def _build(world):
    faces, verts = L.faces_of(world)
    patches, points = L.build_patches(faces, verts, L.face_reflectivity(world))
    samples, first = L.build_samples(faces, verts)
    off, lst = L.build_neighbours(faces, verts)
    return patches.tobytes(), points.tobytes(), samples.tobytes(), first.tobytes(), off.tobytes(), lst.tobytes()


def test_concurrent_callers_get_the_serial_results():
    small = [c for c in (rg.config_batch(i, seed=3) for i in range(64)) if c.side <= 5][:3]
    assert len(small) == 3
    worlds = [rg.generate(c) for c in small]
    want = [_build(w) for w in worlds]
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        for _ in range(2):
            futures = [ex.submit(_build, w) for w in worlds for _ in range(2)]
            got = [f.result() for f in futures]
            for k, g in enumerate(got):
                assert g == want[k // 2], k
