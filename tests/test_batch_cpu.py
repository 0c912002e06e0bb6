"""CPU-side checks of the batch runner's boundary: the ctypes records match
the C header's layout (compiled here with gcc), the entry points refuse bad
arguments and a missing device with a status, and the batched workload's
map list is seeded and within its side range."""
import ctypes
import pathlib
import shutil
import subprocess

import pytest

from hl2sdk_tools_sharp_b200 import batch as B, roomgrid as rg, tracer as T

ROOT = pathlib.Path(__file__).resolve().parent.parent

_FIELDS = {
    "vrad_batch_map": ("triangles", "world", "bounce", "lighting", "lightofs", "capacity", "ntriangles",
                       "extra_passes", "status", "worker", "lighting_bytes", "seconds", "scene_s", "world_s",
                       "bounce_s", "pass_s", "pass", "bounce_stats", "error"),
    "vrad_batch_stats": ("workers", "maps", "failed", "block", "seconds", "busy_seconds", "rays", "luxels",
                         "lighting_bytes", "device_mallocs", "device_malloc_bytes", "device_trims"),
}


def _c_layout(tmp_path):
    if not shutil.which("gcc"):
        pytest.skip("gcc absent")
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "vrad_cuda.h"', "int main(void) {"]
    for s, fields in _FIELDS.items():
        lines.append(f'printf("{s} %zu\\n", sizeof({s}));')
        for f in fields:
            lines.append(f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {k: int(v) for k, v in (ln.split() for ln in out.splitlines())}


def test_records_match_the_header(tmp_path):
    c = _c_layout(tmp_path)
    assert c["vrad_batch_map"] == ctypes.sizeof(B._BatchMap)
    assert c["vrad_batch_stats"] == ctypes.sizeof(B.BatchStats)
    rename = {"pass": "pass_stats"}
    for f in _FIELDS["vrad_batch_map"]:
        assert c[f"vrad_batch_map.{f}"] == getattr(B._BatchMap, rename.get(f, f)).offset, f
    for f in _FIELDS["vrad_batch_stats"]:
        assert c[f"vrad_batch_stats.{f}"] == getattr(B.BatchStats, f).offset, f


def test_create_refuses_worker_counts_out_of_range():
    lib = B._lib()
    out = ctypes.c_void_p()
    for w in (0, -1, B.MAX_WORKERS + 1):
        assert lib.vrad_batch_create(0, w, ctypes.byref(out)) == -1
        assert not out.value


def test_create_without_a_device_fails_with_a_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = B._lib()
    out = ctypes.c_void_p()
    assert lib.vrad_batch_create(0, 2, ctypes.byref(out)) == -7
    assert not out.value
    with pytest.raises(T.VradError):
        B.LightingBatch(2)


def test_null_batch_calls_are_argument_errors():
    lib = B._lib()
    st = B.BatchStats()
    assert lib.vrad_batch_run(None, None, 0, 0, ctypes.byref(st)) == -1
    w, blk = ctypes.c_int32(), ctypes.c_int32()
    assert lib.vrad_batch_autotune(None, None, 0, ctypes.byref(w), ctypes.byref(blk), None) == -1
    assert lib.vrad_batch_destroy(None) == 0


def test_batched_workload_is_seeded_and_in_range():
    a = [rg.config_batch(i, seed=1) for i in range(32)]
    b = [rg.config_batch(i, seed=1) for i in range(32)]
    assert [c.side for c in a] == [c.side for c in b]
    assert all(rg.BATCH_SIDES[0] <= c.side <= rg.BATCH_SIDES[1] for c in a)
    assert len({c.side for c in a}) > 4            # uneven sizes
    assert len({c.seed for c in a}) == 32          # every map its own geometry
    assert [c.side for c in a] != [rg.config_batch(i, seed=2).side for i in range(32)]


def test_map_inputs_size_the_lump_from_the_layout():
    w = rg.generate(rg.config_batch(8, seed=1))
    m = B.map_inputs(w)
    from hl2sdk_tools_sharp_b200 import lighting as L
    _, size = L.lightmap_layout(m.inputs.faces)
    assert m.lighting_bytes == size > 0
    assert m.bounced and len(m.pvs_offsets) == w.pvs.shape[0] + 1
    assert len(m.triangles) == len(w.tri_ids)
    assert not B.map_inputs(w, m.inputs, bounce=False).bounced
