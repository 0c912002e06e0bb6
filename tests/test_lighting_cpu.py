"""Host set-up of the lighting stage, checked on the CPU: the native sample
builder against the oracle's restatement, and the light list's build."""
import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import lighting as L, roomgrid as rg


@pytest.mark.parametrize("cfg", [rg.config_3x3(seed=2), rg.config_8x8(seed=1)], ids=["3x3", "8x8"])
def test_samples_match_the_oracle_bit_for_bit(oracle_mod, cfg):
    w = rg.generate(cfg)
    faces, verts = L.faces_of(w)
    got, first = L.build_samples(faces, verts)
    want, wfirst = oracle_mod.build_samples(faces, verts)
    assert np.array_equal(first, wfirst)
    assert np.array_equal(got.view(np.uint8).reshape(-1), want)


def test_samples_cover_cells_not_luxel_corners():
    # A face whose lightmap is W x H luxel cells gets W*H samples (the
    # luxel grid has (W+1)*(H+1) corners; the last row and column clip to
    # nothing), each at its cell's balance point.
    w = rg.generate(rg.config_3x3(seed=2))
    faces, verts = L.faces_of(w)
    s, first = L.build_samples(faces, verts)
    sizes = (faces["lightmap_size"][:, 0]) * (faces["lightmap_size"][:, 1])
    assert np.array_equal(np.diff(first), sizes)
    full = s["area"] == s["area"].max()
    assert np.allclose(s["coord"][full] - np.floor(s["coord"][full]), 0.5, atol=1e-5)


def test_parse_intensity_gamma_and_brightness():
    # "_light" "255 255 255 255": gamma leaves 255, brightness 255/255.
    v = L.parse_intensity([255, 255, 255, 255])
    assert np.array_equal(v, np.float32([255, 255, 255]))
    # half-grey: (0.5^2.2)*255 in double, narrowed
    v = L.parse_intensity([127.5, 0, 255, 510])
    assert v[0] == np.float32(np.float32((0.5 ** 2.2) * 255) * np.float32(2.0))
    assert v[1] == 0 and v[2] == np.float32(510.0)
    assert not L.parse_intensity([-1, 0, 0, 0]).any()


def test_light_list_order_and_falloff():
    w = rg.generate(rg.config_3x3(seed=2))
    lights, off, flat = L.build_lights(w)
    # Prepending: the last light entity first, then ambient, then the sun.
    assert lights["type"][-1] == L.EMIT_SKY and lights["type"][-2] == L.EMIT_AMBIENT
    assert np.array_equal(lights["origin"][0], w.light_origin[-1])
    # Hammer's _quadratic_attn 1: intensity scaled by 100^2.
    point = lights[0]
    assert point["quadratic_attn"] == 1 and point["constant_attn"] == 0
    assert np.allclose(point["intensity"], L.parse_intensity(w.light_color[-1]) * np.float32(10000))
    # Every cluster sees the sun and the ambient, and its own room's lights.
    assert len(off) == w.pvs.shape[0] + 1
    for c in range(w.pvs.shape[0]):
        lst = flat[off[c]:off[c + 1]]
        assert len(lights) - 1 in lst and len(lights) - 2 in lst
        assert list(lst) == sorted(lst)


@pytest.mark.parametrize("cfg", [rg.config_3x3(seed=2), rg.config_8x8(seed=1)], ids=["3x3", "8x8"])
def test_neighbours_match_the_oracle(oracle_mod, cfg):
    w = rg.generate(cfg)
    faces, verts = L.faces_of(w)
    off, lst = L.build_neighbours(faces, verts)
    woff, wlst = oracle_mod.neighbours(faces, verts)
    assert np.array_equal(off, woff) and np.array_equal(lst, wlst)
    assert len(lst) > 0


def test_layout_puts_the_median_before_lightofs():
    w = rg.generate(rg.config_3x3(seed=2))
    faces, _ = L.faces_of(w)
    ofs, total = L.lightmap_layout(faces)
    luxels = (faces["lightmap_size"][:, 0] + 1) * (faces["lightmap_size"][:, 1] + 1)
    assert ofs[0] == 4
    assert np.array_equal(np.diff(ofs), 4 * luxels[:-1] + 4)
    assert total == ofs[-1] + 4 * luxels[-1]


def test_oracle_encode_known_values(oracle_mod):
    # StockLightColor.Encode: 1.0 -> exponent -7, mantissa 128 (1 * 2^7);
    # 0 -> all zero; 255 -> exponent 0, 255.
    import ctypes
    faces = np.zeros(1, L.FACE_DTYPE)
    faces["normal"] = (0, 0, 1)
    faces["lightmap_vecs"][0, 0] = (1, 0, 0, 0)
    faces["lightmap_vecs"][0, 1] = (0, 1, 0, 0)
    faces["lightmap_size"] = (1, 1)
    faces["first_vertex"] = 0
    faces["num_vertices"] = 4
    verts = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    samples, first = L.build_samples(faces, verts)
    assert len(samples) == 1
    for value, word in ((1.0, (128, 128, 128, -7)), (0.0, (0, 0, 0, 0)), (255.0, (255, 255, 255, 0))):
        light = np.full((1, 4), value, np.float32)
        lump, _ = oracle_mod.final(faces, verts, samples, first, light)
        px = lump[4:8].view(np.int8)
        assert tuple(int(x) & 0xFF for x in px[:3]) == word[:3] and int(px[3]) == word[3], (value, px)
