"""The light list builder (hl2sdk_tools_sharp_b200/lights.py) against the
reference's own known answers: the cases of DirectLightBuilderTests and
EntityKeyTests in src/SourceSharp.Tests/MapTools/Rad/Light/DirectLightTests.cs,
restated with the same entities and the same expected values.  The box map
those tests build has one cluster, so every light's cluster is 0 here."""
import math

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import lighting as L, lights as LT, roomgrid as rg, workload as wl


def build(*ents, hdr=False):
    return LT.build([LT.entity(("classname", "worldspawn"))] + [LT.entity(*e) for e in ents], hdr=hdr)


def test_a_point_light_becomes_one_active_light():
    ls = build([("classname", "light"), ("origin", "128 128 128"), ("_light", "255 255 255 200")])
    (light,) = ls.active
    assert light.type == LT.EMIT_POINT
    assert np.array_equal(light.origin, [128, 128, 128])


def test_light_intensity_is_linearised_and_scaled_by_the_fourth_field():
    (light,) = build([("classname", "light"), ("origin", "128 128 128"), ("_light", "255 255 255 200")]).active
    assert light.intensity[0] == pytest.approx(200.0, abs=5e-4)


def test_light_dynamic_is_not_a_compile_light():
    assert not build([("classname", "light_dynamic"), ("origin", "1 1 1"), ("_light", "255 0 0")]).active


def test_an_unknown_light_class_is_reported_and_skipped():
    ls = build([("classname", "light_glow"), ("origin", "1 1 1")])
    assert not ls.active and "light_glow" in ls.unsupported_class_names


def test_the_active_list_is_in_reverse_creation_order():
    ls = build([("classname", "light"), ("origin", "10 10 10"), ("_light", "255 255 255")],
               [("classname", "light"), ("origin", "20 20 20"), ("_light", "255 255 255")])
    assert np.array_equal(ls.active[0].origin, [20, 20, 20])
    assert np.array_equal(ls.active[1].origin, [10, 10, 10])


def _cos_deg(deg):
    # (float)Math.Cos(deg_f / 180 * Math.PI): a float divide, then double.
    return np.float32(math.cos(float(np.float32(deg) / np.float32(180)) * math.pi))


def test_a_spotlights_cones_become_cosines():
    (light,) = build([("classname", "light_spot"), ("origin", "128 128 200"), ("angles", "-90 0 0"),
                      ("_light", "255 255 255 200"), ("_inner_cone", "30"), ("_cone", "45")]).active
    assert light.type == LT.EMIT_SPOT
    assert light.stop_dot == _cos_deg(30.0) and light.stop_dot2 == _cos_deg(45.0)


def test_a_spotlight_with_no_inner_cone_gets_ten():
    (light,) = build([("classname", "light_spot"), ("origin", "1 1 1"), ("_light", "255 255 255")]).active
    assert light.stop_dot == _cos_deg(10.0) and light.stop_dot2 == light.stop_dot


def test_a_fully_open_spotlight_is_a_point_light_with_zero_cones():
    (light,) = build([("classname", "light_spot"), ("origin", "1 1 1"), ("_light", "255 255 255"),
                      ("_inner_cone", "180"), ("_cone", "180")]).active
    assert light.type == LT.EMIT_POINT and (light.stop_dot, light.stop_dot2) == (0, 0)


def test_a_cone_wider_than_ninety_is_clamped_and_warned():
    ls = build([("classname", "light_spot"), ("origin", "1 1 1"), ("_light", "255 255 255"),
                ("_inner_cone", "100"), ("_cone", "120")])
    (light,) = ls.active
    assert light.stop_dot == _cos_deg(90.0)
    assert sum("larger than 90" in w for w in ls.warnings) == 2


def test_a_target_aims_the_light():
    (light,) = build([("classname", "info_target"), ("targetname", "t"), ("origin", "100 50 0")],
                     [("classname", "light_spot"), ("origin", "100 50 100"), ("target", "t"),
                      ("_light", "255 255 255")]).active
    assert np.array_equal(light.normal, [0, 0, -1])


def test_a_missing_target_warns_and_leaves_the_normal_zero():
    ls = build([("classname", "light_spot"), ("origin", "1 2 3"), ("target", "nobody"), ("_light", "255 255 255")])
    assert not ls.active[0].normal.any()
    assert any("missing target" in w for w in ls.warnings)


def test_hdr_prefers_light_hdr_when_it_parses():
    (light,) = build([("classname", "light"), ("origin", "1 1 1"), ("_light", "255 255 255 100"),
                      ("_lightHDR", "255 255 255 50")], hdr=True).active
    assert light.intensity[0] == pytest.approx(50.0, abs=5e-4)


def test_hdr_falls_back_to_light_when_light_hdr_is_negative():
    (light,) = build([("classname", "light"), ("origin", "1 1 1"), ("_light", "255 255 255 100"),
                      ("_lightHDR", "-1 -1 -1 1")], hdr=True).active
    assert light.intensity[0] == pytest.approx(100.0, abs=5e-4)


def test_light_scale_hdr_applies_only_to_the_hdr_pass():
    e = [("classname", "light"), ("origin", "1 1 1"), ("_light", "255 255 255 100"), ("_lightscaleHDR", "3")]
    assert build(e).active[0].intensity[0] == pytest.approx(100.0, abs=5e-4)
    assert build(e, hdr=True).active[0].intensity[0] == pytest.approx(300.0, abs=5e-4)


def test_a_light_environment_makes_a_sun_and_an_ambient_ambient_first():
    ls = build([("classname", "light_environment"), ("origin", "1 1 1"), ("_light", "255 255 255 200"),
                ("pitch", "-45")])
    assert [l.type for l in ls.active] == [LT.EMIT_AMBIENT, LT.EMIT_SKY]


def test_a_missing_ambient_is_half_the_sun():
    ls = build([("classname", "light_environment"), ("origin", "1 1 1"), ("_light", "255 255 255 200")])
    assert np.array_equal(ls.ambient.intensity, ls.sky_light.intensity * np.float32(0.5))


def test_a_second_light_environment_is_counted_but_dropped():
    ls = build([("classname", "light_environment"), ("origin", "1 1 1"), ("_light", "255 255 255")],
               [("classname", "light_environment"), ("origin", "2 2 2"), ("_light", "255 0 0")])
    assert len(ls.active) == 2 and ls.count == 3 and ls.orphaned_sky_lights == 1


def test_sun_spread_angle_is_stored_as_a_sine():
    ls = build([("classname", "light_environment"), ("origin", "1 1 1"), ("_light", "255 255 255"),
                ("SunSpreadAngle", "5")])
    assert ls.sun_angular_extent == np.float32(math.sin(math.pi / 180.0 * 5))


def test_a_style_is_read_as_a_float_and_truncated():
    (light,) = build([("classname", "light"), ("origin", "1 1 1"), ("_light", "255 255 255"),
                      ("style", "2.9")]).active
    assert light.style == 2


def test_the_last_duplicate_key_wins():
    assert LT.value_for_key(LT.entity(("style", "1"), ("style", "2")), "style") == "2"


def test_a_missing_key_is_empty_or_null_with_default():
    e = LT.entity()
    assert LT.value_for_key(e, "x") == "" and LT.value_for_key_with_default(e, "x") is None
    assert LT.float_for_key_with_default(e, "x", 4.0) == 4.0


def test_a_vector_stops_at_the_first_unparsable_field():
    assert np.array_equal(LT.vector_for_key(LT.entity(("origin", "1 2 x 4")), "origin"), [1, 2, 0])


# ---- the generated maps' lists

@pytest.mark.parametrize("cfg", [rg.config_3x3(seed=2), rg.config_8x8(seed=1)], ids=["3x3", "8x8"])
def test_generated_map_lists_for_both_ranges(cfg):
    w = rg.generate(cfg)
    ldr, off, flat = L.build_lights(w)
    hdr, off_h, flat_h = L.build_lights(w, hdr=True)
    # The ranges differ in intensity only: positions, cones, falloff, order
    # and the per-cluster lists are the same.
    for f in L.LIGHT_DTYPE.names:
        if f != "intensity":
            assert np.array_equal(ldr[f], hdr[f]), f
    assert np.array_equal(off, off_h) and np.array_equal(flat, flat_h)
    n = len(w.light_origin)
    for k in range(n):
        l = n - 1 - k                                  # prepended: the last entity first
        base = L.parse_intensity(w.light_color[l]) * np.float32(10000)   # _quadratic_attn 1
        assert np.array_equal(ldr["intensity"][k], base)
        hc = w.light_color_hdr[l]
        src = L.parse_intensity(w.light_color[l]) if hc[0] < 0 else L.parse_intensity(hc, hdr=True)
        want = (src * np.float32(w.light_scale_hdr[l])) * np.float32(10000)
        assert np.array_equal(hdr["intensity"][k], want.astype(np.float32))
    assert hdr["type"][-1] == L.EMIT_SKY and hdr["type"][-2] == L.EMIT_AMBIENT


def test_sky_directions_are_the_detmath_sampler():
    # DirectionalSampler.NextValue with DetMathF's correctly rounded float
    # functions, which tests/test_detmath_cpu.py pins to the golden table;
    # here the table's first directions are checked to be unit vectors whose
    # z is 2 x Halton(2) - 1 exactly.
    d = wl.ambient_directions()
    assert d.shape == (162, 3)
    z = wl.halton(2, 162)
    assert np.array_equal(d[:, 2], (2.0 * z.astype(np.float64) - 1.0).astype(np.float32))
    assert np.allclose(np.linalg.norm(d.astype(np.float64), axis=1), 1.0, atol=1e-6)
