"""The solved light falloff (_fifty_percent_distance), its solver and a
light's direction: the reference's LightFalloffTests, MathSolverTests and
LightNormalTests (src/SourceSharp.Tests/MapTools/Rad/Light/
LightMathTests.cs:90-289) restated on the host layer (lights._falloff,
lights.solve_inverse_quadratic*, lights.from_props), in the reference's
Correct mode (divides, the slope at the first point, the double cosine)."""
import math

import numpy as np

from hl2sdk_tools_sharp_b200 import detmath as DM, lights as LT

f32 = np.float32


def solve(d50, d0):
    light = LT.DirectLight(index=0, origin=np.zeros(3, f32), cluster=0)
    LT._falloff(LT.entity(("_fifty_percent_distance", repr(float(d50))), ("_zero_percent_distance", repr(float(d0)))),
                light)
    return light


def test_the_solved_curve_is_twice_the_full_brightness_at_the_fifty_percent_distance():
    l = solve(128, 400)
    v50 = f32(l.constant_attn + f32(128 * f32(l.linear_attn + f32(128 * l.quadratic_attn))))
    assert abs(float(v50) - 2.0) < 5e-6


def test_a_zero_distance_shorter_than_the_fifty_percent_one_is_twice_it():
    a, b = solve(100, 50), solve(100, 200)
    assert (a.quadratic_attn, a.linear_attn, a.constant_attn) == (b.quadratic_attn, b.linear_attn, b.constant_attn)


def test_hard_falloff_fades_from_three_quarters_of_the_way():
    light = LT.DirectLight(index=0, origin=np.zeros(3, f32), cluster=0)
    LT._falloff(LT.entity(("_fifty_percent_distance", "100"), ("_zero_percent_distance", "300"),
                          ("_hardfalloff", "1")), light)
    assert light.end_fade_distance == f32(300)
    assert light.start_fade_distance == f32(0.75 * 300 + 0.25 * 100)


def test_literal_coefficients_below_equal_epsilon_are_dropped_and_scale_intensity():
    light = LT.DirectLight(index=0, origin=np.zeros(3, f32), cluster=0, intensity=np.ones(3, f32))
    LT._falloff(LT.entity(("_quadratic_attn", "0.0005")), light)
    assert (light.constant_attn, light.linear_attn, light.quadratic_attn) == (1, 0, 0)
    light = LT.DirectLight(index=0, origin=np.zeros(3, f32), cluster=0, intensity=np.ones(3, f32))
    LT._falloff(LT.entity(("_linear_attn", "1")), light)
    assert np.array_equal(light.intensity, [100, 100, 100])


def test_the_start_point_slope_test_leaves_the_extreme_curve_uncapped():
    light = solve(10, 20)
    assert light.cap_dist == f32(1.0e22) and light.linear_attn >= 0


def test_a_quadratic_through_three_points_is_exact():
    assert LT.solve_inverse_quadratic(0, 1, 1, 2, 2, 5) == (1, 0, 1)


def test_coincident_x_fails_and_keeps_the_seed():
    assert LT.solve_inverse_quadratic(1, 1, 1, 2, 3, 4) is None
    ok, a, b, c = LT.solve_inverse_quadratic_monotonic(0, 1, 100, 2, 100, 256, f32(0), f32(1), f32(0))
    assert not ok and (a, b, c) == (0, 1, 0)


def test_the_monotonic_solve_sorts_its_points_by_x():
    one = LT.solve_inverse_quadratic_monotonic(0, 1, 128, 2, 400, 256, f32(0), f32(1), f32(0))
    two = LT.solve_inverse_quadratic_monotonic(400, 256, 0, 1, 128, 2, f32(0), f32(1), f32(0))
    assert one == two


def test_the_divide_form_gives_the_references_bits():
    # TheDivideFormDiffersInTheLastBits: d50 96 / d0 256 after the rescale.
    light = solve(96, 256)
    assert light.linear_attn == f32(0.00250157318) and light.quadratic_attn == f32(0.000185510071)


def test_a_solved_light_goes_through_the_builder():
    e = LT.entity(("classname", "light"), ("origin", "0 0 64"), ("_light", "255 255 255 200"),
                  ("_fifty_percent_distance", "96"), ("_zero_percent_distance", "256"))
    ls = LT.build([e])
    (light,) = ls.active
    assert light.linear_attn == f32(0.00250157318) and light.quadratic_attn == f32(0.000185510071)
    assert not ls.warnings


# LightNormalTests (LightMathTests.cs:246-289): a light's direction from its
# angle keys (LightNormals.FromProps, Correct mode).

def test_zero_angle_falls_back_to_the_angles_yaw():
    assert LT.from_props((0, 180, 0), 0, 0)[0] == f32(-1)


def test_zero_pitch_falls_back_to_the_angles_pitch():
    assert LT.from_props((-90, 0, 0), 0, 0)[2] == f32(-1)


def test_angle_up_is_overwritten_by_the_pitch():
    assert np.array_equal(LT.from_props((0, 0, 0), -1, 0), [0, 0, 0])


def test_the_correct_cosine_of_a_right_angle_is_the_doubles_distance_from_pi():
    assert f32(DM.cos_d(math.pi / 2)) == f32(6.123234e-17)
