"""The network oracle's own gradient formulas against finite differences
(float64, no BF16 rounding), so the GPU's gradients are checked against
something itself checked."""
import numpy as np


def test_oracle_gradient_matches_finite_differences():
    from oracle import mlp_oracle as MO
    rng = np.random.default_rng(0)
    n = sum(int(np.prod(s)) for _, s in MO.SHAPES)
    p = rng.normal(size=n) * 0.2
    x = rng.normal(size=(5, MO.INPUTS))
    t = rng.normal(size=(5, MO.OUTPUTS))
    g, _ = MO.gradient(p, None, t, rounding=False, x=x)

    def loss(q):
        y, _, _ = MO.forward(q, None, rounding=False, x=x)
        return np.mean((y - t) ** 2)
    idx = rng.choice(n, 60, replace=False)
    for i in idx:
        e = np.zeros(n)
        e[i] = 1e-6
        fd = (loss(p + e) - loss(p - e)) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    from oracle import mlp_oracle as MO
    vals = np.array([1.0, 1.00390625, 1.005859375, 1.0078125 + 2 ** -9, -3.14159], np.float32)
    got = MO.bf16(vals)
    assert got[0] == 1.0 and got[1] == 1.0              # a tie goes to the even mantissa
    assert got[2] == 1.0078125                          # above the tie rounds up
    assert abs(got[4] + 3.140625) < 1e-9
