"""The FP64 network restatement against central finite differences (CPU)."""
import numpy as np

import mlp_reference as M


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = M.init(5).astype(np.float64)
    x = rng.normal(size=(40, 2))
    y = rng.normal(size=40)
    mask = rng.random(40) < 0.7
    g, _ = M.gradient(p, x, y, mask)
    for i in list(range(0, 128, 17)) + list(range(192, 4288, 401)) + [4300, 4360, 4416]:
        h = 1e-6
        e = np.zeros_like(p)
        e[i] = h
        num = (M.gradient(p + e, x, y, mask)[1] - M.gradient(p - e, x, y, mask)[1]) / (2 * h)
        assert abs(num - g[i]) <= 1e-6 * max(1.0, abs(g[i])), i


def test_bf16_rounding_is_nearest_even():
    assert M.bf16(np.float32(1.0)) == 1.0
    assert M.bf16(np.float32(1.0 + 2 ** -8)) == 1.0            # tie -> even
    assert M.bf16(np.float32(1.0 + 3 * 2 ** -8)) == 1.0 + 2 ** -6
    assert M.bf16(np.float32(-3.14159)) == -3.140625
