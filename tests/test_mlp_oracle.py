"""The float64 MLP oracle's gradient against central finite differences."""

import numpy as np

from oracle import mlp as omlp


def _params(rng):
    return {"w1": rng.normal(size=(64, 8)) / 3, "b1": rng.normal(size=64) / 10,
            "w2": rng.normal(size=(64, 64)) / 8, "b2": rng.normal(size=64) / 10,
            "w3": rng.normal(size=64) / 8, "b3": 0.1}


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = _params(rng)
    x = rng.normal(size=(50, 8))
    t = rng.normal(size=50)
    _, g = omlp.loss_and_grad(p, x, t)
    eps = 1e-6
    for name, idx in [("w1", (3, 5)), ("b1", (7,)), ("w2", (10, 20)), ("b2", (33,)),
                      ("w3", (12,)), ("b3", None)]:
        q1 = {k: np.array(v, dtype=np.float64, copy=True) for k, v in p.items()}
        q2 = {k: np.array(v, dtype=np.float64, copy=True) for k, v in p.items()}
        if idx is None:
            q1[name] = p[name] + eps
            q2[name] = p[name] - eps
            ana = g[name]
        else:
            q1[name][idx] += eps
            q2[name][idx] -= eps
            ana = g[name][idx]
        num = (omlp.loss_and_grad(q1, x, t)[0] - omlp.loss_and_grad(q2, x, t)[0]) / (2 * eps)
        assert abs(num - ana) <= 1e-7 * max(1.0, abs(ana)), (name, num, ana)


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.00390625, 1.005859375, -3.1416], dtype=np.float64)
    out = omlp.bf16(vals)
    assert out[0] == 1.0
    assert out[1] == 1.0           # tie -> even
    assert out[2] == 1.0078125     # above the tie -> up
    assert abs(out[3] + 3.140625) < 1e-12
