"""The oracle's proposal network (CPU): its analytic gradient matches FP64
central finite differences of its loss (without BF16 rounding), and the BF16
rounding helper rounds to nearest even."""
import numpy as np

from oracle import proposal as P


def _problem(seed=0, n=64):
    rng = np.random.default_rng(seed)
    params = np.zeros(P.PARAMS)
    for l in range(4):
        w = np.zeros((P.ROWS[l], P.IN))
        fan = 78 if l == 0 else 65
        rows = 2 if l == 3 else P.ROWS[l]
        w[:rows, :fan] = rng.normal(0, 1.0 / np.sqrt(fan), (rows, fan))
        params[P.OFF[l]:P.OFF[l] + P.ROWS[l] * P.IN] = w.reshape(-1)
    o = rng.normal(0, 1, (n, 3))
    o = 3 * o / np.linalg.norm(o, axis=1, keepdims=True)
    d = -o / 3 + rng.normal(0, 0.2, (n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    targets = np.stack([rng.uniform(2, 3, n), rng.uniform(3, 4, n)], 1)
    targets[::5, 0] = -1.0  # rays without hits: no t_near term
    return params, rays, targets


def test_gradient_matches_finite_differences():
    params, rays, targets = _problem()
    kw = dict(origin_scale=1 / 3, t_shift=3.0, t_scale=1.0, near_weight=8.0, far_weight=3.0, bf16_ops=False)
    _, g = P.loss_and_grad(params, rays, targets, **kw)
    rng = np.random.default_rng(1)
    live = np.flatnonzero(np.abs(g) > 1e-6)
    picks = rng.choice(live, 40, replace=False)
    h = 1e-6
    for i in picks:
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        num = (P.loss_and_grad(p1, rays, targets, **kw)[0] - P.loss_and_grad(p2, rays, targets, **kw)[0]) / (2 * h)
        assert abs(num - g[i]) <= 1e-5 * max(abs(g[i]), 1e-3), (i, num, g[i])
    # weights fed by the zero input and unused output rows get no gradient
    G = P.layers(g)
    assert np.all(G[0][:, 79] == 0) and np.all(G[1][:, 65:] == 0) and np.all(G[3][2:] == 0)


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 3e-3], np.float32)
    r = P.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie -> even
    assert r[2] == np.float32(1.0 + 2 ** -6)  # tie -> even (up)
    assert r[3] == 1.0 and r[4] == -2.5
    assert abs(r[5] - 3e-3) <= 3e-3 * 2 ** -8
