"""CPU checks of the W_c interpolator's oracle and host logic (no GPU)."""
import numpy as np

from oracle import mlp


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(mlp.NPARAM) * 0.05
    x = rng.standard_normal((40, 16))
    t = rng.integers(0, 5, 40)
    y = rng.standard_normal(40)
    w = rng.uniform(0.1, 2.0, 40)
    _, g = mlp.loss_and_grad(p, x, t, y, w, rounded=False)
    picks = np.r_[rng.integers(mlp.OFF_W1, mlp.OFF_B1, 4), rng.integers(mlp.OFF_W2, mlp.OFF_B2, 4),
                  mlp.OFF_B1 + 3, mlp.OFF_B2 + 9, mlp.OFF_W3 + 7, mlp.OFF_B3, mlp.OFF_C + 20, mlp.OFF_C + 3]
    h = 1e-6
    for i in picks:
        a, b = p.copy(), p.copy()
        a[i] += h
        b[i] -= h
        fd = (mlp.loss_and_grad(a, x, t, y, w, rounded=False)[0]
              - mlp.loss_and_grad(b, x, t, y, w, rounded=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1e-3, abs(g[i])), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-3], np.float32)
    r = mlp.bf16_round(v)
    assert r[0] == 1.0 and r[1] == 1.0                   # tie -> even mantissa
    assert r[2] == np.float32(1.0 + 2 ** -7)             # above the tie -> up
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-3) <= 2 ** -8 * 3.0e-3                # half an ulp (7 mantissa bits)


def test_oracle_features_layout():
    rng = np.random.default_rng(1)
    proj = rng.normal(size=(2, 6, 4)).astype(np.float32)
    x, tix, y, w, s = mlp.features(proj, [0, 2, 5], [1, 4], [7, 3], np.linspace(0.1, 0.9, 6))
    assert x.shape == (2 * 4 * 2, 16) and tix.tolist()[:2] == [7, 3]
    # sample (q=1, channel=2, target=1): index ((1*4)+2)*2+1
    k = ((1 * 4) + 2) * 2 + 1
    sk = np.abs(proj[1, [0, 2, 5], 2]).max()
    np.testing.assert_allclose(x[k, :3], proj[1, [0, 2, 5], 2] / sk, rtol=1e-6)
    assert x[k, 3] == np.float32(np.linspace(0.1, 0.9, 6)[4]) and x[k, 4] == 1.0 and not x[k, 5:].any()
    np.testing.assert_allclose(y[k], proj[1, 4, 2] / sk, rtol=1e-6)
    np.testing.assert_allclose(w[k], sk * sk, rtol=1e-6)


def test_grid_split_and_linear_head():
    from ecalj_b200 import lib, surrogate, synth
    anchors, targets, held = surrogate.split_grid(48)
    assert len(anchors) == 8 and len(targets) == 40 and len(held) == 8
    assert set(held) <= set(targets) and not set(anchors) & set(targets)
    x = synth.imag_mesh(48)["x"]
    p = surrogate.linear_head_init(x, anchors, targets, np.zeros(lib.wsurr_nparam(), np.float32))
    C = p[mlp.OFF_C:].reshape(mlp.NTMAX, mlp.NIN)
    # the initial head reproduces a function linear in x exactly
    f = 2.0 * x - 0.3
    for j, t in enumerate(targets):
        assert abs(C[j, :8] @ f[anchors] - f[t]) < 1e-5
        np.testing.assert_allclose(C[j].sum(), 1.0, rtol=1e-6)
