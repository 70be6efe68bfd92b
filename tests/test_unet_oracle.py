"""The CPU oracle of the learned preconditioner's network, checked on its own
(no GPU): backward passes against central finite differences in float64,
pooling/upsampling adjoints, the Adam step, bfloat16 rounding and the
energy-norm loss gradient.  The GPU kernels are then checked against this
oracle (tests/test_gpu_learned.py)."""
import numpy as np
import pytest

import unet_oracle as U


def test_bf16_rounding_is_nearest_even():
    one = 1.0
    ulp = 2.0 ** -7  # bfloat16 spacing at 1
    vals = np.array([one, one + ulp / 2, one + 3 * ulp / 2, one + ulp / 4, -2.5, 1e-40, 3.0e38])
    r = U.bf16(vals)
    assert r[0] == 1.0
    assert r[1] == 1.0                     # tie -> even (1.0)
    assert r[2] == one + 2 * ulp           # tie -> even (1 + 2 ulp)
    assert r[3] == 1.0
    assert r[4] == -2.5
    assert np.isfinite(r[6])


def test_param_count_is_about_half_a_million():
    assert 450_000 < U.param_count() < 650_000


def test_pool_and_up_adjoints():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2, 8, 6, 3))
    y = rng.standard_normal((2, 4, 3, 3))
    assert np.isclose(np.sum(U.pool2(x) * y), np.sum(x * U.pool2_bwd(y)))
    z = rng.standard_normal((2, 8, 6, 3))
    assert np.isclose(np.sum(U.up2(y) * z), np.sum(y * U.up2_bwd(z)))


def test_conv_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((2, 5, 7, 4))
    w = rng.standard_normal((3, 3, 3, 4))
    g = rng.standard_normal((2, 5, 7, 3))
    loss = lambda x_, w_: np.sum(U.conv3x3(x_, w_) * g)
    dx, dw = U.conv3x3_dgrad(g, w), U.conv3x3_wgrad(x, g)
    h = 1e-6
    for idx in [(0, 0, 0, 0), (1, 4, 6, 3), (0, 2, 3, 1), (1, 0, 6, 2)]:
        e = np.zeros_like(x)
        e[idx] = h
        fd = (loss(x + e, w) - loss(x - e, w)) / (2 * h)
        assert abs(fd - dx[idx]) < 1e-6 * max(1, abs(fd))
    for idx in [(0, 0, 0, 0), (2, 2, 2, 3), (1, 1, 0, 2), (2, 0, 2, 1)]:
        e = np.zeros_like(w)
        e[idx] = h
        fd = (loss(x, w + e) - loss(x, w - e)) / (2 * h)
        assert abs(fd - dw[idx]) < 1e-6 * max(1, abs(fd))


def test_unet_backward_matches_finite_differences():
    rng = np.random.default_rng(2)
    params = U.init_params(3)
    x = rng.standard_normal((1, 16, 16, 3))
    out, cache = U.forward(params, x)
    G = rng.standard_normal(out.shape)
    gW, gx = U.backward(cache, G)

    def loss(ps, xx):
        return float(np.sum(U.forward(ps, xx)[0] * G))

    h = 1e-5
    for k in range(len(U.LAYERS)):
        co, _, _, ci = params[k].shape
        for _ in range(2):
            idx = (rng.integers(co), rng.integers(3), rng.integers(3), rng.integers(ci))
            pp = [p.copy() for p in params]
            pm = [p.copy() for p in params]
            pp[k][idx] += h
            pm[k][idx] -= h
            fd = (loss(pp, x) - loss(pm, x)) / (2 * h)
            # ReLU kinks are crossed with probability ~0 at this step
            assert abs(fd - gW[k][idx]) <= 1e-5 * max(1.0, abs(fd)), (U.LAYERS[k][0], fd, gW[k][idx])
    for _ in range(4):
        idx = (0, rng.integers(16), rng.integers(16), rng.integers(3))
        e = np.zeros_like(x)
        e[idx] = h
        fd = (loss(params, x + e) - loss(params, x - e)) / (2 * h)
        assert abs(fd - gx[idx]) <= 1e-5 * max(1.0, abs(fd))


def test_unet_is_positively_homogeneous():
    """No biases and ReLU activations: N(c x) = c N(x) for c > 0, so the
    network's correction scales with the residual."""
    rng = np.random.default_rng(4)
    params = U.init_params(5)
    x = rng.standard_normal((1, 16, 16, 3))
    a = U.forward(params, x)[0]
    b = U.forward(params, 1e-3 * x)[0]
    assert np.allclose(b, 1e-3 * a, rtol=1e-9, atol=1e-15)


def test_adam_step():
    p = [np.array([1.0, -2.0])]
    g = [np.array([0.5, -0.25])]
    m = [np.zeros(2)]
    v = [np.zeros(2)]
    P, M, V = U.adam(p, g, m, v, 1, lr=1e-3)
    # first step: m_hat = g, v_hat = g^2 -> update lr * sign(g) (up to eps)
    assert np.allclose(P[0], p[0] - 1e-3 * np.sign(g[0]), rtol=0, atol=1e-9)
    assert np.allclose(M[0], 0.1 * g[0]) and np.allclose(V[0], 0.001 * g[0] ** 2)


def test_energy_loss_gradient():
    import scipy.sparse as sp

    rng = np.random.default_rng(6)
    n = 12
    R = sp.random(n, n, density=0.4, random_state=7)
    A = (R @ R.T + sp.eye(n) * n).tocsr()
    e1 = rng.standard_normal(n)
    y = rng.standard_normal(n)
    L, g = U.energy_loss(A, e1, y)
    assert L > 0
    h = 1e-6
    for i in range(n):
        d = np.zeros(n)
        d[i] = h
        fd = (U.energy_loss(A, e1, y + d)[0] - U.energy_loss(A, e1, y - d)[0]) / (2 * h)
        assert abs(fd - g[i]) < 1e-6 * max(1, abs(fd))
    assert U.energy_loss(A, e1, e1)[0] == 0.0


def test_image_maps_round_trip():
    rng = np.random.default_rng(8)
    Nn, H, W = 10, 4, 5
    node_pixel = rng.permutation(H * W)[:Nn]
    v = rng.standard_normal(3 * Nn)
    cons = np.zeros(3 * Nn, np.uint8)
    cons[4] = 1
    img = U.to_image(v, node_pixel, H, W, [1.0, 2.0, 4.0])
    back = U.from_image(img, node_pixel, [1.0, 0.5, 0.25], cons)
    want = v.copy()
    want[4] = 0
    assert np.allclose(back, want)


def test_smoothed_energy_loss_gradient():
    import scipy.sparse as sp

    rng = np.random.default_rng(12)
    nn = 5
    n = 3 * nn
    R = sp.random(n, n, density=0.5, random_state=3)
    A = (R @ R.T + sp.eye(n) * n).tocsr()
    # symmetric positive 3x3 block inverses
    blocks = []
    for _ in range(nn):
        q = rng.standard_normal((3, 3))
        blocks.append(np.linalg.inv(q @ q.T + 3 * np.eye(3)))
    binv = np.stack(blocks).reshape(-1)
    e1 = rng.standard_normal(n)
    y = rng.standard_normal(n)
    g = U.smoothed_energy_grad(A, binv, 0.7, e1, y)
    h = 1e-6
    for i in range(n):
        d = np.zeros(n)
        d[i] = h
        fd = (U.smoothed_energy_loss(A, binv, 0.7, e1, y + d) -
              U.smoothed_energy_loss(A, binv, 0.7, e1, y - d)) / (2 * h)
        assert abs(fd - g[i]) < 1e-6 * max(1, abs(fd))
    assert U.smoothed_energy_loss(A, binv, 0.7, e1, e1) == 0.0
