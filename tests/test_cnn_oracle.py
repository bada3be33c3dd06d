"""The network oracle (oracle/cnn_ref.py) pinned without a GPU: its analytic
gradient against central finite differences of its own exact forward pass,
its BF16 rounding against known values, and the BF16-emulating form close to
the exact one."""
import numpy as np
import pytest

from oracle import cnn_ref as N


def _case(seed, B=2, H=6, W=7):
    rng = np.random.default_rng(seed)
    w = N.he_init(seed).astype(np.float64)
    inp = rng.standard_normal((B, H, W))
    tgt = rng.standard_normal((B, H, W))
    return w, inp, tgt


def test_bf16_rounding_known_values():
    vals = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, 1.0 + 2.0 ** -7 + 2.0 ** -8, -2.5, 0.0, 3.0e38],
                    dtype=np.float32)
    want = np.array([1.0, 1.0, 1.0 + 2.0 ** -7, 1.0 + 2.0 ** -6, -2.5, 0.0, np.float32(3.0e38)])
    got = N.bf16(vals)
    assert got[0] == 1.0 and got[1] == 1.0  # tie -> even
    assert got[2] == want[2] and got[3] == want[3]  # above half -> up; tie at odd -> up to even
    assert got[4] == -2.5 and got[5] == 0.0
    assert abs(got[6] - 3.0e38) / 3.0e38 < 2.0 ** -8


def test_layout_sizes():
    assert N.NPARAM == 37440
    W1, Wm, W6 = N.split(np.arange(N.NPARAM, dtype=np.float64))
    assert W1.shape == (32, 9) and len(Wm) == 4 and Wm[0].shape == (32, 9, 32) and W6.shape == (9, 32)
    assert np.array_equal(N.join(W1, Wm, W6), np.arange(N.NPARAM))


@pytest.mark.parametrize("seed", [0, 1])
def test_gradient_matches_finite_differences(seed):
    w, inp, tgt = _case(seed)
    scale = 0.7
    _, g = N.loss_grad(w, scale, inp, tgt, bf16_mode=False)
    rng = np.random.default_rng(100 + seed)
    # parameters of every layer
    idx = np.concatenate([rng.choice(N.OFF_WM, 6, replace=False),
                          N.OFF_WM + rng.choice(N.OFF_W6 - N.OFF_WM, 16, replace=False),
                          N.OFF_W6 + rng.choice(N.K, 6, replace=False)])
    eps = 1e-6
    gmax = np.max(np.abs(g))
    for k in idx:
        wp, wm = w.copy(), w.copy()
        wp[k] += eps
        wm[k] -= eps
        lp, _ = N.loss_grad(wp, scale, inp, tgt, bf16_mode=False)
        lm, _ = N.loss_grad(wm, scale, inp, tgt, bf16_mode=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * gmax + 1e-5 * abs(g[k]), (k, fd, g[k])


def test_bf16_form_close_to_exact():
    w, inp, tgt = _case(3, B=1, H=9, W=11)
    y_e, _ = N.forward(w, 1.0, inp, bf16_mode=False)
    y_b, _ = N.forward(w, 1.0, inp, bf16_mode=True)
    assert np.linalg.norm(y_b - y_e) / np.linalg.norm(y_e) < 3e-2
    _, g_e = N.loss_grad(w, 1.0, inp, tgt, bf16_mode=False)
    _, g_b = N.loss_grad(w, 1.0, inp, tgt, bf16_mode=True)
    assert np.linalg.norm(g_b - g_e) / np.linalg.norm(g_e) < 5e-2


def test_positive_homogeneity():
    # no biases and ReLU: net(a x) = a net(x) for a > 0 (the solver's guess
    # relies on it only through the Rayleigh-Ritz scaling)
    w, inp, _ = _case(4, B=1, H=5, W=5)
    y1, _ = N.forward(w, 1.0, inp, bf16_mode=False)
    y2, _ = N.forward(w, 1.0, 3.0 * inp, bf16_mode=False)
    assert np.allclose(y2, 3.0 * y1, rtol=1e-12, atol=1e-12)


def test_residual_loss_gradient_matches_finite_differences():
    # the residual loss on a small stretched cavity's pressure operator
    from oracle import ins2d_ref as R
    from ins2d_b200 import cases
    x = cases.tanh_grid(7, 0.0, 1.0, 1.05)
    y = cases.tanh_grid(6, 0.0, 1.0, 1.05)
    o = R.make_options(x, y, cases.BC_CAVITY, Re=100.0, poisson=4)
    A = o.discretization.A
    H, W = 6, 7
    assert A.shape == (H * W, H * W)
    w, inp, _ = _case(5, B=2, H=H, W=W)
    scale = 0.9
    loss, g = N.loss_grad(w, scale, inp, None, bf16_mode=False, A=A)
    assert loss > 0
    rng = np.random.default_rng(7)
    idx = np.concatenate([rng.choice(N.OFF_WM, 4, replace=False),
                          N.OFF_WM + rng.choice(N.OFF_W6 - N.OFF_WM, 8, replace=False),
                          N.OFF_W6 + rng.choice(N.K, 4, replace=False)])
    eps = 1e-6
    gmax = np.max(np.abs(g))
    for k in idx:
        wp, wm = w.copy(), w.copy()
        wp[k] += eps
        wm[k] -= eps
        fd = (N.loss_grad(wp, scale, inp, None, bf16_mode=False, A=A)[0] -
              N.loss_grad(wm, scale, inp, None, bf16_mode=False, A=A)[0]) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * gmax + 1e-5 * abs(g[k]), (k, fd, g[k])
