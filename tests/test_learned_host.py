"""Host-side logic of the learned guess and the backward-facing-step workload
(no GPU): the explicit-RK4 stability rule of the step size, the detection of
singular pressure operators (centred targets), and the odd part the solver
applies, checked on the CPU oracle of the network."""
import types

import numpy as np

from oracle import cnn_ref as N


def test_bfs_step_respects_the_rk4_stability_limit():
    import bench
    from ins2d_b200 import cases
    x = cases.tanh_grid(1024, 0.0, 30.0, 1.02)
    y = cases.tanh_grid(1024, -0.5, 0.5, 1.02)
    dt = bench.bfs_dt(x, y, 800.0, 1e-3)
    hx, hy = np.min(np.diff(x)), np.min(np.diff(y))
    # diffusive eigenvalue bound 4 nu (1/hx^2 + 1/hy^2) times dt within RK4's 2.78
    assert dt * 4.0 / 800.0 * (1 / hx ** 2 + 1 / hy ** 2) <= 0.7 * 2.78 + 1e-12
    assert 5e-5 < dt < 2e-4
    # a coarse grid keeps the configured step
    xs = cases.tanh_grid(64, 0.0, 30.0, 1.02)
    ys = cases.tanh_grid(64, -0.5, 0.5, 1.02)
    assert bench.bfs_dt(xs, ys, 800.0, 1e-3) == 1e-3


def test_singular_operator_detection():
    from ins2d_b200 import cases, learned
    cav = types.SimpleNamespace(BC=cases.BC_CAVITY)
    per = types.SimpleNamespace(BC=cases.BC_PERIODIC)
    chan = types.SimpleNamespace(BC=cases.BC_CHANNEL)
    assert learned.singular(cav) and learned.singular(per)
    assert not learned.singular(chan)


def test_odd_part_is_odd_and_exact_for_linear_maps():
    rng = np.random.default_rng(0)
    w = N.he_init(2).astype(np.float64)
    v = rng.standard_normal((1, 9, 11))
    yp, _ = N.forward(w, 1.0, v, bf16_mode=False)
    ym, _ = N.forward(w, 1.0, -v, bf16_mode=False)
    odd = 0.5 * (yp - ym)
    # odd in v, homogeneous of degree one
    y2p, _ = N.forward(w, 1.0, -2.0 * v, bf16_mode=False)
    y2m, _ = N.forward(w, 1.0, 2.0 * v, bf16_mode=False)
    assert np.allclose(0.5 * (y2p - y2m), -2.0 * odd, rtol=1e-12, atol=1e-12)
    # ReLU(z) - ReLU(-z) = z: one layer's odd part is linear
    z = rng.standard_normal(100)
    assert np.allclose(np.maximum(z, 0) - np.maximum(-z, 0), z)
