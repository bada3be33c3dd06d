"""The CUDA path against the reference's own logged runs
(results/*/convergence.txt, extracted into tests/golden/ by
tests/golden/make_golden.py): per-step residual max|F|, divergence and kinetic
energy to the printed 9 digits."""
import json
import os

import numpy as np
import pytest

from tests.cases_common import BC_COMBOS

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    with open(os.path.join(GOLDEN, name)) as fh:
        return np.array(json.load(fh)["rows"])


def _lid(x, y, t):
    n = np.size(x) * np.size(y)
    return np.ones(n) if (np.size(y) == 1 and abs(float(y) - 1.0) < 1e-10) else np.zeros(n)


def _history(m, V, p, dt, nsteps):
    import torch
    Vd = torch.tensor(V, dtype=torch.float64, device="cuda")
    pd = torch.tensor(p, dtype=torch.float64, device="cuda")
    hist = [(m.F(Vd, None, pd, 0.0)[0],) + m.check_conservation(Vd, 0.0)]
    for n in range(1, nsteps + 1):
        m.time_ERK(Vd, pd, (n - 1) * dt, dt)
        hist.append((m.F(Vd, None, pd, n * dt)[0],) + m.check_conservation(Vd, n * dt))
    return np.array(hist)  # res, maxdiv, umom, vmom, k


def test_ldc_re100_log():
    import ins2d_b200
    ref = _load("ldc_re100_20x20.json")
    x = np.arange(21) / 20.0
    m = ins2d_b200.Options(x, x.copy(), BC_COMBOS["cavity"], Re=100.0, poisson=4, CG_acc=1e-15, CG_maxit=5000,
                           uBC=_lid, RK="RK33P2")
    V = np.zeros(m.NV)
    p = m.pressure_additional_solve(V, np.zeros(m.Np), 0.0)  # p_initial (input_check.m:126-128)
    h = _history(m, V, p, 0.01, 100)
    np.testing.assert_allclose(h[:, 0], ref[:, 3], rtol=1e-8)
    np.testing.assert_allclose(h[1:, 4], ref[1:, 7], rtol=1e-8)
    assert np.all(h[:, 1] < 1e-14)


def test_shear_layer_log():
    import ins2d_b200
    ref = _load("shear_layer_40x40.json")
    N = 40
    x = 2 * np.pi * np.arange(N + 1) / N
    m = ins2d_b200.Options(x, x.copy(), BC_COMBOS["periodic"], Re=1e100, poisson=6, RK="RK44")
    d, e = np.pi / 15, 0.05
    u = 1 + np.tanh((m.yu - np.pi / 2) / d) * (m.yu <= np.pi) + np.tanh((3 * np.pi / 2 - m.yu) / d) * (m.yu > np.pi)
    v = e * np.sin(m.xv)
    V = np.r_[u, v]
    p = m.pressure_additional_solve(V, np.zeros(m.Np), 0.0)
    h = _history(m, V, p, 0.01, 400)
    np.testing.assert_allclose(h[:, 0], ref[:, 3], rtol=2e-8)
    np.testing.assert_allclose(h[:, 2], ref[:, 5], rtol=1e-8)
    np.testing.assert_allclose(h[:, 4], ref[:, 7], rtol=1e-8)
    assert np.max(h[:, 1]) < 1e-13
