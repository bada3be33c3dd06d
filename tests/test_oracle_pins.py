"""The oracle against the reference's own logged results and the algebraic
invariants the reference checks at run time.  CPU only."""
import json
import os

import numpy as np
import pytest

from oracle import ins2d_ref as R
from tests.cases_common import BC_COMBOS, grid_stretched, grid_uniform, smooth_bc

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    with open(os.path.join(GOLDEN, name)) as fh:
        return np.array(json.load(fh)["rows"])


def _lid(x, y, t):
    n = np.size(x) * np.size(y)
    return np.ones(n) if (np.size(y) == 1 and abs(float(y) - 1.0) < 1e-10) else np.zeros(n)


def test_ldc_re100_log():
    """results/LDC_unsteady_1.000e+02_20x20_0/convergence.txt (101 rows):
    residual, divergence and kinetic energy per step, to the 9 printed digits."""
    ref = _load("ldc_re100_20x20.json")
    x, _ = R.nonuniform_grid(1 / 20, 0, 1, 1)
    cav = BC_COMBOS["cavity"]
    o = R.make_options(x, x.copy(), cav, Re=100.0, poisson=1, uBC=_lid, RK="RK33P2")
    _, _, hist = R.run(o, np.zeros(o.grid.NV), np.zeros(o.grid.Np), 0.01, 100, log=True)
    h = np.array(hist)
    assert h.shape[0] == ref.shape[0]
    np.testing.assert_allclose(h[:, 2], ref[:, 3], rtol=1e-8)      # res
    np.testing.assert_allclose(h[1:, 6], ref[1:, 7], rtol=1e-8)    # k
    assert np.all(h[:, 3] < 1e-15) and np.all(ref[:, 4] < 1e-15)   # maxdiv


def test_shear_layer_log():
    """results/shear_layer01/convergence.txt (401 rows): inviscid periodic
    shear layer on 40x40, RK44 + FFT; energy conserved to 9 digits."""
    ref = _load("shear_layer_40x40.json")
    N = 40
    x, _ = R.nonuniform_grid(2 * np.pi / N, 0, 2 * np.pi, 1)
    o = R.make_options(x, x.copy(), BC_COMBOS["periodic"], Re=1e100, poisson=6, RK="RK44")
    g = o.grid
    d, e = np.pi / 15, 0.05
    u = 1 + np.tanh((g.yu - np.pi / 2) / d) * (g.yu <= np.pi) + np.tanh((3 * np.pi / 2 - g.yu) / d) * (g.yu > np.pi)
    v = e * np.sin(g.xv)
    _, _, hist = R.run(o, np.r_[u, v], np.zeros(g.Np), 0.01, 400, log=True)
    h = np.array(hist)
    np.testing.assert_allclose(h[:, 2], ref[:, 3], rtol=2e-8)   # res
    np.testing.assert_allclose(h[:, 4], ref[:, 5], rtol=1e-8)   # umom
    np.testing.assert_allclose(h[:, 6], ref[:, 7], rtol=1e-8)   # k
    assert np.max(np.abs(h[:, 6] - h[0, 6])) / h[0, 6] < 1e-8


@pytest.mark.parametrize("combo", sorted(BC_COMBOS))
@pytest.mark.parametrize("stretch", [False, True])
def test_operator_invariants(combo, stretch):
    """operator_divergence.m:295-300 (zero row sums of A without 'pres' BC),
    A = M*Om_inv*G, G = -M', and check_symmetry.m (skew-symmetric convection
    for a divergence-free field)."""
    gx = grid_stretched(9, 0, 1.3) if stretch else grid_uniform(9, 0, 1.3)
    gy = grid_stretched(7, -0.5, 0.5) if stretch else grid_uniform(7, -0.5, 0.5)
    bc = BC_COMBOS[combo]
    uBC, vBC = smooth_bc(1)
    o = R.make_options(gx, gy, bc, Re=50.0, poisson=4, uBC=uBC, vBC=vBC)
    d, g = o.discretization, o.grid
    A2 = d.M @ R.diagm(g.Om_inv) @ d.G
    assert abs(A2 - d.A).max() < 1e-12
    assert abs(d.G + d.M.T).max() == 0
    has_pres = "pres" in (bc["u"]["left"], bc["u"]["right"], bc["v"]["low"], bc["v"]["up"])
    if not has_pres:
        assert np.max(np.abs(d.A @ np.ones(g.Np))) < 1e-10
    # a divergence-free field with homogeneous BCs: project a random field
    o0 = R.make_options(gx, gy, bc, Re=50.0, poisson=1)
    rng = np.random.default_rng(0)
    V = R.initial_projection(rng.standard_normal(o0.grid.NV), 0.0, o0)
    ok, err = R.check_symmetry(V, 0.0, o0)
    if not has_pres:  # check_symmetry.m:36-45 flags an error only without outflow
        assert err < 1e-13


def test_cg_dic_matches_direct():
    """The DIC-PCG restatement solves the pressure system to its tolerance."""
    x = grid_stretched(24, 0, 2.0)
    y = grid_uniform(16, 0, 1.0)
    o = R.make_options(x, y, BC_COMBOS["channel"], Re=100.0, poisson=4, CG_acc=1e-13)
    rng = np.random.default_rng(3)
    f = rng.standard_normal(o.grid.Np)
    dp = R.pressure_poisson(f, 0.0, o)
    it = o.solversettings.last_iter
    assert 0 < it < 200
    r = o.discretization.A @ dp - f
    assert np.linalg.norm(r) / np.linalg.norm(f) < 1e-12


def test_periodic_c_restatement_matches_scipy_oracle():
    """oracle/erk_periodic.c (the timed CPU baseline) against the scipy
    restatement of time_ERK on periodic grids: same steps to round-off."""
    import numpy as np
    from oracle import ins2d_ref as R
    for (nx, ny, L, Re) in ((32, 16, (2 * np.pi, 3.0), 1e100), (16, 32, (1.0, 1.0), 300.0)):
        x = L[0] * np.arange(nx + 1) / nx
        y = L[1] * np.arange(ny + 1) / ny
        bc = dict(u=dict(left="per", right="per", low="per", up="per"),
                  v=dict(left="per", right="per", low="per", up="per"))
        o = R.make_options(x, y, bc, Re=Re, poisson=6)
        rng = np.random.default_rng(nx)
        V0 = R.initial_projection(rng.standard_normal(o.grid.NV), 0.0, o)
        p0 = np.zeros(o.grid.Np)
        V, p = V0.copy(), p0.copy()
        for n in range(3):
            V, p = R.time_ERK(V, p, n * 1e-3, 1e-3, o)
        Vc, pc = R.erk_periodic_c(V0, p0, nx, ny, L[0], L[1], Re, 1e-3, 3)
        assert np.max(np.abs(Vc - V)) <= 1e-12 * np.max(np.abs(V))
        assert np.max(np.abs((pc - pc.mean()) - (p - p.mean()))) <= 1e-10 * np.max(np.abs(p))
