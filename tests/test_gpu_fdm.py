"""The fast-diagonalization preconditioner of the device PCG
(INS2D_PRECOND_FDM) on the GPU: solves on stretched grids of every
boundary-condition kind reach cg.F's stopping rule in a few iterations and
agree with the direct solve; periodic uniform grids use the FFT solve as the
preconditioner; time steps agree with the oracle."""
import numpy as np
import pytest

from oracle import ins2d_ref as R
from tests.cases_common import BC_COMBOS, grid_stretched, grid_uniform, is_closed, smooth_bc

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("combo", ["cavity", "channel", "open_x", "per_x_walls", "per_y_open", "open_y_both",
                                   "periodic"])
@pytest.mark.parametrize("shape", [(40, 28), (301, 257)])
def test_fdm_pcg_solve(combo, shape):
    import ins2d_b200
    nx, ny = shape
    x = grid_stretched(nx, 0.0, 1.7)
    y = grid_stretched(ny, -0.5, 0.5, beta=1.2)
    bc = BC_COMBOS[combo]
    uBC, vBC = smooth_bc(3, closed=is_closed(bc))
    m = ins2d_b200.Options(x, y, bc, Re=100.0, poisson=4, CG_acc=1e-12, CG_maxit=500, uBC=uBC, vBC=vBC,
                           precond="fdm")
    o = R.make_options(x, y, bc, Re=100.0, poisson=1, uBC=uBC, vBC=vBC)
    rng = np.random.default_rng(7)
    f = o.discretization.M @ rng.standard_normal(o.grid.NV) + o.discretization.yM
    dp, st = m.pressure_poisson(f, return_stats=True)
    A = o.discretization.A
    assert np.linalg.norm(A @ dp - f) <= 2e-12 * np.linalg.norm(f)
    assert st["iters"] <= 4, st
    if nx < 100:
        ref = R.pressure_poisson(f, 0.0, o)
        if is_closed(bc):
            dp, ref = dp - dp.mean(), ref - ref.mean()
        assert _rel(dp, ref) < 1e-9


def test_fdm_spectral_periodic_uniform():
    import ins2d_b200
    from ins2d_b200 import cases
    N = 256
    x = cases.uniform_grid(N, 0.0, 1.0)
    m = ins2d_b200.Options(x, x.copy(), cases.BC_PERIODIC, Re=2000.0, poisson=4, CG_acc=1e-12, precond="fdm")
    mf = ins2d_b200.Options(x, x.copy(), cases.BC_PERIODIC, Re=2000.0, poisson=6)
    rng = np.random.default_rng(4)
    f = rng.standard_normal(N * N)
    f -= f.mean()
    dp, st = m.pressure_poisson(f, return_stats=True)
    assert st["iters"] <= 2, st
    ref = mf.pressure_poisson(f)
    assert _rel(dp - dp.mean(), ref - ref.mean()) < 1e-11


@pytest.mark.parametrize("combo", ["cavity", "channel"])
def test_fdm_time_steps(combo):
    import ins2d_b200
    x = grid_stretched(48, 0.0, 1.5)
    y = grid_stretched(36, -0.5, 0.5)
    bc = BC_COMBOS[combo]
    uBC, vBC = smooth_bc(9, closed=is_closed(bc))
    o = R.make_options(x, y, bc, Re=300.0, poisson=1, uBC=uBC, vBC=vBC)
    m = ins2d_b200.Options(x, y, bc, Re=300.0, poisson=4, CG_acc=1e-13, CG_maxit=200, uBC=uBC, vBC=vBC,
                           precond="fdm")
    rng = np.random.default_rng(1)
    V0 = R.initial_projection(0.3 * rng.standard_normal(o.grid.NV), 0.0, o)
    p0 = R.pressure_additional_solve(V0, np.zeros(o.grid.Np), 0.0, o)
    V, p = V0.copy(), p0.copy()
    for n in range(4):
        V, p = R.time_ERK(V, p, n * 1e-3, 1e-3, o)
    Vg, pg, st = m.time_ERK(V0, p0, 0.0, 1e-3, nsteps=4, return_stats=True)
    assert _rel(Vg, V) < 1e-10
    assert st["iters_max"] <= 4, st


def test_fdm_too_large_rejected():
    import ins2d_b200
    x = grid_stretched(1100, 0.0, 1.0)
    y = grid_stretched(16, 0.0, 1.0)
    with pytest.raises(ins2d_b200.Ins2dError) as ei:
        ins2d_b200.Options(x, y, BC_COMBOS["cavity"], Re=100.0, poisson=4, precond="fdm")
    assert ei.value.status == 1
