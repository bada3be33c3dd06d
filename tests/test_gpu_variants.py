"""Variants of the time step against the oracle: unsteady boundary
conditions (time_ERK.m:69-71, 108-113, 152-165 with BC_unsteady = 1, with and
without the additional pressure solve), and the FP32-stencil precision mode
against the FP64 path (drift bounded by single-precision rounding)."""
import numpy as np
import pytest

from oracle import ins2d_ref as R
from tests.cases_common import BC_COMBOS, grid_stretched, grid_uniform, smooth_bc, unsteady_bc

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("combo", ["channel", "open_x", "open_y"])
@pytest.mark.parametrize("p_add_solve", [1, 0])
def test_erk_unsteady_bc(combo, p_add_solve):
    import ins2d_b200
    x = grid_stretched(18, 0.0, 1.7)
    y = grid_stretched(14, -0.5, 0.5, beta=1.2)
    bc = dict(BC_COMBOS[combo], BC_unsteady=1)
    uBC, vBC, dudtBC, dvdtBC = unsteady_bc(7)
    kw = dict(Re=60.0, CG_acc=1e-13, uBC=uBC, vBC=vBC, dudtBC=dudtBC, dvdtBC=dvdtBC, p_add_solve=p_add_solve,
              RK="RK44")
    o = R.make_options(x, y, bc, poisson=1, **kw)
    m = ins2d_b200.Options(x, y, bc, poisson=4, CG_maxit=20000, **kw)
    g = o.grid
    rng = np.random.default_rng(4)
    V0 = R.initial_projection(0.3 * rng.standard_normal(g.NV), 0.0, o)
    p0 = R.pressure_additional_solve(V0, np.zeros(g.Np), 0.0, o)
    V, p = V0.copy(), p0.copy()
    for n in range(3):
        V, p = R.time_ERK(V, p, 0.2 + n * 0.01, 0.01, o)
    Vg, pg = m.time_ERK(V0, p0, 0.2, 0.01, nsteps=3)
    assert _rel(Vg, V) < 1e-10
    assert _rel(pg, p) < 1e-8
    # the boundary data moved with t: divergence-free to the solver tolerance at t_end
    assert m.check_conservation(Vg, 0.23)[0] < 1e-9


def test_fp32_stencil_periodic():
    """FP32 convection/diffusion on a 256^2 periodic grid: after 10 RK4 steps
    the velocity stays within 1e-5 (relative) of the FP64 run and the field
    stays divergence-free (the projection is FP64)."""
    import ins2d_b200
    N = 256
    x = grid_uniform(N, 0.0, 1.0)
    bc = BC_COMBOS["periodic"]
    m64 = ins2d_b200.Options(x, x.copy(), bc, Re=2000.0, poisson=6)
    m32 = ins2d_b200.Options(x, x.copy(), bc, Re=2000.0, poisson=6, precision="fp32")
    o = R.make_options(x, x.copy(), bc, Re=2000.0, poisson=6)
    rng = np.random.default_rng(8)
    V0 = R.initial_projection(rng.standard_normal(o.grid.NV), 0.0, o)
    p0 = np.zeros(o.grid.Np)
    V64, p64 = m64.time_ERK(V0, p0, 0.0, 2e-4, nsteps=10)
    V32, p32 = m32.time_ERK(V0, p0, 0.0, 2e-4, nsteps=10)
    assert _rel(V32, V64) < 1e-5
    assert _rel(V32, V64) > 0.0  # the FP32 stencils really ran
    assert m32.check_conservation(V32, 0.0)[0] < 1e-10
    k64 = m64.check_conservation(V64, 0.0)[3]
    k32 = m32.check_conservation(V32, 0.0)[3]
    assert abs(k32 - k64) < 1e-5 * k64


def test_fp32_stencil_channel():
    """FP32 stencils on a stretched channel (table walkers at the boundaries,
    PCG pressure): within 1e-5 of the FP64 run after 5 steps."""
    import ins2d_b200
    x = grid_stretched(96, 0.0, 4.0)
    y = grid_stretched(48, -0.5, 0.5, beta=1.2)
    bc = BC_COMBOS["channel"]
    uBC, vBC = smooth_bc(2)
    kw = dict(Re=100.0, poisson=4, CG_acc=1e-12, CG_maxit=20000, uBC=uBC, vBC=vBC)
    m64 = ins2d_b200.Options(x, y, bc, **kw)
    m32 = ins2d_b200.Options(x, y, bc, precision="fp32", **kw)
    o = R.make_options(x, y, bc, Re=100.0, poisson=1, uBC=uBC, vBC=vBC)
    rng = np.random.default_rng(6)
    V0 = R.initial_projection(0.2 * rng.standard_normal(o.grid.NV), 0.0, o)
    p0 = R.pressure_additional_solve(V0, np.zeros(o.grid.Np), 0.0, o)
    V64, _ = m64.time_ERK(V0, p0, 0.0, 1e-3, nsteps=5)
    V32, _ = m32.time_ERK(V0, p0, 0.0, 1e-3, nsteps=5)
    assert 0.0 < _rel(V32, V64) < 1e-5
