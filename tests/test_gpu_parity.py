"""Parity of the CUDA path (through the C-ABI of libins2d.so) with the CPU
oracle on the same seeded inputs.  FP64 bar: 1e-12 relative for F, the
divergence, the Laplacian and the FFT solve; PCG solves to their stated
tolerance; time steps within 1e-10 relative after several steps."""
import numpy as np
import pytest

from oracle import ins2d_ref as R
from tests.cases_common import BC_COMBOS, grid_stretched, grid_uniform, is_closed, smooth_bc

pytestmark = pytest.mark.gpu


def _ins2d():
    import ins2d_b200
    return ins2d_b200


def _pair(combo, stretch, nx=12, ny=10, Re=45.0, poisson=4, CG_acc=1e-13, RK="RK44", seed=3):
    x = grid_stretched(nx, 0.0, 1.7) if stretch else grid_uniform(nx, 0.0, 1.7)
    y = grid_stretched(ny, -0.5, 0.5, beta=1.2) if stretch else grid_uniform(ny, -0.5, 0.5)
    bc = BC_COMBOS[combo]
    uBC, vBC = smooth_bc(seed, closed=is_closed(bc))
    o = R.make_options(x, y, bc, Re=Re, poisson=poisson if poisson != 4 else 1, CG_acc=CG_acc, uBC=uBC, vBC=vBC,
                       RK=RK)
    m = _ins2d().Options(x, y, bc, Re=Re, poisson=poisson, CG_acc=CG_acc, CG_maxit=20000, uBC=uBC, vBC=vBC, RK=RK)
    return o, m


def _rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


COMBOS = sorted(BC_COMBOS)


@pytest.mark.parametrize("combo", COMBOS)
@pytest.mark.parametrize("stretch", [False, True])
def test_F_divergence_laplacian(combo, stretch):
    o, m = _pair(combo, stretch)
    g = o.grid
    assert (m.Nu, m.Nv, m.Np) == (g.Nu, g.Nv, g.Np)
    rng = np.random.default_rng(11)
    V = rng.standard_normal(g.NV)
    C = rng.standard_normal(g.NV)
    p = rng.standard_normal(g.Np)
    mr_ref, F_ref = R.F(V, V, p, 0.0, o)
    mr, Fg = m.F(V, None, p, 0.0)
    assert _rel(Fg, F_ref) < 1e-12
    assert abs(mr - mr_ref) <= 1e-12 * mr_ref
    # convecting field different from the convected one (F.m:1 C argument)
    cu, cv = R.convection(V, C, 0.0, o)
    d2u, d2v = R.diffusion(V, 0.0, o)
    F_np_ref = np.r_[-cu + d2u, -cv + d2v]
    _, F_np = m.F(V, C, None, 0.0, nopressure=1)
    assert _rel(F_np, F_np_ref) < 1e-12
    # divergence M*V + yM and Laplacian A*p
    f, maxdiv = m.divergence(V)
    f_ref = o.discretization.M @ V + o.discretization.yM
    assert _rel(f, f_ref) < 1e-12
    assert abs(maxdiv - np.max(np.abs(f_ref))) <= 1e-12 * np.max(np.abs(f_ref))
    Ap = m.laplacian(p)
    assert _rel(Ap, o.discretization.A @ p) < 1e-12
    # check_conservation
    cons = m.check_conservation(V, 0.0)
    cons_ref = R.check_conservation(V, 0.0, o)
    for a, b in zip(cons, cons_ref):
        assert abs(a - b) <= 1e-12 * max(abs(b), 1.0)


@pytest.mark.parametrize("combo,nx,ny", [("cavity", 200, 140), ("channel", 200, 140), ("periodic", 128, 96),
                                          ("per_y_open", 130, 96)])
@pytest.mark.parametrize("stretch", [False, True])
def test_F_tiled_walkers(combo, nx, ny, stretch):
    """F with the pressure (C = V) runs through the stage walkers -- shared-
    memory tiles inside, table walker at the boundary -- and a separate
    max|F| reduction: against the oracle at 1e-12."""
    o, m = _pair(combo, stretch, nx=nx, ny=ny)
    g = o.grid
    rng = np.random.default_rng(17)
    V = rng.standard_normal(g.NV)
    p = rng.standard_normal(g.Np)
    mr_ref, F_ref = R.F(V, V, p, 0.0, o)
    mr, Fg = m.F(V, None, p, 0.0)
    assert _rel(Fg, F_ref) < 1e-12
    assert abs(mr - mr_ref) <= 1e-12 * mr_ref


@pytest.mark.parametrize("nx,ny", [(16, 8), (40, 40), (64, 32), (12, 10), (128, 128), (1024, 512), (2048, 2048),
                                   (8192, 64), (64, 8192), (4096, 32), (96, 1024), (256, 4096), (64, 2048)])
def test_fft_poisson(nx, ny):
    x = grid_uniform(nx, 0.0, 2 * np.pi)
    y = grid_uniform(ny, 0.0, 3.0)
    bc = BC_COMBOS["periodic"]
    o = R.make_options(x, y, bc, Re=1e100, poisson=6)
    m = _ins2d().Options(x, y, bc, Re=1e100, poisson=6)
    rng = np.random.default_rng(nx * 7 + ny)
    f = rng.standard_normal(o.grid.Np)
    f -= f.mean()
    dp_ref = R.pressure_poisson(f, 0.0, o)
    dp = m.pressure_poisson(f)
    assert _rel(dp, dp_ref) < 1e-12
    # tiny right-hand side: early return with dp = 0 (pressure_poisson.m:21-32)
    assert np.all(m.pressure_poisson(f * 1e-18) == 0.0)


@pytest.mark.parametrize("combo", ["cavity", "channel", "open_x", "per_y_open", "open_y_both"])
def test_pcg_poisson(combo):
    o, m = _pair(combo, True, nx=24, ny=20, CG_acc=1e-13)
    g = o.grid
    rng = np.random.default_rng(5)
    V = rng.standard_normal(g.NV)
    f = o.discretization.M @ V + o.discretization.yM  # a consistent right-hand side
    dp, st = m.pressure_poisson(f, return_stats=True)
    A = o.discretization.A
    assert np.linalg.norm(A @ dp - f) / np.linalg.norm(f) <= 2e-13  # CG_acc plus residual drift
    assert abs(st["norm1"] - np.linalg.norm(A @ dp - f) / np.linalg.norm(f)) < 1e-13
    assert 0 < st["iters"] < 20000
    dp_ref = R.pressure_poisson(f, 0.0, o)  # direct solve
    singular = not any(t == "pres" for t in (o.BC.u.left, o.BC.u.right, o.BC.v.low, o.BC.v.up))
    if singular:
        dp = dp - dp.mean()
        dp_ref = dp_ref - dp_ref.mean()
    assert _rel(dp, dp_ref) < 1e-10


def test_pcg_not_converged_reports_error():
    o, m = _pair("cavity", False, nx=24, ny=20)
    m2 = _ins2d().Options(o.grid.x, o.grid.y, BC_COMBOS["cavity"], Re=45.0, poisson=4, CG_acc=1e-14, CG_maxit=2,
                          precond="mg")
    f = o.discretization.M @ np.random.default_rng(1).standard_normal(o.grid.NV) + o.discretization.yM
    with pytest.raises(_ins2d().Ins2dError) as ei:
        m2.pressure_poisson(f)
    assert ei.value.status == 2  # INS2D_ENOTCONV (cg.F:262)


@pytest.mark.parametrize("combo", COMBOS)
@pytest.mark.parametrize("rk", ["RK44", "RK33P2"])
def test_erk_steps(combo, rk):
    o, m = _pair(combo, True, nx=14, ny=12, CG_acc=1e-13, RK=rk)
    g = o.grid
    rng = np.random.default_rng(2)
    V0 = R.initial_projection(0.3 * rng.standard_normal(g.NV), 0.0, o)
    p0 = R.pressure_additional_solve(V0, np.zeros(g.Np), 0.0, o)
    V, p = V0.copy(), p0.copy()
    for n in range(3):
        V, p = R.time_ERK(V, p, n * 0.01, 0.01, o)
    Vg, pg = m.time_ERK(V0, p0, 0.0, 0.01, nsteps=3)
    assert _rel(Vg, V) < 1e-10
    singular = not any(t == "pres" for t in (o.BC.u.left, o.BC.u.right, o.BC.v.low, o.BC.v.up))
    if singular:
        pg = pg - pg.mean()
        p = p - p.mean()
    assert _rel(pg, p) < 1e-9
    assert m.check_conservation(Vg, 0.03)[0] < 1e-10


def test_erk_fft_taylor_green():
    N = 32
    x = grid_uniform(N, 0.0, 2 * np.pi)
    bc = BC_COMBOS["periodic"]
    o = R.make_options(x, x.copy(), bc, Re=1e100, poisson=6)
    m = _ins2d().Options(x, x.copy(), bc, Re=1e100, poisson=6)
    g = o.grid
    V0 = np.r_[np.sin(g.xu) * np.cos(g.yu), -np.cos(g.xv) * np.sin(g.yv)]
    p0 = np.zeros(g.Np)
    V, p = V0.copy(), p0.copy()
    for n in range(5):
        V, p = R.time_ERK(V, p, n * 1e-2, 1e-2, o)
    Vg, pg = m.time_ERK(V0, p0, 0.0, 1e-2, nsteps=5)
    assert _rel(Vg, V) < 1e-12
    assert _rel(pg - pg.mean(), p - p.mean()) < 1e-10
    k0 = R.check_conservation(V0, 0.0, o)[3]
    kg = m.check_conservation(Vg, 0.05)[3]
    kr = R.check_conservation(V, 0.05, o)[3]
    assert abs((kg - k0) - (kr - k0)) < 1e-14 * k0 + 1e-3 * abs(kr - k0)


@pytest.mark.parametrize("combo", ["cavity", "periodic", "channel", "open_x", "per_y_open"])
def test_erk_steps_large_grid(combo):
    """Grids with several 64x32 tiles per direction, so the interior tiles
    take the fast stencil path and the boundary tiles the table path."""
    o, m = _pair(combo, True, nx=200, ny=140, CG_acc=1e-12, RK="RK44")
    g = o.grid
    rng = np.random.default_rng(9)
    V0 = R.initial_projection(0.3 * rng.standard_normal(g.NV), 0.0, o)
    p0 = R.pressure_additional_solve(V0, np.zeros(g.Np), 0.0, o)
    V, p = V0.copy(), p0.copy()
    for n in range(2):
        V, p = R.time_ERK(V, p, n * 1e-3, 1e-3, o)
    Vg, pg = m.time_ERK(V0, p0, 0.0, 1e-3, nsteps=2)
    assert _rel(Vg, V) < 1e-9
    # the additional-solve residual (fast walker in residual mode) through p
    if not is_closed(BC_COMBOS[combo]):
        assert _rel(pg, p) < 1e-8


def test_erk_fft_large_grid():
    N = 256
    x = grid_uniform(N, 0.0, 1.0)
    bc = BC_COMBOS["periodic"]
    uBC, vBC = smooth_bc(4, closed=True)
    o = R.make_options(x, x.copy(), bc, Re=500.0, poisson=6)
    m = _ins2d().Options(x, x.copy(), bc, Re=500.0, poisson=6)
    g = o.grid
    rng = np.random.default_rng(12)
    V0 = R.initial_projection(rng.standard_normal(g.NV), 0.0, o)
    V, p = V0.copy(), np.zeros(g.Np)
    for n in range(3):
        V, p = R.time_ERK(V, p, n * 1e-4, 1e-4, o)
    Vg, pg = m.time_ERK(V0, np.zeros(g.Np), 0.0, 1e-4, nsteps=3)
    assert _rel(Vg, V) < 1e-12
    assert _rel(pg - pg.mean(), p - p.mean()) < 1e-10


@pytest.mark.parametrize("rk", ["RK44", "RK33P2"])
@pytest.mark.parametrize("poisson,stretch", [(6, False), (4, False), (4, True)])
def test_erk_whole_tile_grid(rk, poisson, stretch):
    """Periodic grid of whole 64x32 walker tiles: only the tiled walkers run
    (no table-walker launch).  Runs of several steps (first stage from the
    cached residual; CUDA graphs, PCG loops on the device) and single steps
    (first stage from V; host-polled PCG) against the oracle."""
    o, m = _pair("periodic", stretch, nx=128, ny=96, Re=300.0, poisson=poisson, CG_acc=1e-13, RK=rk)
    g = o.grid
    rng = np.random.default_rng(21)
    V0 = R.initial_projection(0.5 * rng.standard_normal(g.NV), 0.0, o)
    p0 = R.pressure_additional_solve(V0, np.zeros(g.Np), 0.0, o)
    dt = 2e-4
    V, p = V0.copy(), p0.copy()
    for n in range(3):
        V, p = R.time_ERK(V, p, n * dt, dt, o)
    Vg, pg = m.time_ERK(V0, p0, 0.0, dt, nsteps=3)
    Vs, ps = V0.copy(), p0.copy()
    for n in range(3):
        Vs, ps = m.time_ERK(Vs, ps, n * dt, dt, nsteps=1)
    tol = 1e-12 if poisson == 6 else 1e-10
    assert _rel(Vg, V) < tol
    assert _rel(Vs, V) < tol
    assert _rel(pg - pg.mean(), p - p.mean()) < 1e2 * tol
    assert _rel(ps - ps.mean(), p - p.mean()) < 1e2 * tol
    assert m.check_conservation(Vg, 3 * dt)[0] < 1e-10


@pytest.mark.parametrize("combo", ["cavity", "channel", "periodic", "per_y_open", "open_x"])
@pytest.mark.parametrize("shape", [(24, 20), (301, 257)])
@pytest.mark.parametrize("precond", ["mg", "jacobi", "fdm"])
def test_pcg_preconditioners(combo, shape, precond):
    """Multigrid, Jacobi and fast-diagonalization preconditioned CG reach the stated tolerance and
    agree with the oracle's direct solve, one thread block (24x20) and
    multi-block (301x257) paths; multigrid needs few iterations on stretched
    grids."""
    nx, ny = shape
    bc = BC_COMBOS[combo]
    perx, pery = bc["u"]["left"] == "per", bc["v"]["low"] == "per"
    x = grid_uniform(nx, 0.0, 1.7) if perx else grid_stretched(nx, 0.0, 1.7)
    y = grid_uniform(ny, -0.5, 0.5) if pery else grid_stretched(ny, -0.5, 0.5, beta=1.2)
    if precond == "jacobi" and nx > 100 and combo != "periodic":
        pytest.skip("Jacobi-preconditioned CG on the large stretched grid takes too many iterations for a test")
    o = R.make_options(x, y, bc, poisson=1)
    m = _ins2d().Options(x, y, bc, poisson=4, CG_acc=1e-11, CG_maxit=50000, precond=precond)
    rng = np.random.default_rng(nx + ny)
    V = rng.standard_normal(o.grid.NV)
    f = o.discretization.M @ V + o.discretization.yM
    dp, st = m.pressure_poisson(f, return_stats=True)
    A = o.discretization.A
    res = np.linalg.norm(A @ dp - f) / np.linalg.norm(f)
    assert res <= 2e-11
    if precond == "mg":
        assert st["iters"] <= 40, st
    if precond == "fdm":
        assert st["iters"] <= 4, st
    dp_ref = R.pressure_poisson(f, 0.0, o)
    if is_closed(bc):
        dp, dp_ref = dp - dp.mean(), dp_ref - dp_ref.mean()
    assert _rel(dp, dp_ref) < 1e-8


@pytest.mark.parametrize("poisson,precond", [(4, "mg"), (4, "jacobi"), (4, "fdm")])
def test_nonfinite_rhs_reports_error(poisson, precond):
    """A NaN in the right-hand side ends the solve with INS2D_ENONFINITE (the
    device path reports it as a status; no fault, the context stays usable)."""
    o, _ = _pair("cavity", False, nx=24, ny=20)
    m = _ins2d().Options(o.grid.x, o.grid.y, BC_COMBOS["cavity"], Re=45.0, poisson=poisson, CG_acc=1e-12,
                         precond=precond)
    f = o.discretization.M @ np.random.default_rng(1).standard_normal(o.grid.NV) + o.discretization.yM
    bad = f.copy()
    bad[7] = np.nan
    with pytest.raises(_ins2d().Ins2dError) as ei:
        m.pressure_poisson(bad)
    assert ei.value.status == 4  # INS2D_ENONFINITE
    dp = m.pressure_poisson(f)  # the context still works
    assert np.linalg.norm(o.discretization.A @ dp - f) <= 2e-12 * np.linalg.norm(f)
