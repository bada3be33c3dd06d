"""Ensembles (ins2d_ens_*): members of different grids, boundary conditions
and Re advanced together must reproduce each member's own single-context
run (the batched launches use the same per-cell arithmetic; the PCG solves
agree to the solver tolerance)."""
import numpy as np
import pytest

from ins2d_b200 import cases

pytestmark = pytest.mark.gpu


def _members(seed, n, sizes, stretch=1.05, precond="default"):
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n):
        nx, ny = (int(v) for v in rng.choice(sizes, 2))
        U = float(rng.uniform(0.5, 1.5))
        Re = float(rng.uniform(100.0, 5000.0))
        if m % 2 == 0:
            x = cases.tanh_grid(nx, 0.0, 1.0, stretch)
            y = cases.tanh_grid(ny, 0.0, 1.0, stretch)
            out.append(dict(x=x, y=y, BC=cases.BC_CAVITY, Re=Re, uBC=cases.lid_uBC(U, 1.0)))
        else:
            x = cases.tanh_grid(nx, 0.0, 4.0, stretch)
            y = cases.tanh_grid(ny, -0.5, 0.5, stretch)
            out.append(dict(x=x, y=y, BC=cases.BC_CHANNEL, Re=Re,
                            uBC=cases.channel_uBC(lambda yy, U=U: U * (1 - 4 * np.asarray(yy) ** 2))))
    # the single contexts the members are compared with take the same
    # preconditioner setting (default: fast diagonalization; mg: multigrid)
    for kw in out:
        kw.update(poisson=4, CG_acc=1e-12, CG_maxit=20000, RK="RK44", precond=precond)
    return out


@pytest.mark.parametrize("seed,n,sizes", [(4, 6, [24, 32, 40, 64]), (5, 9, [16, 48, 96, 130])])
@pytest.mark.parametrize("solver,precond", [(-1, "default"), (0, "default"), (-1, "mg"), (0, "mg"), (512, "mg")])
def test_ensemble_matches_single_runs(seed, n, sizes, solver, precond):
    """solver -1: tuned form; 0: solves batched across members; 512:
    persistent member solve.  precond default: the batched solves with fast
    diagonalization (four products over all members' tiles per application);
    mg: the members' V-cycles."""
    import ins2d_b200
    members = _members(seed, n, sizes, precond=precond)
    ens = ins2d_b200.Ensemble(members)
    ens.set_solver(solver)
    singles, states = [], []
    for m, kw in enumerate(members):
        o = ins2d_b200.Options(**kw)
        V0 = np.zeros(o.NV)
        p0 = o.pressure_additional_solve(V0, np.zeros(o.Np), 0.0)
        ens.set_state(m, V0, p0)
        singles.append(o)
        states.append((V0, p0))
    dt, nsteps = 2e-3, 6
    stats = ens.time_ERK(0.0, dt, nsteps)
    shape = ens.solve_shape()
    assert shape["threads"] in (0, 256, 512)
    if solver >= 0:
        assert shape["threads"] == solver
    for m, o in enumerate(singles):
        V, p = o.time_ERK(*states[m], 0.0, dt, nsteps=nsteps)
        Ve, pe = ens.get_state(m)
        scale = max(np.max(np.abs(V)), 1e-30)
        assert np.max(np.abs(Ve - V)) <= 1e-10 * scale, m
        assert np.max(np.abs(pe - p)) <= 1e-8 * max(np.max(np.abs(p)), 1e-30), m
        assert stats[m]["n_solves"] == 4 * nsteps  # 3 stage solves + 1 additional per RK4 step
        assert stats[m]["iters_max"] <= (4 if precond == "default" else 60)
        # the member context still serves the single-flow API on the ensemble's state
        assert ens.member(m).check_conservation(Ve, nsteps * dt)[0] < 1e-10


def test_ensemble_fdm_solves_batched():
    """An ensemble with the fast-diagonalization preconditioner refuses the
    persistent per-member solve form (its V-cycle is not the same
    preconditioner) and keeps the batched form."""
    import ins2d_b200
    ens = ins2d_b200.Ensemble(_members(2, 3, [24, 32]))
    with pytest.raises(ins2d_b200.Ins2dError) as ei:
        ens.set_solver(512)
    assert ei.value.status == 1
    ens.set_solver(0)
    ens.close()


def test_ensemble_rejects_unsupported_members():
    """Mixed solver settings, unsteady boundary conditions and the FFT solver
    are refused with EINVAL (no member is advanced)."""
    import ins2d_b200
    members = _members(1, 2, [16, 24])
    members[1]["CG_acc"] = 1e-6
    with pytest.raises(ins2d_b200.Ins2dError) as ei:
        ins2d_b200.Ensemble(members)
    assert ei.value.status == 1
    members = _members(1, 2, [16, 24])
    members[0]["BC"] = dict(members[0]["BC"], BC_unsteady=1)
    with pytest.raises(ins2d_b200.Ins2dError) as ei:
        ins2d_b200.Ensemble(members)
    assert ei.value.status == 1
    x = cases.uniform_grid(16, 0.0, 1.0)
    with pytest.raises(ins2d_b200.Ins2dError) as ei:
        ins2d_b200.Ensemble([dict(x=x, y=x.copy(), BC=cases.BC_PERIODIC, Re=100.0, poisson=6)])
    assert ei.value.status == 1


def test_ensemble_reports_failing_member():
    """A member whose state holds a NaN makes the run return ENONFINITE naming
    that member; the other members are still advanced."""
    import ins2d_b200
    members = _members(3, 3, [24, 32])
    ens = ins2d_b200.Ensemble(members)
    ens.set_solver(0)
    for m in range(3):
        o = ens.member(m)
        V = np.zeros(o.NV)
        if m == 1:
            V[5] = np.nan
        ens.set_state(m, V, np.zeros(o.Np))
    with pytest.raises(ins2d_b200.Ins2dError) as ei:
        ens.time_ERK(0.0, 1e-3, 1)
    assert ei.value.status == 4 and "member 1" in str(ei.value)
    V0, _ = ens.get_state(0)
    assert np.all(np.isfinite(V0)) and np.max(np.abs(V0)) > 0.0
