"""Host-side behaviour of the C-ABI on the GPU: ordering after torch's stream,
the host's bounded wait on the PCG convergence flag (INS2D_ETIMEOUT), the
initial projection of input_check.m:95-111, and the skew-symmetry and
energy conservation of the device's convection operator
(check_symmetry.m:42-61; the semi-discrete energy identity V' conv(V) = 0)."""
import numpy as np
import pytest

from oracle import ins2d_ref as R
from tests.cases_common import BC_COMBOS, grid_stretched, grid_uniform, is_closed, smooth_bc

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def test_device_inputs_wait_for_torch_stream():
    """An input tensor still being written by a torch kernel (queued behind a
    long device sleep) is read only after that kernel has finished."""
    import torch
    import ins2d_b200
    N = 256
    x = grid_uniform(N, 0.0, 1.0)
    m = ins2d_b200.Options(x, x.copy(), BC_COMBOS["periodic"], Re=500.0, poisson=6)
    rng = np.random.default_rng(3)
    a = rng.standard_normal(m.NV)
    b = rng.standard_normal(m.NV)
    p = rng.standard_normal(m.Np)
    _, F_ref = m.F(a + b, None, p, 0.0)
    f_ref, _ = m.divergence(a + b)
    ad, bd = torch.tensor(a, device="cuda"), torch.tensor(b, device="cuda")
    pd = torch.tensor(p, device="cuda")
    torch.cuda.synchronize()
    for call in ("F", "divergence"):
        torch.cuda._sleep(200_000_000)  # keeps torch's stream busy well past the library's launch
        Vd = ad + bd                    # queued behind the sleep
        if call == "F":
            _, Fd = m.F(Vd, None, pd, 0.0)
            assert _rel(Fd.cpu().numpy(), F_ref) < 1e-14
        else:
            fd, _ = m.divergence(Vd)
            assert _rel(fd.cpu().numpy(), f_ref) < 1e-14


def test_pcg_poll_limit_timeout():
    """A grid solved by the host-driven multi-launch PCG (more than 65536
    cells): with a zero poll limit the solve returns INS2D_ETIMEOUT instead of
    waiting, and the context stays usable."""
    import ins2d_b200
    from ins2d_b200 import _lib
    x = grid_stretched(300, 0.0, 1.0)
    y = grid_stretched(260, 0.0, 1.0)
    bc = BC_COMBOS["cavity"]
    m = ins2d_b200.Options(x, y, bc, Re=100.0, poisson=4, CG_acc=1e-10)
    rng = np.random.default_rng(2)
    f, _ = m.divergence(rng.standard_normal(m.NV))
    f -= f.mean()
    lib = _lib.load()
    assert lib.ins2d_set_poll_limit(m._ctx, 0) == 0
    with pytest.raises(ins2d_b200.Ins2dError) as ei:
        m.pressure_poisson(f)
    assert ei.value.status == _lib.ETIMEOUT
    assert "iteration limit" in str(ei.value)
    assert lib.ins2d_set_poll_limit(m._ctx, -1) == 0
    dp, st = m.pressure_poisson(f, return_stats=True)
    assert st["norm1"] <= 1e-10
    assert np.linalg.norm(m.laplacian(dp) - f) <= 1.5e-10 * np.linalg.norm(f)


@pytest.mark.parametrize("precond", ["fdm", "mg", "jacobi"])
def test_pcg_step_graph_matches_host_loop(precond):
    """A run of several steps captures each step as a CUDA graph in which the
    PCG iteration loops are conditional WHILE nodes (no host round trip);
    single steps run the host-polled loop.  Both take the same iterations and
    give the same states (grid above the single-block solver's size)."""
    import ins2d_b200
    x = grid_stretched(300, 0.0, 1.0)
    y = grid_stretched(260, 0.0, 1.0)
    bc = BC_COMBOS["cavity"]
    uBC, vBC = smooth_bc(5, closed=True)
    m = ins2d_b200.Options(x, y, bc, Re=200.0, poisson=4, CG_acc=1e-10, CG_maxit=50000, uBC=uBC, vBC=vBC,
                           precond=precond)
    V0 = np.zeros(m.NV)
    p0 = np.zeros(m.Np)
    dt = 1e-4
    Vg, pg, sg = m.time_ERK(V0, p0, 0.0, dt, nsteps=3, return_stats=True)
    Vh, ph = V0.copy(), p0.copy()
    iters = 0
    for n in range(3):
        Vh, ph, sh = m.time_ERK(Vh, ph, n * dt, dt, nsteps=1, return_stats=True)
        iters += sh["iters_total"]
    assert sg["n_solves"] == 12
    assert sg["iters_total"] == iters
    assert _rel(Vg, Vh) < 1e-13
    assert _rel(pg, ph) < 1e-12


def test_pcg_step_graph_loop_limit():
    """The device-side iteration loop of a step graph ends at its pass limit
    (a zero poll limit: no pass) and the run reports INS2D_ETIMEOUT; the
    context stays usable."""
    import ins2d_b200
    from ins2d_b200 import _lib
    x = grid_stretched(300, 0.0, 1.0)
    y = grid_stretched(260, 0.0, 1.0)
    uBC, vBC = smooth_bc(5, closed=True)
    m = ins2d_b200.Options(x, y, BC_COMBOS["cavity"], Re=200.0, poisson=4, CG_acc=1e-10, uBC=uBC, vBC=vBC,
                           precond="mg")
    lib = _lib.load()
    assert lib.ins2d_set_poll_limit(m._ctx, 0) == 0
    with pytest.raises(ins2d_b200.Ins2dError) as ei:
        m.time_ERK(np.zeros(m.NV), np.zeros(m.Np), 0.0, 1e-4, nsteps=2)
    assert ei.value.status == _lib.ETIMEOUT
    assert "iteration-loop limit" in str(ei.value)
    assert lib.ins2d_set_poll_limit(m._ctx, -1) == 0
    V, p, st = m.time_ERK(np.zeros(m.NV), np.zeros(m.Np), 0.0, 1e-4, nsteps=2, return_stats=True)
    assert st["n_solves"] == 8 and st["norm1_max"] <= 1e-10


@pytest.mark.parametrize("combo", ["cavity", "channel", "periodic", "per_x_walls"])
def test_initial_projection(combo):
    """input_check.m:95-111 on the device against the oracle: a random field
    with the case's boundary values is projected to max|div| < 1e-12."""
    import ins2d_b200
    x = grid_stretched(20, 0.0, 1.5) if combo != "periodic" else grid_uniform(20, 0.0, 1.5)
    y = grid_stretched(16, -0.5, 0.5) if combo != "periodic" else grid_uniform(16, -0.5, 0.5)
    bc = BC_COMBOS[combo]
    uBC, vBC = smooth_bc(5, closed=is_closed(bc))
    poisson = 6 if combo == "periodic" else 4
    o = R.make_options(x, y, bc, Re=100.0, poisson=poisson if poisson == 6 else 1, uBC=uBC, vBC=vBC)
    m = ins2d_b200.Options(x, y, bc, Re=100.0, poisson=poisson, CG_acc=1e-14, CG_maxit=20000, uBC=uBC, vBC=vBC)
    V0 = np.random.default_rng(6).standard_normal(o.grid.NV)
    V_ref = R.initial_projection(V0, 0.0, o)
    V, md = m.initial_projection(V0, 0.0, return_maxdiv=True)
    assert md > 1e-12
    assert _rel(V, V_ref) < 1e-11
    assert m.check_conservation(V, 0.0)[0] < 1e-12
    # an already divergence-free field is returned unchanged
    V2, md2 = m.initial_projection(V, 0.0, return_maxdiv=True)
    assert md2 < 1e-12
    assert np.array_equal(V2, V)


def _homogeneous(combo, N=24, stretch=True):
    import ins2d_b200
    x = grid_stretched(N, 0.0, 1.3) if stretch else grid_uniform(N, 0.0, 1.3)
    y = grid_stretched(N - 4, -0.5, 0.5) if stretch else grid_uniform(N - 4, -0.5, 0.5)
    bc = BC_COMBOS[combo]
    poisson = 6 if (combo == "periodic" and not stretch) else 4
    o = R.make_options(x, y, bc, Re=1e300, poisson=poisson if poisson == 6 else 1)
    m = ins2d_b200.Options(x, y, bc, Re=1e300, poisson=poisson, CG_acc=1e-14, CG_maxit=20000)
    return o, m


@pytest.mark.parametrize("combo,stretch", [("periodic", False), ("periodic", True), ("cavity", False),
                                           ("cavity", True), ("per_x_walls", True)])
def test_convection_skew_symmetric(combo, stretch):
    """check_symmetry.m:42-61 through the device's F: for a discretely
    divergence-free convecting field c with zero boundary values the
    convection operator C(c) is skew-symmetric, w1' C(c) w2 = -w2' C(c) w1,
    to round-off (the reference's bound is 1e-14 on the entries of C + C',
    which the oracle's assembled matrices meet).  Cases with an outflow
    ('pres') side are not skew, and the reference does not flag them."""
    o, m = _homogeneous(combo, stretch=stretch)
    rng = np.random.default_rng(9)
    c = R.initial_projection(rng.standard_normal(o.grid.NV), 0.0, o)
    ok, err = R.check_symmetry(c, 0.0, o)
    w1, w2 = rng.standard_normal(o.grid.NV), rng.standard_normal(o.grid.NV)
    _, F2 = m.F(w2, c, None, 0.0, nopressure=1)   # -C(c) w2 (diffusion ~ 1e-300)
    _, F1 = m.F(w1, c, None, 0.0, nopressure=1)
    a, b = w1 @ F2, w2 @ F1
    scale = np.linalg.norm(w1) * np.linalg.norm(F2)
    assert abs(a + b) <= 1e-14 * scale
    assert ok, err


@pytest.mark.parametrize("N", [64, 512])
def test_semidiscrete_energy_periodic(N):
    """Energy conservation of the spatial operator, the round-off form of the
    energy claim: on a periodic grid, for a divergence-free V, the convective energy
    production V' conv(V) vanishes to round-off (|V' F| <= 1e-14 |V| |F|
    with F = -conv(V) at Re = inf)."""
    import ins2d_b200
    from ins2d_b200 import cases
    x = grid_uniform(N, 0.0, 1.0)
    m = ins2d_b200.Options(x, x.copy(), BC_COMBOS["periodic"], Re=1e300, poisson=6)
    V = cases.decaying_turbulence_ic(m, k0=6.0, seed=N)
    assert m.check_conservation(V, 0.0)[0] < 1e-12
    _, F = m.F(V, None, np.zeros(m.Np), 0.0)
    prod = V @ F
    assert abs(prod) <= 1e-14 * np.linalg.norm(V) * np.linalg.norm(F)


@pytest.mark.parametrize("case", ["fft", "fft_fp32", "pcg"])
@pytest.mark.parametrize("nsteps", [1, 3])
def test_host_buffers_match_device_tensors(case, nsteps):
    """A step on host buffers copies p in on a second stream beside the first
    stage and, for a single step, copies V out beside the additional solve;
    its state equals the same steps run on device tensors."""
    import torch
    import ins2d_b200
    if case.startswith("fft"):
        x = grid_uniform(128, 0.0, 1.0)
        m = ins2d_b200.Options(x, x.copy(), BC_COMBOS["periodic"], Re=500.0, poisson=6,
                               precision="fp32" if case == "fft_fp32" else "fp64")
        dt = 1e-3
    else:
        x = grid_stretched(300, 0.0, 1.0)
        y = grid_stretched(260, 0.0, 1.0)
        uBC, vBC = smooth_bc(5, closed=True)
        m = ins2d_b200.Options(x, y, BC_COMBOS["cavity"], Re=200.0, poisson=4, CG_acc=1e-10, uBC=uBC, vBC=vBC)
        dt = 1e-5
    rng = np.random.default_rng(11)
    V0 = 0.1 * rng.standard_normal(m.NV)
    p0 = 0.1 * rng.standard_normal(m.Np)
    Vh, ph = m.time_ERK(V0, p0, 0.0, dt, nsteps=nsteps)
    Vd = torch.tensor(V0, device="cuda")
    pd = torch.tensor(p0, device="cuda")
    m.time_ERK(Vd, pd, 0.0, dt, nsteps=nsteps)
    torch.cuda.synchronize()
    assert _rel(Vh, Vd.cpu().numpy()) < 1e-13
    assert _rel(ph, pd.cpu().numpy()) < 1e-13
    assert not np.array_equal(Vh, V0)
