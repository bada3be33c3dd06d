"""The y-slab decomposition on the GPU (ins2d_b200/slab.py with
DeviceSlabOps): the slab FFT entry points against the context's FFT solve,
and RK44 steps of a single slab (world size 1: the halo exchange wraps
around, the transposes are identities) against the context's own steps.
Several slabs need several GPUs; their exchange logic is covered on CPU ranks
by tests/test_slab.py."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_slab_fft_pieces_match_context_solve():
    import torch
    import ins2d_b200
    from ins2d_b200 import _lib, cases
    Nx, Ny, Lx, Ly = 256, 128, 2 * np.pi, 1.3
    x, y = cases.uniform_grid(Nx, 0.0, Lx), cases.uniform_grid(Ny, 0.0, Ly)
    m = ins2d_b200.Options(x, y, cases.BC_PERIODIC, Re=1e100, poisson=6)
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.ins2d_slab_fft_create(Nx, Ny, Lx / Nx, Ly / Ny, 0, ctypes.byref(h)) == 0
    try:
        rng = np.random.default_rng(3)
        f = rng.standard_normal(Nx * Ny)
        f -= f.mean()
        ref = m.pressure_poisson(f)
        fd = torch.tensor(f.reshape(Ny, Nx), device="cuda")
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        spec = torch.empty((Ny, Nx // 2 + 1), dtype=torch.complex128, device="cuda")
        assert lib.ins2d_slab_fft_rows_forward(h, fd.data_ptr(), Ny, spec.data_ptr(), st) == 0
        spec_ref = np.fft.fft(f.reshape(Ny, Nx), axis=1)[:, :Nx // 2 + 1]
        assert _rel(spec.cpu().numpy(), spec_ref) < 1e-13
        # the columns in two ranges (as two ranks would hold them), width 80
        width = 80
        mxs = []
        out_cols = []
        for I0 in (0, width):
            cols = torch.zeros((Ny, width), dtype=torch.complex128, device="cuda")
            n = min(width, Nx // 2 + 1 - I0)
            cols[:, :n] = spec[:, I0:I0 + n]
            mx = ctypes.c_double()
            assert lib.ins2d_slab_fft_columns(h, cols.data_ptr(), width, I0, ctypes.byref(mx), st) == 0
            mxs.append(mx.value)
            out_cols.append(cols[:, :n])
        full = torch.cat(out_cols, dim=1).contiguous()
        assert abs(max(mxs) - np.max(np.abs(np.fft.fft2(f.reshape(Ny, Nx))))) <= 1e-12 * max(mxs)
        dp = torch.empty((Ny, Nx), dtype=torch.float64, device="cuda")
        assert lib.ins2d_slab_fft_rows_inverse(h, full.data_ptr(), Ny, max(mxs), dp.data_ptr(), st) == 0
        assert _rel(dp.cpu().numpy().ravel(), ref) < 1e-12
        # a vanishing spectrum: dp = 0 (pressure_poisson.m:21-32)
        assert lib.ins2d_slab_fft_rows_inverse(h, full.data_ptr(), Ny, 1e-15, dp.data_ptr(), st) == 0
        assert float(dp.abs().max()) == 0.0
        assert lib.ins2d_slab_fft_create(100, 64, 1.0, 1.0, 0, ctypes.byref(ctypes.c_void_p())) == _lib.EINVAL
    finally:
        lib.ins2d_slab_fft_destroy(h)


@pytest.mark.parametrize("solver", ["fft", "cg"])
def test_single_slab_steps_match_context(solver):
    import torch
    import ins2d_b200
    from ins2d_b200 import cases, slab
    from ins2d_b200.rk import getRKmethod
    N, L, Re = 256, 1.0, 1500.0
    x = cases.uniform_grid(N, 0.0, L)
    m = ins2d_b200.Options(x, x.copy(), cases.BC_PERIODIC, Re=Re, poisson=6)
    V0 = cases.decaying_turbulence_ic(m, k0=8.0, seed=5)
    dt = cases.cfl_dt(m, V0, 0.5)
    p0 = m.pressure_additional_solve(V0, np.zeros(m.Np), 0.0)
    nsteps = 3
    V_ref, p_ref = m.time_ERK(V0, p0, 0.0, dt, nsteps=nsteps)
    part = slab.SlabPartition(N, 1, 0)
    rows = part.global_rows()
    u = torch.tensor(V0[:N * N].reshape(N, N)[rows], device="cuda")
    v = torch.tensor(V0[N * N:].reshape(N, N)[rows], device="cuda")
    p = torch.tensor(p0.reshape(N, N)[rows], device="cuda")
    ops = slab.DeviceSlabOps(N, N, L, L, Re, part)
    A, b, c = getRKmethod("RK44")
    erk = slab.SlabERK(ops, part, slab.Exchange(part), A, b, c, solver=solver, CG_acc=1e-13)
    for n in range(nsteps):
        erk.step(u, v, p, n * dt, dt)
    I = part.interior()
    V = np.r_[u[I].cpu().numpy().ravel(), v[I].cpu().numpy().ravel()]
    pp = p[I].cpu().numpy().ravel()
    tol = 1e-12 if solver == "fft" else 1e-10
    assert _rel(V, V_ref) < tol
    assert _rel(pp - pp.mean(), p_ref - p_ref.mean()) < 10 * tol
    ops.close()
