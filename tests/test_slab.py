"""The y-slab decomposition of a single grid (ins2d_b200/slab.py) on CPU
ranks: world sizes 1 and 2 (gloo), the oracle's operators applied per slab
with halos exchanged, the FFT solve's all-to-all transposes and the
single-reduction CG -- one RK44 step must reproduce the single-grid oracle
step (time_ERK.m) to 1e-13 (FFT), or to the CG tolerance (PCG)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import ins2d_ref as R

NX, NY, LX, LY, RE, DT = 24, 20, 2 * np.pi, 1.7, 300.0, 2e-3


class OracleSlabOps:
    """Local operators of a rank from the oracle: the oracle's matrices of the
    rank's local grid, Nx x nL cells, uniform and periodic, with the global
    grid's spacings.  On interior rows they coincide with the global
    operators."""

    def __init__(self, Nx, Ny, Lx, Ly, Re, part):
        from ins2d_b200 import cases
        self.R = R
        hx, hy = Lx / Nx, Ly / Ny
        x = cases.uniform_grid(Nx, 0.0, Lx)
        y = hy * np.arange(part.nL + 1)
        self.o = R.make_options(x, y, cases.BC_PERIODIC, Re=Re, poisson=6)
        self.Nx, self.nL = Nx, part.nL
        self.hx, self.hy = hx, hy
        # FFT symbol of the global grid (operator_divergence.m:283-284)
        I = np.arange(Nx // 2 + 1)
        J = np.arange(Ny)
        self.ax = np.sin(np.pi * I / Nx) ** 2 / hx ** 2
        self.ay = np.sin(np.pi * J / Ny) ** 2 / hy ** 2
        self.dxdy = hx * hy
        self.diagA = self.o.discretization.A.diagonal().copy()

    @staticmethod
    def _np(t):
        return t.detach().cpu().numpy().ravel()

    def _t(self, a, like, shape):
        import torch
        return torch.as_tensor(np.ascontiguousarray(a).reshape(shape), dtype=like.dtype, device=like.device)

    def rhs(self, u, v, t=0.0):
        """Om^-1 R(V) (F.m without the pressure terms) on the local grid"""
        V = np.r_[self._np(u), self._np(v)]
        cu, cv = self.R.convection(V, V, t, self.o)
        d2u, d2v = self.R.diffusion(V, t, self.o)
        k = self.o.grid.Om_inv * np.r_[-cu + d2u, -cv + d2v]
        n = self.Nx * self.nL
        return self._t(k[:n], u, u.shape), self._t(k[n:], v, v.shape)

    def div(self, u, v):
        """M V (periodic: yM = 0) on the local pressure rows"""
        f = self.o.discretization.M @ np.r_[self._np(u), self._np(v)]
        return self._t(f, u, u.shape)

    def grad(self, p):
        """Om^-1 G p at the u and v points"""
        g = self.o.grid.Om_inv * (self.o.discretization.G @ self._np(p))
        n = self.Nx * self.nL
        return self._t(g[:n], p, p.shape), self._t(g[n:], p, p.shape)

    def lap(self, p):
        return self._t(self.o.discretization.A @ self._np(p), p, p.shape)

    def jacobi(self, r):
        return r / self._t(self.diagA, r, r.shape)

    # FFT pieces (numpy.fft on the local rows / columns)
    def fft_rows(self, f):
        import torch
        a = np.fft.fft(f.detach().cpu().numpy(), axis=1)[:, :self.Nx // 2 + 1]
        return torch.as_tensor(a, dtype=torch.complex128)

    def fft_cols_solve(self, cols, I0):
        """forward FFT along the columns, -1/Ahat scaling (Ahat(0,0) = 1),
        inverse FFT; returns (result, max|fhat| of these columns)"""
        import torch
        a = cols.numpy()
        w = a.shape[1]
        fh = np.fft.fft(a, axis=0)
        I = I0 + np.arange(w)
        valid = I < self.Nx // 2 + 1
        Iv = np.where(valid, I, 0)
        lam = self.dxdy * 4.0 * (self.ax[Iv][None, :] + self.ay[:, None])
        lam[0, :] = np.where(I == 0, 1.0, lam[0, :])
        mx = float(np.max(np.abs(fh[:, valid]))) if valid.any() else 0.0
        out = np.fft.ifft(-fh / lam, axis=0)
        out[:, ~valid] = 0.0
        return torch.as_tensor(out), mx

    def ifft_rows(self, spec):
        """half spectrum rows -> real rows (Hermitian completion)"""
        import torch
        a = spec.numpy()
        Nx = self.Nx
        full = np.zeros((a.shape[0], Nx), dtype=complex)
        full[:, :Nx // 2 + 1] = a
        k = np.arange(Nx // 2 + 1, Nx)
        full[:, k] = np.conj(a[:, Nx - k])
        return torch.as_tensor(np.real(np.fft.ifft(full, axis=1)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _reference(nsteps):
    from ins2d_b200 import cases
    x = cases.uniform_grid(NX, 0.0, LX)
    y = cases.uniform_grid(NY, 0.0, LY)
    o = R.make_options(x, y, cases.BC_PERIODIC, Re=RE, poisson=6)
    rng = np.random.default_rng(12)
    V0 = R.initial_projection(rng.standard_normal(o.grid.NV), 0.0, o)
    p0 = rng.standard_normal(o.grid.Np) * 0.1
    V, p = V0.copy(), p0.copy()
    for n in range(nsteps):
        V, p = R.time_ERK(V, p, n * DT, DT, o)
    return V0, p0, V, p


def _rank(rank, world, port, solver, nsteps, out):
    import torch.distributed as dist
    from ins2d_b200 import slab
    from ins2d_b200.rk import getRKmethod
    if world > 1:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        V0, p0, _, _ = _reference(0)
        part = slab.SlabPartition(NY, world, rank)
        rows = part.global_rows()
        u0 = V0[:NX * NY].reshape(NY, NX)
        v0 = V0[NX * NY:].reshape(NY, NX)
        u = torch.tensor(u0[rows])
        v = torch.tensor(v0[rows])
        p = torch.tensor(p0.reshape(NY, NX)[rows])
        ops = OracleSlabOps(NX, NY, LX, LY, RE, part)
        A, b, c = getRKmethod("RK44")
        erk = slab.SlabERK(ops, part, slab.Exchange(part), A, b, c, solver=solver, CG_acc=1e-13)
        for n in range(nsteps):
            erk.step(u, v, p, n * DT, DT)
        I = part.interior()
        out[rank] = (part.j0, part.j1, u[I].numpy().copy(), v[I].numpy().copy(), p[I].numpy().copy(),
                     list(erk.iters))
    finally:
        if world > 1:
            dist.destroy_process_group()


def _run(world, solver, nsteps):
    if world == 1:
        out = {}
        _rank(0, 1, 0, solver, nsteps, out)
        return out
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, solver, nsteps, out)) for r in range(world)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=300)
    assert all(pr.exitcode == 0 for pr in procs)
    return dict(out)


def _assemble(out):
    u = np.zeros((NY, NX))
    v = np.zeros((NY, NX))
    p = np.zeros((NY, NX))
    for j0, j1, ur, vr, pr, _ in out.values():
        u[j0:j1], v[j0:j1], p[j0:j1] = ur, vr, pr
    return np.r_[u.ravel(), v.ravel()], p.ravel()


@pytest.mark.parametrize("world", [1, 2])
def test_slab_step_fft_matches_single_grid(world):
    nsteps = 3
    _, _, V_ref, p_ref = _reference(nsteps)
    V, p = _assemble(_run(world, "fft", nsteps))
    assert np.max(np.abs(V - V_ref)) <= 1e-13 * np.max(np.abs(V_ref))
    assert np.max(np.abs(p - p_ref)) <= 1e-13 * np.max(np.abs(p_ref))


def test_slab_step_cg_matches_single_grid():
    nsteps = 2
    _, _, V_ref, p_ref = _reference(nsteps)
    out = _run(2, "cg", nsteps)
    V, p = _assemble(out)
    assert np.max(np.abs(V - V_ref)) <= 1e-10 * np.max(np.abs(V_ref))
    dp = (p - p.mean()) - (p_ref - p_ref.mean())
    assert np.max(np.abs(dp)) <= 1e-9 * np.max(np.abs(p_ref))
    its = [o[5] for o in out.values()]
    assert its[0] == its[1] and all(0 < k < 10000 for k in its[0])  # every rank takes the same CG steps


def test_partition_rows():
    from ins2d_b200 import slab
    parts = [slab.SlabPartition(2050, 4, r) for r in range(4)]
    assert [pt.n for pt in parts] == [513, 513, 512, 512]
    assert parts[0].j0 == 0 and parts[-1].j1 == 2050
    assert list(parts[0].global_rows()[:3]) == [2048, 2049, 0]
    with pytest.raises(ValueError):
        slab.SlabPartition(6, 4, 0)
