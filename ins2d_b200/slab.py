"""A single grid split into y-slabs over several processes (one per GPU).

The pressure rows j = 0 .. Ny-1 of a uniform, doubly periodic grid are split
into contiguous slabs, one per rank; rank r owns the u, v and p rows
[j0, j1) and keeps H = 2 halo rows on each side, so its local arrays have
n_local + 2H rows (local row k is global row (j0 - H + k) mod Ny).  One RK
step of time_ERK (unsteady/time_ERK.m:78-168) then needs, per stage:

  * a halo exchange of the stage velocity (H rows of u and v to each
    neighbour; torch.distributed point-to-point, NCCL on GPUs);
  * the right-hand side, divergence and projection on the local rows (every
    interior row's stencil lies inside the local array, so the results there
    equal the single-grid ones; the halo rows' values are discarded);
  * the Poisson solve over the whole grid:
      FFT path (pressure_poisson.m:92-104): forward row transforms on the
      local rows, an all-to-all that gives every rank whole columns of a
      range of wave numbers, the column transforms with the -1/Ahat
      scaling, the all-to-all back and the inverse row transforms; the
      early return (max|fhat| < 1e-14) is an all-reduce of the maximum;
      PCG path (cg.F:158-280's stopping rule): Chronopoulos-Gear CG, one
      halo exchange of the preconditioned residual and ONE all-reduce of
      three dot products (r'z, z'Az, r'r) per iteration;
  * a halo exchange of dp (one row) for the pressure gradient.

The partition, the exchanges and the step are written against a backend of
local operators (right-hand side, divergence, gradient, Laplacian, row and
column transforms) and torch.distributed, so the same code runs on CPU ranks
(gloo) and GPU ranks (NCCL) with any backend that provides those operators;
DeviceSlabOps is the GPU one.  Data never moves between GPUs other than
through these collectives; no rank reads another's memory directly.
"""
from __future__ import annotations

import numpy as np


class SlabPartition:
    """Rows [j0, j1) of rank ``rank`` out of ``world`` contiguous slabs of Ny
    rows (the first Ny % world slabs one row longer), halo H rows."""

    def __init__(self, Ny, world, rank, halo=2):
        if world < 1 or not 0 <= rank < world:
            raise ValueError("bad rank/world")
        base, rem = divmod(Ny, world)
        if base < halo:
            raise ValueError(f"{Ny} rows over {world} ranks leaves slabs thinner than the {halo}-row halo")
        self.Ny, self.world, self.rank, self.H = Ny, world, rank, halo
        self.counts = [base + (1 if r < rem else 0) for r in range(world)]
        self.starts = [sum(self.counts[:r]) for r in range(world)]
        self.j0 = self.starts[rank]
        self.n = self.counts[rank]
        self.j1 = self.j0 + self.n
        self.nL = self.n + 2 * halo
        self.up = (rank + 1) % world
        self.down = (rank - 1) % world

    def global_rows(self):
        """global row of each local row (halo rows wrapped)"""
        return (self.j0 - self.H + np.arange(self.nL)) % self.Ny

    def interior(self):
        return slice(self.H, self.H + self.n)


class Exchange:
    """The collectives of the slab step over a torch.distributed group (or a
    single process when world == 1)."""

    def __init__(self, part, group=None):
        self.part = part
        self.group = group

    def _dist(self):
        import torch.distributed as dist
        return dist

    def halo(self, fields, rows=None):
        """Fills the halo rows of each [nL, Nx] tensor from the neighbours'
        interior rows (periodic ring): the H (or ``rows``) rows below the
        slab from the rank below, those above from the rank above."""
        P = self.part
        H = P.H
        h = H if rows is None else rows
        lo, hi = P.H, P.H + P.n  # interior rows [lo, hi)
        if P.world == 1:
            for f in fields:
                f[H - h:H] = f[hi - h:hi]
                f[hi:hi + h] = f[lo:lo + h]
            return
        dist = self._dist()
        ops, bufs = [], []
        for f in fields:
            top = f[hi - h:hi].contiguous()  # my top interior rows -> rank above's lower halo
            bot = f[lo:lo + h].contiguous()  # my bottom interior rows -> rank below's upper halo
            r_lo = f.new_empty(top.shape)
            r_hi = f.new_empty(top.shape)
            # sends and receives in one order on every rank: matched pairwise
            # (tags 0: going up, 1: going down)
            ops += [dist.P2POp(dist.isend, top, P.up, self.group, 0),
                    dist.P2POp(dist.isend, bot, P.down, self.group, 1),
                    dist.P2POp(dist.irecv, r_lo, P.down, self.group, 0),
                    dist.P2POp(dist.irecv, r_hi, P.up, self.group, 1)]
            bufs.append((f, r_lo, r_hi))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        for f, r_lo, r_hi in bufs:
            f[H - h:H] = r_lo
            f[hi:hi + h] = r_hi

    def _alltoall(self, recv, send):
        """recv[q] <- rank q's send[rank], for every q (point-to-point
        operations in one batch: NCCL groups them into one all-to-all, and
        gloo, which has no all-to-all, runs them as pairwise exchanges)"""
        P = self.part
        dist = self._dist()
        recv[P.rank].copy_(send[P.rank])
        ops = []
        for q in range(P.world):
            if q != P.rank:
                ops.append(dist.P2POp(dist.isend, send[q], q, self.group, 2))
                ops.append(dist.P2POp(dist.irecv, recv[q], q, self.group, 2))
        for req in dist.batch_isend_irecv(ops):
            req.wait()

    def allreduce(self, t, op="sum"):
        if self.part.world == 1:
            return t
        dist = self._dist()
        dist.all_reduce(t, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MAX, group=self.group)
        return t

    def rows_to_cols(self, spec, width):
        """[n_local, Hc] spectrum rows -> [Ny, width] columns [rank*width, (rank+1)*width) of all rows
        (the wave numbers padded to world*width)."""
        import torch
        if spec.is_complex():
            return torch.view_as_complex(self.rows_to_cols(torch.view_as_real(spec), width).contiguous())
        P = self.part
        n, Hc = spec.shape[:2]
        tail = tuple(spec.shape[2:])
        pad = P.world * width - Hc
        if pad:
            spec = torch.cat([spec, spec.new_zeros((n, pad) + tail)], dim=1)
        send = spec.reshape((n, P.world, width) + tail).transpose(0, 1).contiguous()  # [world, n, width, ...]
        if P.world == 1:
            return send.reshape((n, width) + tail)
        recv = [spec.new_empty((c, width) + tail) for c in P.counts]
        self._alltoall(recv, [t.contiguous() for t in send.unbind(0)])
        return torch.cat(recv, dim=0)

    def cols_to_rows(self, cols, Hc):
        """inverse of rows_to_cols: [Ny, width] -> [n_local, Hc]"""
        import torch
        if cols.is_complex():
            return torch.view_as_complex(self.cols_to_rows(torch.view_as_real(cols), Hc).contiguous())
        P = self.part
        width = cols.shape[1]
        tail = tuple(cols.shape[2:])
        if P.world == 1:
            return cols[:, :Hc].contiguous()
        send = [s.contiguous() for s in torch.split(cols, P.counts, dim=0)]
        recv = [cols.new_empty((P.n, width) + tail) for _ in range(P.world)]
        self._alltoall(recv, send)
        return torch.cat(recv, dim=1)[:, :Hc].contiguous()


class SlabERK:
    """time_ERK on a y-slab partition: the rank's local fields u, v, p (each
    [nL, Nx], interior rows the rank's slab) advanced in place."""

    def __init__(self, ops, part, exch, A, b, c, solver="fft", CG_acc=1e-12, CG_maxit=10000):
        s = len(b)
        # shifted tableau (time_ERK.m:29-32)
        self.A = [list(A[i + 1]) for i in range(s - 1)] + [list(b)]
        self.c = list(c[1:]) + [1.0]
        self.s = s
        self.ops, self.part, self.ex = ops, part, exch
        self.solver = solver
        self.tol, self.maxit = CG_acc, CG_maxit
        self.iters = []

    # -- Poisson solve over the whole grid ---------------------------------------
    def solve(self, f):
        """dp (local rows, halo included after the exchange) of A dp = f; f on
        the local rows (interior valid)"""
        if self.solver == "fft":
            return self._solve_fft(f)
        return self._solve_cg(f)

    def _solve_fft(self, f):
        import torch
        P, ops = self.part, self.ops
        I = P.interior()
        spec = ops.fft_rows(f[I])
        Hc = spec.shape[1]
        width = -(-Hc // P.world)
        cols = self.ex.rows_to_cols(spec, width)
        out, mx = ops.fft_cols_solve(cols, P.rank * width)
        mxt = self.ex.allreduce(torch.tensor([mx], dtype=torch.float64, device=f.device), op="max")
        dp = torch.zeros_like(f)
        if float(mxt[0]) < 1e-14:  # pressure_poisson.m:21-32
            return dp
        dp[I] = ops.ifft_rows(self.ex.cols_to_rows(out, Hc)).to(f.dtype)
        self.ex.halo([dp], rows=1)
        return dp

    def _solve_cg(self, f):
        """Chronopoulos-Gear PCG (Jacobi), cg.F's stopping rule r'r <= tol^2 f'f;
        one halo exchange and one all-reduce of three dot products per iteration"""
        import torch
        P, ops, ex = self.part, self.ops, self.ex
        I = P.interior()

        def dots(*pairs):
            t = torch.stack([(a[I] * b[I]).sum() for a, b in pairs]).to(torch.float64)
            return ex.allreduce(t).tolist()

        ff = dots((f, f))[0]
        x = torch.zeros_like(f)
        if ff == 0.0:
            self.iters.append(0)
            return x
        r = f.clone()
        z = ops.jacobi(r)
        ex.halo([z], rows=1)
        w = ops.lap(z)
        gamma, delta, rr = dots((r, z), (z, w), (r, r))
        alpha = gamma / delta
        beta = 0.0
        p = torch.zeros_like(f)
        s = torch.zeros_like(f)
        it = 0
        while True:
            p = z + beta * p
            s = w + beta * s
            x = x + alpha * p
            r = r - alpha * s
            it += 1
            z = ops.jacobi(r)
            ex.halo([z], rows=1)
            w = ops.lap(z)
            g_new, delta, rr = dots((r, z), (z, w), (r, r))
            if rr <= self.tol ** 2 * ff:
                break
            if it >= self.maxit:
                raise RuntimeError(f"CG didn't converge in {self.maxit} iterations")
            beta = g_new / gamma
            alpha = g_new / (delta - beta * g_new / alpha)
            gamma = g_new
        self.iters.append(it)
        ex.halo([x], rows=1)
        return x

    # -- one time step --------------------------------------------------------------
    def step(self, u, v, p, t, dt):
        """[V,p] = time_ERK(V,p,T,t,dt,options) on the local slab, in place"""
        ops, ex = self.ops, self.ex
        ex.halo([u, v])
        ex.halo([p], rows=1)
        un, vn = u.clone(), v.clone()
        us, vs = u, v
        ku, kv = [None] * self.s, [None] * self.s
        dp = p
        for i in range(self.s):
            ku[i], kv[i] = ops.rhs(us, vs, t)
            tu = sum(self.A[i][m] * ku[m] for m in range(i + 1) if self.A[i][m] != 0.0)
            tv = sum(self.A[i][m] * kv[m] for m in range(i + 1) if self.A[i][m] != 0.0)
            if isinstance(tu, int):
                tu, tv = 0.0 * un, 0.0 * vn
            if i > 0:
                # f = (M (Vn/dt + Vtemp) + yM/dt)/c  (time_ERK.m:117; periodic: yM = 0)
                f = ops.div(un / dt + tu, vn / dt + tv) / self.c[i]
                dp = self.solve(f)
            else:
                dp = p  # time_ERK.m:125-127 (p's halo exchanged at the start of the step)
            gu, gv = ops.grad(dp)
            us = un + dt * (tu - self.c[i] * gu)
            vs = vn + dt * (tv - self.c[i] * gv)
            ex.halo([us, vs])
        u.copy_(us)
        v.copy_(vs)
        # p = pressure_additional_solve(V, p, t+dt): f = M Om^-1 (R(V) - G p)
        ku0, kv0 = ops.rhs(u, v, t + dt)
        gu, gv = ops.grad(p)
        f = ops.div(ku0 - gu, kv0 - gv)
        p += self.solve(f)
        ex.halo([p], rows=1)


class DeviceSlabOps:
    """Local operators of a rank on its GPU: a context of the rank's local
    grid (Nx x nL cells, periodic, the global spacings) for the right-hand
    side, divergence, gradient and Laplacian (ins2d_F, ins2d_divergence,
    ins2d_laplacian), and the transform pieces of the global grid
    (ins2d_slab_fft_*).  Fields are torch CUDA tensors of the rank's device."""

    def __init__(self, Nx, Ny, Lx, Ly, Re, part, device=0):
        import ctypes
        import torch
        from . import _lib, api, cases
        self.lib = _lib.load()
        hx, hy = Lx / Nx, Ly / Ny
        x = cases.uniform_grid(Nx, 0.0, Lx)
        y = hy * np.arange(part.nL + 1)
        # the local context's own solver is not used: Jacobi keeps its set-up small
        self.ctx = api.Options(x, y, cases.BC_PERIODIC, Re=Re, poisson=4, precond="jacobi", device=device)
        self.Nx, self.Ny, self.nL = Nx, Ny, part.nL
        self.Hc = Nx // 2 + 1
        self.oi = (1.0 / hy) * (1.0 / hx)  # Om^-1 of the uniform periodic grid
        self.diagA = -2.0 * (hy / hx + hx / hy)  # diagonal of A = M Om^-1 G on that grid
        self.dev = torch.device("cuda", device)
        self.zero = torch.zeros(2 * Nx * part.nL, dtype=torch.float64, device=self.dev)
        self.h = ctypes.c_void_p()
        rc = self.lib.ins2d_slab_fft_create(Nx, Ny, hx, hy, device, ctypes.byref(self.h))
        if rc != 0:
            msg = self.lib.ins2d_slab_fft_last_error(self.h)
            self.lib.ins2d_slab_fft_destroy(self.h)
            raise api.Ins2dError(rc, msg.decode() if msg else "")

    def close(self):
        if self.h:
            self.lib.ins2d_slab_fft_destroy(self.h)
            self.h = None
        self.ctx.close()

    def _stream(self):
        import ctypes
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    def _check(self, rc):
        if rc != 0:
            from .api import Ins2dError
            msg = self.lib.ins2d_slab_fft_last_error(self.h)
            raise Ins2dError(rc, msg.decode() if msg else "")

    def _split(self, V, like):
        n = self.Nx * self.nL
        return V[:n].view(like.shape), V[n:].view(like.shape)

    def rhs(self, u, v, t=0.0):
        """Om^-1 R(V) (F.m without the pressure terms) on the local grid"""
        import torch
        V = torch.cat([u.reshape(-1), v.reshape(-1)])
        _, F = self.ctx.F(V, None, None, t, nopressure=1)
        return self._split(F * self.oi, u)

    def div(self, u, v):
        import torch
        f, _ = self.ctx.divergence(torch.cat([u.reshape(-1), v.reshape(-1)]))
        return f.view(u.shape)

    def grad(self, p):
        """Om^-1 G p at the u and v points (F(0, p) = -G p on a periodic grid)"""
        _, F = self.ctx.F(self.zero, None, p.reshape(-1).contiguous(), 0.0)
        return self._split(F * (-self.oi), p)

    def lap(self, p):
        return self.ctx.laplacian(p.reshape(-1).contiguous()).view(p.shape)

    def jacobi(self, r):
        return r / self.diagA

    def fft_rows(self, f):
        import torch
        f = f.contiguous()
        spec = torch.empty((f.shape[0], self.Hc), dtype=torch.complex128, device=self.dev)
        self._check(self.lib.ins2d_slab_fft_rows_forward(self.h, f.data_ptr(), f.shape[0], spec.data_ptr(),
                                                         self._stream()))
        return spec

    def fft_cols_solve(self, cols, I0):
        import ctypes
        cols = cols.contiguous()
        mx = ctypes.c_double()
        self._check(self.lib.ins2d_slab_fft_columns(self.h, cols.data_ptr(), cols.shape[1], int(I0),
                                                    ctypes.byref(mx), self._stream()))
        return cols, mx.value

    def ifft_rows(self, spec):
        import torch
        spec = spec.contiguous()
        out = torch.empty((spec.shape[0], self.Nx), dtype=torch.float64, device=self.dev)
        # the caller has already taken the early return of a vanishing spectrum
        self._check(self.lib.ins2d_slab_fft_rows_inverse(self.h, spec.data_ptr(), spec.shape[0], 1.0,
                                                         out.data_ptr(), self._stream()))
        return out
