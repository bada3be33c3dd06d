"""CPU oracle for the INS2D explicit-RK + pressure-projection hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (the ``ins2d_b200`` package,
its CUDA library, ``bench.py``'s GPU arm) may import or call this module; only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
it, and there only as the checker / the timed CPU stand-in.

It is a line-by-line restatement in numpy/scipy of the reference MATLAB code
(bsanderse/INS2D).  The sparse operators are assembled with the same
kron/spdiags structure as the reference, so that F, the divergence, the
pressure matrix and the boundary-condition vectors are the reference's own
matrices.  Citations are ``file:line`` inside the reference project.

Parity pin: the reference cannot run here (no MATLAB/Octave) and its testsuite
``*_refdata.mat`` files are not in the checkout.  The restatement is pinned on
the reference's own logged results (``results/*/convergence.txt``), see
``tests/test_oracle_pins.py``.

Vectors follow MATLAB column-major ordering with x fastest:
u(i,j) -> i + j*Nux_in, V = [u; v], p(i,j) -> i + j*Npx.
"""
from __future__ import annotations

import ctypes
import math
import os
from types import SimpleNamespace

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

BC_TYPES = ("dir", "pres", "per", "sym")


# ----------------------------------------------------------------------------
# MATLAB helpers
# ----------------------------------------------------------------------------
def spdiags(B, d, m, n):
    """MATLAB ``spdiags(B,d,m,n)`` (create form), including its rule that the
    diagonal values are indexed by column when m>=n and by row when m<n."""
    B = np.asarray(B, dtype=float)
    if B.ndim == 1:
        B = B[:, None]
    d = np.atleast_1d(np.asarray(d, dtype=int))
    rows, cols, vals = [], [], []
    for k, dk in enumerate(d):
        i = np.arange(max(1, 1 - dk), min(m, n - dk) + 1)  # 1-based rows
        idx = i + (dk if m >= n else 0)
        rows.append(i - 1)
        cols.append(i + dk - 1)
        vals.append(B[idx - 1, k])
    if rows:
        r = np.concatenate(rows)
        c = np.concatenate(cols)
        v = np.concatenate(vals)
    else:
        r = c = np.zeros(0, int)
        v = np.zeros(0)
    return sp.csr_matrix((v, (r, c)), shape=(m, n))


def spdiags_extract(A):
    """MATLAB ``[B,d] = spdiags(A)`` for a square matrix: B(j,k) = A(j-d(k), j)
    (column-indexed), d sorted ascending."""
    A = sp.coo_matrix(A)
    m, n = A.shape
    assert m == n
    nz = A.data != 0
    dd = np.unique(A.col[nz] - A.row[nz])
    B = np.zeros((n, len(dd)))
    Ad = A.tocsr()
    for k, dk in enumerate(dd):
        i = np.arange(max(1, 1 - dk), min(m, n - dk) + 1)
        vals = np.asarray(Ad[i - 1, i + dk - 1]).ravel()
        B[i + dk - 1, k] = vals
    return B, dd


def kron(a, b):
    return sp.kron(a, b, format="csr")


def speye(n):
    return sp.identity(n, format="csr")


def diagm(v):
    v = np.asarray(v, dtype=float).ravel()
    return sp.diags(v, 0, shape=(len(v), len(v)), format="csr")


# ----------------------------------------------------------------------------
# grid generation (preprocessing/mesh_generation.m, libs/nonuniform_grid.m)
# ----------------------------------------------------------------------------
def nonuniform_grid(deltaz, z_low, z_up, sz):
    """libs/nonuniform_grid.m:1-63 (geometric stretching, secant solve)."""
    eps = 1e-12
    if sz == 1:
        n = (z_up - z_low) / deltaz
        if abs(n - round(n)) > eps:
            deltaz = (z_up - z_low) / math.floor(n)
        # MATLAB colon z_low:deltaz:z_up
        nint = int(math.floor((z_up - z_low) / deltaz + 1e-10))
        z = z_low + deltaz * np.arange(nint + 1)
        return z, np.diff(z)
    z = [z_low]
    i = 1
    while z[i - 1] + deltaz * (sz ** i) <= z_up:
        i += 1
        z.append(z[i - 2] + deltaz * (sz ** (i - 2)))
    S = z_up - z[0]
    n = len(z) - 1
    s = [sz, sz ** 2]
    i = 0
    while abs(s[i + 1] - s[i]) > eps:
        g1 = S * (s[i + 1] - 1) - deltaz * (s[i + 1] ** n - 1)
        g0 = S * (s[i] - 1) - deltaz * (s[i] ** n - 1)
        s.append(s[i + 1] - (s[i + 1] - s[i]) * g1 / (g1 - g0))
        i += 1
    sz = s[-1]
    z = np.zeros(n)
    z[0] = z_low
    for k in range(1, n):
        z[k] = z[k - 1] + deltaz * sz ** (k - 1)
    z = np.asarray(z)
    return z, np.diff(z)


def mesh_metrics(x, y):
    """preprocessing/mesh_generation.m:17-49."""
    x = np.asarray(x, float)
    y = np.asarray(y, float)
    xp = (x[:-1] + x[1:]) / 2
    yp = (y[:-1] + y[1:]) / 2
    hx = np.diff(x)
    hy = np.diff(y)
    Nx, Ny = len(hx), len(hy)
    gx = np.zeros(Nx + 1)
    gx[0] = hx[0] / 2
    gx[1:Nx] = (hx[:-1] + hx[1:]) / 2
    gx[Nx] = hx[-1] / 2
    gy = np.zeros(Ny + 1)
    gy[0] = hy[0] / 2
    gy[1:Ny] = (hy[:-1] + hy[1:]) / 2
    gy[Ny] = hy[-1] / 2
    return SimpleNamespace(x=x, y=y, xp=xp, yp=yp, hx=hx, hy=hy, gx=gx, gy=gy,
                           Nx=Nx, Ny=Ny)


# ----------------------------------------------------------------------------
# boundary-condition elimination
# ----------------------------------------------------------------------------
def _finish_bc(Bin, Bb, Bbc, ybc1, ybc2, Nt, Nb):
    Bb = sp.csr_matrix(Bb)
    Bbc = sp.csr_matrix(Bbc)
    small = (Bbc @ Bb).toarray()
    Btemp = sp.csr_matrix(Bb @ np.linalg.solve(small, np.eye(Nb)))
    B1D = sp.csr_matrix(Bin - Btemp @ Bbc @ Bin)
    return SimpleNamespace(B1D=B1D, Btemp=Btemp, ybc1=ybc1, ybc2=ybc2)


def _no_boundary(Nt):
    return SimpleNamespace(B1D=speye(Nt), Btemp=sp.csr_matrix((Nt, 2)),
                           ybc1=np.zeros(2), ybc2=np.zeros(2))


def bc_general(Nt, Nin, Nb, BC1, BC2, h1, h2):
    """spatial/boundaryconditions/proposed/BC_general.m:1-130 (grid lines)."""
    if Nt != Nin + Nb:
        raise ValueError("Number of inner points plus boundary points is not equal to total points")
    if Nb == 0:
        return _no_boundary(Nt)
    Bbc = np.zeros((Nb, Nt))
    ybc1 = np.zeros(Nb)
    ybc2 = np.zeros(Nb)
    if Nb == 2:
        Bin = spdiags(np.ones(Nt), -1, Nt, Nin)
        Bb = np.zeros((Nt, Nb))
        Bb[0, 0] = 1
        Bb[-1, Nb - 1] = 1
        if BC1 == "dir":
            Bbc[0, 0] = 1
            ybc1[0] = 1
        elif BC1 == "pres":
            Bbc[0, 0] = -1
            Bbc[0, 1] = 1
            ybc1[0] = 2 * h1
        elif BC1 == "per":
            Bbc[0, 0] = -1
            Bbc[0, Nt - 2] = 1
            Bbc[Nb - 1, 1] = -1
            Bbc[Nb - 1, Nt - 1] = 1
        else:
            raise NotImplementedError(BC1)
        if BC2 == "dir":
            Bbc[Nb - 1, Nt - 1] = 1
            ybc2[1] = 1
        elif BC2 == "pres":
            Bbc[Nb - 1, Nt - 2] = -1
            Bbc[Nb - 1, Nt - 1] = 1
            ybc2[1] = 2 * h2
        elif BC2 == "per":
            Bbc[0, 0] = -1
            Bbc[0, Nt - 2] = 1
            Bbc[Nb - 1, 1] = -1
            Bbc[Nb - 1, Nt - 1] = 1
        else:
            raise NotImplementedError(BC2)
    elif Nb == 1:
        Bb = np.zeros((Nt, Nb))
        diagpos = -1
        if BC1 == "dir":
            Bbc[0, 0] = 1
            ybc1[0] = 1
            Bb[0, 0] = 1
        elif BC1 == "pres":
            diagpos = 0
        elif BC1 == "per":
            diagpos = 0
            Bbc[0, 0] = -1
            Bbc[0, Nt - 1] = 1
            Bb[Nt - 1, 0] = 1
        else:
            raise NotImplementedError(BC1)
        if BC2 == "dir":
            Bbc[Nb - 1, Nt - 1] = 1
            ybc2[0] = 1
            Bb[Nt - 1, Nb - 1] = 1
        elif BC2 == "pres":
            pass
        elif BC2 == "per":
            diagpos = 0
            Bbc[0, 0] = -1
            Bbc[0, Nt - 1] = 1
            Bb[Nt - 1, 0] = 1
        else:
            raise NotImplementedError(BC2)
        Bin = spdiags(np.ones(Nt), diagpos, Nt, Nin)
    else:
        raise ValueError("Nb must be 0, 1 or 2")
    return _finish_bc(Bin, Bb, Bbc, ybc1, ybc2, Nt, Nb)


def bc_general_stag(Nt, Nin, Nb, BC1, BC2, h1, h2):
    """spatial/boundaryconditions/proposed/BC_general_stag.m:1-138 (staggered
    lines; Dirichlet as the mean of ghost and first inner point)."""
    if Nt != Nin + Nb:
        raise ValueError("Number of inner points plus boundary points is not equal to total points")
    if Nb == 0:
        return _no_boundary(Nt)
    Bbc = np.zeros((Nb, Nt))
    ybc1 = np.zeros(Nb)
    ybc2 = np.zeros(Nb)
    if Nb == 2:
        Bin = spdiags(np.ones(Nt), -1, Nt, Nin)
        Bb = np.zeros((Nt, Nb))
        Bb[0, 0] = 1
        Bb[-1, Nb - 1] = 1
        if BC1 == "dir":
            Bbc[0, 0] = 0.5
            Bbc[0, 1] = 0.5
            ybc1[0] = 1
        elif BC1 == "sym":
            Bbc[0, 0] = -1
            Bbc[0, 1] = 1
            ybc1[0] = h1
        elif BC1 == "per":
            Bbc[0, 0] = -1
            Bbc[0, Nt - 2] = 1
            Bbc[1, 1] = -1
            Bbc[1, Nt - 1] = 1
        else:
            raise NotImplementedError(BC1)
        if BC2 == "dir":
            Bbc[-1, Nt - 2] = 0.5
            Bbc[-1, Nt - 1] = 0.5
            ybc2[1] = 1
        elif BC2 == "sym":
            Bbc[1, Nt - 2] = -1
            Bbc[1, Nt - 1] = 1
            ybc2[1] = h2
        elif BC2 == "per":
            Bbc[0, 0] = -1
            Bbc[0, Nt - 2] = 1
            Bbc[1, 1] = -1
            Bbc[1, Nt - 1] = 1
        else:
            raise NotImplementedError(BC2)
    elif Nb == 1:
        Bb = np.zeros((Nt, Nb))
        diagpos = -1
        if BC1 == "dir":
            Bbc[0, 0] = 0.5
            Bbc[0, 1] = 0.5
            ybc1[0] = 1
            Bb[0, 0] = 1
        elif BC1 == "sym":
            Bbc[0, 0] = -1
            Bbc[0, 1] = 1
            ybc1[0] = h1
        elif BC1 == "per":
            Bbc[0, 0] = -1
            Bbc[0, Nt - 1] = 1
            Bb[0, 0] = 1
        else:
            raise NotImplementedError(BC1)
        if BC2 == "dir":
            Bbc[Nb - 1, Nt - 2] = 0.5
            Bbc[Nb - 1, Nt - 1] = 0.5
            ybc2[0] = 1
            Bb[Nt - 1, Nb - 1] = 1
        elif BC2 == "sym":
            Bbc[Nb - 1, Nt - 2] = -1
            Bbc[Nb - 1, Nt - 1] = 1
            ybc2[0] = h2
        elif BC2 == "per":
            Bbc[0, 0] = -1
            Bbc[0, Nt - 1] = 1
            Bb[0, 0] = 1
        else:
            raise NotImplementedError(BC2)
        Bin = spdiags(np.ones(Nt), diagpos, Nt, Nin)
    else:
        raise ValueError("Nb must be 0, 1 or 2")
    return _finish_bc(Bin, Bb, Bbc, ybc1, ybc2, Nt, Nb)


def bc_diff_stag(Nt, Nin, Nb, BC1, BC2, h1, h2):
    """spatial/boundaryconditions/proposed/BC_diff_stag.m:1-160.  With two
    boundary points (the only case the operators use) it is the zeroth-order
    mirror condition, i.e. identical to BC_general_stag."""
    if Nb not in (0, 2):
        raise NotImplementedError("BC_diff_stag with one boundary point")
    return bc_general_stag(Nt, Nin, Nb, BC1, BC2, h1, h2)


# ----------------------------------------------------------------------------
# operator construction
# ----------------------------------------------------------------------------
class Options(SimpleNamespace):
    pass


def make_options(x, y, BC, Re=1000.0, poisson=6, CG_acc=1e-12, CG_maxit=10000,
                 p_add_solve=1, RK="RK44", uBC=None, vBC=None, dudtBC=None,
                 dvdtBC=None, pLe=0.0, pRi=0.0, pLo=0.0, pUp=0.0):
    """Builds the ``options`` struct the hot path reads: mesh metrics
    (mesh_generation.m), operators (operators.m:1-18) and the BC vectors at
    t=0 (main.m:165 set_bc_vectors)."""
    g = mesh_metrics(x, y)
    o = Options()
    o.grid = g
    o.BC = SimpleNamespace(u=SimpleNamespace(**BC["u"]), v=SimpleNamespace(**BC["v"]),
                           BC_unsteady=int(BC.get("BC_unsteady", 0)),
                           pLe=pLe, pRi=pRi, pLo=pLo, pUp=pUp)
    for comp in ("u", "v"):
        for side in ("left", "right", "low", "up"):
            t = getattr(getattr(o.BC, comp), side)
            if t not in BC_TYPES:
                raise ValueError(f"wrong BC for {comp}-{side}")
    o.fluid = SimpleNamespace(Re=float(Re))
    o.solversettings = SimpleNamespace(poisson=poisson, CG_acc=CG_acc, CG_maxit=CG_maxit,
                                       p_add_solve=p_add_solve, last_iter=0, last_norm1=0.0)
    o.time = SimpleNamespace(RK=RK)
    o.discretization = SimpleNamespace()
    zero = lambda x_, y_, t_: np.zeros(np.size(x_) * np.size(y_))
    o.uBC = uBC or zero
    o.vBC = vBC or zero
    o.dudtBC = dudtBC or zero
    o.dvdtBC = dvdtBC or zero
    operator_mesh(o)
    operator_averaging(o)
    operator_interpolation(o)
    operator_divergence(o)
    operator_convection_diffusion(o)
    set_bc_vectors(0.0, o)
    return o


def operator_mesh(o):
    """spatial/operators/operator_mesh.m:1-110, 171-419 (order4=0)."""
    g, BC = o.grid, o.BC
    Nx, Ny = g.Nx, g.Ny
    x, y, hx, hy, gx, gy, xp, yp = g.x, g.y, g.hx, g.hy, g.gx, g.gy, g.xp, g.yp
    Npx, Npy = Nx, Ny
    Nux_b = 2
    Nux_in = Nx + 1
    if BC.u.left in ("dir", "sym"):
        Nux_in -= 1
    if BC.u.right in ("dir", "sym"):
        Nux_in -= 1
    if BC.u.left == "per" and BC.u.right == "per":
        Nux_in -= 1
    Nux_t = Nux_in + Nux_b
    Nuy_b = 2
    Nuy_in = Ny
    Nuy_t = Nuy_in + Nuy_b
    Nvx_b = 2
    Nvx_in = Nx
    Nvx_t = Nvx_in + Nvx_b
    Nvy_b = 2
    Nvy_in = Ny + 1
    if BC.v.low in ("dir", "sym"):
        Nvy_in -= 1
    if BC.v.up in ("dir", "sym"):
        Nvy_in -= 1
    if BC.v.low == "per" and BC.v.up == "per":
        Nvy_in -= 1
    Nvy_t = Nvy_in + Nvy_b
    Nu = Nux_in * Nuy_in
    Nv = Nvx_in * Nvy_in
    # x-direction metrics (operator_mesh.m:173-249)
    gxd = gx.copy()
    gxd[0] = hx[0]
    gxd[-1] = hx[-1]
    hxi = hx.copy()
    L, R = BC.u.left, BC.u.right
    if L == "dir" and R == "dir":
        xin, hxd, gxi, diagpos = x[1:-1], hx.copy(), gx[1:-1], 1
    elif L == "dir" and R == "pres":
        xin, hxd, gxi, diagpos = x[1:], np.r_[hx, hx[-1]], gx[1:], 1
    elif L == "pres" and R == "dir":
        xin, hxd, gxi, diagpos = x[:-1], np.r_[hx[0], hx], gx[:-1], 0
    elif L == "pres" and R == "pres":
        xin, hxd, gxi, diagpos = x.copy(), np.r_[hx[0], hx, hx[-1]], gx.copy(), 0
    elif L == "per" and R == "per":
        xin = x[:-1]
        hxd = np.r_[hx[-1], hx]
        gxi = np.r_[gx[0] + gx[-1], gx[1:-1]]
        gxd[0] = (hx[0] + hx[-1]) / 2
        gxd[-1] = (hx[0] + hx[-1]) / 2
        diagpos = 0
    else:
        raise NotImplementedError(f"u left/right = {L}/{R}")
    Bvux = spdiags(np.ones(Nvx_t - 1), diagpos, Nux_in, Nvx_t - 1)
    # y-direction metrics (operator_mesh.m:260-327)
    gyd = gy.copy()
    gyd[0] = hy[0]
    gyd[-1] = hy[-1]
    hyi = hy.copy()
    Lo, Up = BC.v.low, BC.v.up
    if Lo == "dir" and Up == "dir":
        yin, hyd, gyi, diagpos = y[1:-1], hy.copy(), gy[1:-1], 1
    elif Lo == "dir" and Up == "pres":
        yin, hyd, gyi, diagpos = y[1:], np.r_[hy, hy[-1]], gy[1:], 1
    elif Lo == "pres" and Up == "dir":
        yin, hyd, gyi, diagpos = y[:-1], np.r_[hy[0], hy], gy[:-1], 0
    elif Lo == "pres" and Up == "pres":
        yin, hyd, gyi, diagpos = y.copy(), np.r_[hy[0], hy, hy[-1]], gy.copy(), 0
    elif Lo == "per" and Up == "per":
        yin = y[:-1]
        hyd = np.r_[hy[-1], hy]
        gyi = np.r_[gy[0] + gy[-1], gy[1:-1]]
        gyd[0] = (hy[0] + hy[-1]) / 2
        gyd[-1] = (hy[0] + hy[-1]) / 2
        diagpos = 0
    else:
        raise NotImplementedError(f"v low/up = {Lo}/{Up}")
    Buvy = spdiags(np.ones(Nuy_t - 1), diagpos, Nvy_in, Nuy_t - 1)
    # volumes (operator_mesh.m:331-352), kron(a,b) of column vectors
    Omp = np.kron(hyi, hxi)
    Omu = np.kron(hyi, gxi)
    Omv = np.kron(gyi, hxi)
    Om = np.r_[Omu, Omv]
    # positions (operator_mesh.m:401-414)
    xu = np.tile(xin, Nuy_in)
    yu = np.repeat(yp, Nux_in)
    xv = np.tile(xp, Nvy_in)
    yv = np.repeat(yin, Nvx_in)
    g.__dict__.update(dict(
        Npx=Npx, Npy=Npy, Np=Npx * Npy, Nux_in=Nux_in, Nux_b=Nux_b, Nux_t=Nux_t,
        Nuy_in=Nuy_in, Nuy_b=Nuy_b, Nuy_t=Nuy_t, Nvx_in=Nvx_in, Nvx_b=Nvx_b,
        Nvx_t=Nvx_t, Nvy_in=Nvy_in, Nvy_b=Nvy_b, Nvy_t=Nvy_t, Nu=Nu, Nv=Nv,
        NV=Nu + Nv, N1=(Nux_in + 1) * Nuy_in, N2=Nux_in * (Nuy_in + 1),
        N3=(Nvx_in + 1) * Nvy_in, N4=Nvx_in * (Nvy_in + 1),
        Omp=Omp, Omp_inv=1 / Omp, Om=Om, Omu=Omu, Omv=Omv, Om_inv=1 / Om,
        Omu_inv=1 / Omu, Omv_inv=1 / Omv, hxi=hxi, hyi=hyi, hxd=hxd, hyd=hyd,
        gxi=gxi, gyi=gyi, gxd=gxd, gyd=gyd, Buvy=Buvy, Bvux=Bvux, xin=xin,
        yin=yin, xu=xu, yu=yu, xv=xv, yv=yv))


def operator_averaging(o):
    """spatial/operators/operator_averaging.m:27-83 (order4=0)."""
    g, BC, d = o.grid, o.BC, o.discretization
    hx, hy = g.hx, g.hy
    w = 0.5
    A1D = spdiags(np.c_[w * np.ones(g.Nux_t), w * np.ones(g.Nux_t)], [0, 1], g.Nux_t - 1, g.Nux_t)
    B = bc_general(g.Nux_t, g.Nux_in, g.Nux_b, BC.u.left, BC.u.right, hx[0], hx[-1])
    d.Au_ux = kron(speye(g.Nuy_in), A1D @ B.B1D)
    B.Bbc = kron(speye(g.Nuy_in), A1D @ B.Btemp)
    d.Au_ux_BC = B
    A1D = spdiags(np.c_[w * np.ones(g.Nuy_t), w * np.ones(g.Nuy_t)], [0, 1], g.Nuy_t - 1, g.Nuy_t)
    B = bc_general_stag(g.Nuy_t, g.Nuy_in, g.Nuy_b, BC.u.low, BC.u.up, hy[0], hy[-1])
    d.Au_uy = kron(A1D @ B.B1D, speye(g.Nux_in))
    B.Bbc = kron(A1D @ B.Btemp, speye(g.Nux_in))
    d.Au_uy_BC = B
    A1D = spdiags(np.c_[w * np.ones(g.Nvx_t), w * np.ones(g.Nvx_t)], [0, 1], g.Nvx_t - 1, g.Nvx_t)
    B = bc_general_stag(g.Nvx_t, g.Nvx_in, g.Nvx_b, BC.v.left, BC.v.right, hx[0], hx[-1])
    d.Av_vx = kron(speye(g.Nvy_in), A1D @ B.B1D)
    B.Bbc = kron(speye(g.Nvy_in), A1D @ B.Btemp)
    d.Av_vx_BC = B
    A1D = spdiags(np.c_[w * np.ones(g.Nvy_t), w * np.ones(g.Nvy_t)], [0, 1], g.Nvy_t - 1, g.Nvy_t)
    B = bc_general(g.Nvy_t, g.Nvy_in, g.Nvy_b, BC.v.low, BC.v.up, hy[0], hy[-1])
    d.Av_vy = kron(A1D @ B.B1D, speye(g.Nvx_in))
    B.Bbc = kron(A1D @ B.Btemp, speye(g.Nvx_in))
    d.Av_vy_BC = B


def operator_interpolation(o):
    """spatial/operators/operator_interpolation.m:1-322 (order4=0), including
    the 2022 outflow half-cell fix (:85-90, :125-130)."""
    g, BC, d = o.grid, o.BC, o.discretization
    Nx, Ny = g.Nx, g.Ny
    hx, hy, hxi, hyi = g.hx, g.hy, g.hxi, g.hyi
    w = 0.5
    mat_hx = diagm(hxi)
    mat_hy = diagm(hyi)
    if BC.u.left == "per" and BC.u.right == "per":
        mat_hx2 = diagm(np.r_[hx[-1], hx, hx[0]])
    else:
        mat_hx2 = diagm(np.r_[hx[0], hx, hx[-1]])
    if BC.v.low == "per" and BC.v.up == "per":
        mat_hy2 = diagm(np.r_[hy[-1], hy, hy[0]])
    else:
        mat_hy2 = diagm(np.r_[hy[0], hy, hy[-1]])
    # Iu_ux
    I1D = spdiags(np.c_[w * np.ones(g.Nux_t), w * np.ones(g.Nux_t)], [0, 1], g.Nux_t - 1, g.Nux_t)
    B = bc_general(g.Nux_t, g.Nux_in, g.Nux_b, BC.u.left, BC.u.right, hx[0], hx[-1])
    d.Iu_ux = kron(mat_hy, I1D @ B.B1D)
    B.Bbc = kron(mat_hy, I1D @ B.Btemp)
    d.Iu_ux_BC = B
    # Iv_uy
    I1D = spdiags(np.c_[w * np.ones(g.Nvx_t), w * np.ones(g.Nvx_t)], [0, 1], g.Nvx_t - 1, g.Nvx_t).tolil()
    if BC.u.right == "pres":
        I1D[I1D.shape[0] - 1, :] = I1D[I1D.shape[0] - 1, :] / 2
    if BC.u.left == "pres":
        I1D[0, :] = I1D[0, :] / 2
    I1D = g.Bvux @ sp.csr_matrix(I1D) @ mat_hx2
    I2D = kron(speye(g.Nuy_t - 1), I1D)
    Nb = g.Nuy_in + 1 - g.Nvy_in
    lu = bc_general(g.Nuy_in + 1, g.Nvy_in, Nb, BC.v.low, BC.v.up, hy[0], hy[-1])
    lu.B2D = kron(lu.B1D, speye(g.Nvx_in))
    lu.Bbc = kron(lu.Btemp, speye(g.Nvx_in))
    lr = bc_general_stag(g.Nvx_t, g.Nvx_in, g.Nvx_b, BC.v.left, BC.v.right, hx[0], hx[-1])
    lr.B2D = I2D @ kron(speye(g.Nuy_t - 1), lr.B1D)
    lr.Bbc = I2D @ kron(speye(g.Nuy_t - 1), lr.Btemp)
    d.Iv_uy = lr.B2D @ lu.B2D
    d.Iv_uy_BC_lr, d.Iv_uy_BC_lu = lr, lu
    # Iu_vx
    I1D = spdiags(np.c_[w * np.ones(g.Nuy_t), w * np.ones(g.Nuy_t)], [0, 1], g.Nuy_t - 1, g.Nuy_t).tolil()
    if BC.v.up == "pres":
        I1D[I1D.shape[0] - 1, :] = I1D[I1D.shape[0] - 1, :] / 2
    if BC.v.low == "pres":
        I1D[0, :] = I1D[0, :] / 2
    I1D = g.Buvy @ sp.csr_matrix(I1D) @ mat_hy2
    I2D = kron(I1D, speye(g.Nvx_t - 1))
    lu = bc_general_stag(g.Nuy_t, g.Nuy_in, g.Nuy_b, BC.u.low, BC.u.up, hy[0], hy[-1])
    lu.B2D = I2D @ kron(lu.B1D, speye(g.Nvx_t - 1))
    lu.Bbc = I2D @ kron(lu.Btemp, speye(g.Nvx_t - 1))
    Nb = g.Nvx_in + 1 - g.Nux_in
    lr = bc_general(g.Nvx_in + 1, g.Nux_in, Nb, BC.u.left, BC.u.right, hx[0], hx[-1])
    lr.B2D = kron(speye(g.Nuy_in), lr.B1D)
    lr.Bbc = kron(speye(g.Nuy_in), lr.Btemp)
    d.Iu_vx = lu.B2D @ lr.B2D
    d.Iu_vx_BC_lr, d.Iu_vx_BC_lu = lr, lu
    # Iv_vy
    I1D = spdiags(np.c_[w * np.ones(g.Nvy_t), w * np.ones(g.Nvy_t)], [0, 1], g.Nvy_t - 1, g.Nvy_t)
    B = bc_general(g.Nvy_t, g.Nvy_in, g.Nvy_b, BC.v.low, BC.v.up, hy[0], hy[-1])
    d.Iv_vy = kron(I1D @ B.B1D, mat_hx)
    B.Bbc = kron(I1D @ B.Btemp, mat_hx)
    d.Iv_vy_BC = B


def operator_divergence(o):
    """spatial/operators/operator_divergence.m:46-167, 207-208, 268-291."""
    g, BC, d = o.grid, o.BC, o.discretization
    Nx, Ny, Npx, Npy = g.Nx, g.Ny, g.Npx, g.Npy
    hx, hy = g.hx, g.hy
    mat_hx = diagm(hx)
    mat_hy = diagm(hy)
    M1D = spdiags(np.c_[-np.ones(g.Nux_t), np.ones(g.Nux_t)], [0, 1], g.Nux_t - 1, g.Nux_t)
    diagpos = 0
    if BC.u.right == "pres" and BC.u.left == "pres":
        diagpos = 1
    if BC.u.right != "pres" and BC.u.left == "pres":
        diagpos = 1
    if BC.u.right == "pres" and BC.u.left != "pres":
        diagpos = 0
    if BC.u.right == "per" and BC.u.left == "per":
        diagpos = 1
    BMx = spdiags(np.ones(Npx), diagpos, Npx, g.Nux_t - 1)
    M1D = BMx @ M1D
    B = bc_general(g.Nux_t, g.Nux_in, g.Nux_b, BC.u.left, BC.u.right, hx[0], hx[-1])
    B.Bbc = kron(mat_hy, M1D @ B.Btemp)
    d.Mx = kron(mat_hy, M1D @ B.B1D)
    d.Mx_BC = B
    d.M1Dx = M1D @ B.B1D
    M1D = spdiags(np.c_[-np.ones(g.Nvy_t), np.ones(g.Nvy_t)], [0, 1], g.Nvy_t - 1, g.Nvy_t)
    diagpos = 0
    if BC.v.up == "pres" and BC.v.low == "pres":
        diagpos = 1
    if BC.v.up != "pres" and BC.v.low == "pres":
        diagpos = 1
    if BC.v.up == "pres" and BC.v.low != "pres":
        diagpos = 0
    if BC.v.up == "per" and BC.v.low == "per":
        diagpos = 1
    BMy = spdiags(np.ones(Npy), diagpos, Npy, g.Nvy_t - 1)
    M1D = BMy @ M1D
    B = bc_general(g.Nvy_t, g.Nvy_in, g.Nvy_b, BC.v.low, BC.v.up, hy[0], hy[-1])
    B.Bbc = kron(M1D @ B.Btemp, mat_hx)
    d.My = kron(M1D @ B.B1D, mat_hx)
    d.My_BC = B
    d.M = sp.hstack([d.Mx, d.My], format="csr")
    d.Gx = sp.csr_matrix(-d.Mx.T)
    d.Gy = sp.csr_matrix(-d.My.T)
    d.G = sp.vstack([d.Gx, d.Gy], format="csr")
    d.A = sp.csr_matrix(d.M @ diagm(g.Om_inv) @ d.G)
    if o.solversettings.poisson == 6:
        if not (BC.v.low == "per" and BC.v.up == "per" and BC.u.left == "per" and BC.u.right == "per"):
            raise ValueError("Fourier transform for pressure Poisson only implemented for periodic boundary conditions")
        if max(abs(np.diff(hx))) > 1e-14 or max(abs(np.diff(hy))) > 1e-14:
            raise ValueError("grid needs to be uniform to use Fourier transform for pressure matrix")
        dx, dy = hx[0], hy[0]
        I, J = np.meshgrid(np.arange(Npx), np.arange(Npy), indexing="ij")
        Ahat = (dx * dy) * 4 * ((1 / dx ** 2) * np.sin(I * np.pi / Npx) ** 2
                                + (1 / dy ** 2) * np.sin(J * np.pi / Npy) ** 2)
        Ahat[0, 0] = 1
        o.solversettings.Ahat = Ahat  # indexed [I (x), J (y)] as in MATLAB


def operator_convection_diffusion(o):
    """spatial/operators/operator_convection_diffusion.m:81-254, 454-461
    (order4=0, laminar)."""
    g, BC, d = o.grid, o.BC, o.discretization
    Nx, Ny = g.Nx, g.Ny
    hx, hy = g.hx, g.hy
    Re = o.fluid.Re
    D1D = spdiags(np.c_[-np.ones(g.Nux_t), np.ones(g.Nux_t)], [0, 1], g.Nux_t - 2, g.Nux_t - 1)
    d.Cux = kron(speye(g.Nuy_in), D1D)
    d.Dux = kron(diagm(g.hyi), D1D)
    D1D = spdiags(np.c_[-np.ones(g.Nuy_t), np.ones(g.Nuy_t)], [0, 1], g.Nuy_t - 2, g.Nuy_t - 1)
    d.Cuy = kron(D1D, speye(g.Nux_in))
    d.Duy = kron(D1D, diagm(g.gxi))
    D1D = spdiags(np.c_[-np.ones(g.Nvx_t), np.ones(g.Nvx_t)], [0, 1], g.Nvx_t - 2, g.Nvx_t - 1)
    d.Cvx = kron(speye(g.Nvy_in), D1D)
    d.Dvx = kron(diagm(g.gyi), D1D)
    D1D = spdiags(np.c_[-np.ones(g.Nvy_t), np.ones(g.Nvy_t)], [0, 1], g.Nvy_t - 2, g.Nvy_t - 1)
    d.Cvy = kron(D1D, speye(g.Nvx_in))
    d.Dvy = kron(D1D, diagm(g.hxi))
    # Su_ux
    S1D = spdiags(np.c_[-1 / g.hxd, 1 / g.hxd], [0, 1], g.Nux_t - 1, g.Nux_t)
    B = bc_general(g.Nux_t, g.Nux_in, g.Nux_b, BC.u.left, BC.u.right, hx[0], hx[-1])
    d.Su_ux = kron(speye(Ny), S1D @ B.B1D)
    B.Bbc = kron(speye(Ny), S1D @ B.Btemp)
    d.Su_ux_BC = B
    # Su_uy
    S1D = spdiags(np.c_[-1 / g.gyd, 1 / g.gyd], [0, 1], g.Nuy_t - 1, g.Nuy_t)
    B = bc_diff_stag(g.Nuy_t, g.Nuy_in, g.Nuy_b, BC.u.low, BC.u.up, hy[0], hy[-1])
    d.Su_uy = kron(S1D @ B.B1D, speye(g.Nux_in))
    B.Bbc = kron(S1D @ B.Btemp, speye(g.Nux_in))
    d.Su_uy_BC = B
    # Sv_vx
    S1D = spdiags(np.c_[-1 / g.gxd, 1 / g.gxd], [0, 1], g.Nvx_t - 1, g.Nvx_t)
    B = bc_diff_stag(g.Nvx_t, g.Nvx_in, g.Nvx_b, BC.v.left, BC.v.right, hx[0], hx[-1])
    d.Sv_vx = kron(speye(g.Nvy_in), S1D @ B.B1D)
    B.Bbc = kron(speye(g.Nvy_in), S1D @ B.Btemp)
    d.Sv_vx_BC = B
    # Sv_vy
    S1D = spdiags(np.c_[-1 / g.hyd, 1 / g.hyd], [0, 1], g.Nvy_t - 1, g.Nvy_t)
    B = bc_general(g.Nvy_t, g.Nvy_in, g.Nvy_b, BC.v.low, BC.v.up, hy[0], hy[-1])
    d.Sv_vy = kron(S1D @ B.B1D, speye(Nx))
    B.Bbc = kron(S1D @ B.Btemp, speye(Nx))
    d.Sv_vy_BC = B
    d.Diffu = d.Dux @ ((1 / Re) * d.Su_ux) + d.Duy @ ((1 / Re) * d.Su_uy)
    d.Diffv = d.Dvx @ ((1 / Re) * d.Sv_vx) + d.Dvy @ ((1 / Re) * d.Sv_vy)


# ----------------------------------------------------------------------------
# boundary-condition vectors (set_bc_vectors.m, order4=0, laminar)
# ----------------------------------------------------------------------------
def bc_samples(t, o):
    """The BC values set_bc_vectors.m:52-79 samples from uBC/vBC."""
    g = o.grid
    x, y, xp, yp, xin, yin = g.x, g.y, g.xp, g.yp, g.xin, g.yin
    uBC, vBC = o.uBC, o.vBC
    s = SimpleNamespace(
        uLo=uBC(x, y[0], t), uUp=uBC(x, y[-1], t),
        uLo_i=uBC(xin, y[0], t), uUp_i=uBC(xin, y[-1], t),
        uLe_i=uBC(x[0], yp, t), uRi_i=uBC(x[-1], yp, t),
        vLe=vBC(x[0], y, t), vRi=vBC(x[-1], y, t),
        vLo_i=vBC(xp, y[0], t), vUp_i=vBC(xp, y[-1], t),
        vLe_i=vBC(x[0], yin, t), vRi_i=vBC(x[-1], yin, t))
    if o.BC.BC_unsteady == 1:
        s.dudtLe_i = o.dudtBC(x[0], yp, t)
        s.dudtRi_i = o.dudtBC(x[-1], yp, t)
        s.dvdtLo_i = o.dvdtBC(xp, y[0], t)
        s.dvdtUp_i = o.dvdtBC(xp, y[-1], t)
    return s


def _k(a, b):
    return np.kron(np.asarray(a, float).ravel(), np.asarray(b, float).ravel())


def set_bc_vectors(t, o):
    """spatial/boundaryconditions/set_bc_vectors.m:1-345, 415-539 (order4=0,
    laminar)."""
    g, BC, d = o.grid, o.BC, o.discretization
    Re = o.fluid.Re
    s = bc_samples(t, o)
    hx, hy = g.hx, g.hy
    # divergence (:87-118)
    ybc = _k(s.uLe_i, d.Mx_BC.ybc1) + _k(s.uRi_i, d.Mx_BC.ybc2)
    yMx = d.Mx_BC.Bbc @ ybc
    ybc = _k(d.My_BC.ybc1, s.vLo_i) + _k(d.My_BC.ybc2, s.vUp_i)
    yMy = d.My_BC.Bbc @ ybc
    d.yM = yMx + yMy
    # time derivative of divergence (:121-147)
    if BC.BC_unsteady == 1:
        ybc = _k(s.dudtLe_i, d.Mx_BC.ybc1) + _k(s.dudtRi_i, d.Mx_BC.ybc2)
        ydMx = d.Mx_BC.Bbc @ ybc
        ybc = _k(d.My_BC.ybc1, s.dvdtLo_i) + _k(d.My_BC.ybc2, s.dvdtUp_i)
        ydMy = d.My_BC.Bbc @ ybc
        d.ydM = ydMx + ydMy
    else:
        d.ydM = np.zeros(g.Np)
    # pressure (:154-180)
    y1D_le = np.zeros(g.Nux_in)
    y1D_ri = np.zeros(g.Nux_in)
    if BC.u.left == "pres":
        y1D_le[0] = -1
    if BC.u.right == "pres":
        y1D_ri[-1] = 1
    d.y_px = _k(hy * BC.pLe, y1D_le) + _k(hy * BC.pRi, y1D_ri)
    y1D_lo = np.zeros(g.Nvy_in)
    y1D_up = np.zeros(g.Nvy_in)
    if BC.v.low == "pres":
        y1D_lo[0] = -1
    if BC.v.up == "pres":
        y1D_up[-1] = 1
    d.y_py = _k(y1D_lo, hx * BC.pLo) + _k(y1D_up, hx * BC.pUp)
    # averaging (:183-235)
    B = d.Au_ux_BC
    d.yAu_ux = B.Bbc @ (_k(s.uLe_i, B.ybc1) + _k(s.uRi_i, B.ybc2))
    B = d.Au_uy_BC
    d.yAu_uy = B.Bbc @ (_k(B.ybc1, s.uLo_i) + _k(B.ybc2, s.uUp_i))
    B = d.Av_vx_BC
    d.yAv_vx = B.Bbc @ (_k(s.vLe_i, B.ybc1) + _k(s.vRi_i, B.ybc2))
    B = d.Av_vy_BC
    d.yAv_vy = B.Bbc @ (_k(B.ybc1, s.vLo_i) + _k(B.ybc2, s.vUp_i))
    # diffusion (:258-345)
    B = d.Su_ux_BC
    ySu_ux = B.Bbc @ (_k(s.uLe_i, B.ybc1) + _k(s.uRi_i, B.ybc2))
    B = d.Su_uy_BC
    ySu_uy = B.Bbc @ (_k(B.ybc1, s.uLo_i) + _k(B.ybc2, s.uUp_i))
    B = d.Sv_vx_BC
    ySv_vx = B.Bbc @ (_k(s.vLe_i, B.ybc1) + _k(s.vRi_i, B.ybc2))
    B = d.Sv_vy_BC
    ySv_vy = B.Bbc @ (_k(B.ybc1, s.vLo_i) + _k(B.ybc2, s.vUp_i))
    d.yDiffu = d.Dux @ ((1 / Re) * ySu_ux) + d.Duy @ ((1 / Re) * ySu_uy)
    d.yDiffv = d.Dvx @ ((1 / Re) * ySv_vx) + d.Dvy @ ((1 / Re) * ySv_vy)
    # interpolation (:415-539)
    B = d.Iu_ux_BC
    d.yIu_ux = B.Bbc @ (_k(s.uLe_i, B.ybc1) + _k(s.uRi_i, B.ybc2))
    lr, lu = d.Iv_uy_BC_lr, d.Iv_uy_BC_lu
    yIv_uy_lr = lr.Bbc @ (_k(s.vLe, lr.ybc1) + _k(s.vRi, lr.ybc2))
    yIv_uy_lu = lr.B2D @ (lu.Bbc @ (_k(lu.ybc1, s.vLo_i) + _k(lu.ybc2, s.vUp_i)))
    d.yIv_uy = yIv_uy_lr + yIv_uy_lu
    lr, lu = d.Iu_vx_BC_lr, d.Iu_vx_BC_lu
    yIu_vx_lu = lu.Bbc @ (_k(lu.ybc1, s.uLo) + _k(lu.ybc2, s.uUp))
    yIu_vx_lr = lu.B2D @ (lr.Bbc @ (_k(s.uLe_i, lr.ybc1) + _k(s.uRi_i, lr.ybc2)))
    d.yIu_vx = yIu_vx_lr + yIu_vx_lu
    B = d.Iv_vy_BC
    d.yIv_vy = B.Bbc @ (_k(B.ybc1, s.vLo_i) + _k(B.ybc2, s.vUp_i))
    return o


# ----------------------------------------------------------------------------
# right-hand side
# ----------------------------------------------------------------------------
def convection(V, C, t, o):
    """spatial/convection.m:124-215 (convection_components, order4=0,
    regularize=0)."""
    g, d = o.grid, o.discretization
    uh, vh = V[:g.Nu], V[g.Nu:]
    cu, cv = C[:g.Nu], C[g.Nu:]
    u_ux = d.Au_ux @ uh + d.yAu_ux
    uf_ux = d.Iu_ux @ cu + d.yIu_ux
    du2dx = d.Cux @ (uf_ux * u_ux)
    u_uy = d.Au_uy @ uh + d.yAu_uy
    vf_uy = d.Iv_uy @ cv + d.yIv_uy
    duvdy = d.Cuy @ (vf_uy * u_uy)
    v_vx = d.Av_vx @ vh + d.yAv_vx
    uf_vx = d.Iu_vx @ cu + d.yIu_vx
    duvdx = d.Cvx @ (uf_vx * v_vx)
    v_vy = d.Av_vy @ vh + d.yAv_vy
    vf_vy = d.Iv_vy @ cv + d.yIv_vy
    dv2dy = d.Cvy @ (vf_vy * v_vy)
    return du2dx + duvdy, duvdx + dv2dy


def diffusion(V, t, o):
    """spatial/diffusion.m:22-30 (laminar)."""
    g, d = o.grid, o.discretization
    return (d.Diffu @ V[:g.Nu] + d.yDiffu, d.Diffv @ V[g.Nu:] + d.yDiffv)


def F(V, C, p, t, o, nopressure=0):
    """spatial/F.m:1-187 (no force, no temperature, no Jacobian)."""
    g, d = o.grid, o.discretization
    if o.BC.BC_unsteady == 1:
        set_bc_vectors(t, o)
    convu, convv = convection(V, C, t, o)
    d2u, d2v = diffusion(V, t, o)
    Fu = -convu + d2u
    Fv = -convv + d2v
    if nopressure == 0:
        Fu = Fu - (d.Gx @ p + d.y_px)
        Fv = Fv - (d.Gy @ p + d.y_py)
    Fr = np.r_[Fu, Fv]
    return float(np.max(np.abs(Fr))), Fr


# ----------------------------------------------------------------------------
# pressure Poisson
# ----------------------------------------------------------------------------
_CG_LIB = None


def _cg_lib():
    global _CG_LIB
    if _CG_LIB is None:
        here = os.path.dirname(os.path.abspath(__file__))
        path = os.path.join(here, "_build", "libins2d_oracle.so")
        if not os.path.exists(path):
            from . import build as _b  # noqa: F401  (oracle/build.py)
            _b.build()
        lib = ctypes.CDLL(path)
        lib.oracle_cg_dic.restype = ctypes.c_int
        lib.oracle_cg_dic.argtypes = [
            ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long,
            ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_long,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _CG_LIB = lib
    return _CG_LIB


class CGNotConverged(RuntimeError):
    pass


def erk_periodic_c(V, p, Nx, Ny, Lx, Ly, Re, dt, nsteps, RK="RK44", threads=0):
    """oracle/erk_periodic.c: the same explicit RK steps as time_ERK for a
    uniform, doubly periodic grid with the FFT pressure solve, matrix-free and
    OpenMP-parallel (threads = 0: all).  V (2 Nx Ny) and p (Nx Ny) are
    returned as new arrays."""
    lib = _cg_lib()
    if not hasattr(lib, "_erk_ready"):
        lib.oracle_erk_periodic.restype = ctypes.c_int
        lib.oracle_erk_periodic.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_int]
        lib.oracle_max_threads.restype = ctypes.c_int
        lib._erk_ready = True
    A, b, c = getRKmethod(RK)
    A = np.ascontiguousarray(A, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    c = np.ascontiguousarray(c, dtype=np.float64)
    V = np.array(V, dtype=np.float64)
    p = np.array(p, dtype=np.float64)
    rc = lib.oracle_erk_periodic(Nx, Ny, Lx, Ly, Re, len(b), A.ctypes.data, b.ctypes.data, c.ctypes.data, dt,
                                 nsteps, V.ctypes.data, p.ctypes.data, threads)
    if rc != 0:
        raise RuntimeError(f"oracle_erk_periodic failed ({rc})")
    return V, p


def oracle_threads():
    """Threads the OpenMP restatement uses by default."""
    erk = _cg_lib()
    erk.oracle_max_threads.restype = ctypes.c_int
    return int(erk.oracle_max_threads())


def lower_diagonals(A):
    """The storage cg.F / cg_matlab.m use: [B,d]=spdiags(A), the main and lower
    diagonals in order of distance (cg_matlab.m:30-34,
    operator_divergence.m:221-224)."""
    B, dd = spdiags_extract(A)
    nd = (len(dd) + 1) // 2
    Bl = np.ascontiguousarray(B[:, nd - 1::-1])
    dia = dd[nd - 1:].astype(np.int64)
    return Bl, dia


def cg_dic(A, y, tol, x_in, maxit, storage=None):
    """Fortran MEX solvers/pressure/cg.F:158-280 (PCG with a
    diagonal-incomplete-Cholesky preconditioner, cg.F:317-429), restated in C
    (oracle/cg_dic.c) and called through ctypes.  Returns x, iter, norm1,
    norm2."""
    if storage is None:
        storage = lower_diagonals(A)
    Bl, dia = storage
    N = Bl.shape[0]
    nd = Bl.shape[1]
    Bf = np.asfortranarray(Bl)
    y = np.ascontiguousarray(y, dtype=float)
    x_in = np.ascontiguousarray(x_in, dtype=float)
    x = np.zeros(N)
    it = np.zeros(1, np.int64)
    n1 = np.zeros(1)
    n2 = np.zeros(1)
    lib = _cg_lib()
    st = lib.oracle_cg_dic(N, Bf.ctypes.data, dia.ctypes.data, nd, y.ctypes.data, tol,
                           x_in.ctypes.data, maxit, x.ctypes.data, it.ctypes.data,
                           n1.ctypes.data, n2.ctypes.data)
    if st != 0:
        raise CGNotConverged("CG didn't converge in maxiter iterations")
    return x, int(it[0]), float(n1[0]), float(n2[0])


def pressure_poisson(f, t, o):
    """solvers/pressure/pressure_poisson.m:1-106.  Branch 6 (FFT) exactly;
    branches 3/4 (PCG with DIC) via cg_dic; branch 1 (direct) via a sparse LU
    with one pressure value fixed when A is singular (the velocity only sees
    G*dp, which is blind to that constant)."""
    g, d, ss = o.grid, o.discretization, o.solversettings
    Np = g.Np
    dp = np.zeros(Np)
    poisson = ss.poisson
    if poisson == 6:
        Ahat = ss.Ahat
        fhat = np.fft.fft2(f.reshape(g.Npy, g.Npx).T)
        if np.max(np.abs(Ahat * 0 + fhat)) < 1e-14:
            ss.last_iter, ss.last_norm1 = 0, 0.0
            return dp
        phat = -fhat / Ahat
        dp = np.real(np.fft.ifft2(phat)).T.ravel()
        ss.last_iter, ss.last_norm1 = 0, 0.0
        return dp
    A = d.A
    if np.max(np.abs(A @ dp - f)) < 1e-14:
        ss.last_iter, ss.last_norm1 = 0, 0.0
        return dp
    if poisson == 1:
        if not hasattr(ss, "_lu"):
            singular = not any(s == "pres" for s in (o.BC.u.left, o.BC.u.right, o.BC.v.low, o.BC.v.up))
            ss._singular = singular
            As = A[1:, 1:] if singular else A
            ss._lu = spla.splu(sp.csc_matrix(As))
        if ss._singular:
            dp[1:] = ss._lu.solve(f[1:])
        else:
            dp = ss._lu.solve(f)
        ss.last_iter, ss.last_norm1 = 0, 0.0
        return dp
    if poisson in (2, 3, 4, 5):
        if not hasattr(ss, "_cg_storage"):
            ss._cg_storage = lower_diagonals(A)
        dp, it, n1, n2 = cg_dic(A, f, ss.CG_acc, dp, ss.CG_maxit, ss._cg_storage)
        ss.last_iter, ss.last_norm1 = it, n1
        return dp
    raise ValueError("wrong poisson method")


def pressure_additional_solve(V, p, t, o):
    """solvers/pressure/pressure_additional_solve.m:1-25."""
    g, d = o.grid, o.discretization
    if o.BC.BC_unsteady == 1:
        set_bc_vectors(t, o)
    _, R = F(V, V, p, t, o)
    f = d.M @ (g.Om_inv * R) + d.ydM
    dp = pressure_poisson(f, t, o)
    return p + dp


# ----------------------------------------------------------------------------
# time integration
# ----------------------------------------------------------------------------
RK_TABLES = {
    # unsteady/getRKmethod.m (A, b; c = row sums unless given)
    "FE11": ([[0]], [1], None),
    "SSP22": ([[0, 0], [1, 0]], [0.5, 0.5], None),
    "SSP33": ([[0, 0, 0], [1, 0, 0], [0.25, 0.25, 0]], [1 / 6, 1 / 6, 2 / 3], None),
    "Heun33": ([[0, 0, 0], [1 / 3, 0, 0], [0, 2 / 3, 0]], [0.25, 0, 0.75], None),
    "RK33C2": ([[0, 0, 0], [2 / 3, 0, 0], [1 / 3, 1 / 3, 0]], [0.25, 0, 0.75], [0, 2 / 3, 2 / 3]),
    "RK33P2": ([[0, 0, 0], [1 / 3, 0, 0], [-1, 2, 0]], [0, 0.75, 0.25], [0, 1 / 3, 1]),
    "Wray3": ([[0, 0, 0], [8 / 15, 0, 0], [8 / 15 - 17 / 60, 5 / 12, 0]], [8 / 15 - 17 / 60, 0, 0.75],
              [0, 8 / 15, 8 / 15 - 17 / 60 + 5 / 12]),
    "RK44": ([[0, 0, 0, 0], [0.5, 0, 0, 0], [0, 0.5, 0, 0], [0, 0, 1, 0]],
             [1 / 6, 1 / 3, 1 / 3, 1 / 6], None),
    "RK44C2": ([[0, 0, 0, 0], [0.25, 0, 0, 0], [0, 0.5, 0, 0], [1, -2, 2, 0]],
               [1 / 6, 0, 2 / 3, 1 / 6], [0, 0.25, 0.5, 1]),
    "RK44C23": ([[0, 0, 0, 0], [0.5, 0, 0, 0], [0.25, 0.25, 0, 0], [0, -1, 2, 0]],
                [1 / 6, 0, 2 / 3, 1 / 6], [0, 0.5, 0.5, 1]),
    "RK44P2": ([[0, 0, 0, 0], [1, 0, 0, 0], [3 / 8, 1 / 8, 0, 0], [-1 / 8, -3 / 8, 3 / 2, 0]],
               [1 / 6, -1 / 18, 2 / 3, 2 / 9], [0, 1, 0.5, 1]),
}


def getRKmethod(name):
    """unsteady/getRKmethod.m (table data for the explicit methods above)."""
    A, b, c = RK_TABLES[name]
    A = np.array(A, float)
    b = np.array(b, float)
    c = A.sum(axis=1) if c is None else np.array(c, float)
    return A, b, c


def time_ERK(Vn, pn, tn, dt, o):
    """unsteady/time_ERK.m:1-173 (no temperature)."""
    g, d = o.grid, o.discretization
    A_RK, b_RK, c_RK = getRKmethod(o.time.RK)
    s = len(b_RK)
    A_RK = np.vstack([A_RK[1:, :], b_RK[None, :]])
    c_RK = np.r_[c_RK[1:], 1.0]
    V = Vn.copy()
    p = pn.copy()
    kV = np.zeros((g.NV, s))
    kp = np.zeros((g.Np, s))
    if o.BC.BC_unsteady == 1:
        set_bc_vectors(tn, o)
    G, M = d.G, d.M
    yM = d.yM
    ti = tn
    stats = []
    for i in range(s):
        _, F_rhs = F(V, V, p, ti, o)
        kV[:, i] = g.Om_inv * (F_rhs + G @ p)
        Vtemp = kV @ A_RK[i, :]
        ti = tn + c_RK[i] * dt
        if o.BC.BC_unsteady == 1:
            set_bc_vectors(ti, o)
            yM = d.yM
        f = (M @ (Vn / dt + Vtemp) + yM / dt) / c_RK[i]
        if o.BC.BC_unsteady == 1 or i > 0:
            dp = pressure_poisson(f, ti, o)
            stats.append((o.solversettings.last_iter, o.solversettings.last_norm1))
        else:
            dp = pn
        kp[:, i] = dp
        V = Vn + dt * (Vtemp - c_RK[i] * g.Om_inv * (G @ dp))
    if o.BC.BC_unsteady == 1:
        if o.solversettings.p_add_solve == 1:
            p = pressure_additional_solve(V, p, tn + dt, o)
            stats.append((o.solversettings.last_iter, o.solversettings.last_norm1))
        else:
            p = kp[:, -1].copy()
    else:
        p = pressure_additional_solve(V, p, tn + dt, o)
        stats.append((o.solversettings.last_iter, o.solversettings.last_norm1))
    o.last_step_stats = stats
    return V, p


# ----------------------------------------------------------------------------
# diagnostics and initialisation
# ----------------------------------------------------------------------------
def check_conservation(V, t, o):
    """spatial/check_conservation.m:1-76."""
    g, d, BC = o.grid, o.discretization, o.BC
    uh, vh = V[:g.Nu], V[g.Nu:]
    if BC.BC_unsteady == 1:
        set_bc_vectors(t, o)
    s = bc_samples(t, o)
    maxdiv = float(np.max(np.abs(d.M @ V + d.yM)))
    umom = float(np.sum(g.Omu * uh))
    vmom = float(np.sum(g.Omv * vh))
    if BC.u.left == "dir":
        umom += np.sum(s.uLe_i * g.hy) * g.gx[0]
    if BC.u.right == "dir":
        umom += np.sum(s.uRi_i * g.hy) * g.gx[-1]
    if BC.v.low == "dir":
        vmom += np.sum(s.vLo_i * g.hx) * g.gy[0]
    if BC.v.up == "dir":
        vmom += np.sum(s.vUp_i * g.hx) * g.gy[-1]
    k = 0.5 * np.sum(g.Omu * uh ** 2) + 0.5 * np.sum(g.Omv * vh ** 2)
    if BC.u.left == "dir":
        k += 0.5 * np.sum((s.uLe_i ** 2) * g.hy) * g.gx[0]
    if BC.u.right == "dir":
        k += 0.5 * np.sum((s.uRi_i ** 2) * g.hy) * g.gx[-1]
    if BC.v.low == "dir":
        k += 0.5 * np.sum((s.vLo_i ** 2) * g.hx) * g.gy[0]
    if BC.v.up == "dir":
        k += 0.5 * np.sum((s.vUp_i ** 2) * g.hx) * g.gy[-1]
    return maxdiv, float(umom), float(vmom), float(k)


def convection_matrices(V, o):
    """The convection operators Cu, Cv of set_timestep.m:8-12 / check_symmetry.m
    (convection of V by the field V, linear in the convected field)."""
    g, d = o.grid, o.discretization
    uh, vh = V[:g.Nu], V[g.Nu:]
    Cu = (d.Cux @ diagm(d.Iu_ux @ uh + d.yIu_ux) @ d.Au_ux
          + d.Cuy @ diagm(d.Iv_uy @ vh + d.yIv_uy) @ d.Au_uy)
    Cv = (d.Cvx @ diagm(d.Iu_vx @ uh + d.yIu_vx) @ d.Av_vx
          + d.Cvy @ diagm(d.Iv_vy @ vh + d.yIv_vy) @ d.Av_vy)
    return Cu, Cv


def check_symmetry(V, t, o, tol=1e-14):
    """spatial/check_symmetry.m:42-61: the convection operator must be
    skew-symmetric."""
    Cu, Cv = convection_matrices(V, o)
    eu = abs(Cu + Cu.T).max() if Cu.nnz else 0.0
    ev = abs(Cv + Cv.T).max() if Cv.nnz else 0.0
    err = float(max(eu, ev))
    return err <= tol, err


def initial_projection(V, t, o):
    """preprocessing/input_check.m:95-111: project the initial field when its
    divergence exceeds 1e-12."""
    g, d = o.grid, o.discretization
    maxdiv = check_conservation(V, t, o)[0]
    if maxdiv > 1e-12:
        f = d.M @ V + d.yM
        dp = pressure_poisson(f, t, o)
        V = V - g.Om_inv * (d.G @ dp)
    return V


def velocity_from_streamfunction(psi, o):
    """postprocessing/get_velocity_from_streamfunction.m (periodic grids):
    V = W' psi with W = [-Wu_uy Wv_vx]."""
    g = o.grid
    Nx, Ny = g.Nx, g.Ny
    d1 = 1 / g.hy
    W1D = spdiags(np.c_[-d1, d1], [-1, 0], Ny, Ny).tolil()
    W1D[0, Ny - 1] = -W1D[0, 0]
    Wu_uy = kron(sp.csr_matrix(W1D), speye(Nx))
    d1 = 1 / g.hx
    W1D = spdiags(np.c_[-d1, d1], [-1, 0], Nx, Nx).tolil()
    W1D[0, Nx - 1] = -W1D[0, 0]
    Wv_vx = kron(speye(Ny), sp.csr_matrix(W1D))
    W = sp.hstack([-Wu_uy, Wv_vx], format="csr")
    return W.T @ psi


def run(o, V0, p0, dt, nsteps, t0=0.0, p_initial=True, log=None):
    """solver_unsteady.m:72-120 for method 20 (ERK) with the per-step
    check_conservation and residual of process_iteration.m:4,22."""
    V = initial_projection(np.asarray(V0, float).copy(), t0, o)
    p = np.asarray(p0, float).copy()
    if p_initial:
        p = pressure_additional_solve(V, p, t0, o)
    t = t0
    hist = []
    res = F(V, V, p, t, o)[0]
    hist.append((0, t, res) + check_conservation(V, t, o))
    for n in range(1, nsteps + 1):
        V, p = time_ERK(V, p, t, dt, o)
        t = t0 + n * dt
        if log is not None:
            res = F(V, V, p, t, o)[0]
            hist.append((n, t, res) + check_conservation(V, t, o))
    return V, p, hist
