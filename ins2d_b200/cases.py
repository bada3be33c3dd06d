"""Case definitions for the benchmark configurations: grids, boundary
functions and initial fields (the roles of a reference case's
``<case>_mesh.m``, ``<case>_uBC.m``/``_vBC.m`` and ``<case>_IC.m``).

Setup-only host code: nothing here is on the time-stepping path.
"""
from __future__ import annotations

import math

import numpy as np

BC_CAVITY = {"u": dict(left="dir", right="dir", low="dir", up="dir"),
             "v": dict(left="dir", right="dir", low="dir", up="dir")}
BC_PERIODIC = {"u": dict(left="per", right="per", low="per", up="per"),
               "v": dict(left="per", right="per", low="per", up="per")}
# channel / backward-facing step: inflow left (dir), outflow right (pres,
# p = 0), walls low/up (BFS_unsteady_BCtype.m)
BC_CHANNEL = {"u": dict(left="dir", right="pres", low="dir", up="dir"),
              "v": dict(left="dir", right="sym", low="dir", up="dir")}


def uniform_grid(N, a, b):
    """Uniform grid lines (nonuniform_grid.m with stretch factor 1)."""
    return a + (b - a) * np.arange(N + 1) / N


def nonuniform_grid(deltaz, z_low, z_up, sz):
    """libs/nonuniform_grid.m:1-63: geometric stretching from z_low with first
    spacing deltaz and a stretch factor adapted by a secant iteration so the
    grid ends at z_up."""
    eps = 1e-12
    if sz == 1:
        n = (z_up - z_low) / deltaz
        if abs(n - round(n)) > eps:
            deltaz = (z_up - z_low) / math.floor(n)
        nint = int(math.floor((z_up - z_low) / deltaz + 1e-10))
        return z_low + deltaz * np.arange(nint + 1)
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
    out = np.zeros(n)
    out[0] = z_low
    for k in range(1, n):
        out[k] = out[k - 1] + deltaz * sz ** (k - 1)
    return out


def tanh_grid(N, a, b, stretch):
    """Grid lines clustered towards both ends by the tanh map
    z(s) = tanh(stretch * s) / tanh(stretch), s uniform in [-1, 1] (the
    reference has no tanh stretching; this is the map the benchmark
    configurations name, with ``stretch`` its parameter: 1.05 makes the
    end cells about 2.6 times narrower than the middle ones).  stretch <= 0
    gives the uniform grid."""
    if stretch <= 0.0:
        return uniform_grid(N, a, b)
    s = np.linspace(-1.0, 1.0, N + 1)
    z = np.tanh(stretch * s) / np.tanh(stretch)
    z[0], z[-1] = -1.0, 1.0
    return a + (b - a) * (z + 1) / 2


def lid_uBC(U=1.0, y_lid=1.0):
    """uBC of a lid-driven cavity (LDC_unsteady_uBC.m): u = U on the lid."""
    def uBC(x, y, t):
        n = np.size(x) * np.size(y)
        if np.size(y) == 1 and abs(float(np.ravel(y)[0]) - y_lid) < 1e-10:
            return np.full(n, float(U))
        return np.zeros(n)
    return uBC


def channel_uBC(profile):
    """uBC for a channel: profile(y) on the left boundary, zero elsewhere
    (the right boundary is an outflow with zero normal derivative)."""
    def uBC(x, y, t):
        x = np.atleast_1d(np.asarray(x, float))
        y = np.atleast_1d(np.asarray(y, float))
        n = x.size * y.size
        if x.size == 1 and abs(x[0] - channel_uBC.x_left) < 1e-12 and y.size > 0:
            return profile(y)
        return np.zeros(n)
    return uBC


channel_uBC.x_left = 0.0


def taylor_green(opts):
    """u = sin x cos y, v = -cos x sin y at the staggered points."""
    return np.r_[np.sin(opts.xu) * np.cos(opts.yu), -np.cos(opts.xv) * np.sin(opts.yv)]


def streamfunction_velocity(psi, opts):
    """get_velocity_from_streamfunction.m for periodic grids: V = W' psi with
    W = [-Wu_uy Wv_vx] (discrete curl; discretely divergence free).  psi is
    given at the Nx x Ny corner points, x fastest."""
    Nx, Ny = opts.Nx, opts.Ny
    hx, hy = np.diff(opts.x), np.diff(opts.y)
    P = psi.reshape(Ny, Nx)
    # Wu_uy = kron(W1D_y, I): (W1D_y psi)(j) = (psi(j) - psi(j-1))/hy(j-1) (cyclic), u = -Wu_uy' psi
    # W1D(i,i) = 1/h(i), W1D(i+1,i) = -1/h(i), W1D(1,end) = -1/h(1)
    # (W1D' q)(i) = q(i)/h(i) - q(i+1)/h(i)  for i<N;  (W1D' q)(N) = q(N)/h(N) - q(1)/h(1)
    def w1d_t(q, h, axis):
        qn = np.roll(q, -1, axis=axis)
        shape = [1, 1]
        shape[axis] = -1
        hh = h.reshape(shape)
        out = q / hh - qn / hh
        # last entry uses h(1) for the wrapped term
        idx = [slice(None), slice(None)]
        idx[axis] = -1
        last_q = np.take(q, -1, axis=axis)
        first_q = np.take(q, 0, axis=axis)
        out[tuple(idx)] = last_q / h[-1] - first_q / h[0]
        return out
    u = -w1d_t(P, hy, 0)
    v = w1d_t(P, hx, 1)
    return np.r_[u.ravel(), v.ravel()]


def _turbulence_velocity(opts, k0, seed):
    Nx, Ny = opts.Nx, opts.Ny
    rng = np.random.default_rng(seed)
    kx = np.fft.rfftfreq(Nx, d=1.0 / Nx)   # integer wave numbers, x (halved axis)
    ky = np.fft.fftfreq(Ny, d=1.0 / Ny)
    KX, KY = np.meshgrid(kx, ky)          # shape (Ny, Nx//2+1)
    K = np.sqrt(KX ** 2 + KY ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        E = K ** 4 * np.exp(-2.0 * (K / k0) ** 2)
        amp = np.where(K > 0, np.sqrt(E / (np.pi * K)) / K, 0.0)
    spec = amp * np.exp(2j * np.pi * rng.random(amp.shape))
    psi = np.fft.irfft2(spec, s=(Ny, Nx)).ravel()  # (j, i) -> x fastest
    return streamfunction_velocity(psi, opts)


def decaying_turbulence_ic(opts, k0=10.0, seed=2048, energy=1.0):
    """Random-phase streamfunction with energy spectrum E(k) ~ k^4 exp(-2 (k/k0)^2)
    on a periodic grid, turned into a discretely divergence-free velocity and
    scaled to kinetic energy ``energy`` (check_conservation.m k)."""
    V = _turbulence_velocity(opts, k0, seed)
    k = opts.check_conservation(V, 0.0)[3]
    return V * math.sqrt(energy / k)


def decaying_turbulence_ic_host(N, L=1.0, k0=10.0, seed=2048, energy=1.0):
    """The same field on the uniform periodic N x N grid of side L, computed
    on the host alone (no device context): on that grid every u and v point
    has the volume hx*hy, so check_conservation.m's k is hx*hy*sum(V^2)/2."""
    from types import SimpleNamespace
    x = uniform_grid(N, 0.0, L)
    g = SimpleNamespace(Nx=N, Ny=N, x=x, y=x.copy())
    V = _turbulence_velocity(g, k0, seed)
    h = L / N
    k = 0.5 * h * h * float(np.dot(V, V))
    return V * math.sqrt(energy / k)


def cfl_dt(opts, V, cfl=0.5):
    """dt = cfl * min(h) / max|u| (the CFL rule the turbulence configuration
    names; set_timestep.m has no branch for explicit RK)."""
    h = min(np.min(np.diff(opts.x)), np.min(np.diff(opts.y)))
    return cfl * h / float(np.max(np.abs(V)))
