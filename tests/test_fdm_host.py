"""Host side of the fast-diagonalization preconditioner (fdm_host.cpp),
through the test probe: the generalized eigen-decompositions T Q = diag(h) Q
Lambda of the pressure matrix's 1D factors (Q' diag(h) Q = I), and the
resulting exact inverse of A = M Om^-1 G on the range of A, against the
oracle's assembled matrix (operator_divergence.m:208) on stretched grids and
every boundary-condition kind."""
import numpy as np
import pytest

from oracle import ins2d_ref as R
from tests.cases_common import BC_COMBOS, grid_stretched, grid_uniform
from tests.test_host_tables import Tables, probe  # noqa: F401  (module fixture)


def _fdm(probe_lib, T, nx, ny):
    import ctypes
    probe_lib.probe_fdm.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    out = []
    for d, n in ((0, nx), (1, ny)):
        Q = np.zeros(n * n)
        lam = np.zeros(n)
        got = probe_lib.probe_fdm(T.h, d, Q.ctypes.data, lam.ctypes.data)
        assert got == n, probe_lib.probe_error()
        out.append((Q.reshape(n, n), lam))
    return out


@pytest.mark.parametrize("combo", ["cavity", "periodic", "channel", "open_x", "per_x_walls", "open_y_both"])
@pytest.mark.parametrize("stretch", [False, True])
def test_fdm_inverse(probe, combo, stretch):
    nx, ny = 23, 17
    x = grid_stretched(nx, 0.0, 1.7) if stretch else grid_uniform(nx, 0.0, 1.7)
    y = grid_stretched(ny, -0.5, 0.5, beta=1.3) if stretch else grid_uniform(ny, -0.5, 0.5)
    bc = BC_COMBOS[combo]
    T = Tables(probe, x, y, bc, 100.0)
    (Qx, lx), (Qy, ly) = _fdm(probe, T, nx, ny)
    o = R.make_options(x, y, bc, Re=100.0, poisson=1)
    hx, hy = np.diff(x), np.diff(y)
    # Q' diag(h) Q = I, eigenvalues >= 0
    assert np.max(np.abs(Qx.T @ (hx[:, None] * Qx) - np.eye(nx))) < 1e-12
    assert np.max(np.abs(Qy.T @ (hy[:, None] * Qy) - np.eye(ny))) < 1e-12
    assert lx.min() >= 0.0 and ly.min() >= 0.0
    # A^+ f through the transforms, for a consistent right-hand side
    A = o.discretization.A.toarray()
    rng = np.random.default_rng(2)
    f = o.discretization.M @ rng.standard_normal(o.grid.NV)
    F = f.reshape(ny, nx)  # memory order: rows j, x fastest
    Y = Qy.T @ F @ Qx      # [b, a]
    lam = lx[None, :] + ly[:, None]
    scale = np.where(lam > 1e-12 * lam.max(), -1.0 / np.where(lam > 0, lam, 1.0), 0.0)
    z = (Qy @ (Y * scale) @ Qx.T).ravel()
    assert np.linalg.norm(A @ z - f) <= 1e-11 * np.linalg.norm(f)
