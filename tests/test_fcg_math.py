"""The flexible CG recurrence of the network-preconditioned solve (FCG(1):
alpha = p'r / p'Ap, beta = -z'Ap / p'Ap, as in the context's fcg_learned),
restated in numpy (no GPU): with a fixed SPD preconditioner it takes the
iterations of preconditioned CG; with a nonlinear, odd and homogeneous
preconditioner (the form of the network's odd part) it still reaches the
stopping rule ||r|| <= tol ||f||."""
import numpy as np


def laplacian_1d2d(n):
    """negative-definite 5-point Laplacian with Dirichlet walls, n x n cells"""
    T = np.diag(-2.0 * np.ones(n)) + np.diag(np.ones(n - 1), 1) + np.diag(np.ones(n - 1), -1)
    I = np.eye(n)
    return np.kron(I, T) + np.kron(T, I)


def fcg1(A, f, M, tol, maxit=2000):
    x = np.zeros_like(f)
    r = f.copy()
    ff = f @ f
    z = M(r)
    p = z.copy()
    for it in range(1, maxit + 1):
        q = A @ p
        pq = p @ q
        a = (p @ r) / pq
        x += a * p
        r -= a * q
        if r @ r <= tol * tol * ff:
            return x, it
        z = M(r)
        p = z - ((z @ q) / pq) * p
    return x, maxit


def pcg(A, f, M, tol, maxit=2000):
    x = np.zeros_like(f)
    r = f.copy()
    ff = f @ f
    z = M(r)
    p = z.copy()
    rz = r @ z
    for it in range(1, maxit + 1):
        q = A @ p
        a = rz / (p @ q)
        x += a * p
        r -= a * q
        if r @ r <= tol * tol * ff:
            return x, it
        z = M(r)
        rz, rz_old = r @ z, rz
        p = z + (rz / rz_old) * p
    return x, maxit


def test_fcg1_with_a_fixed_preconditioner_takes_pcg_iterations():
    A = laplacian_1d2d(16)
    f = np.random.default_rng(0).standard_normal(A.shape[0])
    d = np.diag(A)
    M = lambda r: r / d  # Jacobi (A is negative definite, so is M)
    x1, it1 = fcg1(A, f, M, 1e-10)
    x2, it2 = pcg(A, f, M, 1e-10)
    assert abs(it1 - it2) <= 1
    assert np.linalg.norm(A @ x1 - f) <= 1e-10 * np.linalg.norm(f) * (1 + 1e-6)


def test_fcg1_with_a_nonlinear_odd_preconditioner_converges():
    A = laplacian_1d2d(16)
    f = np.random.default_rng(1).standard_normal(A.shape[0])
    d = np.diag(A)

    def M(r):  # odd and homogeneous of degree one, but not linear
        s = np.sqrt(np.mean(r * r)) or 1.0
        v = r / s
        return s * (v + 0.3 * v ** 3 / (1 + v * v)) / d

    x, it = fcg1(A, f, M, 1e-10)
    assert it < 2000
    assert np.linalg.norm(A @ x - f) <= 1e-10 * np.linalg.norm(f) * (1 + 1e-6)
