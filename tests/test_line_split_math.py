"""The algebra of the multigrid line solves split over several warps
(mg_line_split, mg_ycols_block), restated in numpy and checked against a
direct tridiagonal solve (no GPU): Thomas factors, the forward and backward
recurrences as affine maps, 32-cell chunks scanned per warp, range composites
chained across warps, and the re-walk of each range from its carry."""
import numpy as np
import pytest


def thomas_factors(a, b, c):
    """fi = 1/pivot, fc = c' of the Thomas algorithm (mg_factor_xline without
    the cyclic correction)."""
    n = len(b)
    fi, fc = np.zeros(n), np.zeros(n)
    cp = 0.0
    for i in range(n):
        inv = 1.0 / (b[i] - (a[i] * cp if i > 0 else 0.0))
        cp = c[i] * inv if i < n - 1 else 0.0
        fi[i], fc[i] = inv, cp
    return fi, fc


def split_solve(a, fi, fc, r, P, chunk=32):
    """Forward d_i = A_i d_{i-1} + B_i (A_i = -a_i fi_i, B_i = r_i fi_i) and
    backward x_i = -fc_i x_{i+1} + d_i, each over P ranges of chunks: pass 1
    composes a range's maps, the composites give each range its carry, pass 2
    re-walks the range."""
    n = len(r)
    A = np.where(np.arange(n) > 0, -a * fi, 0.0)
    B = r * fi
    chunks = (n + chunk - 1) // chunk
    per = (chunks + P - 1) // P
    ranges = [(min(chunks, q * per), min(chunks, q * per + per)) for q in range(P)]

    def cells(c):
        return range(c * chunk, min(n, (c + 1) * chunk))

    # forward, pass 1: composite (SA, SB) of each range
    comp = []
    for lo, hi in ranges:
        SA, SB = 1.0, 0.0
        for c in range(lo, hi):
            for i in cells(c):
                SA, SB = A[i] * SA, A[i] * SB + B[i]
        comp.append((SA, SB))
    d = np.zeros(n)
    for q, (lo, hi) in enumerate(ranges):
        carry = 0.0
        for SA, SB in comp[:q]:
            carry = SA * carry + SB
        for c in range(lo, hi):
            for i in cells(c):
                carry = A[i] * carry + B[i]
                d[i] = carry
    # backward, pass 1 (right to left)
    Ab, Bb = -fc, d
    comp = []
    for lo, hi in ranges:
        SA, SB = 1.0, 0.0
        for c in range(hi - 1, lo - 1, -1):
            for i in reversed(cells(c)):
                SA, SB = Ab[i] * SA, Ab[i] * SB + Bb[i]
        comp.append((SA, SB))
    x = np.zeros(n)
    for q, (lo, hi) in enumerate(ranges):
        carry = 0.0
        for SA, SB in reversed(comp[q + 1:]):
            carry = SA * carry + SB
        for c in range(hi - 1, lo - 1, -1):
            for i in reversed(cells(c)):
                carry = Ab[i] * carry + Bb[i]
                x[i] = carry
    return x


@pytest.mark.parametrize("n", [1, 5, 31, 33, 76, 151, 301, 1024])
@pytest.mark.parametrize("P", [1, 2, 4, 8])
def test_split_solve_matches_direct_solve(n, P):
    rng = np.random.default_rng(n * 10 + P)
    a = -rng.uniform(0.5, 1.5, n)
    c = -rng.uniform(0.5, 1.5, n)
    b = -(a + c) + rng.uniform(0.1, 1.0, n)  # diagonally dominant, like a relaxed Laplacian line
    r = rng.standard_normal(n)
    fi, fc = thomas_factors(a, b, c)
    x = split_solve(a, fi, fc, r, P)
    T = np.diag(b) + np.diag(a[1:], -1) + np.diag(c[:-1], 1)
    assert np.allclose(T @ x, r, rtol=0, atol=1e-12 * np.max(np.abs(r)) * n)
