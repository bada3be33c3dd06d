"""The multigrid hierarchy of the pressure preconditioner (mg_host.cpp), on
the CPU: level 0 rebuilt from its 1D rows equals the oracle's pressure
matrix A = M Om^-1 G (operator_divergence.m:208), every coarse level equals
the Galerkin product P' A P of the level above for piecewise-constant
aggregation, and the coarsest level's dense pseudo-inverse matches numpy's."""
import ctypes
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import ins2d_ref as R
from tests.cases_common import BC_COMBOS, grid_stretched, grid_uniform

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BCCODE = {"dir": 0, "pres": 1, "per": 2, "sym": 3}


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    out = tmp_path_factory.mktemp("probe_mg") / "libprobe_mg.so"
    csrc = os.path.join(ROOT, "ins2d_b200", "csrc")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I", csrc,
                           os.path.join(ROOT, "tests", "native", "probe.cpp"), os.path.join(csrc, "setup.cpp"),
                           os.path.join(csrc, "mg_host.cpp"), os.path.join(csrc, "fdm_host.cpp"), "-o", str(out)])
    lib = ctypes.CDLL(str(out))
    lib.probe_build.restype = ctypes.c_void_p
    lib.probe_build.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_double]
    lib.probe_free.argtypes = [ctypes.c_void_p]
    lib.probe_error.restype = ctypes.c_char_p
    lib.probe_mg_build.restype = ctypes.c_void_p
    lib.probe_mg_build.argtypes = [ctypes.c_void_p]
    lib.probe_mg_free.argtypes = [ctypes.c_void_p]
    lib.probe_mg_nlev.argtypes = [ctypes.c_void_p]
    lib.probe_mg_level.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_void_p)]
    lib.probe_mg_pinv.restype = ctypes.c_void_p
    lib.probe_mg_pinv.argtypes = [ctypes.c_void_p]
    return lib


def _levels(lib, x, y, bc):
    codes = np.array([BCCODE[bc[c][s]] for c in ("u", "v") for s in ("left", "right", "low", "up")], np.int32)
    x = np.ascontiguousarray(x, float)
    y = np.ascontiguousarray(y, float)
    h = lib.probe_build(len(x) - 1, len(y) - 1, x.ctypes.data, y.ctypes.data, codes.ctypes.data, 1.0)
    assert h, lib.probe_error()
    m = lib.probe_mg_build(h)
    assert m, lib.probe_error()
    out = []
    for l in range(lib.probe_mg_nlev(m)):
        dims = np.zeros(6, np.int32)
        vecs = []
        for w in range(8):
            p = ctypes.c_void_p()
            assert lib.probe_mg_level(m, l, dims.ctypes.data, w, ctypes.byref(p)) == 0
            n = dims[0] if w < 4 else dims[1]
            vecs.append(np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_double)), shape=(n,)).copy())
        out.append((dims.copy(), vecs))
    nc = out[-1][0][0] * out[-1][0][1]
    pinv = np.ctypeslib.as_array(ctypes.cast(lib.probe_mg_pinv(m), ctypes.POINTER(ctypes.c_double)),
                                 shape=(nc * nc,)).copy().reshape(nc, nc)
    lib.probe_mg_free(m)
    lib.probe_free(h)
    return out, pinv


def _tri(m, z0, p, per):
    n = len(z0)
    T = sp.lil_matrix((n, n))
    for i in range(n):
        T[i, i] += z0[i]
        if i > 0 or per:
            T[i, (i - 1) % n] += m[i]
        if i < n - 1 or per:
            T[i, (i + 1) % n] += p[i]
    return T.tocsr()


def _matrix(dims, v):
    nx, ny, perx, pery = dims[:4]
    xm, x0, xp, hx, ym, y0, yp, hy = v
    TX = _tri(xm, x0, xp, perx)
    TY = _tri(ym, y0, yp, pery)
    return -(sp.kron(sp.diags(hy), TX) + sp.kron(TY, sp.diags(hx)))


def _agg(nx, ny, cx, cy):
    ncx = (nx + cx - 1) // cx
    ncy = (ny + cy - 1) // cy
    i = np.tile(np.arange(nx), ny)
    j = np.repeat(np.arange(ny), nx)
    return sp.csr_matrix((np.ones(nx * ny), (i + j * nx, i // cx + (j // cy) * ncx)), shape=(nx * ny, ncx * ncy))


@pytest.mark.parametrize("combo", sorted(BC_COMBOS))
@pytest.mark.parametrize("shape", [(24, 20), (37, 9), (7, 64)])
def test_mg_hierarchy(probe, combo, shape):
    nx, ny = shape
    x = grid_stretched(nx, 0.0, 1.7)
    y = grid_stretched(ny, -0.5, 0.5, beta=1.2)
    bc = BC_COMBOS[combo]
    if "per" in (bc["u"]["left"], bc["v"]["low"]):
        x = grid_uniform(nx, 0.0, 1.7) if bc["u"]["left"] == "per" else x
        y = grid_uniform(ny, -0.5, 0.5) if bc["v"]["low"] == "per" else y
    o = R.make_options(x, y, bc, poisson=4)
    levels, pinv = _levels(probe, x, y, bc)
    A = _matrix(*levels[0])
    ref = o.discretization.A
    assert abs(A - ref).max() <= 1e-12 * abs(ref).max()
    for l in range(len(levels) - 1):
        dims, v = levels[l]
        P = _agg(dims[0], dims[1], dims[4], dims[5])
        Ac = _matrix(*levels[l + 1])
        G = P.T @ A @ P
        assert abs(Ac - G).max() <= 1e-12 * abs(G).max()
        A = Ac
    last = levels[-1][0]
    assert last[0] * last[1] <= 64
    np.testing.assert_allclose(pinv, np.linalg.pinv(A.toarray(), rcond=1e-10, hermitian=True),
                               atol=1e-10 * np.abs(pinv).max())
