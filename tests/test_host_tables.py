"""The C++ operator derivation (ins2d_b200/csrc/setup.cpp) against the
oracle's assembled operators, on the CPU: every 2D operator and BC vector of
the reference is rebuilt from the 1D row tables the device kernels use and
compared with the oracle's sparse matrices, for every boundary-condition
combination and for uniform and stretched grids."""
import ctypes
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import ins2d_ref as R
from tests.cases_common import BC_COMBOS, grid_stretched, grid_uniform, smooth_bc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BCCODE = {"dir": 0, "pres": 1, "per": 2, "sym": 3}


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    out = tmp_path_factory.mktemp("probe") / "libprobe.so"
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
    lib.probe_table.argtypes = [ctypes.c_void_p, ctypes.c_char_p] + [ctypes.c_void_p] * 6
    lib.probe_sizes.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    return lib


class Tables:
    def __init__(self, lib, x, y, bc, Re):
        self.lib = lib
        codes = np.array([BCCODE[bc[c][s]] for c in ("u", "v") for s in ("left", "right", "low", "up")], np.int32)
        x = np.ascontiguousarray(x, float)
        y = np.ascontiguousarray(y, float)
        self.h = lib.probe_build(len(x) - 1, len(y) - 1, x.ctypes.data, y.ctypes.data, codes.ctypes.data, Re)
        assert self.h, lib.probe_error()

    def __del__(self):
        self.lib.probe_free(self.h)

    def get(self, name):
        nr, nc = ctypes.c_int(), ctypes.c_int()
        col, w, b1, b2 = (ctypes.c_void_p() for _ in range(4))
        assert self.lib.probe_table(self.h, name.encode(), ctypes.byref(nr), ctypes.byref(nc), ctypes.byref(col),
                                    ctypes.byref(w), ctypes.byref(b1), ctypes.byref(b2)) == 0
        n, m = nr.value, nc.value
        C = np.ctypeslib.as_array(ctypes.cast(col, ctypes.POINTER(ctypes.c_int32)), shape=(n * 3,)).copy()
        W = np.ctypeslib.as_array(ctypes.cast(w, ctypes.POINTER(ctypes.c_double)), shape=(n * 3,)).copy()
        B1 = np.ctypeslib.as_array(ctypes.cast(b1, ctypes.POINTER(ctypes.c_double)), shape=(n,)).copy()
        B2 = np.ctypeslib.as_array(ctypes.cast(b2, ctypes.POINTER(ctypes.c_double)), shape=(n,)).copy()
        rows = np.repeat(np.arange(n), 3)
        T = sp.csr_matrix((W, (rows, C)), shape=(n, m))
        return T, B1, B2


def _close(A, B, tol=1e-13):
    A = sp.csr_matrix(A)
    B = sp.csr_matrix(B)
    assert A.shape == B.shape, (A.shape, B.shape)
    d = abs(A - B)
    scale = max(abs(B).max() if B.nnz else 1.0, 1.0)
    assert (d.max() if d.nnz else 0.0) <= tol * scale


def _vclose(a, b, tol=1e-13):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    assert a.shape == b.shape
    scale = max(np.max(np.abs(b)) if b.size else 1.0, 1.0)
    assert np.max(np.abs(a - b)) <= tol * scale if a.size else True


@pytest.mark.parametrize("combo", sorted(BC_COMBOS))
@pytest.mark.parametrize("stretch", [False, True])
def test_tables_match_oracle(probe, combo, stretch):
    x = grid_stretched(10, 0.0, 1.7) if stretch else grid_uniform(10, 0.0, 1.7)
    y = grid_stretched(8, -0.5, 0.5, beta=1.2) if stretch else grid_uniform(8, -0.5, 0.5)
    bc = BC_COMBOS[combo]
    uBC, vBC = smooth_bc(7)
    Re = 37.0
    o = R.make_options(x, y, bc, Re=Re, poisson=4, uBC=uBC, vBC=vBC)
    g, d = o.grid, o.discretization
    s = R.bc_samples(0.0, o)
    T = Tables(probe, x, y, bc, Re)
    I = lambda n: sp.identity(n, format="csr")
    D = lambda v: sp.diags(np.asarray(v, float))
    # u-component
    AUX, a1, a2 = T.get("AUX")
    _close(sp.kron(I(g.Nuy_in), AUX), d.Au_ux)
    _vclose(np.kron(s.uLe_i, a1) + np.kron(s.uRi_i, a2), d.yAu_ux)
    _close(sp.kron(D(g.hy), AUX), d.Iu_ux)
    AUY, a1, a2 = T.get("AUY")
    _close(sp.kron(AUY, I(g.Nux_in)), d.Au_uy)
    _vclose(np.kron(a1, s.uLo_i) + np.kron(a2, s.uUp_i), d.yAu_uy)
    IVX, x1, x2 = T.get("IVX")
    IVY, y1, y2 = T.get("IVY")
    _close(sp.kron(IVY, IVX), d.Iv_uy)
    _vclose(np.kron(s.vLe, x1) + np.kron(s.vRi, x2) + np.kron(y1, IVX @ s.vLo_i) + np.kron(y2, IVX @ s.vUp_i),
            d.yIv_uy)
    SUX, s1, s2 = T.get("SUX")
    SUY, t1, t2 = T.get("SUY")
    _close(sp.kron(I(g.Ny), SUX), d.Su_ux)
    _close(sp.kron(SUY, I(g.Nux_in)), d.Su_uy)
    yDiffu = d.Dux @ ((1 / Re) * (np.kron(s.uLe_i, s1) + np.kron(s.uRi_i, s2))) + \
        d.Duy @ ((1 / Re) * (np.kron(t1, s.uLo_i) + np.kron(t2, s.uUp_i)))
    _vclose(yDiffu, d.yDiffu)
    MX, m1, m2 = T.get("MX")
    _close(sp.kron(D(g.hy), MX), d.Mx)
    MXT, _, _ = T.get("MXT")
    _close(-sp.kron(D(g.hy), MXT), d.Gx)
    # v-component
    AVX, a1, a2 = T.get("AVX")
    _close(sp.kron(I(g.Nvy_in), AVX), d.Av_vx)
    _vclose(np.kron(s.vLe_i, a1) + np.kron(s.vRi_i, a2), d.yAv_vx)
    AVY, a1, a2 = T.get("AVY")
    _close(sp.kron(AVY, I(g.Nvx_in)), d.Av_vy)
    _vclose(np.kron(a1, s.vLo_i) + np.kron(a2, s.vUp_i), d.yAv_vy)
    _close(sp.kron(AVY, D(g.hx)), d.Iv_vy)
    IUX, x1, x2 = T.get("IUX")
    IUY, y1, y2 = T.get("IUY")
    _close(sp.kron(IUY, IUX), d.Iu_vx)
    _vclose(np.kron(y1, s.uLo) + np.kron(y2, s.uUp) + np.kron(IUY @ s.uLe_i, x1) + np.kron(IUY @ s.uRi_i, x2),
            d.yIu_vx)
    SVX, s1, s2 = T.get("SVX")
    SVY, t1, t2 = T.get("SVY")
    _close(sp.kron(I(g.Nvy_in), SVX), d.Sv_vx)
    _close(sp.kron(SVY, I(g.Nx)), d.Sv_vy)
    yDiffv = d.Dvx @ ((1 / Re) * (np.kron(s.vLe_i, s1) + np.kron(s.vRi_i, s2))) + \
        d.Dvy @ ((1 / Re) * (np.kron(t1, s.vLo_i) + np.kron(t2, s.vUp_i)))
    _vclose(yDiffv, d.yDiffv)
    MY, n1, n2 = T.get("MY")
    _close(sp.kron(MY, D(g.hx)), d.My)
    _vclose(np.kron(s.uLe_i * 0 + 1, 0 * m1) + (np.kron(g.hy, np.ones(g.Npx)) * (np.kron(s.uLe_i, m1) + np.kron(s.uRi_i, m2))
            + np.kron(np.ones(g.Npy), g.hx) * (np.kron(n1, s.vLo_i) + np.kron(n2, s.vUp_i))), d.yM)
    MYT, _, _ = T.get("MYT")
    _close(-sp.kron(MYT, D(g.hx)), d.Gy)
    # Laplacian
    TX, _, _ = T.get("TX")
    TY, _, _ = T.get("TY")
    _close(-(sp.kron(D(g.hy), TX) + sp.kron(TY, D(g.hx))), d.A, tol=1e-12)
