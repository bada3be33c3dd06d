"""The allocation-free FFT pressure solve (ins2d_fft_poisson_noalloc), for
callers that cannot allocate device memory, checked through the C-ABI
against the context path (ins2d_pressure_poisson with poisson = 6) on two
calls in a row.  Its scratch is a static device array shared by every call,
so the second call must not see anything left over from the first.

This file is named to be collected last: a run that stops at the first
failure has run every other test by then.  It passes alone in a fresh
process and after the other tests."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


# sizes at the static scratch's limits: the longest rows and columns (4096)
# at the cell limit 2^20, the largest size of the generic (non-power-of-two)
# transform, and a generic size close to the cell limit
@pytest.mark.parametrize("Nx,Ny,Lx,Ly", [(256, 128, 2 * np.pi, 1.0), (40, 40, 1.0, 1.0), (4096, 256, 4.0, 1.0),
                                         (256, 4096, 1.0, 4.0), (2048, 512, 2.0, 1.0), (1536, 640, 3.0, 1.25)])
def test_noalloc_matches_context_path(Nx, Ny, Lx, Ly):
    import torch
    import ins2d_b200
    from ins2d_b200 import _lib, cases
    lib = _lib.load()
    x = cases.uniform_grid(Nx, 0.0, Lx)
    y = cases.uniform_grid(Ny, 0.0, Ly)
    opts = ins2d_b200.Options(x, y, cases.BC_PERIODIC, Re=1e100, poisson=6)
    rng = np.random.default_rng(Nx + Ny)
    stream = torch.cuda.current_stream()
    for call in range(2):  # two calls in a row on the shared scratch
        f = rng.standard_normal(opts.Np)
        f -= f.mean()
        fd = torch.tensor(f, dtype=torch.float64, device="cuda")
        ref = opts.pressure_poisson(fd).cpu().numpy()
        out = torch.full((opts.Np,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.ins2d_fft_poisson_noalloc(fd.data_ptr(), out.data_ptr(), Nx, Ny, Lx / Nx, Ly / Ny,
                                           ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert _rel(got, ref) < 1e-12, f"call {call}"


def test_noalloc_rejects_oversize():
    import torch
    from ins2d_b200 import _lib
    lib = _lib.load()
    fd = torch.zeros(8, dtype=torch.float64, device="cuda")
    # larger than the static scratch: a clear error, no device work
    assert lib.ins2d_fft_poisson_noalloc(fd.data_ptr(), fd.data_ptr(), 8192, 8192, 1.0, 1.0, None) == _lib.EINVAL
    assert lib.ins2d_fft_poisson_noalloc(fd.data_ptr(), fd.data_ptr(), 1, 8, 1.0, 1.0, None) == _lib.EINVAL
