// FFT pressure solve of a grid split into y-slabs over several GPUs (one
// process per GPU): the three passes of the context's FFT solve
// (pressure_poisson.m:92-104) split at the transposes, so that the caller can
// move the half spectrum between the row layout (each rank its rows) and the
// column layout (each rank a range of wave numbers over all Ny rows) with an
// all-to-all in between.  The arithmetic is the context path's: the same
// kernels, twiddle tables and symbol factors.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "ins2d.h"
#include "kernels.cuh"

namespace ins2d {
bool slab_fft_supported(int Nx, int Ny);
cudaError_t slab_rows_forward(int Nx, const double2 *twx, const double *f, int nrows, double2 *spec, cudaStream_t s);
cudaError_t slab_columns(int Ny, const double2 *twy, const double *ax, const double *ay, double dxdy, double2 *cols,
                         int width, int ncols, int I0, unsigned long long *maxbits, cudaStream_t s);
cudaError_t slab_rows_inverse(int Nx, const double2 *twx, const double2 *spec, int nrows, double *out,
                              const unsigned long long *maxbits, cudaStream_t s);
}  // namespace ins2d

using namespace ins2d;

struct ins2d_slab_fft {
  int device = 0, Nx = 0, Ny = 0;
  double dx = 0.0, dy = 0.0;
  double2 *twx = nullptr, *twy = nullptr;
  double *ax = nullptr, *ay = nullptr;
  unsigned long long *maxbits = nullptr;  // device word: max |fhat| as ordered bits
  unsigned long long *h_bits = nullptr;   // pinned
  std::string err;
  std::vector<void *> allocs;
};

namespace {

int sfail(ins2d_slab_fft *s, int code, const std::string &m) {
  if (s) s->err = m;
  return code;
}

bool sok(ins2d_slab_fft *s, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  if (s) s->err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

}  // namespace

extern "C" {

int ins2d_slab_fft_create(int32_t Nx, int32_t Ny, double dx, double dy, int32_t device, ins2d_slab_fft **out) {
  if (!out) return INS2D_EINVAL;
  *out = nullptr;
  ins2d_slab_fft *s = new (std::nothrow) ins2d_slab_fft();
  if (!s) return INS2D_ENOMEM;
  *out = s;
  if (!slab_fft_supported(Nx, Ny) || !(dx > 0) || !(dy > 0))
    return sfail(s, INS2D_EINVAL, "slab FFT: Nx, Ny must be powers of two from 64 to 8192 and dx, dy positive");
  s->device = device;
  s->Nx = Nx;
  s->Ny = Ny;
  s->dx = dx;
  s->dy = dy;
  DeviceGuard dg(device);
  if (!sok(s, dg.err, "cudaSetDevice")) return INS2D_ECUDA;
  const std::vector<double> tx = fft_twiddle_table(Nx), ty = fft_twiddle_table(Ny);
  // symbol factors (1/dx^2) sin^2(I pi/Nx), (1/dy^2) sin^2(J pi/Ny) of
  // operator_divergence.m:283, as in the context path
  std::vector<double> ax((size_t)Nx), ay((size_t)Ny);
  for (size_t k = 0; k < ax.size(); ++k) {
    const double sn = std::sin((double)k * M_PI / Nx);
    ax[k] = (1.0 / (dx * dx)) * (sn * sn);
  }
  for (size_t k = 0; k < ay.size(); ++k) {
    const double sn = std::sin((double)k * M_PI / Ny);
    ay[k] = (1.0 / (dy * dy)) * (sn * sn);
  }
  auto alloc = [&](void **p, size_t bytes) {
    if (!sok(s, cudaMalloc(p, bytes), "cudaMalloc")) return false;
    s->allocs.push_back(*p);
    return true;
  };
  if (!alloc((void **)&s->twx, tx.size() * sizeof(double)) || !alloc((void **)&s->twy, ty.size() * sizeof(double)) ||
      !alloc((void **)&s->ax, ax.size() * sizeof(double)) || !alloc((void **)&s->ay, ay.size() * sizeof(double)) ||
      !alloc((void **)&s->maxbits, sizeof(unsigned long long)))
    return INS2D_ENOMEM;
  if (!sok(s, cudaMallocHost((void **)&s->h_bits, sizeof(unsigned long long)), "cudaMallocHost")) return INS2D_ENOMEM;
  if (!sok(s, cudaMemcpy(s->twx, tx.data(), tx.size() * sizeof(double), cudaMemcpyHostToDevice), "copy") ||
      !sok(s, cudaMemcpy(s->twy, ty.data(), ty.size() * sizeof(double), cudaMemcpyHostToDevice), "copy") ||
      !sok(s, cudaMemcpy(s->ax, ax.data(), ax.size() * sizeof(double), cudaMemcpyHostToDevice), "copy") ||
      !sok(s, cudaMemcpy(s->ay, ay.data(), ay.size() * sizeof(double), cudaMemcpyHostToDevice), "copy") ||
      !sok(s, fft_prepare(), "fft_prepare"))
    return INS2D_ECUDA;
  return INS2D_OK;
}

int ins2d_slab_fft_destroy(ins2d_slab_fft *s) {
  if (!s) return INS2D_OK;
  DeviceGuard dg(s->device);
  for (void *p : s->allocs) cudaFree(p);
  if (s->h_bits) cudaFreeHost(s->h_bits);
  delete s;
  return INS2D_OK;
}

const char *ins2d_slab_fft_last_error(const ins2d_slab_fft *s) { return s ? s->err.c_str() : "null slab FFT"; }

int ins2d_slab_fft_rows_forward(ins2d_slab_fft *s, const double *f, int32_t nrows, double *spec, void *stream) {
  if (!s || !f || !spec || nrows < 1) return sfail(s, INS2D_EINVAL, "rows_forward: bad argument");
  s->err.clear();
  DeviceGuard dg(s->device);
  if (!sok(s, dg.err, "cudaSetDevice")) return INS2D_ECUDA;
  const cudaStream_t st = (cudaStream_t)stream;
  if (!sok(s, slab_rows_forward(s->Nx, s->twx, f, nrows, (double2 *)spec, st), "rows_forward")) return INS2D_ECUDA;
  if (!sok(s, cudaStreamSynchronize(st), "rows_forward")) return INS2D_ECUDA;
  return INS2D_OK;
}

int ins2d_slab_fft_columns(ins2d_slab_fft *s, double *cols, int32_t width, int32_t I0, double *maxabs,
                           void *stream) {
  if (!s || !cols || width < 1 || I0 < 0) return sfail(s, INS2D_EINVAL, "columns: bad argument");
  s->err.clear();
  DeviceGuard dg(s->device);
  if (!sok(s, dg.err, "cudaSetDevice")) return INS2D_ECUDA;
  const cudaStream_t st = (cudaStream_t)stream;
  const int Hc = s->Nx / 2 + 1;
  const int ncols = std::min(width, Hc - I0);
  if (!sok(s, cudaMemsetAsync(s->maxbits, 0, sizeof(unsigned long long), st), "columns")) return INS2D_ECUDA;
  if (ncols > 0 && !sok(s, slab_columns(s->Ny, s->twy, s->ax, s->ay, s->dx * s->dy, (double2 *)cols, width, ncols,
                                        I0, s->maxbits, st),
                        "columns"))
    return INS2D_ECUDA;
  if (!sok(s, cudaMemcpyAsync(s->h_bits, s->maxbits, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st),
           "columns") ||
      !sok(s, cudaStreamSynchronize(st), "columns"))
    return INS2D_ECUDA;
  if (maxabs) {
    const unsigned long long b = *s->h_bits;
    double m;
    std::memcpy(&m, &b, sizeof m);
    *maxabs = m;
  }
  return INS2D_OK;
}

int ins2d_slab_fft_rows_inverse(ins2d_slab_fft *s, const double *spec, int32_t nrows, double maxabs, double *dp,
                                void *stream) {
  if (!s || !spec || !dp || nrows < 1 || !(maxabs >= 0.0))
    return sfail(s, INS2D_EINVAL, "rows_inverse: bad argument");
  s->err.clear();
  DeviceGuard dg(s->device);
  if (!sok(s, dg.err, "cudaSetDevice")) return INS2D_ECUDA;
  const cudaStream_t st = (cudaStream_t)stream;
  unsigned long long b;
  std::memcpy(&b, &maxabs, sizeof b);  // maxabs >= 0: bit order = value order
  *s->h_bits = b;
  if (!sok(s, cudaMemcpyAsync(s->maxbits, s->h_bits, sizeof b, cudaMemcpyHostToDevice, st), "rows_inverse") ||
      !sok(s, slab_rows_inverse(s->Nx, s->twx, (const double2 *)spec, nrows, dp, s->maxbits, st), "rows_inverse") ||
      !sok(s, cudaStreamSynchronize(st), "rows_inverse"))
    return INS2D_ECUDA;
  return INS2D_OK;
}

}  // extern "C"
