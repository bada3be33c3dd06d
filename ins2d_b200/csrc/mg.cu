// Device side of the multigrid preconditioner (see mg.cuh): upload of the
// level hierarchy built by mg_host.cpp, the per-line factors (one thread per
// line), and the multi-block V-cycle launches.
#include <algorithm>
#include <cmath>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "mg.cuh"
#include "mg_host.hpp"

static_assert(ins2d::kMgMaxLevels == ins2d::kMgMaxLevelsHost && ins2d::kMgCoarseMax == ins2d::kMgCoarseMaxHost,
              "host and device multigrid limits");

namespace ins2d {

namespace {

__global__ void k_factor_x(MgLevelD L) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < L.ny) mg_factor_xline(L, j);
}
__global__ void k_factor_y(MgLevelD L) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < L.nx) mg_factor_yline(L, i);
}

constexpr int kLineThreads = 128;
#ifndef INS2D_MG_TAIL_THREADS
#define INS2D_MG_TAIL_THREADS 512
#endif
constexpr int kTailThreads = INS2D_MG_TAIL_THREADS;
// levels with at most this many cells run in the single-block tail
#ifndef INS2D_MG_TAIL_CELLS
#define INS2D_MG_TAIL_CELLS 4096
#endif
constexpr long long kTailMaxCells = INS2D_MG_TAIL_CELLS;

__device__ __forceinline__ bool is_done(const int *done) { return done && *(volatile const int *)done; }

// unrolling of the chunk loops of the multi-block x-line kernel (the
// in-block solvers keep 2)
#ifndef INS2D_MG_XUNROLL
#define INS2D_MG_XUNROLL 2
#endif
constexpr int kXlineUnroll = INS2D_MG_XUNROLL;
// x-lines split over kXlineSplit warps each (1 = a warp per row, the
// original kernel); blocks of one line each
#ifndef INS2D_MG_XSPLIT
#define INS2D_MG_XSPLIT 8
#endif
constexpr int kXlineSplit = INS2D_MG_XSPLIT;
template <int P>
__global__ void __launch_bounds__(32 * P) k_mg_xline_split(const MgLevelD L, const double *__restrict__ b,
                                                           const double *__restrict__ xold,
                                                           double *__restrict__ xnew, double omega, const int *done) {
  __shared__ double sh[4 * P];
  if (is_done(done)) return;
  mg_line_split<P>(mg_make_xline(L, blockIdx.x), b, xold, xnew, omega, threadIdx.x >> 5, sh);
}

__global__ void __launch_bounds__(kLineThreads) k_mg_xline(const MgLevelD L, const double *__restrict__ b,
                                                           const double *__restrict__ xold, double *__restrict__ xnew,
                                                           double omega, const int *done) {
  if (is_done(done)) return;
  mg_xline<kXlineUnroll>(L, b, xold, xnew, omega, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}
__global__ void __launch_bounds__(256) k_mg_restrict(const MgLevelD F, const MgLevelD C, const double *__restrict__ b,
                                                     const double *__restrict__ x, double *__restrict__ bc,
                                                     const int *done) {
  if (is_done(done)) return;
  mg_restrict(F, C, b, x, bc, blockIdx.x * (long long)blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x);
}
__global__ void __launch_bounds__(256) k_mg_prolong(const MgLevelD F, const MgLevelD C, double *__restrict__ x,
                                                    const double *__restrict__ xc, double alpha, const int *done) {
  if (is_done(done)) return;
  mg_prolong(F, C, x, xc, alpha, blockIdx.x * (long long)blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x);
}
__global__ void __launch_bounds__(kTailThreads, 1) k_mg_tail(const __grid_constant__ MgD M, int l0,
                                                            const double *__restrict__ b0, const int *done) {
  __shared__ double ysh[2 * kTailThreads];
  if (is_done(done)) return;
  mg_vcycle_block(M, b0, l0, ysh);
}

// unrolling of the segment walks in the multi-block y-line kernel (the
// in-block solvers keep kMgUnroll)
#ifndef INS2D_MG_YCOLS_UNROLL
#define INS2D_MG_YCOLS_UNROLL 8
#endif
constexpr int kYcolsUnroll = INS2D_MG_YCOLS_UNROLL;
// columns per block of the multi-block y-line kernel (32, or 16: two row
// segments per warp)
#ifndef INS2D_MG_YCW
#define INS2D_MG_YCW 16
#endif
constexpr int kYcolsCols = INS2D_MG_YCW;
// y-lines of 32 columns per block (kColThreads threads: one segment of rows per warp)
constexpr int kColThreads = 1024;
__global__ void __launch_bounds__(kColThreads) k_mg_ycols(const MgLevelD L, const double *__restrict__ b,
                                                          const double *__restrict__ xold, double *__restrict__ xnew,
                                                          double omega, const int *done) {
  __shared__ double ysh[2 * kColThreads];
  if (is_done(done)) return;
  mg_ycols_block<kYcolsUnroll, kYcolsCols>(L, b, xold, xnew, omega, blockIdx.x * kYcolsCols, ysh);
}

// warps per column block: one segment of about INS2D_MG_YSEG rows each, at
// most 32
#ifndef INS2D_MG_YSEG
#define INS2D_MG_YSEG 8
#endif
int col_threads(int ny) {
  int w = ny / (INS2D_MG_YSEG * (32 / kYcolsCols));
  if (w < 1) w = 1;
  if (w > kColThreads / 32) w = kColThreads / 32;
  return 32 * w;
}

unsigned blocks_for(long long n, int t) {
  long long b = (n + t - 1) / t;
  if (b > 148LL * 32) b = 148LL * 32;
  return (unsigned)(b < 1 ? 1 : b);
}

void launch_xline(const MgLevelD &L, const double *b, const double *xold, double *xnew, double omega, const int *done,
                  cudaStream_t s) {
  if (kXlineSplit > 1)
    k_mg_xline_split<kXlineSplit><<<L.ny, 32 * kXlineSplit, 0, s>>>(L, b, xold, xnew, omega, done);
  else
    k_mg_xline<<<blocks_for((long long)L.ny * kMgLineThreads, kLineThreads), kLineThreads, 0, s>>>(L, b, xold, xnew,
                                                                                                  omega, done);
}

}  // namespace

int mg_tail_level(const MgD &M) {
  for (int l = 0; l < M.nlev; ++l)
    if ((long long)M.L[l].nx * M.L[l].ny <= kTailMaxCells) return l;
  return M.nlev - 1;
}

void mg_vcycle_launch(const MgD &M, const double *r0, const int *done, cudaStream_t s) {
  const int lt = mg_tail_level(M);
  for (int l = 0; l < lt; ++l) {
    const MgLevelD &L = M.L[l];
    const double *b = (l == 0) ? r0 : L.b;
    launch_xline(L, b, nullptr, L.x, M.omega, done, s);
    k_mg_ycols<<<(L.nx + kYcolsCols - 1) / kYcolsCols, col_threads(L.ny), 0, s>>>(L, b, L.x, L.t, M.omega, done);
    const MgLevelD &C = M.L[l + 1];
    k_mg_restrict<<<blocks_for((long long)C.nx * C.ny, 256), 256, 0, s>>>(L, C, b, L.t, C.b, done);
  }
  k_mg_tail<<<1, kTailThreads, 0, s>>>(M, lt, lt == 0 ? r0 : M.L[lt].b, done);
  for (int l = lt - 1; l >= 0; --l) {
    const MgLevelD &L = M.L[l];
    const double *b = (l == 0) ? r0 : L.b;
    const MgLevelD &C = M.L[l + 1];
    k_mg_prolong<<<blocks_for((long long)L.nx * L.ny, 256), 256, 0, s>>>(L, C, L.t,
                                                                         (l + 1 == M.nlev - 1) ? C.x : C.t,
                                                                         M.alpha, done);
    k_mg_ycols<<<(L.nx + kYcolsCols - 1) / kYcolsCols, col_threads(L.ny), 0, s>>>(L, b, L.t, L.x, M.omega, done);
    launch_xline(L, b, L.x, L.t, M.omega, done, s);
  }
}

void mg_setup_device(const std::vector<MgHostLevel> &lv, MgD &M, const std::function<double *(size_t)> &alloc,
                     cudaStream_t s) {
  M.nlev = (int)lv.size();
  M.omega = 0.8;
  M.alpha = 2.0;
  auto up = [&](const std::vector<double> &v) {
    double *d = alloc(v.size());
    if (cudaMemcpy(d, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
      throw std::runtime_error("multigrid: upload failed");
    return d;
  };
  for (int l = 0; l < M.nlev; ++l) {
    const MgHostLevel &H = lv[l];
    MgLevelD &D = M.L[l];
    D = MgLevelD{};
    D.nx = H.nx;
    D.ny = H.ny;
    D.perx = H.perx;
    D.pery = H.pery;
    D.cx = H.cx;
    D.cy = H.cy;
    D.xm = up(H.xm);
    D.x0 = up(H.x0);
    D.xp = up(H.xp);
    D.hx = up(H.hx);
    D.ym = up(H.ym);
    D.y0 = up(H.y0);
    D.yp = up(H.yp);
    D.hy = up(H.hy);
    const size_t n = (size_t)H.nx * H.ny;
    D.fxc = alloc(n);
    D.fxi = alloc(n);
    D.fyc = alloc(n);
    D.fyi = alloc(n);
    if (H.perx) {
      D.zx = alloc(n);
      D.gx = alloc(H.ny);
      D.kx = alloc(H.ny);
    }
    if (H.pery) {
      D.zy = alloc(n);
      D.gy = alloc(H.nx);
      D.ky = alloc(H.nx);
    }
    D.b = (l > 0) ? alloc(n) : nullptr;
    D.x = alloc(n);
    D.t = alloc(n);
    k_factor_x<<<(H.ny + 127) / 128, 128, 0, s>>>(D);
    k_factor_y<<<(H.nx + 127) / 128, 128, 0, s>>>(D);
  }
  const MgHostLevel &Cst = lv.back();
  M.ncoarse = Cst.nx * Cst.ny;
  M.cinv = up(mg_pinv(mg_dense(Cst), M.ncoarse));
  if (cudaGetLastError() != cudaSuccess) throw std::runtime_error("multigrid: factor kernels failed");
}

}  // namespace ins2d
