// Fast-diagonalization preconditioner applied by ONE thread block (the
// single-block PCG of small grids): z = A^+ r = -Qy [(Qy' R Qx) ./ lam] Qx',
// the four products of fdm_apply, each split into 8 x 8 output fragments
// that the block's warps take in turn, every fragment a chain of FP64 MMAs
// (mma.sync m8n8k4 .f64) whose operands are read straight from memory.
// Small grids only (kFdmBlockMaxN cells per direction): the operands
// (Qx, Qy and the nx x ny intermediates) stay in L1/L2.  The intermediates
// are written by the same kernel, so they are read with plain loads; the
// bases are read-only.
#pragma once

#include "kernels.cuh"

namespace ins2d {

constexpr int kFdmBlockMaxN = 128;

__device__ __forceinline__ void fdm_block_mma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// C (M x N) = op(A) op(B) (layouts as fdm.cu's gemm_tile); SCALE: entry
// (b, a) times -1/(lx[a] + ly[b]), 0 where that sum is <= thr.  AC / BC: A / B
// are read-only bases (read through the non-coherent cache).
template <bool TA, bool TB, bool SCALE, bool AC, bool BC>
__device__ __forceinline__ void fdm_block_gemm(int M, int N, int K, const double *A, int lda, const double *B, int ldb,
                                               double *C, int ldc, const double *__restrict__ lx,
                                               const double *__restrict__ ly, double thr) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int fm = (M + 7) / 8, fn = (N + 7) / 8;
  for (int f = warp; f < fm * fn; f += nw) {
    const int bm = (f / fn) * 8, bn = (f - (f / fn) * fn) * 8;
    const int m = bm + g, n = bn + g;
    double d0 = 0.0, d1 = 0.0;
    for (int k = 0; k < K; k += 4) {
      const int kk = k + t;
      double a = 0.0, b = 0.0;
      if (m < M && kk < K) {
        const double *pa = TA ? A + (size_t)kk * lda + m : A + (size_t)m * lda + kk;
        a = AC ? __ldg(pa) : *pa;
      }
      if (n < N && kk < K) {
        const double *pb = TB ? B + (size_t)n * ldb + kk : B + (size_t)kk * ldb + n;
        b = BC ? __ldg(pb) : *pb;
      }
      fdm_block_mma(d0, d1, a, b);
    }
    const int row = bm + g;
    if (row < M) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int col = bn + 2 * t + h;
        if (col >= N) continue;
        double v = h ? d1 : d0;
        if (SCALE) {
          const double lam = __ldg(lx + col) + __ldg(ly + row);
          v = lam > thr ? -v / lam : 0.0;
        }
        C[(size_t)row * ldc + col] = v;
      }
    }
  }
}

// z = A^+ r by the whole block; r must be complete (the caller synchronised
// after writing it); z is complete for every thread on return
__device__ __forceinline__ void fdm_apply_block(const FdmD &F, const double *r, double *z) {
  const int nx = F.nx, ny = F.ny;
  fdm_block_gemm<false, false, false, false, true>(ny, nx, nx, r, nx, F.Qx, nx, F.t1, nx, F.lx, F.ly, F.thr);
  __syncthreads();
  fdm_block_gemm<true, false, true, true, false>(ny, nx, ny, F.Qy, ny, F.t1, nx, F.t2, nx, F.lx, F.ly, F.thr);
  __syncthreads();
  fdm_block_gemm<false, false, false, true, false>(ny, nx, ny, F.Qy, ny, F.t2, nx, F.t1, nx, F.lx, F.ly, F.thr);
  __syncthreads();
  fdm_block_gemm<false, true, false, false, true>(ny, nx, nx, F.t1, nx, F.Qx, nx, z, nx, F.lx, F.ly, F.thr);
  __syncthreads();
}

}  // namespace ins2d
