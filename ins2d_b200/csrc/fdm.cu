// Fast-diagonalization preconditioner of the device PCG.
//
// The pressure matrix is separable, A = M Om^-1 G = -(diag(hy) (x) TX + TY (x)
// diag(hx)) (operator_divergence.m:208 with the 1D factors of setup.cpp), so
// with the generalized eigen-decompositions TX Qx = diag(hx) Qx Lx,
// TY Qy = diag(hy) Qy Ly (Q' diag(h) Q = I, fdm_host.cpp)
//   A^+ r = -Qy . [ (Qy' R Qx) ./ (lx_a + ly_b) ] . Qx'
// where R is r as an Npy x Npx matrix (rows j, x fastest) and the null mode of
// a singular A (closed or periodic domains) is left out.  Applied exactly this
// is the inverse on the range of A, so the PCG -- which keeps cg.F's control
// flow and stopping rule -- converges in one or two iterations.  Four dense
// products per application, run by a tiled FP64 GEMM (CUDA cores).
#include "kernels.cuh"

namespace ins2d {

namespace {

constexpr int kBM = 64, kBN = 64, kBK = 16, kGemmThreads = 256;

// C (M x N, row-major, ldc) = op(A) op(B), op(A) M x K, op(B) K x N.
// TA: A stored K x M (element (m,k) at A[k*lda + m]); else A[m*lda + k].
// TB: B stored N x K (element (k,n) at B[n*ldb + k]); else B[k*ldb + n].
// SCALE: C(b, a) *= -1/(lx[a] + ly[b]), 0 where lx[a] + ly[b] <= thr.
template <bool TA, bool TB, bool SCALE>
__global__ void __launch_bounds__(kGemmThreads) k_gemm(int M, int N, int K, const double *__restrict__ A, int lda,
                                                       const double *__restrict__ B, int ldb, double *__restrict__ C,
                                                       int ldc, const double *__restrict__ lx,
                                                       const double *__restrict__ ly, double thr,
                                                       const int *__restrict__ done) {
  if (done && *(volatile const int *)done) return;
  __shared__ double As[kBK][kBM];
  __shared__ double Bs[kBK][kBN];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  double acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += kBK) {
#pragma unroll
    for (int q = 0; q < (kBM * kBK) / kGemmThreads; ++q) {
      const int e = tid + kGemmThreads * q;
      int m, k;
      if (TA) {
        k = e / kBM;
        m = e - k * kBM;
      } else {
        m = e / kBK;
        k = e - m * kBK;
      }
      const int gm = m0 + m, gk = k0 + k;
      double a = 0.0;
      if (gm < M && gk < K) a = TA ? __ldg(A + (size_t)gk * lda + gm) : __ldg(A + (size_t)gm * lda + gk);
      As[k][m] = a;
    }
#pragma unroll
    for (int q = 0; q < (kBN * kBK) / kGemmThreads; ++q) {
      const int e = tid + kGemmThreads * q;
      int n, k;
      if (TB) {
        n = e / kBK;
        k = e - n * kBK;
      } else {
        k = e / kBN;
        n = e - k * kBN;
      }
      const int gn = n0 + n, gk = k0 + k;
      double b = 0.0;
      if (gn < N && gk < K) b = TB ? __ldg(B + (size_t)gn * ldb + gk) : __ldg(B + (size_t)gk * ldb + gn);
      Bs[k][n] = b;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kBK; ++k) {
      double a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = As[k][ty + 16 * r];
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = Bs[k][tx + 16 * c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int gm = m0 + ty + 16 * r;
    if (gm >= M) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int gn = n0 + tx + 16 * c;
      if (gn >= N) continue;
      double v = acc[r][c];
      if (SCALE) {
        const double lam = __ldg(lx + gn) + __ldg(ly + gm);
        v = lam > thr ? -v / lam : 0.0;
      }
      C[(size_t)gm * ldc + gn] = v;
    }
  }
}

template <bool TA, bool TB, bool SCALE>
void gemm(int M, int N, int K, const double *A, int lda, const double *B, int ldb, double *C, int ldc,
          const FdmD &F, const int *done, cudaStream_t s) {
  const dim3 g((N + kBN - 1) / kBN, (M + kBM - 1) / kBM);
  k_gemm<TA, TB, SCALE><<<g, kGemmThreads, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, F.lx, F.ly, F.thr, done);
}

}  // namespace

void fdm_apply(const FdmD &F, const double *r, double *z, const int *done, cudaStream_t s) {
  const int nx = F.nx, ny = F.ny;
  gemm<false, false, false>(ny, nx, nx, r, nx, F.Qx, nx, F.t1, nx, F, done, s);        // T1 = R Qx
  gemm<true, false, true>(ny, nx, ny, F.Qy, ny, F.t1, nx, F.t2, nx, F, done, s);       // T2 = -(Qy' T1) ./ lam
  gemm<false, false, false>(ny, nx, ny, F.Qy, ny, F.t2, nx, F.t1, nx, F, done, s);     // T1 = Qy T2
  gemm<false, true, false>(ny, nx, nx, F.t1, nx, F.Qx, nx, z, nx, F, done, s);         // Z = T1 Qx'
}

}  // namespace ins2d
