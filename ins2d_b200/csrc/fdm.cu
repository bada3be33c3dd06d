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
// products per application, run by a tiled FP64 GEMM on the FP64 tensor cores
// (mma.sync m8n8k4 .f64; a CUDA-core form of the same tile stays available
// with INS2D_FDM_DMMA=0).
#include "kernels.cuh"

namespace ins2d {

namespace {

#ifndef INS2D_FDM_BM
#define INS2D_FDM_BM 64
#endif
constexpr int kBM = INS2D_FDM_BM, kBN = 64, kBK = 16, kCoreThreads = 256;

// C (M x N, row-major, ldc) = op(A) op(B), op(A) M x K, op(B) K x N.
// TA: A stored K x M (element (m,k) at A[k*lda + m]); else A[m*lda + k].
// TB: B stored N x K (element (k,n) at B[n*ldb + k]); else B[k*ldb + n].
// SCALE: C(b, a) *= -1/(lx[a] + ly[b]), 0 where lx[a] + ly[b] <= thr.
// one kBM x kBN tile (rows m0.., columns n0..) of C by a block of kCoreThreads.
// Thread (ty, tx) of 16 x 16 owns rows {2ty, 2ty+1, 32+2ty, 33+2ty} and the
// same columns with tx, so its operands of one k are two 16-byte shared
// loads each (conflict-free); the next k-slab's global loads are issued into
// registers before the current slab's products (INS2D_FDM_PREFETCH).
#ifndef INS2D_FDM_PREFETCH
#define INS2D_FDM_PREFETCH 1
#endif
template <bool TA, bool TB, bool SCALE>
__device__ __forceinline__ void gemm_tile(int M, int N, int K, const double *__restrict__ A, int lda,
                                          const double *__restrict__ B, int ldb, double *__restrict__ C, int ldc,
                                          const double *__restrict__ lx, const double *__restrict__ ly, double thr,
                                          int m0, int n0) {
  __shared__ __align__(16) double As[kBK][kBM];
  __shared__ __align__(16) double Bs[kBK][kBN];
  constexpr int QA = (kBM * kBK) / kCoreThreads, QB = (kBN * kBK) / kCoreThreads;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  // global -> registers of the k-slab starting at k0
  auto load = [&](int k0, double (&ra)[QA], double (&rb)[QB]) {
#pragma unroll
    for (int q = 0; q < QA; ++q) {
      const int e = tid + kCoreThreads * q;
      const int m = TA ? e % kBM : e / kBK, k = TA ? e / kBM : e % kBK;
      const int gm = m0 + m, gk = k0 + k;
      ra[q] = (gm < M && gk < K) ? (TA ? __ldg(A + (size_t)gk * lda + gm) : __ldg(A + (size_t)gm * lda + gk)) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < QB; ++q) {
      const int e = tid + kCoreThreads * q;
      const int n = TB ? e / kBK : e % kBN, k = TB ? e % kBK : e / kBN;
      const int gn = n0 + n, gk = k0 + k;
      rb[q] = (gn < N && gk < K) ? (TB ? __ldg(B + (size_t)gn * ldb + gk) : __ldg(B + (size_t)gk * ldb + gn)) : 0.0;
    }
  };
  auto store = [&](const double (&ra)[QA], const double (&rb)[QB]) {
#pragma unroll
    for (int q = 0; q < QA; ++q) {
      const int e = tid + kCoreThreads * q;
      As[TA ? e / kBM : e % kBK][TA ? e % kBM : e / kBK] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < QB; ++q) {
      const int e = tid + kCoreThreads * q;
      Bs[TB ? e % kBK : e / kBN][TB ? e / kBK : e % kBN] = rb[q];
    }
  };
  double acc[4][4] = {};
  double ra[QA], rb[QB];
  load(0, ra, rb);
  for (int k0 = 0; k0 < K; k0 += kBK) {
    store(ra, rb);
    __syncthreads();
#if INS2D_FDM_PREFETCH
    if (k0 + kBK < K) load(k0 + kBK, ra, rb);
#endif
#pragma unroll
    for (int k = 0; k < kBK; ++k) {
      const double2 a0 = *reinterpret_cast<const double2 *>(&As[k][2 * ty]);
      const double2 a1 = *reinterpret_cast<const double2 *>(&As[k][32 + 2 * ty]);
      const double2 b0 = *reinterpret_cast<const double2 *>(&Bs[k][2 * tx]);
      const double2 b1 = *reinterpret_cast<const double2 *>(&Bs[k][32 + 2 * tx]);
      const double a[4] = {a0.x, a0.y, a1.x, a1.y}, b[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
    __syncthreads();
#if !INS2D_FDM_PREFETCH
    if (k0 + kBK < K) load(k0 + kBK, ra, rb);
#endif
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int gm = m0 + (r >> 1) * 32 + 2 * ty + (r & 1);
    if (gm >= M) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int gn = n0 + (c >> 1) * 32 + 2 * tx + (c & 1);
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

// The same tile on the FP64 tensor cores (INS2D_FDM_DMMA): mma.sync
// m8n8k4 .f64, each warp a 32 x kTcWarpN block of C (4 x kTcWarpN/8
// fragments of 8 x 8; INS2D_FDM_WARP_N 32: four warps per tile, 16: eight).
// Fragment layout of m8n8k4 .f64 (group g = lane / 4, t = lane % 4): A holds
// (row g, col t), B (row t, col g), C/D (row g, cols 2t, 2t+1).  The operand
// slabs are staged with padded rows (kBM + 4) so a warp's fragment loads hit
// distinct banks.
#ifndef INS2D_FDM_DMMA
#define INS2D_FDM_DMMA 1
#endif
#ifndef INS2D_FDM_WARP_N
#define INS2D_FDM_WARP_N 32
#endif
constexpr int kTcWarpN = INS2D_FDM_WARP_N, kTcThreads = 32 * (kBM / 32) * (kBN / kTcWarpN);
static_assert(INS2D_FDM_DMMA || (kBM == 64 && kBN == 64), "the CUDA-core tile is 64 x 64");
constexpr int kGemmThreads = INS2D_FDM_DMMA ? kTcThreads : kCoreThreads;
__device__ __forceinline__ void dmma_884(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}
template <bool TA, bool TB, bool SCALE>
__device__ __forceinline__ void gemm_tile_tc(int M, int N, int K, const double *__restrict__ A, int lda,
                                             const double *__restrict__ B, int ldb, double *__restrict__ C, int ldc,
                                             const double *__restrict__ lx, const double *__restrict__ ly,
                                             double thr, int m0, int n0) {
  constexpr int PA = kBM + 4, PB = kBN + 4;
  __shared__ __align__(16) double As[kBK][PA];
  __shared__ __align__(16) double Bs[kBK][PB];
  constexpr int QA = (kBM * kBK) / kTcThreads, QB = (kBN * kBK) / kTcThreads;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  constexpr int NJ = kTcWarpN / 8;  // fragments per warp along n
  constexpr int WM = kBM / 32;  // warps along m
  const int wm = (warp % WM) * 32, wn = (warp / WM) * kTcWarpN;
  double ra[QA], rb[QB];
  auto load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < QA; ++q) {
      const int e = tid + kTcThreads * q;
      const int m = TA ? e % kBM : e / kBK, k = TA ? e / kBM : e % kBK;
      const int gm = m0 + m, gk = k0 + k;
      ra[q] = (gm < M && gk < K) ? (TA ? __ldg(A + (size_t)gk * lda + gm) : __ldg(A + (size_t)gm * lda + gk)) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < QB; ++q) {
      const int e = tid + kTcThreads * q;
      const int n = TB ? e / kBK : e % kBN, k = TB ? e % kBK : e / kBN;
      const int gn = n0 + n, gk = k0 + k;
      rb[q] = (gn < N && gk < K) ? (TB ? __ldg(B + (size_t)gn * ldb + gk) : __ldg(B + (size_t)gk * ldb + gn)) : 0.0;
    }
  };
  double acc[4][NJ][2] = {};
  load(0);
  for (int k0 = 0; k0 < K; k0 += kBK) {
#pragma unroll
    for (int q = 0; q < QA; ++q) {
      const int e = tid + kTcThreads * q;
      As[TA ? e / kBM : e % kBK][TA ? e % kBM : e / kBK] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < QB; ++q) {
      const int e = tid + kTcThreads * q;
      Bs[TB ? e % kBK : e / kBN][TB ? e / kBK : e % kBN] = rb[q];
    }
    __syncthreads();
    if (k0 + kBK < K) load(k0 + kBK);
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 4) {
      double a[4], b[NJ];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk + t][wm + 8 * i + g];
#pragma unroll
      for (int j = 0; j < NJ; ++j) b[j] = Bs[kk + t][wn + 8 * j + g];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) dmma_884(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gm = m0 + wm + 8 * i + g;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gn = n0 + wn + 8 * j + 2 * t + h;
        if (gn >= N) continue;
        double v = acc[i][j][h];
        if (SCALE) {
          const double lam = __ldg(lx + gn) + __ldg(ly + gm);
          v = lam > thr ? -v / lam : 0.0;
        }
        C[(size_t)gm * ldc + gn] = v;
      }
  }
}

template <bool TA, bool TB, bool SCALE>
__global__ void __launch_bounds__(kGemmThreads) k_gemm(int M, int N, int K, const double *__restrict__ A, int lda,
                                                       const double *__restrict__ B, int ldb, double *__restrict__ C,
                                                       int ldc, const double *__restrict__ lx,
                                                       const double *__restrict__ ly, double thr,
                                                       const int *__restrict__ done) {
  if (done && *(volatile const int *)done) return;
#if INS2D_FDM_DMMA
  gemm_tile_tc<TA, TB, SCALE>(M, N, K, A, lda, B, ldb, C, ldc, lx, ly, thr, blockIdx.y * kBM, blockIdx.x * kBN);
#else
  gemm_tile<TA, TB, SCALE>(M, N, K, A, lda, B, ldb, C, ldc, lx, ly, thr, blockIdx.y * kBM, blockIdx.x * kBN);
#endif
}

// The four products of fdm_apply for many members in one launch per product:
// work items {member, tile row, tile column}; members whose CG has converged
// (cg[m].done) skip their tiles.  OP 0: T1 = R Qx; 1: T2 = -(Qy' T1) ./ lam;
// 2: T1 = Qy T2; 3: Z = T1 Qx'.
#if INS2D_FDM_DMMA
#define GEMM_TILE gemm_tile_tc
#else
#define GEMM_TILE gemm_tile
#endif
template <int OP>
__global__ void __launch_bounds__(kGemmThreads) k_gemm_ens(const EnsFdmD *__restrict__ F,
                                                           const int4 *__restrict__ tiles,
                                                           const EnsCg *__restrict__ cg) {
  const int4 t = tiles[blockIdx.x];
  const int m = t.x;
  if (*(volatile const int *)&cg[m].done) return;
  const EnsFdmD &D = F[m];
  const int nx = D.nx, ny = D.ny, m0 = t.y * kBM, n0 = t.z * kBN;
  if (OP == 0)
    GEMM_TILE<false, false, false>(ny, nx, nx, D.r, nx, D.Qx, nx, D.t1, nx, D.lx, D.ly, D.thr, m0, n0);
  else if (OP == 1)
    GEMM_TILE<true, false, true>(ny, nx, ny, D.Qy, ny, D.t1, nx, D.t2, nx, D.lx, D.ly, D.thr, m0, n0);
  else if (OP == 2)
    GEMM_TILE<false, false, false>(ny, nx, ny, D.Qy, ny, D.t2, nx, D.t1, nx, D.lx, D.ly, D.thr, m0, n0);
  else
    GEMM_TILE<false, true, false>(ny, nx, nx, D.t1, nx, D.Qx, nx, D.z, nx, D.lx, D.ly, D.thr, m0, n0);
}

template <bool TA, bool TB, bool SCALE>
void gemm(int M, int N, int K, const double *A, int lda, const double *B, int ldb, double *C, int ldc,
          const FdmD &F, const int *done, cudaStream_t s) {
  const dim3 g((N + kBN - 1) / kBN, (M + kBM - 1) / kBM);
  k_gemm<TA, TB, SCALE><<<g, kGemmThreads, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, F.lx, F.ly, F.thr, done);
}

}  // namespace

void fdm_tiles(int member, int nx, int ny, std::vector<int4> &out) {
  for (int bm = 0; bm < (ny + kBM - 1) / kBM; ++bm)
    for (int bn = 0; bn < (nx + kBN - 1) / kBN; ++bn) out.push_back(make_int4(member, bm, bn, 0));
}

void fdm_apply_ens(const EnsFdmD *F, const int4 *tiles, int ntiles, const EnsCg *cg, cudaStream_t s) {
  if (ntiles <= 0) return;
  k_gemm_ens<0><<<ntiles, kGemmThreads, 0, s>>>(F, tiles, cg);
  k_gemm_ens<1><<<ntiles, kGemmThreads, 0, s>>>(F, tiles, cg);
  k_gemm_ens<2><<<ntiles, kGemmThreads, 0, s>>>(F, tiles, cg);
  k_gemm_ens<3><<<ntiles, kGemmThreads, 0, s>>>(F, tiles, cg);
}

void fdm_apply(const FdmD &F, const double *r, double *z, const int *done, cudaStream_t s) {
  const int nx = F.nx, ny = F.ny;
  gemm<false, false, false>(ny, nx, nx, r, nx, F.Qx, nx, F.t1, nx, F, done, s);        // T1 = R Qx
  gemm<true, false, true>(ny, nx, ny, F.Qy, ny, F.t1, nx, F.t2, nx, F, done, s);       // T2 = -(Qy' T1) ./ lam
  gemm<false, false, false>(ny, nx, ny, F.Qy, ny, F.t2, nx, F.t1, nx, F, done, s);     // T1 = Qy T2
  gemm<false, true, false>(ny, nx, nx, F.t1, nx, F.Qx, nx, z, nx, F, done, s);         // Z = T1 Qx'
}

}  // namespace ins2d
