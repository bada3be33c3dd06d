// Preconditioned conjugate gradients for A dp = f, A = M Om^-1 G, with the
// control flow and stopping rule of the reference's cg.F:158-280:
//   x0 = 0, r0 = f, z = M^-1 r, p = z, rr0 = f'f; stop at once if rr0 <= tol^2;
//   per iteration: q = A p; alpha = r'z / p'q; x += alpha p; r -= alpha q;
//   converged when r'r / rr0 <= tol^2 (iter = that iteration);
//   else z = M^-1 r; beta = r'z_new / r'z_old; p = z + beta p;
//   error after maxit iterations;  norm1 = sqrt(r'r/rr0),
//   norm2 = max|r| / (max x - min x) of the last iteration.
// pressure_poisson.m:33-38's early return (max|A*0 - f| < 1e-14 -> dp = 0)
// is folded into the first kernel.
//
// The reference preconditions with a diagonal incomplete Cholesky factor
// whose forward/backward sweeps are sequential (cg.F:317-390).  Here the
// preconditioner is a multigrid V-cycle (mg.cuh, the default) or the
// diagonal of A (Jacobi), both parallel; iteration counts therefore differ
// from the reference, the converged solution agrees to the stated tolerance.
//
// Three kernels per iteration (SpMV + p'q; x/r update + r'r, r'z and the
// norm2 extrema; p update); scalars live on the device and each kernel's last
// block advances them, so the host only polls the convergence flag every few
// iterations.
#include "ins2d.h"
#include "kernels.cuh"
#include "mg.cuh"
#include "fdm_block.cuh"
#include "reduce.cuh"

namespace ins2d {

namespace {

constexpr int BX = 32, BY = 8;

inline dim3 pgrid(const DevOps &P) { return dim3((P.Npx + BX - 1) / BX, (P.Npy + BY - 1) / BY); }

__device__ __forceinline__ RedScratch red_of(const PcgWork &W) {
  RedScratch r;
  r.partials = W.partials;
  r.counter = &W.sc->counter;
  r.result = W.partials + (size_t)W.blocks * 8;  // 8 slots after the partials
  r.max_blocks = W.blocks;
  return r;
}

// q = A p and p'q (alpha), walking columns: a thread takes one column i and
// kSpmvRows rows, so the x-row of TX at i (columns and weights) is read once,
// the TY row of each j is a warp-uniform read, and the p values of a column
// reach the thread through L1.  Same arithmetic per cell as lap().
constexpr int kSpmvRows = 16;
__global__ void __launch_bounds__(256) k_spmv_cols(const __grid_constant__ DevOps P, const PcgWork W) {
  if (*(volatile int *)&W.sc->done) return;
  const int i = blockIdx.x * BX + threadIdx.x;
  const int j0 = (blockIdx.y * BY + threadIdx.y) * kSpmvRows;
  double q1[1] = {0.0};
  const int ops[1] = {R_SUM};
  if (i < P.Npx && j0 < P.Npy) {
    const int32_t *cx = P.TX.c + kT * i;
    const double *wx = P.TX.w + kT * i;
    const int cx0 = __ldg(cx), cx1 = __ldg(cx + 1), cx2 = __ldg(cx + 2);
    const double wx0 = __ldg(wx), wx1 = __ldg(wx + 1), wx2 = __ldg(wx + 2);
    const double hxi = __ldg(P.hx + i);
    const int j1 = min(j0 + kSpmvRows, P.Npy);
    const double *__restrict__ p = W.p;
#pragma unroll 4
    for (int j = j0; j < j1; ++j) {
      const long long base = (long long)j * P.Npx;
      const double tx = wx0 * __ldg(p + base + cx0) + wx1 * __ldg(p + base + cx1) + wx2 * __ldg(p + base + cx2);
      const int32_t *cy = P.TY.c + kT * j;
      const double *wy = P.TY.w + kT * j;
      const double ty = __ldg(wy) * __ldg(p + (long long)__ldg(cy) * P.Npx + i) +
                        __ldg(wy + 1) * __ldg(p + (long long)__ldg(cy + 1) * P.Npx + i) +
                        __ldg(wy + 2) * __ldg(p + (long long)__ldg(cy + 2) * P.Npx + i);
      const double aq = -(__ldg(P.hy + j) * tx + hxi * ty);
      W.q[base + i] = aq;
      q1[0] += __ldg(p + base + i) * aq;
    }
  }
  double out[1];
  if (grid_reduce<1>(q1, ops, red_of(W), out)) {
    PcgScalars *s = W.sc;
    s->pq = out[0];
    if (!isfinite(out[0])) {
      s->status = INS2D_ENONFINITE;
      s->done = 1;
    } else if (out[0] == 0.0) {
      s->status = INS2D_EBREAKDOWN;
      s->done = 1;
    } else {
      s->alpha = s->rz / out[0];
    }
  }
}
inline dim3 spmv_grid(const DevOps &P) {
  return dim3((P.Npx + BX - 1) / BX, (P.Npy + BY * kSpmvRows - 1) / (BY * kSpmvRows));
}

__global__ void __launch_bounds__(256) k_update(const __grid_constant__ DevOps P, const PcgWork W) {
  if (*(volatile int *)&W.sc->done) return;
  const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
  const double alpha = W.sc->alpha;
  double q[5] = {0.0, 0.0, -DBL_MAX, DBL_MAX, 0.0};
  const int ops[5] = {R_SUM, R_SUM, R_MAX, R_MIN, R_MAX};
  if (i < P.Npx && j < P.Npy) {
    const long long k = (long long)j * P.Npx + i;
    const double x = W.x[k] + alpha * W.p[k];
    const double r = W.r[k] - alpha * W.q[k];
    W.x[k] = x;
    W.r[k] = r;
    q[0] = r * r;
    q[1] = r * (r / lap_diag(P, i, j));
    q[2] = x;
    q[3] = x;
    q[4] = fabs(r);
  }
  double out[5];
  if (grid_reduce<5>(q, ops, red_of(W), out)) {
    PcgScalars *s = W.sc;
    s->it += 1;
    s->rr = out[0] / s->rr0;
    s->maxx = out[2];
    s->minx = out[3];
    s->maxres = out[4];
    if (!isfinite(s->rr) || !isfinite(out[1])) {
      s->status = INS2D_ENONFINITE;
      s->done = 1;
    } else if (s->rr <= s->tol2) {
      s->done = 1;
    } else if (s->it >= s->maxit) {
      s->status = INS2D_ENOTCONV;
      s->done = 1;
    } else {
      s->beta = out[1] / s->rz;
      s->rz = out[1];
    }
  }
}

__global__ void __launch_bounds__(256) k_pupdate(const __grid_constant__ DevOps P, const PcgWork W) {
  if (*(volatile int *)&W.sc->done) return;
  const int i = blockIdx.x * BX + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
  if (i < P.Npx && j < P.Npy) {
    const long long k = (long long)j * P.Npx + i;
    W.p[k] = W.r[k] / lap_diag(P, i, j) + W.sc->beta * W.p[k];
  }
}

__global__ void k_copy_out(const double *__restrict__ x, double *__restrict__ dp, long long n, int accumulate) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    dp[k] = accumulate ? dp[k] + x[k] : x[k];
}


// ---------------------------------------------------------------------------
// Whole solve in one thread block (small grids): same algorithm and stopping
// rule, block-level reductions in a fixed order, no host round trips.
constexpr int kBlockThreads = 1024;

template <int NQ>
__device__ void block_reduce(double (&v)[NQ], const int (&ops)[NQ], double (*sh)[NQ]) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q)
    for (int off = 16; off > 0; off >>= 1) v[q] = red_combine(v[q], __shfl_down_sync(0xffffffffu, v[q], off), ops[q]);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NQ; ++q) sh[warp][q] = v[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double a = sh[0][q];
    for (int w = 1; w < nw; ++w) a = red_combine(a, sh[w][q], ops[q]);
    v[q] = a;  // every thread gets the block result
  }
  __syncthreads();
}

// The whole solve by one thread block.  PK 0: Jacobi preconditioner
// (z = r / diag A); 1: one multigrid V-cycle per application (mg.cuh);
// 2: fast diagonalization (fdm_block.cuh).  Results go to out (the
// PcgScalars of this solve).
template <int PK>
__device__ void pcg_block_body(const DevOps &P, const MgD *M, const FdmD *F, const PcgWork &W,
                               const double *__restrict__ f, double *__restrict__ dp, double tol2, long long maxit,
                               int accumulate, PcgScalars *out, double (*sh)[5], double *ysh) {
  constexpr bool MG = PK != 0;  // a preconditioner with its own z buffer
  const int Npx = P.Npx;
  const long long Np = P.Np;
  const int tid = threadIdx.x, nt = blockDim.x;
  double *__restrict__ x = W.x, *__restrict__ r = W.r, *__restrict__ p = W.p, *__restrict__ q = W.q;
  double *zw = PK == 1 ? mg_result(*M, 0) : (PK == 2 ? F->z : nullptr);
  const double *z = zw;
  auto precond = [&]() {
    if constexpr (PK == 1)
      mg_vcycle_block(*M, r, 0, ysh);
    else if constexpr (PK == 2)
      fdm_apply_block(*F, r, zw);
  };
  // init (cg.F:207-229 with x_in = 0)
  double a3[3] = {0.0, 0.0, 0.0};
  const int op3[3] = {R_SUM, R_SUM, R_MAX};
  for (long long k = tid; k < Np; k += nt) {
    const int i = (int)(k % Npx), j = (int)(k / Npx);
    const double fv = f[k];
    x[k] = 0.0;
    r[k] = fv;
    if (!MG) {
      const double zv = fv / lap_diag(P, i, j);
      p[k] = zv;
      a3[1] += fv * zv;
    }
    a3[0] += fv * fv;
    a3[2] = fmax(a3[2], fabs(fv));
  }
  block_reduce<3>(a3, op3, (double(*)[3])sh);
  const double rr0 = a3[0];
  double rz = a3[1];
  double rr = 0.0, maxx = 0.0, minx = 0.0, maxres = 0.0;
  long long it = 0;
  int status = 0;
  bool done = (a3[2] < 1e-14 || rr0 <= tol2);  // pressure_poisson.m:33-38, cg.F:222-227
  if (!isfinite(rr0)) {
    status = INS2D_ENONFINITE;
    done = true;
  }
  const int op1[1] = {R_SUM};
  if (MG && !done) {
    __syncthreads();
    precond();
    double a1[1] = {0.0};
    for (long long k = tid; k < Np; k += nt) {
      p[k] = z[k];
      a1[0] += r[k] * z[k];
    }
    block_reduce<1>(a1, op1, (double(*)[1])sh);
    rz = a1[0];
  }
  if (!isfinite(rz)) {
    status = INS2D_ENONFINITE;
    done = true;
  }
  const int op5[5] = {R_SUM, R_SUM, R_MAX, R_MIN, R_MAX};
  MG_T0();
  while (!done) {
    double a1[1] = {0.0};
    for (long long k = tid; k < Np; k += nt) {
      const int i = (int)(k % Npx), j = (int)(k / Npx);
      const double aq = lap(P, p, i, j);
      q[k] = aq;
      a1[0] += p[k] * aq;
    }
    block_reduce<1>(a1, op1, (double(*)[1])sh);
    MG_TICK(120);
    const double pq = a1[0];
    if (!isfinite(pq)) {
      status = INS2D_ENONFINITE;
      break;
    }
    if (pq == 0.0) {
      status = INS2D_EBREAKDOWN;
      break;
    }
    const double alpha = rz / pq;
    double a5[5] = {0.0, 0.0, -DBL_MAX, DBL_MAX, 0.0};
    for (long long k = tid; k < Np; k += nt) {
      const int i = (int)(k % Npx), j = (int)(k / Npx);
      const double xv = x[k] + alpha * p[k];
      const double rv = r[k] - alpha * q[k];
      x[k] = xv;
      r[k] = rv;
      a5[0] += rv * rv;
      if (!MG) a5[1] += rv * (rv / lap_diag(P, i, j));
      a5[2] = fmax(a5[2], xv);
      a5[3] = fmin(a5[3], xv);
      a5[4] = fmax(a5[4], fabs(rv));
    }
    block_reduce<5>(a5, op5, (double(*)[5])sh);
    MG_TICK(121);
    ++it;
    rr = a5[0] / rr0;
    maxx = a5[2];
    minx = a5[3];
    maxres = a5[4];
    if (!isfinite(rr)) {
      status = INS2D_ENONFINITE;
      break;
    }
    if (rr <= tol2) break;
    if (it >= maxit) {
      status = INS2D_ENOTCONV;
      break;
    }
    double rz_new = a5[1];
    if (MG) {
      MG_TICK(124);
      precond();
      MG_TICK(125);
      double b1[1] = {0.0};
      for (long long k = tid; k < Np; k += nt) b1[0] += r[k] * z[k];
      block_reduce<1>(b1, op1, (double(*)[1])sh);
      rz_new = b1[0];
      MG_TICK(122);
    }
    if (!isfinite(rz_new)) {
      status = INS2D_ENONFINITE;
      break;
    }
    const double beta = rz_new / rz;
    rz = rz_new;
    for (long long k = tid; k < Np; k += nt) {
      const int i = (int)(k % Npx), j = (int)(k / Npx);
      const double zv = MG ? z[k] : r[k] / lap_diag(P, i, j);
      p[k] = zv + beta * p[k];
    }
    __syncthreads();
    MG_TICK(123);
  }
  if (status == 0)
    for (long long k = tid; k < Np; k += nt) dp[k] = accumulate ? dp[k] + x[k] : x[k];
  if (tid == 0) {
    out->rr0 = rr0;
    out->rr = rr;
    out->it = it;
    out->maxx = maxx;
    out->minx = minx;
    out->maxres = maxres;
    out->status = status;
    out->done = 1;
    out->tol2 = tol2;
    out->maxit = maxit;
  }
}

__global__ void __launch_bounds__(kBlockThreads, 1) k_pcg_block(const __grid_constant__ DevOps P, const PcgWork W,
                                                               const double *__restrict__ f, double *__restrict__ dp,
                                                               double tol2, long long maxit, int accumulate) {
  __shared__ double sh[kBlockThreads / 32][5];
  pcg_block_body<0>(P, nullptr, nullptr, W, f, dp, tol2, maxit, accumulate, W.sc, sh, nullptr);
}

// multigrid variant: 512 threads (the chunked line solves need ~128 registers)
#ifndef INS2D_MG_THREADS
#define INS2D_MG_THREADS 512
#endif
constexpr int kBlockThreadsMg = INS2D_MG_THREADS;
__global__ void __launch_bounds__(kBlockThreadsMg, 1) k_pcg_block_mg(const __grid_constant__ DevOps P,
                                                                  const __grid_constant__ MgD M, const PcgWork W,
                                                                  const double *__restrict__ f,
                                                                  double *__restrict__ dp, double tol2,
                                                                  long long maxit, int accumulate) {
  __shared__ double sh[kBlockThreads / 32][5];
  __shared__ double ysh[2 * kBlockThreadsMg];
  pcg_block_body<1>(P, &M, nullptr, W, f, dp, tol2, maxit, accumulate, W.sc, sh, ysh);
}

// fast-diagonalization variant for grids up to kFdmBlockMaxN cells per direction
constexpr int kBlockThreadsFdm = 512;
__global__ void __launch_bounds__(kBlockThreadsFdm, 1) k_pcg_block_fdm(const __grid_constant__ DevOps P,
                                                                    const __grid_constant__ FdmD F, const PcgWork W,
                                                                    const double *__restrict__ f,
                                                                    double *__restrict__ dp, double tol2,
                                                                    long long maxit, int accumulate) {
  __shared__ double sh[kBlockThreads / 32][5];
  pcg_block_body<2>(P, nullptr, &F, W, f, dp, tol2, maxit, accumulate, W.sc, sh, nullptr);
}

// Grid-stride CG kernels of the multigrid path for large grids: the SpMV uses
// the 3-point 1D rows of the hierarchy's level 0 (the same operator as A,
// without table indirection), and each thread handles many cells, so the
// block partials of the reductions stay few.
constexpr int kVecThreads = 256;
__global__ void __launch_bounds__(kVecThreads) k_spmv_g(const MgLevelD L0, const PcgWork W, long long n) {
  if (*(volatile int *)&W.sc->done) return;
  double q[1] = {0.0};
  const int ops[1] = {R_SUM};
  const int nx = L0.nx;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % nx), j = (int)(k / nx);
    const double aq = mg_apply(L0, W.p, i, j);
    W.q[k] = aq;
    q[0] += W.p[k] * aq;
  }
  double out[1];
  if (grid_reduce<1>(q, ops, red_of(W), out)) {
    PcgScalars *s = W.sc;
    s->pq = out[0];
    if (!isfinite(out[0])) {
      s->status = INS2D_ENONFINITE;
      s->done = 1;
    } else if (out[0] == 0.0) {
      s->status = INS2D_EBREAKDOWN;
      s->done = 1;
    } else {
      s->alpha = s->rz / out[0];
    }
  }
}

// PCG initialisation over a grid-stride loop (a few blocks per SM, so the final
// reduction combines few partials): x = 0, r = f, p = f / diag A; f'f,
// f'(f / diag A), max|f|
__global__ void __launch_bounds__(kVecThreads) k_init_g(const __grid_constant__ DevOps P, const PcgWork W,
                                                      const double *__restrict__ f, double tol2, long long maxit) {
  double q[3] = {0.0, 0.0, 0.0};
  const int ops[3] = {R_SUM, R_SUM, R_MAX};
  const int Npx = P.Npx;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < P.Np;
       k += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(k / Npx), i = (int)(k - (long long)j * Npx);
    const double fv = f[k];
    const double z = fv / lap_diag(P, i, j);
    W.x[k] = 0.0;
    W.r[k] = fv;
    W.p[k] = z;
    q[0] += fv * fv;
    q[1] += fv * z;
    q[2] = fmax(q[2], fabs(fv));
  }
  double out[3];
  if (grid_reduce<3>(q, ops, red_of(W), out)) {
    PcgScalars *s = W.sc;
    s->tol2 = tol2;
    s->maxit = maxit;
    s->rr0 = out[0];
    s->rz = out[1];
    s->rr = 0.0;
    s->it = 0;
    s->status = 0;
    s->maxx = s->minx = s->maxres = 0.0;
    s->loops = 0;
    // pressure_poisson.m:33-38 and cg.F:222-227
    s->done = (out[2] < 1e-14 || out[0] <= tol2) ? 1 : 0;
    if (!isfinite(out[0]) || !isfinite(out[1])) {
      s->status = INS2D_ENONFINITE;
      s->done = 1;
    }
  }
}

__global__ void __launch_bounds__(kVecThreads) k_update_g(const PcgWork W, long long n) {
  if (*(volatile int *)&W.sc->done) return;
  const double alpha = W.sc->alpha;
  double q[4] = {0.0, -DBL_MAX, DBL_MAX, 0.0};
  const int ops[4] = {R_SUM, R_MAX, R_MIN, R_MAX};
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double x = W.x[k] + alpha * W.p[k];
    const double r = W.r[k] - alpha * W.q[k];
    W.x[k] = x;
    W.r[k] = r;
    q[0] += r * r;
    q[1] = fmax(q[1], x);
    q[2] = fmin(q[2], x);
    q[3] = fmax(q[3], fabs(r));
  }
  double out[4];
  if (grid_reduce<4>(q, ops, red_of(W), out)) {
    PcgScalars *s = W.sc;
    s->it += 1;
    s->rr = out[0] / s->rr0;
    s->maxx = out[1];
    s->minx = out[2];
    s->maxres = out[3];
    if (!isfinite(s->rr)) {
      s->status = INS2D_ENONFINITE;
      s->done = 1;
    } else if (s->rr <= s->tol2) {
      s->done = 1;
    } else if (s->it >= s->maxit) {
      s->status = INS2D_ENOTCONV;
      s->done = 1;
    }
  }
}

__global__ void __launch_bounds__(kVecThreads) k_rz_g(const PcgWork W, const double *__restrict__ z, long long n,
                                                      int init) {
  if (*(volatile int *)&W.sc->done) return;
  double q[1] = {0.0};
  const int ops[1] = {R_SUM};
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    q[0] += W.r[k] * z[k];
    if (init) W.p[k] = z[k];
  }
  double out[1];
  if (grid_reduce<1>(q, ops, red_of(W), out)) {
    PcgScalars *s = W.sc;
    if (!isfinite(out[0])) {
      s->status = INS2D_ENONFINITE;
      s->done = 1;
    } else if (init) {
      s->rz = out[0];
    } else {
      s->beta = out[0] / s->rz;
      s->rz = out[0];
    }
  }
}

__global__ void __launch_bounds__(kVecThreads) k_pupdate_g(const PcgWork W, const double *__restrict__ z, long long n) {
  if (*(volatile int *)&W.sc->done) return;
  const double beta = W.sc->beta;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    W.p[k] = z[k] + beta * W.p[k];
}

// Ensemble solves: a persistent launch whose blocks take members from a
// queue (largest first) and run the whole PCG of each.
__global__ void __launch_bounds__(kBlockThreadsMg, 1) k_pcg_members(const EnsMemberD *__restrict__ mem,
                                                                  const int *__restrict__ order, int n, int which,
                                                                  double tol2, long long maxit,
                                                                  unsigned *queue, EnsStats *stats) {
  __shared__ __align__(16) DevOps sP;
  __shared__ __align__(16) MgD sM;
  __shared__ double sh[kBlockThreads / 32][5];
  __shared__ double ysh[2 * kBlockThreadsMg];
  __shared__ int s_k;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (;;) {
    if (tid == 0) s_k = (int)atomicAdd(&queue[0], 1u);
    __syncthreads();
    const int k = s_k;
    if (k >= n) break;
    const int m = order[k];
    const EnsMemberD &E = mem[m];
    for (int w = tid; w < (int)(sizeof(DevOps) / 8); w += nt) ((long long *)&sP)[w] = ((const long long *)&E.P)[w];
    const bool mg = E.mg != nullptr;
    if (mg)
      for (int w = tid; w < (int)(sizeof(MgD) / 8); w += nt) ((long long *)&sM)[w] = ((const long long *)E.mg)[w];
    __syncthreads();
    double *dst = which ? E.p : E.dp;
    if (mg)
      pcg_block_body<1>(sP, &sM, nullptr, E.W, E.f, dst, tol2, maxit, which, E.W.sc, sh, ysh);
    else
      pcg_block_body<0>(sP, nullptr, nullptr, E.W, E.f, dst, tol2, maxit, which, E.W.sc, sh, ysh);
    __syncthreads();
    if (tid == 0) {
      const PcgScalars &o = *E.W.sc;
      EnsStats &st = stats[m];
      st.n_solves += 1;
      st.iters_total += o.it;
      st.iters_max = o.it > st.iters_max ? o.it : st.iters_max;
      const double n1 = sqrt(o.rr);
      st.norm1_max = n1 > st.norm1_max ? n1 : st.norm1_max;
      if (o.status != 0 && st.status == 0) st.status = o.status;
    }
    __syncthreads();  // s_k and the shared descriptors are reused
  }
  if (tid == 0) {
    __threadfence();
    const unsigned d = atomicAdd(&queue[1], 1u);
    if (d == gridDim.x - 1) {  // last block out: reset the queue for the next launch
      queue[0] = 0;
      queue[1] = 0;
      __threadfence();
    }
  }
}

}  // namespace

bool pcg_use_block(const DevOps &P) { return P.Np <= kPcgBlockMaxCells; }

void pcg_solve_block(const DevOps &P, const PcgWork &W, const double *f, double *dp, double tol, long long maxit,
                     bool accumulate, cudaStream_t s) {
  k_pcg_block<<<1, kBlockThreads, 0, s>>>(P, W, f, dp, tol * tol, maxit, accumulate ? 1 : 0);
}

#ifdef INS2D_MG_TIMING
extern "C" int ins2d_debug_mg_clocks(unsigned long long out[128], int reset) {
  if (cudaMemcpyFromSymbol(out, g_mg_clk, sizeof(unsigned long long) * 128) != cudaSuccess) return 1;
  if (reset) {
    static const unsigned long long z[128] = {};
    cudaMemcpyToSymbol(g_mg_clk, z, sizeof z);
  }
  return 0;
}
#endif

void pcg_solve_block_mg(const DevOps &P, const MgD &M, const PcgWork &W, const double *f, double *dp, double tol,
                        long long maxit, bool accumulate, cudaStream_t s) {
  k_pcg_block_mg<<<1, kBlockThreadsMg, 0, s>>>(P, M, W, f, dp, tol * tol, maxit, accumulate ? 1 : 0);
}

bool pcg_use_block_fdm(const FdmD &F) { return !F.spectral && F.nx <= kFdmBlockMaxN && F.ny <= kFdmBlockMaxN; }

void pcg_solve_block_fdm(const DevOps &P, const FdmD &F, const PcgWork &W, const double *f, double *dp, double tol,
                         long long maxit, bool accumulate, cudaStream_t s) {
  k_pcg_block_fdm<<<1, kBlockThreadsFdm, 0, s>>>(P, F, W, f, dp, tol * tol, maxit, accumulate ? 1 : 0);
}

int pcg_blocks(const DevOps &P) {
  dim3 g = pgrid(P);
  return (int)(g.x * g.y);
}

namespace {
// blocks of the grid-stride kernels: at most 8 per SM and at most the
// reduction scratch's capacity
unsigned vec_blocks(const DevOps &P, const PcgWork &W) {
  long long b = (P.Np + kVecThreads - 1) / kVecThreads;
  if (b > 148LL * 8) b = 148LL * 8;
  if (b > W.blocks) b = W.blocks;
  return (unsigned)(b < 1 ? 1 : b);
}
}  // namespace

void pcg_init(const DevOps &P, const PcgWork &W, const double *f, double tol, long long maxit, cudaStream_t s) {
  k_init_g<<<vec_blocks(P, W), kVecThreads, 0, s>>>(P, W, f, tol * tol, maxit);
}

void pcg_iterations(const DevOps &P, const PcgWork &W, int n, cudaStream_t s) {
  const dim3 g = pgrid(P), b(BX, BY);
  for (int it = 0; it < n; ++it) {
    k_spmv_cols<<<spmv_grid(P), b, 0, s>>>(P, W);
    k_update<<<g, b, 0, s>>>(P, W);
    k_pupdate<<<g, b, 0, s>>>(P, W);
  }
}


void pcg_init_mg(const DevOps &P, const MgD &M, const PcgWork &W, const double *f, double tol, long long maxit,
                 cudaStream_t s) {
  k_init_g<<<vec_blocks(P, W), kVecThreads, 0, s>>>(P, W, f, tol * tol, maxit);
  mg_vcycle_launch(M, W.r, &W.sc->done, s);
  k_rz_g<<<vec_blocks(P, W), kVecThreads, 0, s>>>(W, mg_result_host(M, 0), P.Np, 1);
}

void pcg_iterations_mg(const DevOps &P, const MgD &M, const PcgWork &W, int n, cudaStream_t s) {
  const unsigned g = vec_blocks(P, W);
  const double *z = mg_result_host(M, 0);
  for (int it = 0; it < n; ++it) {
    k_spmv_g<<<g, kVecThreads, 0, s>>>(M.L[0], W, P.Np);
    k_update_g<<<g, kVecThreads, 0, s>>>(W, P.Np);
    mg_vcycle_launch(M, W.r, &W.sc->done, s);
    k_rz_g<<<g, kVecThreads, 0, s>>>(W, z, P.Np, 0);
    k_pupdate_g<<<g, kVecThreads, 0, s>>>(W, z, P.Np);
  }
}

namespace {
void precond_fdm(const DevOps &P, const FdmD &F, const PcgWork &W, cudaStream_t s) {
  if (F.spectral)
    launch_fft_precond(P, *F.fft, W.r, F.z, F.gate, &W.sc->done, s);
  else
    fdm_apply(F, W.r, F.z, &W.sc->done, s);
}
}  // namespace

void pcg_init_fdm(const DevOps &P, const FdmD &F, const PcgWork &W, const double *f, double tol, long long maxit,
                  cudaStream_t s) {
  k_init_g<<<vec_blocks(P, W), kVecThreads, 0, s>>>(P, W, f, tol * tol, maxit);
  precond_fdm(P, F, W, s);
  k_rz_g<<<vec_blocks(P, W), kVecThreads, 0, s>>>(W, F.z, P.Np, 1);
}

void pcg_iterations_fdm(const DevOps &P, const FdmD &F, const PcgWork &W, int n, cudaStream_t s) {
  const unsigned g = vec_blocks(P, W);
  for (int it = 0; it < n; ++it) {
    k_spmv_cols<<<spmv_grid(P), dim3(BX, BY), 0, s>>>(P, W);
    k_update_g<<<g, kVecThreads, 0, s>>>(W, P.Np);
    precond_fdm(P, F, W, s);
    k_rz_g<<<g, kVecThreads, 0, s>>>(W, F.z, P.Np, 0);
    k_pupdate_g<<<g, kVecThreads, 0, s>>>(W, F.z, P.Np);
  }
}

namespace {
__global__ void k_pcg_cond(PcgScalars *sc, cudaGraphConditionalHandle h, int limit, int count) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int n = sc->loops;
  if (count) sc->loops = ++n;
  const int done = *(volatile int *)&sc->done;
  cudaGraphSetConditional(h, (!done && n < limit) ? 1u : 0u);
}
__global__ void k_solve_accum(const PcgScalars *sc, SolveAccum *a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const long long it = sc->it;
  a->n_solves += 1;
  a->iters_total += it;
  if (it > a->iters_max) a->iters_max = it;
  const double n1 = sqrt(sc->rr);
  if (n1 > a->norm1_max) a->norm1_max = n1;
  const int st = sc->done ? sc->status : INS2D_ETIMEOUT;
  if (st != 0 && a->status == 0) {
    a->status = st;
    a->fail_rr = sc->rr;
    a->fail_maxit = sc->maxit;
  }
}
}  // namespace

void launch_pcg_cond(PcgScalars *sc, cudaGraphConditionalHandle h, int limit, int count, cudaStream_t s) {
  k_pcg_cond<<<1, 32, 0, s>>>(sc, h, limit, count);
}
void launch_solve_accum(const PcgScalars *sc, SolveAccum *acc, cudaStream_t s) {
  k_solve_accum<<<1, 32, 0, s>>>(sc, acc);
}

void pcg_finish(const DevOps &P, const PcgWork &W, double *dp, bool accumulate, cudaStream_t s) {
  long long n = P.Np;
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_copy_out<<<(unsigned)blocks, 256, 0, s>>>(W.x, dp, n, accumulate ? 1 : 0);
}

}  // namespace ins2d

namespace ins2d {

void launch_pcg_members(const EnsMemberD *mem, const int *order, int n, int which, double tol2, long long maxit,
                        unsigned *queue, EnsStats *stats, int threads, int blocks, cudaStream_t s) {
  if (n <= 0) return;
  k_pcg_members<<<blocks, threads, 0, s>>>(mem, order, n, which, tol2, maxit, queue, stats);
}

}  // namespace ins2d
