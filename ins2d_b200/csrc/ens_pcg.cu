// Ensemble Poisson solves batched across members: the same PCG (cg.F's
// control flow and stopping rule) and multigrid V-cycle as a single context,
// but every phase is ONE launch over the work of all members that have not
// converged yet: CG vector operations over 256-cell tiles of the members'
// grids (one member per tile, block reductions, one atomic per tile), the
// line relaxations over all members' lines of a level (one thread per line),
// restriction, prolongation and the coarsest-level products over all
// members' cells.  Member parallelism keeps the whole GPU busy and hides the
// latency of the sequential line solves, which a one-block-per-member solve
// cannot do for large members.  The per-member scalars (alpha, beta,
// convergence) are advanced by one small kernel per step of the iteration.
#include <cfloat>

#include "ins2d.h"
#include "kernels.cuh"
#include "mg.cuh"

namespace ins2d {

namespace {

constexpr int kTile = 256;

__device__ __forceinline__ double warp_sum(double v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
  return v;
}

// block sum (or max) of one value; the result is valid in thread 0
template <bool MAX>
__device__ double block_red1(double v, double *sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = MAX ? warp_max(v) : warp_sum(v);
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double a = sh[0];
  if (threadIdx.x == 0)
    for (int k = 1; k < nw; ++k) a = MAX ? fmax(a, sh[k]) : a + sh[k];
  __syncthreads();
  return a;
}

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
  atomicMax((unsigned long long *)addr, (unsigned long long)__double_as_longlong(v));
}

// member of global work index g (start has n+1 entries, increasing)
__device__ __forceinline__ int seg_find(const long long *__restrict__ start, int n, long long g) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= g)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ const MgLevelD &lev(const EnsMgD &G, int m, int l) { return G.lev[m * kMgMaxLevels + l]; }
__device__ __forceinline__ const double *mg_res(const EnsMgD &G, int m, int l) {
  return (l == G.nlev[m] - 1) ? lev(G, m, l).x : lev(G, m, l).t;
}
__device__ __forceinline__ const double *level_rhs(const EnsMemberD *mem, const EnsMgD &G, int m, int l) {
  return l == 0 ? mem[m].W.r : lev(G, m, l).b;
}

// ---------------------------------------------------------------------------
// CG vector phases over 256-cell tiles {member, first cell}
__global__ void __launch_bounds__(kTile) k_ecg_vec(const EnsMemberD *__restrict__ mem, const EnsMgD G,
                                                  const int2 *__restrict__ tiles, EnsCg *__restrict__ cg, int op) {
  __shared__ __align__(16) DevOps sP;
  __shared__ double sh[kTile / 32];
  const int2 t = tiles[blockIdx.x];
  const int m = t.x;
  EnsCg &C = cg[m];
  if (op != 0 && *(volatile int *)&C.done) return;
  const EnsMemberD &E = mem[m];
  const long long k = (long long)t.y + threadIdx.x;
  const bool in = k < E.P.Np;
  const PcgWork &W = E.W;
  const double *z = E.zf ? E.zf : mg_res(G, m, 0);
  double a = 0.0, b = 0.0;
  if (op == 1) {  // q = A p, p'q
    for (int w = threadIdx.x; w < (int)(sizeof(DevOps) / 8); w += blockDim.x)
      ((long long *)&sP)[w] = ((const long long *)&E.P)[w];
    __syncthreads();
    if (in) {
      const int i = (int)(k % sP.Npx), j = (int)(k / sP.Npx);
      const double aq = lap(sP, W.p, i, j);
      W.q[k] = aq;
      a = W.p[k] * aq;
    }
    a = block_red1<false>(a, sh);
    if (threadIdx.x == 0) atomicAdd(&C.acc_pq, a);
    return;
  }
  if (op == 0) {  // init: x = 0, r = f; f'f, max|f|
    if (in) {
      const double fv = E.f[k];
      W.x[k] = 0.0;
      W.r[k] = fv;
      a = fv * fv;
      b = fabs(fv);
    }
    a = block_red1<false>(a, sh);
    b = block_red1<true>(b, sh);
    if (threadIdx.x == 0) {
      atomicAdd(&C.acc_rr, a);
      atomic_max_nonneg(&C.maxf, b);
    }
  } else if (op == 2) {  // x += alpha p, r -= alpha q; r'r
    const double al = C.alpha;
    if (in) {
      W.x[k] += al * W.p[k];
      const double rv = W.r[k] - al * W.q[k];
      W.r[k] = rv;
      a = rv * rv;
    }
    a = block_red1<false>(a, sh);
    if (threadIdx.x == 0) atomicAdd(&C.acc_rr, a);
  } else if (op == 3 || op == 4) {  // r'z (op 4: first iteration, p = z)
    if (in) {
      a = W.r[k] * z[k];
      if (op == 4) W.p[k] = z[k];
    }
    a = block_red1<false>(a, sh);
    if (threadIdx.x == 0) atomicAdd(&C.acc_rz, a);
  } else if (op == 5) {  // p = z + beta p
    if (in) W.p[k] = z[k] + C.beta * W.p[k];
  }
}

// Per-member scalar steps (one thread per member, one block).  Counts the
// members still iterating into *active.
__global__ void k_ecg_scalar(EnsCg *__restrict__ cg, int n, int op, int *active) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int mine = 0;
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    EnsCg &C = cg[m];
    if (op == 0) {  // after init (pressure_poisson.m:33-38, cg.F:222-227)
      C.rr0 = C.acc_rr;
      C.acc_rr = 0.0;
      C.it = 0;
      C.status = 0;
      C.rr = 0.0;
      C.done = (C.maxf < 1e-14 || C.rr0 <= C.tol2) ? 1 : 0;
      if (!isfinite(C.rr0)) {
        C.status = INS2D_ENONFINITE;
        C.done = 1;
      }
    } else if (C.done) {
      continue;
    } else if (op == 1) {  // r'z of the first iteration
      C.rz = C.acc_rz;
      C.acc_rz = 0.0;
      if (!isfinite(C.rz)) {
        C.status = INS2D_ENONFINITE;
        C.done = 1;
      }
    } else if (op == 2) {  // alpha
      const double pq = C.acc_pq;
      C.acc_pq = 0.0;
      if (!isfinite(pq)) {
        C.status = INS2D_ENONFINITE;
        C.done = 1;
      } else if (pq == 0.0) {
        C.status = INS2D_EBREAKDOWN;
        C.done = 1;
      } else {
        C.alpha = C.rz / pq;
      }
    } else if (op == 3) {  // convergence (cg.F:240-262)
      C.it += 1;
      C.rr = C.acc_rr / C.rr0;
      C.acc_rr = 0.0;
      if (!isfinite(C.rr)) {
        C.status = INS2D_ENONFINITE;
        C.done = 1;
      } else if (C.rr <= C.tol2) {
        C.done = 1;
      } else if (C.it >= C.maxit) {
        C.status = INS2D_ENOTCONV;
        C.done = 1;
      }
    } else if (op == 4) {  // beta
      const double rz = C.acc_rz;
      C.acc_rz = 0.0;
      if (!isfinite(rz)) {
        C.status = INS2D_ENONFINITE;
        C.done = 1;
      } else {
        C.beta = rz / C.rz;
        C.rz = rz;
      }
    }
    if (!C.done) ++mine;
  }
  if (mine) atomicAdd(&cnt, mine);
  __syncthreads();
  if (threadIdx.x == 0 && active) *active = cnt;
}

// WHILE condition of the graph form of the batched solve: some member still
// iterating and fewer than `limit` passes (count: this launch ends a pass;
// the first launch resets the pass count)
__global__ void k_ecg_loop_cond(const EnsCg *__restrict__ cg, int n, int *loops, int limit, int count,
                                cudaGraphConditionalHandle h) {
  __shared__ int act;
  if (threadIdx.x == 0) act = 0;
  __syncthreads();
  int mine = 0;
  for (int m = threadIdx.x; m < n; m += blockDim.x) mine += cg[m].done ? 0 : 1;
  if (mine) atomicAdd(&act, mine);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int k = count ? *loops + 1 : 0;
    *loops = k;
    cudaGraphSetConditional(h, (act > 0 && k < limit) ? 1u : 0u);
  }
}

// dst = x (which = 0: dp) or dst += x (which = 1: p); statistics
__global__ void __launch_bounds__(kTile) k_ecg_finish(const EnsMemberD *__restrict__ mem,
                                                     const int2 *__restrict__ tiles, const EnsCg *__restrict__ cg,
                                                     int which) {
  const int2 t = tiles[blockIdx.x];
  const int m = t.x;
  const EnsMemberD &E = mem[m];
  if (cg[m].status != 0) return;
  const long long k = (long long)t.y + threadIdx.x;
  if (k >= E.P.Np) return;
  if (which)
    E.p[k] += E.W.x[k];
  else
    E.dp[k] = E.W.x[k];
}

__global__ void k_ecg_stats(EnsCg *__restrict__ cg, int n, EnsStats *__restrict__ stats) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
    EnsCg &C = cg[m];
    EnsStats &st = stats[m];
    st.n_solves += 1;
    st.iters_total += C.it;
    st.iters_max = C.it > st.iters_max ? C.it : st.iters_max;
    const double n1 = sqrt(C.rr);
    st.norm1_max = n1 > st.norm1_max ? n1 : st.norm1_max;
    if (C.status != 0 && st.status == 0) st.status = C.status;
    C.maxf = 0.0;
  }
}

// ---------------------------------------------------------------------------
// V-cycle phases over all members (work index -> member by binary search)
// kind: 0 x-line from zero (x), 1 y-line x->t, 2 y-line t->x, 3 x-line x->t
__global__ void __launch_bounds__(128) k_emg_line(const EnsMemberD *__restrict__ mem, const EnsMgD G,
                                                  const EnsCg *__restrict__ cg, EnsSeg S, int l, int kind,
                                                  double omega) {
  const long long g = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / kMgLineThreads;  // line of this warp
  if (g >= S.total) return;
  const int s = seg_find(S.start, S.n, g);
  const int m = S.mem[s];
  if (cg[m].done) return;
  const int line = (int)(g - S.start[s]);
  const MgLevelD &L = lev(G, m, l);
  const double *b = level_rhs(mem, G, m, l);
  const bool xl = (kind == 0 || kind == 3);
  const MgLine ln = xl ? mg_make_xline(L, line) : mg_make_yline(L, line);
  const double *xold = kind == 0 ? nullptr : (kind == 2 ? L.t : L.x);
  double *xnew = (kind == 0 || kind == 2) ? L.x : L.t;
  mg_line_warp(ln, b, xold, xnew, omega);
}

// x-lines split over P warps each (mg_line_split), one thread block per line
// of any member; kind 0: from zero (x), 3: x -> t
template <int P>
__global__ void __launch_bounds__(32 * P) k_emg_xline_split(const EnsMemberD *__restrict__ mem, const EnsMgD G,
                                                            const EnsCg *__restrict__ cg, EnsSeg S, int l, int kind,
                                                            double omega) {
  __shared__ double sh[4 * P];
  const long long g = blockIdx.x;
  const int s = seg_find(S.start, S.n, g);
  const int m = S.mem[s];
  if (cg[m].done) return;
  const int line = (int)(g - S.start[s]);
  const MgLevelD &L = lev(G, m, l);
  const double *b = level_rhs(mem, G, m, l);
  const double *xold = kind == 0 ? nullptr : L.x;
  double *xnew = kind == 0 ? L.x : L.t;
  mg_line_split<P>(mg_make_xline(L, line), b, xold, xnew, omega, threadIdx.x >> 5, sh);
}

// y-lines in groups of kEnsYcols columns, one thread block per (member, group);
// kind 1: x -> t, 2: t -> x
constexpr int kColThreadsEns = 256;
__global__ void __launch_bounds__(kColThreadsEns) k_emg_ycols(const EnsMemberD *__restrict__ mem, const EnsMgD G,
                                                              const EnsCg *__restrict__ cg, EnsSeg S, int l, int kind,
                                                              double omega) {
  __shared__ double ysh[2 * kColThreadsEns];
  const long long g = blockIdx.x;
  const int s = seg_find(S.start, S.n, g);
  const int m = S.mem[s];
  if (cg[m].done) return;
  const int grp = (int)(g - S.start[s]);
  const MgLevelD &L = lev(G, m, l);
  const double *b = level_rhs(mem, G, m, l);
  if (kind == 1)
    mg_ycols_block<kMgUnroll, kEnsYcols>(L, b, L.x, L.t, omega, grp * kEnsYcols, ysh);
  else
    mg_ycols_block<kMgUnroll, kEnsYcols>(L, b, L.t, L.x, omega, grp * kEnsYcols, ysh);
}

// kind 0: restriction into level l+1; 1: prolongation into level l;
// 2: coarsest-level product
__global__ void __launch_bounds__(256) k_emg_cells(const EnsMemberD *__restrict__ mem, const EnsMgD G,
                                                   const EnsCg *__restrict__ cg, EnsSeg S, int l, int kind,
                                                   double alpha) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= S.total) return;
  const int s = seg_find(S.start, S.n, g);
  const int m = S.mem[s];
  if (cg[m].done) return;
  const long long k = g - S.start[s];
  if (kind == 0) {
    const MgLevelD &F = lev(G, m, l);
    mg_restrict(F, lev(G, m, l + 1), level_rhs(mem, G, m, l), F.t, lev(G, m, l + 1).b, k, 1LL << 40);
  } else if (kind == 1) {
    const MgLevelD &F = lev(G, m, l);
    mg_prolong(F, lev(G, m, l + 1), F.t, mg_res(G, m, l + 1), alpha, k, 1LL << 40);
  } else {
    const int lc = G.nlev[m] - 1;
    const int n = G.ncoarse[m];
    const double *b = level_rhs(mem, G, m, lc);
    const double *ci = G.cinv[m];
    double s2 = 0.0;
    for (int c = 0; c < n; ++c) s2 += ci[k * n + c] * b[c];
    lev(G, m, lc).x[k] = s2;
  }
}

// The coarse part of the V-cycle (levels >= ltail, a few thousand cells per
// member at most) for all members at once: one thread block per member runs
// the single-block V-cycle from its level ltail down and back.
constexpr int kTailThreadsEns = 256;
__global__ void __launch_bounds__(kTailThreadsEns) k_emg_tail(const EnsMemberD *__restrict__ mem,
                                                             const MgD *const *__restrict__ mgs,
                                                             const EnsCg *__restrict__ cg, int ltail) {
  __shared__ __align__(16) MgD sM;
  __shared__ double ysh[2 * kTailThreadsEns];
  const int m = blockIdx.x;
  if (cg[m].done) return;
  const MgD *src = mgs[m];
  for (int w = threadIdx.x; w < (int)(sizeof(MgD) / 8); w += blockDim.x)
    ((long long *)&sM)[w] = ((const long long *)src)[w];
  __syncthreads();
  const int l0 = min(ltail, sM.nlev - 1);
  const double *b0 = (l0 == 0) ? mem[m].W.r : sM.L[l0].b;
  mg_vcycle_block(sM, b0, l0, ysh);
}

unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// warps per x-line of the batched solves (1 = a warp per line)
#ifndef INS2D_ENS_XSPLIT
#define INS2D_ENS_XSPLIT 1
#endif
constexpr int kEnsXsplit = INS2D_ENS_XSPLIT;

void launch_ens_xline(const EnsMemberD *mem, const EnsMgD &G, const EnsCg *cg, const EnsSeg &X, int l, int kind,
                      double omega, cudaStream_t s) {
  if (kEnsXsplit > 1)
    k_emg_xline_split<kEnsXsplit><<<(unsigned)X.total, 32 * kEnsXsplit, 0, s>>>(mem, G, cg, X, l, kind, omega);
  else
    k_emg_line<<<nblk(X.total * kMgLineThreads, 128), 128, 0, s>>>(mem, G, cg, X, l, kind, omega);
}

}  // namespace

void ens_vcycle(const EnsMemberD *mem, const EnsMgD &G, const EnsCg *cg, const EnsMgPlan &pl, double omega,
                double alpha, cudaStream_t s) {
  const int lb = pl.ltail;  // batched levels 0 .. lb-1
  for (int l = 0; l < lb; ++l) {
    const EnsSeg &X = pl.xl[l], &Y = pl.yg[l], &R = pl.rs[l];
    if (X.total) launch_ens_xline(mem, G, cg, X, l, 0, omega, s);
    if (Y.total) k_emg_ycols<<<(unsigned)Y.total, kColThreadsEns, 0, s>>>(mem, G, cg, Y, l, 1, omega);
    if (R.total) k_emg_cells<<<nblk(R.total, 256), 256, 0, s>>>(mem, G, cg, R, l, 0, alpha);
  }
  k_emg_tail<<<pl.co.n, kTailThreadsEns, 0, s>>>(mem, pl.mgs, cg, lb);
  for (int l = lb - 1; l >= 0; --l) {
    const EnsSeg &X = pl.xl[l], &Y = pl.yg[l], &P = pl.pr[l];
    if (P.total) k_emg_cells<<<nblk(P.total, 256), 256, 0, s>>>(mem, G, cg, P, l, 1, alpha);
    if (Y.total) k_emg_ycols<<<(unsigned)Y.total, kColThreadsEns, 0, s>>>(mem, G, cg, Y, l, 2, omega);
    if (X.total) launch_ens_xline(mem, G, cg, X, l, 3, omega, s);
  }
}

void ens_cg_vec(const EnsMemberD *mem, const EnsMgD &G, const int2 *tiles, int ntiles, EnsCg *cg, int op,
                cudaStream_t s) {
  if (ntiles > 0) k_ecg_vec<<<ntiles, kTile, 0, s>>>(mem, G, tiles, cg, op);
}
void ens_loop_cond(const EnsCg *cg, int n, int *loops, int limit, int count, cudaGraphConditionalHandle h,
                   cudaStream_t s) {
  k_ecg_loop_cond<<<1, 256, 0, s>>>(cg, n, loops, limit, count, h);
}
void ens_cg_scalar(EnsCg *cg, int n, int op, int *active, cudaStream_t s) {
  k_ecg_scalar<<<1, 256, 0, s>>>(cg, n, op, active);
}
void ens_cg_finish(const EnsMemberD *mem, const int2 *tiles, int ntiles, EnsCg *cg, int n, int which,
                   EnsStats *stats, cudaStream_t s) {
  if (ntiles > 0) k_ecg_finish<<<ntiles, kTile, 0, s>>>(mem, tiles, cg, which);
  k_ecg_stats<<<nblk(n, 128), 128, 0, s>>>(cg, n, stats);
}

}  // namespace ins2d
