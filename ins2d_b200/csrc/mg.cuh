// Multigrid V-cycle used as the preconditioner of the pressure PCG.
//
// The pressure matrix of the reference, A = M Om^-1 G (operator_divergence.m:208),
// is separable: A = -(diag(hy) (x) TX + TY (x) diag(hx)) with TX, TY 1D
// tridiagonal operators (periodic wraps included).  Coarse levels are the
// Galerkin products P' A P for piecewise-constant aggregation of 2x2 (or 2x1)
// cells, which keep the same separable form: TXc = Px' TX Px and the weights
// summed over the aggregate (hxc = Px' hx).  So every level is described by
// O(nx + ny) numbers: per row i of the 1D x operator its entries at i-1, i,
// i+1 (xm, x0, xp) and per row j of the y operator (ym, y0, yp), with the
// 5-point couplings
//   W = -hy_j xm_i, E = -hy_j xp_i, S = -hx_i ym_j, N = -hx_i yp_j,
//   C = -(hy_j x0_i + hx_i y0_j).
// Smoother: alternating line relaxation (block Jacobi over x-lines, then over
// y-lines, damped by omega), which stays robust on the strongly stretched
// grids of the channel and cavity cases where point Jacobi stalls.  The
// post-smoother applies the two sweeps in the reverse order, so the V-cycle
// is a symmetric operator (as the preconditioner of CG must be).  The
// coarsest level (<= kMgCoarseMax cells) is solved with a dense
// pseudo-inverse, so singular (all-Neumann or periodic) problems are handled.
// The coarse correction is scaled by alpha (over-correction of unsmoothed
// aggregation).
//
// Line solves use per-cell Thomas factors computed once at set-up (periodic
// lines in the Sherman-Morrison form T = T' + u v', z = T'^-1 u stored per
// cell).  The Thomas recurrences are first-order linear, so a row is solved
// by a warp as a scan of affine maps (mg_line_warp) and 32 columns by a thread
// block whose warps compose segments of rows (mg_ycols_block).
//
// The phase functions take (first line/cell, stride) so the same code runs
// inside one thread block (small grids, ensembles: one block per solve) and
// across a grid of blocks (large grids: one launch per phase).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <vector>

namespace ins2d {

constexpr int kMgMaxLevels = 20;
constexpr int kMgCoarseMax = 64;

struct MgLevelD {
  int nx, ny, perx, pery;
  int cx, cy;  // aggregation factors to the next level (1 or 2)
  const double *xm, *x0, *xp, *hx;  // nx
  const double *ym, *y0, *yp, *hy;  // ny
  // line factors per cell: x-lines (fxc = c', fxi = 1/pivot), y-lines
  double *fxc, *fxi, *fyc, *fyi;
  // periodic lines: z = T'^-1 u per cell; per line g = a0/gamma, k = 1/(1 + v'z)
  double *zx, *zy, *gx, *kx, *gy, *ky;
  // vectors: right-hand side, iterate and its relaxed copy
  double *b, *x, *t;
};

struct MgD {
  int nlev;
  int ncoarse;         // cells of the coarsest level
  const double *cinv;  // ncoarse x ncoarse pseudo-inverse of the coarsest matrix
  double omega, alpha;
  MgLevelD L[kMgMaxLevels];
};

// ---------------------------------------------------------------------------
__device__ __forceinline__ int mg_wrap_lo(int i, int n, int per) { return i > 0 ? i - 1 : (per ? n - 1 : 0); }
__device__ __forceinline__ int mg_wrap_hi(int i, int n, int per) { return i < n - 1 ? i + 1 : (per ? 0 : n - 1); }

// (A x)(i,j) at one cell of level L
__device__ __forceinline__ double mg_apply(const MgLevelD &L, const double *__restrict__ x, int i, int j) {
  const int nx = L.nx;
  const double hx = L.hx[i], hy = L.hy[j];
  const int im = mg_wrap_lo(i, nx, L.perx), ip = mg_wrap_hi(i, nx, L.perx);
  const int jm = mg_wrap_lo(j, L.ny, L.pery), jp = mg_wrap_hi(j, L.ny, L.pery);
  const long long r = (long long)j * nx;
  return -(hy * (L.xm[i] * x[r + im] + L.x0[i] * x[r + i] + L.xp[i] * x[r + ip]) +
           hx * (L.ym[j] * x[(long long)jm * nx + i] + L.y0[j] * x[r + i] + L.yp[j] * x[(long long)jp * nx + i]));
}

// Factors of the x-line of row j: T = tridiag(a, b, c), a_i = W(i,j),
// b_i = C(i,j), c_i = E(i,j) (cyclic: corners a_0 and c_{n-1}).
__device__ inline void mg_factor_xline(const MgLevelD &L, int j) {
  const int n = L.nx;
  const double hy = L.hy[j], y0 = L.y0[j];
  const long long r = (long long)j * n;
  auto A = [&](int i) { return -hy * L.xm[i]; };
  auto B = [&](int i) { return -(hy * L.x0[i] + L.hx[i] * y0); };
  auto C = [&](int i) { return -hy * L.xp[i]; };
  const bool cyc = L.perx && n >= 3;
  const double gamma = -B(0);
  double cp = 0.0;
  for (int i = 0; i < n; ++i) {
    double bi = B(i);
    if (cyc && i == 0) bi -= gamma;
    if (cyc && i == n - 1) bi -= C(n - 1) * A(0) / gamma;
    const double ai = (i > 0) ? A(i) : 0.0;
    const double inv = 1.0 / (bi - ai * cp);
    cp = (i < n - 1) ? C(i) * inv : 0.0;
    L.fxi[r + i] = inv;
    L.fxc[r + i] = cp;
  }
  if (cyc) {
    // z = T'^-1 u, u = (gamma, 0, ..., 0, c_{n-1})
    double d = 0.0;
    for (int i = 0; i < n; ++i) {
      const double ui = (i == 0) ? gamma : (i == n - 1 ? C(n - 1) : 0.0);
      const double ai = (i > 0) ? A(i) : 0.0;
      d = (ui - ai * d) * L.fxi[r + i];
      L.zx[r + i] = d;
    }
    double z = 0.0;
    for (int i = n - 1; i >= 0; --i) {
      z = L.zx[r + i] - L.fxc[r + i] * z;
      L.zx[r + i] = z;
    }
    const double g = A(0) / gamma;
    L.gx[j] = g;
    L.kx[j] = 1.0 / (1.0 + L.zx[r] + g * L.zx[r + n - 1]);
  }
}

__device__ inline void mg_factor_yline(const MgLevelD &L, int i) {
  const int n = L.ny, nx = L.nx;
  const double hx = L.hx[i], x0 = L.x0[i];
  auto A = [&](int j) { return -hx * L.ym[j]; };
  auto B = [&](int j) { return -(L.hy[j] * x0 + hx * L.y0[j]); };
  auto C = [&](int j) { return -hx * L.yp[j]; };
  const bool cyc = L.pery && n >= 3;
  const double gamma = -B(0);
  double cp = 0.0;
  for (int j = 0; j < n; ++j) {
    double bj = B(j);
    if (cyc && j == 0) bj -= gamma;
    if (cyc && j == n - 1) bj -= C(n - 1) * A(0) / gamma;
    const double aj = (j > 0) ? A(j) : 0.0;
    const double inv = 1.0 / (bj - aj * cp);
    cp = (j < n - 1) ? C(j) * inv : 0.0;
    const long long k = (long long)j * nx + i;
    L.fyi[k] = inv;
    L.fyc[k] = cp;
  }
  if (cyc) {
    double d = 0.0;
    for (int j = 0; j < n; ++j) {
      const double uj = (j == 0) ? gamma : (j == n - 1 ? C(n - 1) : 0.0);
      const double aj = (j > 0) ? A(j) : 0.0;
      const long long k = (long long)j * nx + i;
      d = (uj - aj * d) * L.fyi[k];
      L.zy[k] = d;
    }
    double z = 0.0;
    for (int j = n - 1; j >= 0; --j) {
      const long long k = (long long)j * nx + i;
      z = L.zy[k] - L.fyc[k] * z;
      L.zy[k] = z;
    }
    const double g = A(0) / gamma;
    L.gy[i] = g;
    L.ky[i] = 1.0 / (1.0 + L.zy[i] + g * L.zy[(long long)(n - 1) * nx + i]);
  }
}

// One line of a level: cell q at base + q*st (st = 1 for x-lines, nx for
// y-lines); the couplings to the neighbouring lines (at +lo, +hi) enter the
// right-hand side with the old iterate:
//   xnew = (1-omega) xold + omega T^-1 (b - X xold),   xold == nullptr: zero.
struct MgLine {
  long long base, st, lo, hi;  // cell q at base + q*st; neighbours at +lo, +hi
  int n;
  const double *cross_w;       // per cell of the line: weight of the cross couplings (hx or hy)
  double cm, cp;               // cross-coupling entries (ym/yp or xm/xp) of this line
  const double *am;            // per cell: entry at q-1 of the line operator (xm or ym)
  double ascale;               // the line's weight (hy or hx)
  const double *fi, *fc;       // Thomas factors
  const double *z;             // periodic lines: T'^-1 u
  double g, k;                 // periodic lines: v'/(1+v'z) terms
  bool cyc;
};

__device__ __forceinline__ MgLine mg_make_xline(const MgLevelD &L, int j) {
  const int nx = L.nx, ny = L.ny;
  MgLine ln;
  ln.base = (long long)j * nx;
  ln.st = 1;
  ln.lo = (long long)(mg_wrap_lo(j, ny, L.pery) - j) * nx;
  ln.hi = (long long)(mg_wrap_hi(j, ny, L.pery) - j) * nx;
  ln.n = nx;
  ln.cross_w = L.hx;
  ln.cm = L.ym[j];
  ln.cp = L.yp[j];
  ln.am = L.xm;
  ln.ascale = L.hy[j];
  ln.fi = L.fxi;
  ln.fc = L.fxc;
  ln.cyc = L.perx && nx >= 3;
  ln.z = L.zx;
  ln.g = ln.cyc ? L.gx[j] : 0.0;
  ln.k = ln.cyc ? L.kx[j] : 0.0;
  return ln;
}
__device__ __forceinline__ MgLine mg_make_yline(const MgLevelD &L, int i) {
  const int nx = L.nx, ny = L.ny;
  MgLine ln;
  ln.base = i;
  ln.st = nx;
  ln.lo = mg_wrap_lo(i, nx, L.perx) - i;
  ln.hi = mg_wrap_hi(i, nx, L.perx) - i;
  ln.n = ny;
  ln.cross_w = L.hy;
  ln.cm = L.xm[i];
  ln.cp = L.xp[i];
  ln.am = L.ym;
  ln.ascale = L.hx[i];
  ln.fi = L.fyi;
  ln.fc = L.fyc;
  ln.cyc = L.pery && ny >= 3;
  ln.z = L.zy;
  ln.g = ln.cyc ? L.gy[i] : 0.0;
  ln.k = ln.cyc ? L.ky[i] : 0.0;
  return ln;
}

// One line solved by a whole warp: the Thomas recurrences are first-order
// linear (forward d_q = al_q d_{q-1} + be_q with al = -a/pivot, be = rhs/pivot;
// backward x_q = -c'_q x_{q+1} + d_q), so each chunk of 32 cells is one
// warp-wide scan of affine maps (5 shuffle steps) carried from chunk to chunk.
// The dependent chain is n/32 chunk steps instead of n cell steps, and the
// loads of a chunk are coalesced along x-lines.  All 32 lanes must call it.
template <int U = 2>
static __device__ __forceinline__ void mg_line_warp(const MgLine ln, const double *__restrict__ b,
                                                    const double *__restrict__ xold, double *__restrict__ xnew,
                                                    double omega) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int n = ln.n;
  const long long base = ln.base, st = ln.st;
  const bool hasold = xold != nullptr, cyc = ln.cyc;
  double carry = 0.0;
#pragma unroll U
  for (int c0 = 0; c0 < n; c0 += 32) {
    const int q = c0 + lane;
    const long long k = base + (long long)q * st;
    double A = 1.0, B = 0.0;
    if (q < n) {
      double rhs = b[k];
      if (hasold) rhs += ln.cross_w[q] * (ln.cm * xold[k + ln.lo] + ln.cp * xold[k + ln.hi]);
      const double f = ln.fi[k];
      A = (q > 0) ? (ln.ascale * ln.am[q]) * f : 0.0;
      B = rhs * f;
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double Ap = __shfl_up_sync(FULL, A, off), Bp = __shfl_up_sync(FULL, B, off);
      if (lane >= off) {
        B = A * Bp + B;
        A = A * Ap;
      }
    }
    const double d = A * carry + B;
    if (q < n) xnew[k] = d;
    carry = __shfl_sync(FULL, d, 31);
  }
  carry = 0.0;
#pragma unroll U
  for (int c0 = ((n - 1) >> 5) << 5; c0 >= 0; c0 -= 32) {
    const int q = c0 + lane;
    const long long k = base + (long long)q * st;
    double A = 1.0, B = 0.0;
    if (q < n) {
      A = -ln.fc[k];
      B = xnew[k];
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double An = __shfl_down_sync(FULL, A, off), Bn = __shfl_down_sync(FULL, B, off);
      if (lane + off < 32) {
        B = A * Bn + B;
        A = A * An;
      }
    }
    const double x = A * carry + B;
    carry = __shfl_sync(FULL, x, 0);
    if (q < n) {
      if (cyc)
        xnew[k] = x;
      else
        xnew[k] = hasold ? (1.0 - omega) * xold[k] + omega * x : omega * x;
    }
  }
  if (cyc) {
    __syncwarp();
    const double s = (xnew[base] + ln.g * xnew[base + (long long)(n - 1) * st]) * ln.k;
    __syncwarp();
    for (int q = lane; q < n; q += 32) {
      const long long k = base + (long long)q * st;
      const double v = xnew[k] - s * ln.z[k];
      xnew[k] = hasold ? (1.0 - omega) * xold[k] + omega * v : omega * v;
    }
  }
}

// One line relaxed by P warps of a thread block (warps q = 0..P-1 of the
// calling group own consecutive ranges of the line's 32-cell chunks).  Each
// warp first composes the affine maps of the Thomas recurrence over its
// range (forward: lane 31's inclusive scan of every chunk; backward: lane
// 0's), the range composites are chained through shared memory (sh: 4 P
// doubles of this line), then each warp re-walks its range from the value
// entering it.  The dependent chain per warp is about 2 chunks / P + P chunk
// steps in each direction instead of chunks.  Every thread of the block must
// call it (block barriers).
template <int P>
__device__ inline void mg_line_split(const MgLine ln, const double *__restrict__ b, const double *__restrict__ xold,
                                     double *__restrict__ xnew, double omega, int q, double *sh) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int n = ln.n;
  const long long base = ln.base, st = ln.st;
  const bool hasold = xold != nullptr, cyc = ln.cyc;
  const int chunks = (n + 31) >> 5, per = (chunks + P - 1) / P;
  const int c_lo = min(chunks, q * per), c_hi = min(chunks, c_lo + per);
  // forward map of one chunk at lane level (inclusive scan), cell c*32+lane
  auto fscan = [&](int c, double &A, double &B) {
    const int i = c * 32 + lane;
    const long long k = base + (long long)i * st;
    A = 1.0;
    B = 0.0;
    if (i < n) {
      double rhs = b[k];
      if (hasold) rhs += ln.cross_w[i] * (ln.cm * xold[k + ln.lo] + ln.cp * xold[k + ln.hi]);
      const double f = ln.fi[k];
      A = (i > 0) ? (ln.ascale * ln.am[i]) * f : 0.0;
      B = rhs * f;
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double Ap = __shfl_up_sync(FULL, A, off), Bp = __shfl_up_sync(FULL, B, off);
      if (lane >= off) {
        B = A * Bp + B;
        A = A * Ap;
      }
    }
  };
  // backward map of one chunk (suffix scan): x_i = -fc_i x_{i+1} + xnew_i
  auto bscan = [&](int c, double &A, double &B) {
    const int i = c * 32 + lane;
    const long long k = base + (long long)i * st;
    A = 1.0;
    B = 0.0;
    if (i < n) {
      A = -ln.fc[k];
      B = xnew[k];
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double An = __shfl_down_sync(FULL, A, off), Bn = __shfl_down_sync(FULL, B, off);
      if (lane + off < 32) {
        B = A * Bn + B;
        A = A * An;
      }
    }
  };
  double *fA = sh, *fB = sh + P, *gA = sh + 2 * P, *gB = sh + 3 * P;
  // forward, pass 1: composite of the range
  double SA = 1.0, SB = 0.0;
  for (int c = c_lo; c < c_hi; ++c) {
    double A, B;
    fscan(c, A, B);
    const double Ac = __shfl_sync(FULL, A, 31), Bc = __shfl_sync(FULL, B, 31);
    SB = Ac * SB + Bc;
    SA = Ac * SA;
  }
  if (lane == 0) {
    fA[q] = SA;
    fB[q] = SB;
  }
  __syncthreads();
  double carry = 0.0;
  for (int r = 0; r < q; ++r) carry = fA[r] * carry + fB[r];
  // forward, pass 2
  for (int c = c_lo; c < c_hi; ++c) {
    double A, B;
    fscan(c, A, B);
    const double d = A * carry + B;
    const int i = c * 32 + lane;
    if (i < n) xnew[base + (long long)i * st] = d;
    carry = __shfl_sync(FULL, d, 31);
  }
  __syncthreads();
  // backward, pass 1: composite of the range (right to left)
  SA = 1.0;
  SB = 0.0;
  for (int c = c_hi - 1; c >= c_lo; --c) {
    double A, B;
    bscan(c, A, B);
    const double Ac = __shfl_sync(FULL, A, 0), Bc = __shfl_sync(FULL, B, 0);
    SB = Ac * SB + Bc;
    SA = Ac * SA;
  }
  if (lane == 0) {
    gA[q] = SA;
    gB[q] = SB;
  }
  __syncthreads();
  carry = 0.0;
  for (int r = P - 1; r > q; --r) carry = gA[r] * carry + gB[r];
  // backward, pass 2: solution and relaxation
  for (int c = c_hi - 1; c >= c_lo; --c) {
    double A, B;
    bscan(c, A, B);
    const double x = A * carry + B;
    carry = __shfl_sync(FULL, x, 0);
    const int i = c * 32 + lane;
    if (i < n) {
      const long long k = base + (long long)i * st;
      xnew[k] = cyc ? x : (hasold ? (1.0 - omega) * xold[k] + omega * x : omega * x);
    }
  }
  if (cyc) {
    // the line's first and last values are read by every warp before any
    // warp updates its range
    __syncthreads();
    const double s = (xnew[base] + ln.g * xnew[base + (long long)(n - 1) * st]) * ln.k;
    __syncthreads();
    for (int c = c_lo; c < c_hi; ++c) {
      const int i = c * 32 + lane;
      if (i < n) {
        const long long k = base + (long long)i * st;
        const double v = xnew[k] - s * ln.z[k];
        xnew[k] = hasold ? (1.0 - omega) * xold[k] + omega * v : omega * v;
      }
    }
  }
}

// x-line relaxations: a warp per row (first = warp index j0 >> 5, step =
// warps (js + 31) >> 5 when called with thread indices)
template <int U = 2>
__device__ inline void mg_xline(const MgLevelD &L, const double *__restrict__ b, const double *__restrict__ xold,
                                double *__restrict__ xnew, double omega, int j0, int js) {
  for (int j = j0 >> 5; j < L.ny; j += (js + 31) >> 5) mg_line_warp<U>(mg_make_xline(L, j), b, xold, xnew, omega);
}
// threads per line of the warp solves
constexpr int kMgLineThreads = 32;

#ifndef INS2D_MG_UNROLL
#define INS2D_MG_UNROLL 4
#endif
constexpr int kMgUnroll = INS2D_MG_UNROLL;  // unrolling of the column segment walks

// y-lines (columns) i0 .. i0+31 of a level solved by a whole thread block:
// lane = column (loads coalesced along rows), warp w = a segment of rows.
// Each thread first composes the affine maps of the Thomas recurrences over
// its segment, the segments' composites are chained through shared memory
// (sh: 2 x warps x 32 doubles), then each thread re-walks its segment.  The
// dependent chain per thread is about 4 n / warps + 2 warps steps.  All
// threads of the block must call it.
// CW = columns per block (32, or 16: each warp then walks two segments, one
// per half-warp, so twice as many blocks share a level's columns).
template <int U = kMgUnroll, int CW = 32>
__device__ inline void mg_ycols_block(const MgLevelD &L, const double *__restrict__ b,
                                      const double *__restrict__ xold, double *__restrict__ xnew, double omega,
                                      int i0, double *sh) {
  static_assert(CW == 32 || CW == 16 || CW == 8, "columns per block");
  constexpr int SPW = 32 / CW;  // segments per warp
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, W = blockDim.x >> 5;
  const int cl = lane % CW, seg = w * SPW + lane / CW, S = W * SPW;
  const int nx = L.nx, n = L.ny;
  const int i = i0 + cl;
  const bool col = i < nx;
  const int m = (n + S - 1) / S;
  const int j0 = min(n, seg * m), j1 = min(n, j0 + m);
  const bool hasold = xold != nullptr, cyc = L.pery && n >= 3;
  double hx = 0.0, xmv = 0.0, xpv = 0.0;
  int im = 0, ip = 0;
  if (col) {
    hx = L.hx[i];
    xmv = L.xm[i];
    xpv = L.xp[i];
    im = mg_wrap_lo(i, nx, L.perx);
    ip = mg_wrap_hi(i, nx, L.perx);
  }
  auto fwd = [&](int j, double &al, double &be) {
    const long long k = (long long)j * nx + i;
    double rhs = b[k];
    if (hasold) rhs += L.hy[j] * (xmv * xold[(long long)j * nx + im] + xpv * xold[(long long)j * nx + ip]);
    const double f = L.fyi[k];
    al = (j > 0) ? (hx * L.ym[j]) * f : 0.0;
    be = rhs * f;
  };
  // forward pass 1: composite of the segment, d_{j1-1} = A d_{j0-1} + B
  double A = 1.0, B = 0.0;
  if (col)
#pragma unroll U
    for (int j = j0; j < j1; ++j) {
      double al, be;
      fwd(j, al, be);
      B = al * B + be;
      A = al * A;
    }
  double *sA = sh, *sB = sh + W * 32;  // [segment][column], S * CW = W * 32 entries each
  sA[seg * CW + cl] = A;
  sB[seg * CW + cl] = B;
  __syncthreads();
  if (w == 0 && lane < CW) {
    double d = 0.0;
    for (int q = 0; q < S; ++q) {
      const double Aq = sA[q * CW + lane], Bq = sB[q * CW + lane];
      sA[q * CW + lane] = d;  // value entering segment q
      d = Aq * d + Bq;
    }
  }
  __syncthreads();
  double d = sA[seg * CW + cl];
  __syncthreads();
  if (col)
#pragma unroll U
    for (int j = j0; j < j1; ++j) {
      double al, be;
      fwd(j, al, be);
      d = al * d + be;
      xnew[(long long)j * nx + i] = d;
    }
  // backward pass 1: x_{j0} = A x_{j1} + B over the segment
  A = 1.0;
  B = 0.0;
  if (col)
#pragma unroll U
    for (int j = j1 - 1; j >= j0; --j) {
      const long long k = (long long)j * nx + i;
      const double ga = -L.fyc[k];
      B = ga * B + xnew[k];
      A = ga * A;
    }
  sA[seg * CW + cl] = A;
  sB[seg * CW + cl] = B;
  __syncthreads();
  if (w == 0 && lane < CW) {
    double x = 0.0;
    for (int q = S - 1; q >= 0; --q) {
      const double Aq = sA[q * CW + lane], Bq = sB[q * CW + lane];
      sA[q * CW + lane] = x;  // value above segment q
      x = Aq * x + Bq;
    }
  }
  __syncthreads();
  double x = sA[seg * CW + cl];
  __syncthreads();
  if (col)
#pragma unroll U
    for (int j = j1 - 1; j >= j0; --j) {
      const long long k = (long long)j * nx + i;
      x = -L.fyc[k] * x + xnew[k];
      xnew[k] = cyc ? x : (hasold ? (1.0 - omega) * xold[k] + omega * x : omega * x);
    }
  if (cyc) {
    // every segment reads the column's first and last values before any
    // segment overwrites them
    __syncthreads();
    const double s = col ? (xnew[i] + L.gy[i] * xnew[(long long)(n - 1) * nx + i]) * L.ky[i] : 0.0;
    __syncthreads();
    if (col) {
      for (int j = j0; j < j1; ++j) {
        const long long k = (long long)j * nx + i;
        const double v = xnew[k] - s * L.zy[k];
        xnew[k] = hasold ? (1.0 - omega) * xold[k] + omega * v : omega * v;
      }
    }
    __syncthreads();
  }
}

// all y-lines of a level by one thread block (groups of 32 columns)
__device__ inline void mg_yline_block(const MgLevelD &L, const double *__restrict__ b,
                                      const double *__restrict__ xold, double *__restrict__ xnew, double omega,
                                      double *sh) {
  for (int i0 = 0; i0 < L.nx; i0 += 32) {
    mg_ycols_block(L, b, xold, xnew, omega, i0, sh);
    __syncthreads();
  }
}

// bc = P' (b - A x) over the coarse cells k0, k0+ks, ...
__device__ inline void mg_restrict(const MgLevelD &F, const MgLevelD &Cl, const double *__restrict__ b,
                                   const double *__restrict__ x, double *__restrict__ bc, long long k0, long long ks) {
  const long long nc = (long long)Cl.nx * Cl.ny;
  for (long long k = k0; k < nc; k += ks) {
    const int I = (int)(k % Cl.nx), J = (int)(k / Cl.nx);
    double s = 0.0;
    for (int dj = 0; dj < F.cy; ++dj) {
      const int j = J * F.cy + dj;
      if (j >= F.ny) break;
      for (int di = 0; di < F.cx; ++di) {
        const int i = I * F.cx + di;
        if (i >= F.nx) break;
        s += b[(long long)j * F.nx + i] - mg_apply(F, x, i, j);
      }
    }
    bc[k] = s;
  }
}

// x += alpha * P xc over the fine cells k0, k0+ks, ...
__device__ inline void mg_prolong(const MgLevelD &F, const MgLevelD &Cl, double *__restrict__ x,
                                  const double *__restrict__ xc, double alpha, long long k0, long long ks) {
  const long long n = (long long)F.nx * F.ny;
  for (long long k = k0; k < n; k += ks) {
    const int i = (int)(k % F.nx), j = (int)(k / F.nx);
    x[k] += alpha * xc[(long long)(j / F.cy) * Cl.nx + i / F.cx];
  }
}

// x = Cinv b at the coarsest level (rows k0, k0+ks, ...)
__device__ inline void mg_coarse(const MgD &M, const double *__restrict__ b, double *__restrict__ x, int k0, int ks) {
  const int n = M.ncoarse;
  for (int r = k0; r < n; r += ks) {
    double s = 0.0;
    for (int c = 0; c < n; ++c) s += M.cinv[(long long)r * n + c] * b[c];
    x[r] = s;
  }
}

// Optional per-phase clock counters (timing builds only: -DINS2D_MG_TIMING)
#ifdef INS2D_MG_TIMING
static __device__ unsigned long long g_mg_clk[128];
#define MG_T0() long long _mg_t0 = clock64()
#define MG_TICK(k)                                                        \
  do {                                                                    \
    if (threadIdx.x == 0) {                                               \
      const long long _t1 = clock64();                                    \
      atomicAdd(&g_mg_clk[(k) & 127], (unsigned long long)(_t1 - _mg_t0)); \
      _mg_t0 = _t1;                                                       \
    }                                                                     \
  } while (0)
#else
#define MG_T0() \
  do {          \
  } while (0)
#define MG_TICK(k) \
  do {             \
  } while (0)
#endif

// Result location of a V-cycle at level l: the relaxed copy t (levels above
// the coarsest) or x (the coarsest).
__device__ __forceinline__ double *mg_result(const MgD &M, int l) {
  return (l == M.nlev - 1) ? M.L[l].x : M.L[l].t;
}

// One V-cycle inside a thread block from level l0 down to the coarsest and
// back: z = B b with b = b0 the right-hand side of level l0; the result is at
// mg_result(M, l0).  ysh: shared memory of 2 x 32 x (block warps) doubles for
// the column solves.  All threads of the block must call it.
__device__ inline void mg_vcycle_block(const MgD &M, const double *__restrict__ b0, int l0, double *ysh) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int nl = M.nlev;
  MG_T0();
  for (int l = l0; l < nl - 1; ++l) {
    const MgLevelD &L = M.L[l];
    const double *b = (l == l0) ? b0 : L.b;
    mg_xline(L, b, nullptr, L.x, M.omega, tid, nt);
    __syncthreads();
    MG_TICK(l * 8 + 0);
    mg_yline_block(L, b, L.x, L.t, M.omega, ysh);
    MG_TICK(l * 8 + 1);
    mg_restrict(L, M.L[l + 1], b, L.t, M.L[l + 1].b, tid, nt);
    __syncthreads();
    MG_TICK(l * 8 + 2);
  }
  mg_coarse(M, (l0 == nl - 1) ? b0 : M.L[nl - 1].b, M.L[nl - 1].x, tid, nt);
  __syncthreads();
  MG_TICK((nl - 1) * 8 + 3);
  for (int l = nl - 2; l >= l0; --l) {
    const MgLevelD &L = M.L[l];
    const double *b = (l == l0) ? b0 : L.b;
    mg_prolong(L, M.L[l + 1], L.t, mg_result(M, l + 1), M.alpha, tid, nt);
    __syncthreads();
    MG_TICK(l * 8 + 4);
    mg_yline_block(L, b, L.t, L.x, M.omega, ysh);
    MG_TICK(l * 8 + 5);
    mg_xline(L, b, L.x, L.t, M.omega, tid, nt);
    __syncthreads();
    MG_TICK(l * 8 + 6);
  }
}

// Multi-block V-cycle (mg.cu): one launch per phase on the levels above
// mg_tail_level(M), one thread block for the rest.  Every kernel returns at
// once when *done is set (the PCG has converged), so whole iterations can be
// queued ahead.
int mg_tail_level(const MgD &M);
// Allocates (through alloc, in doubles) and fills the device hierarchy of the
// host levels (mg_host.hpp); the factor kernels run on stream s.
struct MgHostLevel;
void mg_setup_device(const std::vector<MgHostLevel> &lv, MgD &M, const std::function<double *(size_t)> &alloc,
                     cudaStream_t s);
inline double *mg_result_host(const MgD &M, int l) { return (l == M.nlev - 1) ? M.L[l].x : M.L[l].t; }
void mg_vcycle_launch(const MgD &M, const double *r0, const int *done, cudaStream_t s);

}  // namespace ins2d
