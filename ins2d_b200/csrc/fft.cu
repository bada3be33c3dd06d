// FFT pressure-Poisson solve for periodic uniform grids:
//   dp = real(ifft2(-fft2(f) ./ Ahat)),  Ahat(0,0) = 1
// (solvers/pressure/pressure_poisson.m:92-104, Ahat from
// operator_divergence.m:283-284), including the early return when
// max|fft2(f)| < 1e-14 (pressure_poisson.m:21-32).
//
// Three passes over HBM, each a batched 1D transform in shared memory (FP64):
//  1. rows, real -> complex half spectrum: two real rows packed as one complex
//     row, one complex FFT, split by Hermitian symmetry;
//  2. columns of the half spectrum: forward FFT, multiply by -1/Ahat, inverse
//     FFT (scaled 1/Ny), and the max |fhat| reduction;
//  3. rows, complex half spectrum -> real: two rows packed as one complex
//     inverse FFT (scaled 1/Nx).
// Power-of-two lengths use radix-2 DIT/DIF with a twiddle table; other
// lengths use a shared-memory DFT (O(N^2), small grids).
#include <cmath>
#include <type_traits>
#include <vector>

#include "kernels.cuh"

namespace ins2d {

namespace {

#ifndef INS2D_FFT_THREADS
#define INS2D_FFT_THREADS 256
#endif
#ifndef INS2D_FFT_COLS_MINB
#define INS2D_FFT_COLS_MINB 1
#endif
#ifndef INS2D_FFT_ROWS_MINB
#define INS2D_FFT_ROWS_MINB 4
#endif
#ifndef INS2D_FFT_COLS_BUDGET
#define INS2D_FFT_COLS_BUDGET 80  // KB of shared memory per column block (two 2048-point columns)
#endif
#ifndef INS2D_FFT_COLS_G
#define INS2D_FFT_COLS_G 2
#endif
constexpr int kThreads = INS2D_FFT_THREADS;
constexpr int kMaxPow2 = 8192;
constexpr int kMaxGeneric = 2048;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 twid(const double2 *tw, int k, bool inv) {
  double2 w = __ldg(tw + k);
  if (inv) w.y = -w.y;
  return w;
}
__device__ __forceinline__ int brev(int k, int logn) { return (int)(__brev((unsigned)k) >> (32 - logn)); }

// Shared-memory layout: complex value i sits at i + i/8 + i/64 + i/512 +
// i/4096.  A 16-byte access is served eight lanes at a time, so the eight
// lanes must fall on distinct 16-byte bank groups (slot mod 8): the i/8 term
// does that for the strided butterfly accesses, the others for the
// bit-reversed readouts (eight lanes 2^(L-3) apart).  Line strides are 4 mod 8,
// so two lines interleaved in one warp (column blocks) use disjoint groups.
__host__ __device__ __forceinline__ int pd(int i) { return i + (i >> 3) + (i >> 6) + (i >> 9) + (i >> 12); }
__host__ __device__ __forceinline__ int padded(int n) {
  const int p = pd(n - 1) + 1;
  return p + ((4 - p) & 7);
}

// In-place radix-2 decimation in time on G lines of length n (input in
// bit-reversed order, output natural), three stages per pass: each thread
// loads 8 values spaced by the first stage's half size, applies the stages in
// registers and writes them back.  tw has n entries e^{-2 pi i k/n}.
__device__ void dit(double2 *a, int G, int n, int logn, const double2 *tw, bool inv) {
  const int t = threadIdx.x, nt = blockDim.x, ld = padded(n);
  for (int s0 = 0; s0 < logn; s0 += 3) {
    const int ns = min(3, logn - s0), R = 1 << ns, h = 1 << s0, per = n >> ns;
    for (int g = t; g < G * per; g += nt) {
      const int line = g / per, gg = g - line * per;
      const int k = gg & (h - 1), blk = gg >> s0;
      const int base = blk * R * h + k;
      double2 *L = a + (size_t)line * ld;
      double2 x[8];
#pragma unroll
      for (int m = 0; m < 8; ++m)
        if (m < R) x[m] = L[pd(base + m * h)];
#pragma unroll
      for (int st = 0; st < 3; ++st) {
        if (st >= ns) break;
        const int hh = 1 << st, sh = logn - (s0 + st + 1);
#pragma unroll
        for (int m = 0; m < 8; ++m) {
          if (m >= R || (m & (2 * hh - 1)) >= hh) continue;
          const int off = k + (m & (hh - 1)) * h;
          const double2 y = cmul(twid(tw, off << sh, inv), x[m + hh]);
          x[m + hh] = make_double2(x[m].x - y.x, x[m].y - y.y);
          x[m] = make_double2(x[m].x + y.x, x[m].y + y.y);
        }
      }
#pragma unroll
      for (int m = 0; m < 8; ++m)
        if (m < R) L[pd(base + m * h)] = x[m];
    }
    __syncthreads();
  }
}

// In-place radix-2 decimation in frequency (input natural, output
// bit-reversed), three stages per pass from the largest half size down.
__device__ void dif(double2 *a, int G, int n, int logn, const double2 *tw, bool inv) {
  const int t = threadIdx.x, nt = blockDim.x, ld = padded(n);
  for (int s_hi = logn; s_hi >= 1; s_hi -= 3) {
    const int ns = min(3, s_hi), s_lo = s_hi - ns + 1;
    const int R = 1 << ns, h = 1 << (s_lo - 1), per = n >> ns;
    for (int g = t; g < G * per; g += nt) {
      const int line = g / per, gg = g - line * per;
      const int k = gg & (h - 1), blk = gg >> (s_lo - 1);
      const int base = blk * R * h + k;
      double2 *L = a + (size_t)line * ld;
      double2 x[8];
#pragma unroll
      for (int m = 0; m < 8; ++m)
        if (m < R) x[m] = L[pd(base + m * h)];
#pragma unroll
      for (int st = 2; st >= 0; --st) {
        if (st >= ns) continue;
        const int hh = 1 << st, sh = logn - (s_lo + st);
#pragma unroll
        for (int m = 0; m < 8; ++m) {
          if (m >= R || (m & (2 * hh - 1)) >= hh) continue;
          const int off = k + (m & (hh - 1)) * h;
          const double2 x0 = x[m], x1 = x[m + hh];
          x[m] = make_double2(x0.x + x1.x, x0.y + x1.y);
          x[m + hh] = cmul(make_double2(x0.x - x1.x, x0.y - x1.y), twid(tw, off << sh, inv));
        }
      }
#pragma unroll
      for (int m = 0; m < 8; ++m)
        if (m < R) L[pd(base + m * h)] = x[m];
    }
    __syncthreads();
  }
}

// Plain DFT of G lines from a into b (natural order, padded layout), any n.
__device__ void dft(const double2 *a, double2 *b, int G, int n, const double2 *tw, bool inv) {
  const int ld = padded(n);
  for (int o = threadIdx.x; o < G * n; o += blockDim.x) {
    const int line = o / n, k = o - line * n;
    const double2 *L = a + (size_t)line * ld;
    double2 s = make_double2(0.0, 0.0);
    int idx = 0;
    for (int m = 0; m < n; ++m) {
      const double2 p = cmul(L[pd(m)], twid(tw, idx, inv));
      s.x += p.x;
      s.y += p.y;
      idx += k;
      if (idx >= n) idx -= n;
    }
    b[(size_t)line * ld + pd(k)] = s;
  }
  __syncthreads();
}

// Pass 1: rows j0=2*blockIdx.x, j1=j0+1 -> half spectra.
__global__ void __launch_bounds__(kThreads) k_rows_r2c(int Nx, int Ny, int logx, const double2 *__restrict__ tw,
                                                       const double *__restrict__ f, double2 *__restrict__ spec) {
  extern __shared__ double2 sm[];
  const int j0 = 2 * blockIdx.x, j1 = j0 + 1;
  const bool has1 = j1 < Ny;
  const int H = Nx / 2 + 1;
  for (int k = threadIdx.x; k < Nx; k += blockDim.x) {
    const double a = f[(size_t)j0 * Nx + k];
    const double b = has1 ? f[(size_t)j1 * Nx + k] : 0.0;
    sm[pd(logx >= 0 ? brev(k, logx) : k)] = make_double2(a, b);
  }
  __syncthreads();
  const double2 *Z = sm;
  if (logx >= 0) {
    dit(sm, 1, Nx, logx, tw, false);
  } else {
    dft(sm, sm + padded(Nx), 1, Nx, tw, false);
    Z = sm + padded(Nx);
  }
  for (int I = threadIdx.x; I < H; I += blockDim.x) {
    const double2 z = Z[pd(I)], m = Z[pd((Nx - I) % Nx)];
    spec[(size_t)j0 * H + I] = make_double2(0.5 * (z.x + m.x), 0.5 * (z.y - m.y));
    if (has1) spec[(size_t)j1 * H + I] = make_double2(0.5 * (z.y + m.y), 0.5 * (m.x - z.x));
  }
}

// Pass 2: G consecutive spectrum columns per block.
__global__ void __launch_bounds__(kThreads) k_cols(int Nx, int Ny, int logy, int G, const double2 *__restrict__ tw,
                                                   const double *__restrict__ ax, const double *__restrict__ ay,
                                                   double dxdy, double2 *__restrict__ spec,
                                                   unsigned long long *__restrict__ maxbits) {
  extern __shared__ double2 sm[];
  __shared__ double wmax[kThreads / 32];
  const int H = Nx / 2 + 1;
  const int c0 = blockIdx.x * G;
  const int g_here = min(G, H - c0);
  // power-of-two columns: forward decimation in frequency (natural order in,
  // bit-reversed out), scaling in bit-reversed order, inverse decimation in
  // time (bit-reversed in, natural out) -- no permutation pass is needed
  const int ldy = padded(Ny);
  for (int o = threadIdx.x; o < g_here * Ny; o += blockDim.x) {
    const int j = o / g_here, g = o - j * g_here;
    sm[(size_t)g * ldy + pd(j)] = spec[(size_t)j * H + c0 + g];
  }
  __syncthreads();
  double2 *A = sm;
  if (logy >= 0) {
    dif(sm, g_here, Ny, logy, tw, false);
  } else {
    dft(sm, sm + (size_t)G * ldy, g_here, Ny, tw, false);
    A = sm + (size_t)G * ldy;
  }
  double lmax = 0.0;
  for (int o = threadIdx.x; o < g_here * Ny; o += blockDim.x) {
    const int g = o / Ny, pos = o - g * Ny;
    const int J = logy >= 0 ? brev(pos, logy) : pos;
    const int I = c0 + g;
    double2 *slot = A + (size_t)g * ldy + pd(pos);
    const double2 F = *slot;
    lmax = fmax(lmax, sqrt(F.x * F.x + F.y * F.y));
    const double lam = (I == 0 && J == 0) ? 1.0 : (dxdy * 4.0) * (__ldg(ax + I) + __ldg(ay + J));
    const double r = -1.0 / lam;
    *slot = make_double2(F.x * r, F.y * r);
  }
  __syncthreads();
  double2 *Bout = A;
  if (logy >= 0) {
    dit(A, g_here, Ny, logy, tw, true);
  } else {
    dft(A, sm, g_here, Ny, tw, true);
    Bout = sm;
  }
  const double sc = 1.0 / Ny;
  for (int o = threadIdx.x; o < g_here * Ny; o += blockDim.x) {
    const int j = o / g_here, g = o - j * g_here;
    const double2 v = Bout[(size_t)g * ldy + pd(j)];
    spec[(size_t)j * H + c0 + g] = make_double2(v.x * sc, v.y * sc);
  }
  for (int off = 16; off > 0; off >>= 1) lmax = fmax(lmax, __shfl_down_sync(0xffffffffu, lmax, off));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = lmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = wmax[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, wmax[w]);
    atomicMax(maxbits, (unsigned long long)__double_as_longlong(m));  // m >= 0: bit order = value order
  }
}

// Pass 3: half spectra of rows j0, j1 -> real rows (scaled 1/Nx).
__global__ void __launch_bounds__(kThreads) k_rows_c2r(int Nx, int Ny, int logx, const double2 *__restrict__ tw,
                                                       const double2 *__restrict__ spec, double *__restrict__ out,
                                                       int accumulate, const unsigned long long *__restrict__ maxbits) {
  extern __shared__ double2 sm[];
  const int j0 = 2 * blockIdx.x, j1 = j0 + 1;
  const bool has1 = j1 < Ny;
  const int H = Nx / 2 + 1;
  const double mx = __longlong_as_double((long long)*maxbits);
  if (mx < 1e-14) {  // pressure_poisson.m:21-32: dp stays zero
    if (!accumulate)
      for (int k = threadIdx.x; k < Nx; k += blockDim.x) {
        out[(size_t)j0 * Nx + k] = 0.0;
        if (has1) out[(size_t)j1 * Nx + k] = 0.0;
      }
    return;
  }
  for (int k = threadIdx.x; k < Nx; k += blockDim.x) {
    double2 g0, g1;
    if (k < H) {
      g0 = spec[(size_t)j0 * H + k];
      g1 = has1 ? spec[(size_t)j1 * H + k] : make_double2(0.0, 0.0);
    } else {
      const double2 a = spec[(size_t)j0 * H + (Nx - k)];
      const double2 b = has1 ? spec[(size_t)j1 * H + (Nx - k)] : make_double2(0.0, 0.0);
      g0 = make_double2(a.x, -a.y);
      g1 = make_double2(b.x, -b.y);
    }
    sm[pd(logx >= 0 ? brev(k, logx) : k)] = make_double2(g0.x - g1.y, g0.y + g1.x);
  }
  __syncthreads();
  const double2 *W = sm;
  if (logx >= 0) {
    dit(sm, 1, Nx, logx, tw, true);
  } else {
    dft(sm, sm + padded(Nx), 1, Nx, tw, true);
    W = sm + padded(Nx);
  }
  const double sc = 1.0 / Nx;
  for (int k = threadIdx.x; k < Nx; k += blockDim.x) {
    const double2 w = W[pd(k)];
    if (accumulate) {
      out[(size_t)j0 * Nx + k] += w.x * sc;
      if (has1) out[(size_t)j1 * Nx + k] += w.y * sc;
    } else {
      out[(size_t)j0 * Nx + k] = w.x * sc;
      if (has1) out[(size_t)j1 * Nx + k] = w.y * sc;
    }
  }
}


// ---------------------------------------------------------------------------
// Register groups of up to three radix-2 stages on 8 values x[m] at positions
// base + m*h (h = half size of the smallest stage of the group, k = base mod h).
// The stage with half size hh*h multiplies by W_{2 hh h}^(k + j h), j < hh,
// = W_{2 hh h}^k * W_{2 hh}^j: the first factor is a power of the group's top
// twiddle W_{R h}^k (R = 2^ns values; read once from the pyramid table, whose
// level of length Lt holds W_Lt^k, k < Lt/2, at Lt/2 + k, so lanes with
// consecutive k read consecutive entries), the second one of the eighth roots
// of unity, applied as adds and one scaling.

// a * W_{2 hh}^j (conjugate root when inv), j < hh <= 4
__device__ __forceinline__ double2 rot(double2 a, int hh, int j, bool inv) {
  constexpr double r = 0.70710678118654752440;  // 1/sqrt(2)
  if (j == 0) return a;
  if (2 * j == hh) return inv ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);  // +i / -i
  if (j == 1)  // (1 + i)/sqrt(2) / (1 - i)/sqrt(2)
    return inv ? make_double2((a.x - a.y) * r, (a.x + a.y) * r) : make_double2((a.x + a.y) * r, (a.y - a.x) * r);
  // j == 3: (-1 + i)/sqrt(2) / (-1 - i)/sqrt(2)
  return inv ? make_double2(-(a.x + a.y) * r, (a.x - a.y) * r) : make_double2((a.y - a.x) * r, -(a.x + a.y) * r);
}
__device__ __forceinline__ double2 csq(double2 a) { return make_double2(a.x * a.x - a.y * a.y, 2.0 * a.x * a.y); }

// base twiddles W_{2^(st+1) h}^k of the group's stages st = 0, 1, 2
__device__ __forceinline__ void group_twiddles(int ns, int k, int h, const double2 *pyr, bool inv, double2 &w0,
                                               double2 &w1, double2 &w2) {
  double2 wt = __ldg(pyr + (((1 << ns) * h) >> 1) + k);
  if (inv) wt.y = -wt.y;
  if (ns == 3) {
    w2 = wt;
    w1 = csq(w2);
    w0 = csq(w1);
  } else if (ns == 2) {
    w1 = w2 = wt;
    w0 = csq(w1);
  } else {
    w0 = w1 = w2 = wt;
  }
}

// UNIT: k = 0, h = 1 (all twiddles are roots of unity of order <= 8)
template <bool UNIT>
__device__ __forceinline__ void group_dif(double2 (&x)[8], int ns, int k, int h, const double2 *pyr, bool inv) {
  double2 w0 = make_double2(1.0, 0.0), w1 = w0, w2 = w0;
  if (!UNIT) group_twiddles(ns, k, h, pyr, inv, w0, w1, w2);
#pragma unroll
  for (int st = 2; st >= 0; --st) {
    if (st >= ns) continue;
    const int hh = 1 << st;
    double2 tw[4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (j < hh) tw[j] = rot(st == 2 ? w2 : (st == 1 ? w1 : w0), hh, j, inv);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      if ((m & (2 * hh - 1)) >= hh || m + hh >= (1 << ns)) continue;
      const double2 x0 = x[m], x1 = x[m + hh];
      const double2 d = make_double2(x0.x - x1.x, x0.y - x1.y);
      x[m] = make_double2(x0.x + x1.x, x0.y + x1.y);
      x[m + hh] = UNIT ? rot(d, hh, m & (hh - 1), inv) : cmul(d, tw[m & (hh - 1)]);
    }
  }
}
template <bool UNIT>
__device__ __forceinline__ void group_dit(double2 (&x)[8], int ns, int k, int h, const double2 *pyr, bool inv) {
  double2 w0 = make_double2(1.0, 0.0), w1 = w0, w2 = w0;
  if (!UNIT) group_twiddles(ns, k, h, pyr, inv, w0, w1, w2);
#pragma unroll
  for (int st = 0; st < 3; ++st) {
    if (st >= ns) break;
    const int hh = 1 << st;
    double2 tw[4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (j < hh) tw[j] = rot(st == 2 ? w2 : (st == 1 ? w1 : w0), hh, j, inv);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      if ((m & (2 * hh - 1)) >= hh || m + hh >= (1 << ns)) continue;
      const double2 y = UNIT ? rot(x[m + hh], hh, m & (hh - 1), inv) : cmul(tw[m & (hh - 1)], x[m + hh]);
      x[m + hh] = make_double2(x[m].x - y.x, x[m].y - y.y);
      x[m] = make_double2(x[m].x + y.x, x[m].y + y.y);
    }
  }
}

// Groups of NS <= 4 radix-2 stages on 16 values (the column pass's outer
// passes, INS2D_FFT_COLS_R16): as group_dif / group_dit with NS a
// compile-time count; the top stage of a four-stage group multiplies by
// sixteenth roots of unity.

// a * W_16^j (conjugate root when inv), j < 8; W_16^j = cos(pi j/8) - i sin(pi j/8)
__device__ __forceinline__ double2 rot16(double2 a, int j, bool inv) {
  if ((j & 1) == 0) return rot(a, 4, j >> 1, inv);  // W_16^(2i) = W_8^i
  constexpr double c = 0.92387953251128675613, s = 0.38268343236508977173;  // cos(pi/8), sin(pi/8)
  double wr, wi;
  if (j == 1) {
    wr = c;
    wi = -s;
  } else if (j == 3) {
    wr = s;
    wi = -c;
  } else if (j == 5) {
    wr = -s;
    wi = -c;
  } else {
    wr = -c;
    wi = -s;
  }
  if (inv) wi = -wi;
  return make_double2(a.x * wr - a.y * wi, a.x * wi + a.y * wr);
}
// w times W_{2 hh}^j, hh <= 8
__device__ __forceinline__ double2 rot_any(double2 w, int hh, int j, bool inv) {
  return hh == 8 ? rot16(w, j, inv) : rot(w, hh, j, inv);
}
// base twiddles W_{2^(st+1) h}^k of stages st < NS from the top one W_{2^NS h}^k
template <int NS>
__device__ __forceinline__ void group_twiddles16(int k, int h, const double2 *pyr, bool inv, double2 (&w)[4]) {
  double2 wt = __ldg(pyr + (((1 << NS) * h) >> 1) + k);
  if (inv) wt.y = -wt.y;
  w[NS - 1] = wt;
#pragma unroll
  for (int st = NS - 2; st >= 0; --st) w[st] = csq(w[st + 1]);
}
template <bool UNIT, int NS>
__device__ __forceinline__ void group_dif16(double2 (&x)[16], int k, int h, const double2 *pyr, bool inv) {
  double2 w[4];
  if constexpr (!UNIT) group_twiddles16<NS>(k, h, pyr, inv, w);
#pragma unroll
  for (int st = NS - 1; st >= 0; --st) {
    const int hh = 1 << st;
    double2 tw[8];
    if constexpr (!UNIT) {
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (j < hh) tw[j] = rot_any(w[st], hh, j, inv);
    }
#pragma unroll
    for (int m = 0; m < (1 << NS); ++m) {
      if ((m & (2 * hh - 1)) >= hh) continue;
      const double2 x0 = x[m], x1 = x[m + hh];
      const double2 d = make_double2(x0.x - x1.x, x0.y - x1.y);
      x[m] = make_double2(x0.x + x1.x, x0.y + x1.y);
      x[m + hh] = UNIT ? rot_any(d, hh, m & (hh - 1), inv) : cmul(d, tw[m & (hh - 1)]);
    }
  }
}
template <bool UNIT, int NS>
__device__ __forceinline__ void group_dit16(double2 (&x)[16], int k, int h, const double2 *pyr, bool inv) {
  double2 w[4];
  if constexpr (!UNIT) group_twiddles16<NS>(k, h, pyr, inv, w);
#pragma unroll
  for (int st = 0; st < NS; ++st) {
    const int hh = 1 << st;
    double2 tw[8];
    if constexpr (!UNIT) {
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (j < hh) tw[j] = rot_any(w[st], hh, j, inv);
    }
#pragma unroll
    for (int m = 0; m < (1 << NS); ++m) {
      if ((m & (2 * hh - 1)) >= hh) continue;
      const double2 y = UNIT ? rot_any(x[m + hh], hh, m & (hh - 1), inv) : cmul(tw[m & (hh - 1)], x[m + hh]);
      x[m + hh] = make_double2(x[m].x - y.x, x[m].y - y.y);
      x[m] = make_double2(x[m].x + y.x, x[m].y + y.y);
    }
  }
}

// --- power-of-two lengths 2^L, 6 <= L <= 13: every shape a compile-time
// constant; the first and last radix-8 passes fused with the global loads and
// stores, no permutation passes; tw is the table of fft_twiddle_table (the
// pyramid at tw + 2^L) ---------------------------------------------------------

// Slot of complex value i in a line of length 2^L: the general layout above,
// or for L >= 9 the cheaper i + i/8 + i/2^(L-3), conflict-free for the same
// accesses at those lengths (the last term spreads the bit-reversed readouts,
// whose eight lanes lie 2^(L-3) apart).
template <int L>
__host__ __device__ constexpr int pdl(int i) {
  return L >= 9 ? i + (i >> 3) + (i >> (L - 3)) : i + (i >> 3) + (i >> 6) + (i >> 9) + (i >> 12);
}
template <int L>
__host__ __device__ constexpr int paddedl() {
  return (pdl<L>((1 << L) - 1) + 1) + ((4 - (pdl<L>((1 << L) - 1) + 1)) & 7);
}
// spectrum columns per column block: two 2048-point columns (32-byte row
// segments) in the shared-memory budget, more for short columns
template <int L>
constexpr int cols_per_block() {
  constexpr int per = paddedl<L>() * 16;
  constexpr int g = (INS2D_FFT_COLS_BUDGET * 1024) / per;
  constexpr int g8 = g > 8 ? 8 : (g < 1 ? 1 : g);
  return (L >= 10 && g8 > INS2D_FFT_COLS_G) ? INS2D_FFT_COLS_G : g8;
}

// The column scaling's y factors ay staged in shared memory (INS2D_FFT_COLS_SAY,
// lengths up to 4096): each block copies ay once, coalesced, to slots
// i + i/8 after its columns, and reads them at the bit-reversed J of its
// values (32 lanes 2^(L-8) apart: two-way bank conflicts with the padding,
// against one sector per lane for the same reads from global memory).
#ifndef INS2D_FFT_COLS_SAY
#define INS2D_FFT_COLS_SAY 1
#endif
template <int L>
__host__ __device__ constexpr bool cols_say() {
  return INS2D_FFT_COLS_SAY && L <= 12;
}
// dynamic shared memory of a column block
template <int L, int G>
constexpr size_t cols_smem() {
  return (size_t)G * paddedl<L>() * sizeof(double2) +
         (cols_say<L>() ? (size_t)((1 << L) + ((1 << L) >> 3)) * sizeof(double) : 0);
}

// DIF passes over stages S_HI down to S_BOT (three per pass) on the first
// `lines` of G lines of stride ld
template <int L, int S_HI, int S_BOT, int G>
__device__ __forceinline__ void dif_passes(double2 *a, int ld, int lines, const double2 *pyr, bool inv) {
  if constexpr (S_HI >= S_BOT) {
    constexpr int NS = (S_HI - S_BOT + 1) < 3 ? (S_HI - S_BOT + 1) : 3;
    constexpr int S_LO = S_HI - NS + 1, R = 1 << NS, H = 1 << (S_LO - 1), PER = (1 << L) >> NS;
    const unsigned lim = (G > 1 ? lines : 1) * PER;
    for (unsigned g = threadIdx.x; g < lim; g += kThreads) {
      const int line = (int)(g / PER), gg = (int)(g % PER);
      const int k = gg & (H - 1), blk = gg >> (S_LO - 1);
      const int base = blk * R * H + k;
      double2 *Lp = a + line * ld;
      double2 x[8];
#pragma unroll
      for (int m = 0; m < R; ++m) x[m] = Lp[pdl<L>(base + m * H)];
      group_dif<false>(x, NS, k, H, pyr, inv);
#pragma unroll
      for (int m = 0; m < R; ++m) Lp[pdl<L>(base + m * H)] = x[m];
    }
    __syncthreads();
    dif_passes<L, S_HI - 3, S_BOT, G>(a, ld, lines, pyr, inv);
  }
}
// DIT passes over stages S0 + 1 up to S_TOP (three per pass)
template <int L, int S0, int S_TOP, int G>
__device__ __forceinline__ void dit_passes(double2 *a, int ld, int lines, const double2 *pyr, bool inv) {
  if constexpr (S0 < S_TOP) {
    constexpr int NS = (S_TOP - S0) < 3 ? (S_TOP - S0) : 3;
    constexpr int R = 1 << NS, H = 1 << S0, PER = (1 << L) >> NS;
    const unsigned lim = (G > 1 ? lines : 1) * PER;
    for (unsigned g = threadIdx.x; g < lim; g += kThreads) {
      const int line = (int)(g / PER), gg = (int)(g % PER);
      const int k = gg & (H - 1), blk = gg >> S0;
      const int base = blk * R * H + k;
      double2 *Lp = a + line * ld;
      double2 x[8];
#pragma unroll
      for (int m = 0; m < R; ++m) x[m] = Lp[pdl<L>(base + m * H)];
      group_dit<false>(x, NS, k, H, pyr, inv);
#pragma unroll
      for (int m = 0; m < R; ++m) Lp[pdl<L>(base + m * H)] = x[m];
    }
    __syncthreads();
    dit_passes<L, S0 + 3, S_TOP, G>(a, ld, lines, pyr, inv);
  }
}

// the same with up to four stages per pass (the column pass's outer passes
// with INS2D_FFT_COLS_R16; every pass's smallest half size H >= 8)
template <int L, int S_HI, int S_BOT, int G>
__device__ __forceinline__ void dif16_passes(double2 *a, int ld, int lines, const double2 *pyr, bool inv) {
  if constexpr (S_HI >= S_BOT) {
    constexpr int NS = (S_HI - S_BOT + 1) < 4 ? (S_HI - S_BOT + 1) : 4;
    constexpr int S_LO = S_HI - NS + 1, R = 1 << NS, H = 1 << (S_LO - 1), PER = (1 << L) >> NS;
    const unsigned lim = (G > 1 ? lines : 1) * PER;
    for (unsigned g = threadIdx.x; g < lim; g += kThreads) {
      const int line = (int)(g / PER), gg = (int)(g % PER);
      const int k = gg & (H - 1), blk = gg >> (S_LO - 1);
      const int base = blk * R * H + k;
      double2 *Lp = a + line * ld;
      double2 x[16];
#pragma unroll
      for (int m = 0; m < R; ++m) x[m] = Lp[pdl<L>(base + m * H)];
      group_dif16<false, NS>(x, k, H, pyr, inv);
#pragma unroll
      for (int m = 0; m < R; ++m) Lp[pdl<L>(base + m * H)] = x[m];
    }
    __syncthreads();
    dif16_passes<L, S_HI - NS, S_BOT, G>(a, ld, lines, pyr, inv);
  }
}
template <int L, int S0, int S_TOP, int G>
__device__ __forceinline__ void dit16_passes(double2 *a, int ld, int lines, const double2 *pyr, bool inv) {
  if constexpr (S0 < S_TOP) {
    constexpr int NS = (S_TOP - S0) < 4 ? (S_TOP - S0) : 4;
    constexpr int R = 1 << NS, H = 1 << S0, PER = (1 << L) >> NS;
    const unsigned lim = (G > 1 ? lines : 1) * PER;
    for (unsigned g = threadIdx.x; g < lim; g += kThreads) {
      const int line = (int)(g / PER), gg = (int)(g % PER);
      const int k = gg & (H - 1), blk = gg >> S0;
      const int base = blk * R * H + k;
      double2 *Lp = a + line * ld;
      double2 x[16];
#pragma unroll
      for (int m = 0; m < R; ++m) x[m] = Lp[pdl<L>(base + m * H)];
      group_dit16<false, NS>(x, k, H, pyr, inv);
#pragma unroll
      for (int m = 0; m < R; ++m) Lp[pdl<L>(base + m * H)] = x[m];
    }
    __syncthreads();
    dit16_passes<L, S0 + NS, S_TOP, G>(a, ld, lines, pyr, inv);
  }
}

// rows j0, j1 -> half spectra (forward DIF; bit-reversed result read back
// during the Hermitian split)
// DIV: the rows are not read from f but computed on the fly as the
// divergence (M W + alpha yM + beta ydM) * gamma of the velocity-sized W
// (time_ERK.m:117, pressure_additional_solve.m:11-13), fusing that kernel in.
// fastdiv: every cell is a regular two-point row of Mx and My (the periodic
// grids this solver takes): the row weights of j0, j1 and the three v rows
// they share are set up once, the column weights once per column.
// SRC 0: the rows of f; 1: the divergence of W = f; 2: the divergence of
// W = ws.Vn ws.sv + ws.sa ws.T (FP32-storage stages)
template <int L, int SRC>
__global__ void __launch_bounds__(kThreads, INS2D_FFT_ROWS_MINB)
    k_rows_r2c_t(int Ny, const double2 *__restrict__ tw, const double *__restrict__ f, const WSplit ws,
                 double2 *__restrict__ spec, const __grid_constant__ DevOps P, double alpha, double beta,
                 double gamma, int fastdiv, const int *__restrict__ skip, unsigned long long *__restrict__ zero_max) {
  constexpr int N = 1 << L, PER = N >> 3, H = N / 2 + 1;
  constexpr bool DIV = SRC != 0;
  pdl_wait();
  pdl_trigger();
  if (zero_max && blockIdx.x == 0 && threadIdx.x == 0) *zero_max = 0ull;  // the column pass's max |fhat|
  if (skip && *(volatile const int *)skip) return;  // preconditioner of a converged CG: nothing to do
  extern __shared__ double2 sm[];
  const double2 *pyr = tw + N;
  const int j0 = 2 * blockIdx.x, j1 = j0 + 1;
  const bool has1 = j1 < Ny;
  auto W = [&](long long k) -> double {
    if constexpr (SRC == 2)
      return ws(k);
    else
      return __ldg(f + k);
  };
  if (DIV && fastdiv) {
    const double hy0 = __ldg(P.hy + j0), hy1 = has1 ? __ldg(P.hy + j1) : 0.0;
    const double m00 = __ldg(P.rMY.w0 + j0), m01 = __ldg(P.rMY.w1 + j0);
    const double m10 = has1 ? __ldg(P.rMY.w0 + j1) : 0.0, m11 = has1 ? __ldg(P.rMY.w1 + j1) : 0.0;
    const int r0 = wrapn(j0 + P.rMY.s, P.rMY.n), r1 = wrapn(r0 + 1, P.rMY.n), r2 = wrapn(r1 + 1, P.rMY.n);
    const long long ua = (long long)j0 * P.Nux, ub = (long long)(has1 ? j1 : j0) * P.Nux;
    const long long va = P.Nu + (long long)r0 * P.Nvx, vb = P.Nu + (long long)r1 * P.Nvx,
                    vc = P.Nu + (long long)r2 * P.Nvx;
    for (int k = threadIdx.x; k < PER; k += kThreads) {
      double2 x[8];
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const int i = k + m * PER;
        const double w0 = __ldg(P.rMX.w0 + i), w1 = __ldg(P.rMX.w1 + i), hx = __ldg(P.hx + i);
        const int c0 = wrapn(i + P.rMX.s, P.rMX.n), c1 = wrapn(c0 + 1, P.rMX.n);
        const double vb_i = W(vb + i);
        const double d0 = hy0 * (w0 * W(ua + c0) + w1 * W(ua + c1)) + hx * (m00 * W(va + i) + m01 * vb_i);
        const double d1 = hy1 * (w0 * W(ub + c0) + w1 * W(ub + c1)) + hx * (m10 * vb_i + m11 * W(vc + i));
        x[m] = make_double2(d0 * gamma, has1 ? d1 * gamma : 0.0);
      }
      group_dif<false>(x, 3, k, PER, pyr, false);
#pragma unroll
      for (int m = 0; m < 8; ++m) sm[pdl<L>(k + m * PER)] = x[m];
    }
  } else {
    const double *r0 = f + (size_t)j0 * N, *r1 = f + (size_t)j1 * N;
    for (int k = threadIdx.x; k < PER; k += kThreads) {
      double2 x[8];
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        if constexpr (SRC == 2)
          x[m] = make_double2(div_cell_f(P, ws, alpha, beta, gamma, k + m * PER, j0),
                              has1 ? div_cell_f(P, ws, alpha, beta, gamma, k + m * PER, j1) : 0.0);
        else if constexpr (SRC == 1)
          x[m] = make_double2(div_cell(P, f, alpha, beta, gamma, k + m * PER, j0),
                              has1 ? div_cell(P, f, alpha, beta, gamma, k + m * PER, j1) : 0.0);
        else
          x[m] = make_double2(__ldg(r0 + k + m * PER), has1 ? __ldg(r1 + k + m * PER) : 0.0);
      }
      group_dif<false>(x, 3, k, PER, pyr, false);
#pragma unroll
      for (int m = 0; m < 8; ++m) sm[pdl<L>(k + m * PER)] = x[m];
    }
  }
  __syncthreads();
  dif_passes<L, L - 3, 1, 1>(sm, 0, 1, pyr, false);
  for (int I = threadIdx.x; I < H; I += kThreads) {
    const double2 z = sm[pdl<L>(brev(I, L))], m = sm[pdl<L>(brev((N - I) & (N - 1), L))];
    spec[(size_t)j0 * H + I] = make_double2(0.5 * (z.x + m.x), 0.5 * (z.y - m.y));
    if (has1) spec[(size_t)j1 * H + I] = make_double2(0.5 * (z.y + m.y), 0.5 * (m.x - z.x));
  }
}

// G spectrum columns of length 2^L: forward DIF, -1/Ahat scaling fused with
// the last DIF and first DIT passes, inverse DIT; max |fhat| reduction
// The columns are the first ncols of a spectrum with row stride H (complex
// values); column c holds wave number I0 + c (I0 > 0 for a slab's column range).
// RX: 8, or 16 for outer passes of four stages (the global load and store
// and the shared-memory passes beside them; fewer shared-memory round trips,
// L >= 9).
template <int L, int G, int RX = 8>
__global__ void __launch_bounds__(kThreads, RX == 16 ? 2 : INS2D_FFT_COLS_MINB)
    k_cols_t(int H, int ncols, int I0, const double2 *__restrict__ tw, const double *__restrict__ ax,
             const double *__restrict__ ay, double dxdy, double2 *__restrict__ spec,
             unsigned long long *__restrict__ maxbits, const int *__restrict__ skip) {
  constexpr int N = 1 << L, PER = N >> 3, LD = paddedl<L>();
  pdl_wait();
  pdl_trigger();
  if (skip && *(volatile const int *)skip) return;
  extern __shared__ double2 sm[];
  __shared__ double wmax[kThreads / 32];
  const double2 *pyr = tw + N;
  const int c0 = blockIdx.x * G;
  const int g_here = min(G, ncols - c0);
  static_assert(RX == 8 || (RX == 16 && L >= 9), "radix-16 outer passes need L >= 9");
  double *say = reinterpret_cast<double *>(sm + G * LD);
  if constexpr (cols_say<L>()) {
    for (int i = threadIdx.x; i < N; i += kThreads) say[i + (i >> 3)] = __ldg(ay + i);
  }  // read after the __syncthreads that ends the first pass
  if constexpr (RX == 16) {
    constexpr int P16 = N >> 4;
    for (unsigned gidx = threadIdx.x; gidx < G * P16; gidx += kThreads) {
      const int k = (int)(gidx / G), line = (int)(gidx % G);
      if (line >= g_here) continue;
      double2 x[16];
#pragma unroll
      for (int m = 0; m < 16; ++m) x[m] = spec[(size_t)(k + m * P16) * H + c0 + line];
      group_dif16<false, 4>(x, k, P16, pyr, false);
#pragma unroll
      for (int m = 0; m < 16; ++m) sm[line * LD + pdl<L>(k + m * P16)] = x[m];
    }
    __syncthreads();
    dif16_passes<L, L - 4, 4, G>(sm, LD, g_here, pyr, false);
  } else {
    for (unsigned gidx = threadIdx.x; gidx < G * PER; gidx += kThreads) {
      const int k = (int)(gidx / G), line = (int)(gidx % G);
      if (line >= g_here) continue;
      double2 x[8];
#pragma unroll
      for (int m = 0; m < 8; ++m) x[m] = spec[(size_t)(k + m * PER) * H + c0 + line];
      group_dif<false>(x, 3, k, PER, pyr, false);
#pragma unroll
      for (int m = 0; m < 8; ++m) sm[line * LD + pdl<L>(k + m * PER)] = x[m];
    }
    __syncthreads();
    dif_passes<L, L - 3, 4, G>(sm, LD, g_here, pyr, false);
  }
  double lmax = 0.0;
  for (unsigned gidx = threadIdx.x; gidx < g_here * PER; gidx += kThreads) {
    const int line = (int)(gidx / PER), k = (int)(gidx % PER);
    double2 *Ls = sm + line * LD;
    const int I = I0 + c0 + line;
    double2 x[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) x[m] = Ls[pdl<L>(8 * k + m)];
    group_dif<true>(x, 3, 0, 1, pyr, false);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int J = brev(8 * k + m, L);
      const double2 F = x[m];
      lmax = fmax(lmax, F.x * F.x + F.y * F.y);  // squared; one square root per block
      double ayJ;
      if constexpr (cols_say<L>())
        ayJ = say[J + (J >> 3)];
      else
        ayJ = __ldg(ay + J);
      const double lam = (I == 0 && J == 0) ? 1.0 : (dxdy * 4.0) * (__ldg(ax + I) + ayJ);
      // the correctly rounded reciprocal: the same value as -1.0 / lam
      const double r = INS2D_FFT_COLS_SAY ? -__drcp_rn(lam) : -1.0 / lam;
      x[m] = make_double2(F.x * r, F.y * r);
    }
    group_dit<true>(x, 3, 0, 1, pyr, true);
#pragma unroll
    for (int m = 0; m < 8; ++m) Ls[pdl<L>(8 * k + m)] = x[m];
  }
  __syncthreads();
  const double sc = 1.0 / N;
  if constexpr (RX == 16) {
    constexpr int P16 = N >> 4;
    dit16_passes<L, 3, L - 4, G>(sm, LD, g_here, pyr, true);
    for (unsigned gidx = threadIdx.x; gidx < G * P16; gidx += kThreads) {
      const int k = (int)(gidx / G), line = (int)(gidx % G);
      if (line >= g_here) continue;
      double2 x[16];
#pragma unroll
      for (int m = 0; m < 16; ++m) x[m] = sm[line * LD + pdl<L>(k + m * P16)];
      group_dit16<false, 4>(x, k, P16, pyr, true);
#pragma unroll
      for (int m = 0; m < 16; ++m)
        spec[(size_t)(k + m * P16) * H + c0 + line] = make_double2(x[m].x * sc, x[m].y * sc);
    }
  } else {
    dit_passes<L, 3, L - 3, G>(sm, LD, g_here, pyr, true);
    for (unsigned gidx = threadIdx.x; gidx < G * PER; gidx += kThreads) {
      const int k = (int)(gidx / G), line = (int)(gidx % G);
      if (line >= g_here) continue;
      double2 x[8];
#pragma unroll
      for (int m = 0; m < 8; ++m) x[m] = sm[line * LD + pdl<L>(k + m * PER)];
      group_dit<false>(x, 3, k, PER, pyr, true);
#pragma unroll
      for (int m = 0; m < 8; ++m)
        spec[(size_t)(k + m * PER) * H + c0 + line] = make_double2(x[m].x * sc, x[m].y * sc);
    }
  }
  for (int off = 16; off > 0; off >>= 1) lmax = fmax(lmax, __shfl_down_sync(0xffffffffu, lmax, off));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = lmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = wmax[0];
    for (int w = 1; w < kThreads / 32; ++w) mm = fmax(mm, wmax[w]);
    atomicMax(maxbits, (unsigned long long)__double_as_longlong(sqrt(mm)));
  }
}

// half spectra of rows j0, j1 -> real rows (inverse DIF, bit-reversed result
// read back in natural order)
template <int L>
__global__ void __launch_bounds__(kThreads, INS2D_FFT_ROWS_MINB)
    k_rows_c2r_t(int Ny, const double2 *__restrict__ tw, const double2 *__restrict__ spec, double *__restrict__ out,
                 int accumulate, const unsigned long long *__restrict__ maxbits, const int *__restrict__ skip) {
  constexpr int N = 1 << L, PER = N >> 3, H = N / 2 + 1;
  pdl_wait();
  pdl_trigger();
  if (skip && *(volatile const int *)skip) return;
  extern __shared__ double2 sm[];
  const int j0 = 2 * blockIdx.x, j1 = j0 + 1;
  const bool has1 = j1 < Ny;
  const double mx = __longlong_as_double((long long)*maxbits);
  if (mx < 1e-14) {  // pressure_poisson.m:21-32: dp stays zero
    if (!accumulate)
      for (int k = threadIdx.x; k < N; k += kThreads) {
        out[(size_t)j0 * N + k] = 0.0;
        if (has1) out[(size_t)j1 * N + k] = 0.0;
      }
    return;
  }
  const double2 *pyr = tw + N;
  const double2 *s0 = spec + (size_t)j0 * H, *s1 = spec + (size_t)j1 * H;
  for (int k = threadIdx.x; k < PER; k += kThreads) {
    double2 x[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int q = k + m * PER;
      double2 g0, g1;
      if (q < H) {
        g0 = s0[q];
        g1 = has1 ? s1[q] : make_double2(0.0, 0.0);
      } else {
        const double2 a = s0[N - q];
        const double2 b = has1 ? s1[N - q] : make_double2(0.0, 0.0);
        g0 = make_double2(a.x, -a.y);
        g1 = make_double2(b.x, -b.y);
      }
      x[m] = make_double2(g0.x - g1.y, g0.y + g1.x);
    }
    group_dif<false>(x, 3, k, PER, pyr, true);
#pragma unroll
    for (int m = 0; m < 8; ++m) sm[pdl<L>(k + m * PER)] = x[m];
  }
  __syncthreads();
  dif_passes<L, L - 3, 1, 1>(sm, 0, 1, pyr, true);
  const double sc = 1.0 / N;
  for (int k = threadIdx.x; k < N; k += kThreads) {
    const double2 w = sm[pdl<L>(brev(k, L))];
    if (accumulate) {
      out[(size_t)j0 * N + k] += w.x * sc;
      if (has1) out[(size_t)j1 * N + k] += w.y * sc;
    } else {
      out[(size_t)j0 * N + k] = w.x * sc;
      if (has1) out[(size_t)j1 * N + k] = w.y * sc;
    }
  }
}

// calls f(std::integral_constant<int, L>) for the runtime l in [LO, 13]
template <int L, typename Fn>
bool with_log2(int l, Fn &&fn) {
  if constexpr (L > 13) {
    return false;
  } else {
    if (l == L) {
      fn(std::integral_constant<int, L>{});
      return true;
    }
    return with_log2<L + 1>(l, fn);
  }
}
constexpr int kFusedMinLog = 6;
// outer radix of the column pass for length 2^L
#ifndef INS2D_FFT_COLS_R16
#define INS2D_FFT_COLS_R16 1
#endif
template <int L>
constexpr int cols_radix() {
  return (INS2D_FFT_COLS_R16 && L >= 9) ? 16 : 8;
}

int ilog2_exact(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return ((1 << l) == n) ? l : -1;
}

int cols_group(int Ny, bool pow2) {
  // two columns (32-byte row segments) per block; more for short columns
  const size_t per = (size_t)padded(Ny) * sizeof(double2) * (pow2 ? 1 : 2);
  int G = (int)((INS2D_FFT_COLS_BUDGET * 1024) / per);
  if (G > 8) G = 8;
  if (G < 1) G = 1;
  if (Ny >= 1024 && G > INS2D_FFT_COLS_G) G = INS2D_FFT_COLS_G;
  return G;
}

}  // namespace

std::vector<double> fft_twiddle_table(int n) {
  std::vector<double> v(4 * (size_t)n, 0.0);
  for (int k = 0; k < n; ++k) {
    const double ang = 2.0 * M_PI * (double)k / (double)n;
    v[2 * k] = std::cos(ang);
    v[2 * k + 1] = -std::sin(ang);
  }
  if (ilog2_exact(n) >= 0)
    for (int Lt = 2; Lt <= n; Lt *= 2)
      for (int k = 0; k < Lt / 2; ++k) {
        const double ang = 2.0 * M_PI * (double)k / (double)Lt;
        v[2 * ((size_t)n + Lt / 2 + k)] = std::cos(ang);
        v[2 * ((size_t)n + Lt / 2 + k) + 1] = -std::sin(ang);
      }
  return v;
}

bool fft_supported(int Nx, int Ny) {
  auto ok = [](int n) { return n >= 2 && ((ilog2_exact(n) >= 0 && n <= kMaxPow2) || n <= kMaxGeneric); };
  return ok(Nx) && ok(Ny);
}

// Opt the transform kernels in to large dynamic shared memory on the current
// device (called once per context); returns the first failure.
cudaError_t fft_prepare() {
  cudaError_t first = cudaSuccess;
  auto opt_in = [&](const void *k) {
    const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (first == cudaSuccess) first = e;
  };
  for (int l = kFusedMinLog; l <= 13; ++l)
    with_log2<kFusedMinLog>(l, [&](auto c) {
      constexpr int L = decltype(c)::value;
      opt_in((const void *)k_rows_r2c_t<L, 0>);
      opt_in((const void *)k_rows_r2c_t<L, 1>);
      opt_in((const void *)k_rows_r2c_t<L, 2>);
      opt_in((const void *)k_cols_t<L, cols_per_block<L>(), cols_radix<L>()>);
      opt_in((const void *)k_rows_c2r_t<L>);
    });
  opt_in((const void *)k_rows_r2c);
  opt_in((const void *)k_cols);
  opt_in((const void *)k_rows_c2r);
  return first;
}

namespace {
// gate: the word the last pass reads for the early return (null: the
// spectrum's own max |fhat|)
cudaError_t fft_passes(const DevOps &P, const FftPlan &plan, const double *src, const WSplit *ws, bool div,
                       double alpha, double beta, double gamma, double *dp, bool accumulate, cudaStream_t s,
                       const unsigned long long *gate = nullptr, const int *skip = nullptr) {
  const int Nx = plan.Nx, Ny = plan.Ny;
  const int pairs = (Ny + 1) / 2;
  const int H = Nx / 2 + 1;
  unsigned long long *maxbits = (unsigned long long *)plan.maxabs;
  // the fused row pass zeroes max |fhat| itself (no memset node between the
  // passes, so the step's kernels chain by programmatic launch)
  if (!(plan.logx >= kFusedMinLog && plan.logx <= 13)) {
    const cudaError_t ms = cudaMemsetAsync(plan.maxabs, 0, sizeof(double), s);
    if (ms != cudaSuccess) return ms;
  }
  // rows, real -> half spectrum
  const int fastdiv = P.rMX.lo <= 0 && P.rMX.hi >= Nx && P.rMY.lo <= 0 && P.rMY.hi >= Ny && P.rMX.two && P.rMY.two;
  const bool fx = with_log2<kFusedMinLog>(plan.logx, [&](auto c) {
    constexpr int L = decltype(c)::value;
    const size_t sm = (size_t)paddedl<L>() * sizeof(double2);
    const WSplit w0{};
    const double *none = nullptr;
    if (ws)
      launch_k(k_rows_r2c_t<L, 2>, dim3(pairs), dim3(kThreads), sm, s, Ny, plan.twx, none, *ws, plan.spec, P, alpha,
               beta, gamma, fastdiv, skip, maxbits);
    else if (div)
      launch_k(k_rows_r2c_t<L, 1>, dim3(pairs), dim3(kThreads), sm, s, Ny, plan.twx, src, w0, plan.spec, P, alpha,
               beta, gamma, fastdiv, skip, maxbits);
    else
      launch_k(k_rows_r2c_t<L, 0>, dim3(pairs), dim3(kThreads), sm, s, Ny, plan.twx, src, w0, plan.spec, P, 0.0,
               0.0, 0.0, 0, skip, maxbits);
  });
  const size_t smx = (size_t)padded(Nx) * sizeof(double2) * (plan.logx >= 0 ? 1 : 2);
  if (!fx) k_rows_r2c<<<pairs, kThreads, smx, s>>>(Nx, Ny, plan.logx, plan.twx, src, plan.spec);
  // columns: forward, scaling, inverse
  const bool fy = with_log2<kFusedMinLog>(plan.logy, [&](auto c) {
    constexpr int L = decltype(c)::value, G = cols_per_block<L>();
    const size_t sm = cols_smem<L, G>();
    launch_k(k_cols_t<L, G, cols_radix<L>()>, dim3((H + G - 1) / G), dim3(kThreads), sm, s, H, H, 0, plan.twy,
             P.fft_ax, P.fft_ay, P.fft_dxdy, plan.spec, maxbits, skip);
  });
  if (!fy) {
    const int G = cols_group(Ny, plan.logy >= 0);
    const size_t smy = (size_t)G * padded(Ny) * sizeof(double2) * (plan.logy >= 0 ? 1 : 2);
    k_cols<<<(H + G - 1) / G, kThreads, smy, s>>>(Nx, Ny, plan.logy, G, plan.twy, P.fft_ax, P.fft_ay, P.fft_dxdy,
                                                  plan.spec, maxbits);
  }
  // rows, half spectrum -> real
  const bool fx2 = with_log2<kFusedMinLog>(plan.logx, [&](auto c) {
    constexpr int L = decltype(c)::value;
    const size_t sm = (size_t)paddedl<L>() * sizeof(double2);
    const unsigned long long *g = gate ? gate : maxbits;
    launch_k(k_rows_c2r_t<L>, dim3(pairs), dim3(kThreads), sm, s, Ny, plan.twx, plan.spec, dp, accumulate ? 1 : 0, g,
             skip);
  });
  if (!fx2)
    k_rows_c2r<<<pairs, kThreads, smx, s>>>(Nx, Ny, plan.logx, plan.twx, plan.spec, dp, accumulate ? 1 : 0,
                                            gate ? gate : maxbits);
  return cudaSuccess;
}
}  // namespace

cudaError_t launch_fft_poisson(const DevOps &P, const FftPlan &plan, const double *f, double *dp, bool accumulate,
                               cudaStream_t s) {
  return fft_passes(P, plan, f, nullptr, false, 0.0, 0.0, 0.0, dp, accumulate, s);
}

bool fft_fuses_div(const FftPlan &plan) { return plan.logx >= kFusedMinLog && plan.logx <= 13; }

int fft_kernels(const FftPlan &) { return 3; }

cudaError_t launch_fft_poisson_div(const DevOps &P, const FftPlan &plan, const double *W, double alpha,
                                   double beta, double gamma, double *dp, bool accumulate, cudaStream_t s) {
  return fft_passes(P, plan, W, nullptr, true, alpha, beta, gamma, dp, accumulate, s);
}

cudaError_t launch_fft_precond(const DevOps &P, const FftPlan &plan, const double *r, double *z,
                               const unsigned long long *gate, const int *skip, cudaStream_t s) {
  return fft_passes(P, plan, r, nullptr, false, 0.0, 0.0, 0.0, z, false, s, gate, skip);
}

cudaError_t launch_fft_poisson_div_split(const DevOps &P, const FftPlan &plan, const double *Vn, const float *T,
                                         double sv, double sa, double alpha, double beta, double gamma, double *dp,
                                         bool accumulate, cudaStream_t s) {
  const WSplit ws{Vn, T, sv, sa};
  return fft_passes(P, plan, nullptr, &ws, true, alpha, beta, gamma, dp, accumulate, s);
}

// --- pieces of the transform for a grid split into y-slabs ----------------------
bool slab_fft_supported(int Nx, int Ny) {
  const int lx = ilog2_exact(Nx), ly = ilog2_exact(Ny);
  return lx >= kFusedMinLog && lx <= 13 && ly >= kFusedMinLog && ly <= 13;
}

cudaError_t slab_rows_forward(int Nx, const double2 *twx, const double *f, int nrows, double2 *spec, cudaStream_t s) {
  const int pairs = (nrows + 1) / 2;
  DevOps P{};
  const WSplit w0{};
  with_log2<kFusedMinLog>(ilog2_exact(Nx), [&](auto c) {
    constexpr int L = decltype(c)::value;
    const size_t sm = (size_t)paddedl<L>() * sizeof(double2);
    k_rows_r2c_t<L, 0><<<pairs, kThreads, sm, s>>>(nrows, twx, f, w0, spec, P, 0.0, 0.0, 0.0, 0, nullptr, nullptr);
  });
  return cudaPeekAtLastError();
}

cudaError_t slab_columns(int Ny, const double2 *twy, const double *ax, const double *ay, double dxdy, double2 *cols,
                         int width, int ncols, int I0, unsigned long long *maxbits, cudaStream_t s) {
  with_log2<kFusedMinLog>(ilog2_exact(Ny), [&](auto c) {
    constexpr int L = decltype(c)::value, G = cols_per_block<L>();
    const size_t sm = cols_smem<L, G>();
    k_cols_t<L, G, cols_radix<L>()><<<(ncols + G - 1) / G, kThreads, sm, s>>>(width, ncols, I0, twy, ax, ay, dxdy,
                                                                              cols, maxbits, nullptr);
  });
  return cudaPeekAtLastError();
}

cudaError_t slab_rows_inverse(int Nx, const double2 *twx, const double2 *spec, int nrows, double *out,
                              const unsigned long long *maxbits, cudaStream_t s) {
  const int pairs = (nrows + 1) / 2;
  with_log2<kFusedMinLog>(ilog2_exact(Nx), [&](auto c) {
    constexpr int L = decltype(c)::value;
    const size_t sm = (size_t)paddedl<L>() * sizeof(double2);
    k_rows_c2r_t<L><<<pairs, kThreads, sm, s>>>(nrows, twx, spec, out, 0, maxbits, nullptr);
  });
  return cudaPeekAtLastError();
}

}  // namespace ins2d
