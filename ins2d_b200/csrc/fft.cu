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

// Shared-memory passes over stages s_top down to s_bot (DIF) / s_bot up to
// s_top (DIT), three stages per pass.
__device__ void dif_range(double2 *a, int G, int n, const double2 *pyr, bool inv, int s_top, int s_bot) {
  const int t = threadIdx.x, nt = blockDim.x, ld = padded(n);
  for (int s_hi = s_top; s_hi >= s_bot; s_hi -= 3) {
    const int ns = min(3, s_hi - s_bot + 1), s_lo = s_hi - ns + 1;
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
      group_dif<false>(x, ns, k, h, pyr, inv);
#pragma unroll
      for (int m = 0; m < 8; ++m)
        if (m < R) L[pd(base + m * h)] = x[m];
    }
    __syncthreads();
  }
}
__device__ void dit_range(double2 *a, int G, int n, const double2 *pyr, bool inv, int s_bot, int s_top) {
  const int t = threadIdx.x, nt = blockDim.x, ld = padded(n);
  for (int s0 = s_bot - 1; s0 < s_top; s0 += 3) {
    const int ns = min(3, s_top - s0), R = 1 << ns, h = 1 << s0, per = n >> ns;
    for (int g = t; g < G * per; g += nt) {
      const int line = g / per, gg = g - line * per;
      const int k = gg & (h - 1), blk = gg >> s0;
      const int base = blk * R * h + k;
      double2 *L = a + (size_t)line * ld;
      double2 x[8];
#pragma unroll
      for (int m = 0; m < 8; ++m)
        if (m < R) x[m] = L[pd(base + m * h)];
      group_dit<false>(x, ns, k, h, pyr, inv);
#pragma unroll
      for (int m = 0; m < 8; ++m)
        if (m < R) L[pd(base + m * h)] = x[m];
    }
    __syncthreads();
  }
}

// --- power-of-two lengths >= 64: first and last radix-8 passes fused with
// the global loads/stores, no permutation passes; tw is the table of
// fft_twiddle_table (the pyramid at tw + N) ----------------------------------

// rows j0, j1 -> half spectra (forward DIF; bit-reversed result read back
// during the Hermitian split)
// DIV: the rows are not read from f but computed on the fly as the
// divergence (M W + alpha yM + beta ydM) * gamma of the velocity-sized W
// (time_ERK.m:117, pressure_additional_solve.m:11-13), fusing that kernel in.
template <bool DIV>
__global__ void __launch_bounds__(kThreads, INS2D_FFT_ROWS_MINB) k_rows_r2c_f(int Nx, int Ny, int L, const double2 *__restrict__ tw,
                                                         const double *__restrict__ f, double2 *__restrict__ spec,
                                                         const __grid_constant__ DevOps P, double alpha, double beta,
                                                         double gamma) {
  extern __shared__ double2 sm[];
  const double2 *pyr = tw + Nx;
  const int j0 = 2 * blockIdx.x, j1 = j0 + 1;
  const bool has1 = j1 < Ny;
  const int H = Nx / 2 + 1, per = Nx >> 3;
  const double *r0 = f + (size_t)j0 * Nx, *r1 = f + (size_t)j1 * Nx;
  for (int k = threadIdx.x; k < per; k += blockDim.x) {
    double2 x[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      if (DIV)
        x[m] = make_double2(div_cell(P, f, alpha, beta, gamma, k + m * per, j0),
                            has1 ? div_cell(P, f, alpha, beta, gamma, k + m * per, j1) : 0.0);
      else
        x[m] = make_double2(__ldg(r0 + k + m * per), has1 ? __ldg(r1 + k + m * per) : 0.0);
    }
    group_dif<false>(x, 3, k, per, pyr, false);
#pragma unroll
    for (int m = 0; m < 8; ++m) sm[pd(k + m * per)] = x[m];
  }
  __syncthreads();
  dif_range(sm, 1, Nx, pyr, false, L - 3, 1);
  for (int I = threadIdx.x; I < H; I += blockDim.x) {
    const double2 z = sm[pd(brev(I, L))], m = sm[pd(brev((Nx - I) & (Nx - 1), L))];
    spec[(size_t)j0 * H + I] = make_double2(0.5 * (z.x + m.x), 0.5 * (z.y - m.y));
    if (has1) spec[(size_t)j1 * H + I] = make_double2(0.5 * (z.y + m.y), 0.5 * (m.x - z.x));
  }
}

// G spectrum columns: forward DIF, -1/Ahat scaling fused with the last DIF and
// first DIT passes, inverse DIT; max |fhat| reduction
__global__ void __launch_bounds__(kThreads, INS2D_FFT_COLS_MINB) k_cols_f(int Nx, int Ny, int L, int G, const double2 *__restrict__ tw,
                                                     const double *__restrict__ ax, const double *__restrict__ ay,
                                                     double dxdy, double2 *__restrict__ spec,
                                                     unsigned long long *__restrict__ maxbits) {
  extern __shared__ double2 sm[];
  __shared__ double wmax[kThreads / 32];
  const double2 *pyr = tw + Ny;
  const int H = Nx / 2 + 1, per = Ny >> 3, ld = padded(Ny);
  const int c0 = blockIdx.x * G;
  const int g_here = min(G, H - c0);
  for (int gidx = threadIdx.x; gidx < g_here * per; gidx += blockDim.x) {
    const int k = gidx / g_here, line = gidx - k * g_here;
    double2 x[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) x[m] = spec[(size_t)(k + m * per) * H + c0 + line];
    group_dif<false>(x, 3, k, per, pyr, false);
#pragma unroll
    for (int m = 0; m < 8; ++m) sm[(size_t)line * ld + pd(k + m * per)] = x[m];
  }
  __syncthreads();
  dif_range(sm, g_here, Ny, pyr, false, L - 3, 4);
  double lmax = 0.0;
  for (int gidx = threadIdx.x; gidx < g_here * per; gidx += blockDim.x) {
    const int line = gidx / per, k = gidx - line * per;
    double2 *Ls = sm + (size_t)line * ld;
    const int I = c0 + line;
    double2 x[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) x[m] = Ls[pd(8 * k + m)];
    group_dif<true>(x, 3, 0, 1, pyr, false);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int J = brev(8 * k + m, L);
      const double2 F = x[m];
      lmax = fmax(lmax, F.x * F.x + F.y * F.y);  // squared; one square root per block
      const double lam = (I == 0 && J == 0) ? 1.0 : (dxdy * 4.0) * (__ldg(ax + I) + __ldg(ay + J));
      const double r = -1.0 / lam;
      x[m] = make_double2(F.x * r, F.y * r);
    }
    group_dit<true>(x, 3, 0, 1, pyr, true);
#pragma unroll
    for (int m = 0; m < 8; ++m) Ls[pd(8 * k + m)] = x[m];
  }
  __syncthreads();
  dit_range(sm, g_here, Ny, pyr, true, 4, L - 3);
  const double sc = 1.0 / Ny;
  for (int gidx = threadIdx.x; gidx < g_here * per; gidx += blockDim.x) {
    const int k = gidx / g_here, line = gidx - k * g_here;
    double2 x[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) x[m] = sm[(size_t)line * ld + pd(k + m * per)];
    group_dit<false>(x, 3, k, per, pyr, true);
#pragma unroll
    for (int m = 0; m < 8; ++m)
      spec[(size_t)(k + m * per) * H + c0 + line] = make_double2(x[m].x * sc, x[m].y * sc);
  }
  for (int off = 16; off > 0; off >>= 1) lmax = fmax(lmax, __shfl_down_sync(0xffffffffu, lmax, off));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = lmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = wmax[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mm = fmax(mm, wmax[w]);
    atomicMax(maxbits, (unsigned long long)__double_as_longlong(sqrt(mm)));
  }
}

// half spectra of rows j0, j1 -> real rows (inverse DIF, bit-reversed result
// read back in natural order)
__global__ void __launch_bounds__(kThreads, INS2D_FFT_ROWS_MINB) k_rows_c2r_f(int Nx, int Ny, int L, const double2 *__restrict__ tw,
                                                         const double2 *__restrict__ spec, double *__restrict__ out,
                                                         int accumulate, const unsigned long long *__restrict__ maxbits) {
  extern __shared__ double2 sm[];
  const int j0 = 2 * blockIdx.x, j1 = j0 + 1;
  const bool has1 = j1 < Ny;
  const int H = Nx / 2 + 1, per = Nx >> 3;
  const double mx = __longlong_as_double((long long)*maxbits);
  if (mx < 1e-14) {  // pressure_poisson.m:21-32: dp stays zero
    if (!accumulate)
      for (int k = threadIdx.x; k < Nx; k += blockDim.x) {
        out[(size_t)j0 * Nx + k] = 0.0;
        if (has1) out[(size_t)j1 * Nx + k] = 0.0;
      }
    return;
  }
  const double2 *pyr = tw + Nx;
  const double2 *s0 = spec + (size_t)j0 * H, *s1 = spec + (size_t)j1 * H;
  for (int k = threadIdx.x; k < per; k += blockDim.x) {
    double2 x[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int q = k + m * per;
      double2 g0, g1;
      if (q < H) {
        g0 = s0[q];
        g1 = has1 ? s1[q] : make_double2(0.0, 0.0);
      } else {
        const double2 a = s0[Nx - q];
        const double2 b = has1 ? s1[Nx - q] : make_double2(0.0, 0.0);
        g0 = make_double2(a.x, -a.y);
        g1 = make_double2(b.x, -b.y);
      }
      x[m] = make_double2(g0.x - g1.y, g0.y + g1.x);
    }
    group_dif<false>(x, 3, k, per, pyr, true);
#pragma unroll
    for (int m = 0; m < 8; ++m) sm[pd(k + m * per)] = x[m];
  }
  __syncthreads();
  dif_range(sm, 1, Nx, pyr, true, L - 3, 1);
  const double sc = 1.0 / Nx;
  for (int k = threadIdx.x; k < Nx; k += blockDim.x) {
    const double2 w = sm[pd(brev(k, L))];
    if (accumulate) {
      out[(size_t)j0 * Nx + k] += w.x * sc;
      if (has1) out[(size_t)j1 * Nx + k] += w.y * sc;
    } else {
      out[(size_t)j0 * Nx + k] = w.x * sc;
      if (has1) out[(size_t)j1 * Nx + k] = w.y * sc;
    }
  }
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
// device (called once per context).
void fft_prepare() {
  cudaFuncSetAttribute(k_rows_r2c_f<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_rows_r2c_f<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_cols_f, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_rows_c2r_f, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_rows_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_rows_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

namespace {
void fft_passes(const DevOps &P, const FftPlan &plan, const double *src, bool div, double alpha, double beta,
                double gamma, double *dp, bool accumulate, cudaStream_t s) {
  const int Nx = plan.Nx, Ny = plan.Ny;
  const size_t smx = (size_t)padded(Nx) * sizeof(double2) * (plan.logx >= 0 ? 1 : 2);
  const int G = cols_group(Ny, plan.logy >= 0);
  const size_t smy = (size_t)G * padded(Ny) * sizeof(double2) * (plan.logy >= 0 ? 1 : 2);
  const int pairs = (Ny + 1) / 2;
  const int H = Nx / 2 + 1;
  cudaMemsetAsync(plan.maxabs, 0, sizeof(double), s);
  const bool fx = plan.logx >= 6, fy = plan.logy >= 6;  // fused-pass kernels
  if (fx && div)
    k_rows_r2c_f<true><<<pairs, kThreads, smx, s>>>(Nx, Ny, plan.logx, plan.twx, src, plan.spec, P, alpha, beta,
                                                    gamma);
  else if (fx)
    k_rows_r2c_f<false><<<pairs, kThreads, smx, s>>>(Nx, Ny, plan.logx, plan.twx, src, plan.spec, P, 0.0, 0.0, 0.0);
  else
    k_rows_r2c<<<pairs, kThreads, smx, s>>>(Nx, Ny, plan.logx, plan.twx, src, plan.spec);
  if (fy)
    k_cols_f<<<(H + G - 1) / G, kThreads, smy, s>>>(Nx, Ny, plan.logy, G, plan.twy, P.fft_ax, P.fft_ay, P.fft_dxdy,
                                                    plan.spec, (unsigned long long *)plan.maxabs);
  else
    k_cols<<<(H + G - 1) / G, kThreads, smy, s>>>(Nx, Ny, plan.logy, G, plan.twy, P.fft_ax, P.fft_ay, P.fft_dxdy,
                                                  plan.spec, (unsigned long long *)plan.maxabs);
  if (fx)
    k_rows_c2r_f<<<pairs, kThreads, smx, s>>>(Nx, Ny, plan.logx, plan.twx, plan.spec, dp, accumulate ? 1 : 0,
                                              (const unsigned long long *)plan.maxabs);
  else
    k_rows_c2r<<<pairs, kThreads, smx, s>>>(Nx, Ny, plan.logx, plan.twx, plan.spec, dp, accumulate ? 1 : 0,
                                            (const unsigned long long *)plan.maxabs);
}
}  // namespace

void launch_fft_poisson(const DevOps &P, const FftPlan &plan, const double *f, double *dp, bool accumulate,
                        cudaStream_t s) {
  fft_passes(P, plan, f, false, 0.0, 0.0, 0.0, dp, accumulate, s);
}

bool fft_fuses_div(const FftPlan &plan) { return plan.logx >= 6; }

void launch_fft_poisson_div(const DevOps &P, const FftPlan &plan, const double *W, double alpha, double beta,
                            double gamma, double *dp, bool accumulate, cudaStream_t s) {
  fft_passes(P, plan, W, true, alpha, beta, gamma, dp, accumulate, s);
}

}  // namespace ins2d
