/* CPU oracle / timed CPU baseline: the reference's explicit RK step on a
 * uniform, doubly periodic staggered grid, matrix-free, OpenMP-parallel.
 *
 * TEST INFRASTRUCTURE ONLY: the checker and the timed CPU stand-in of the
 * reference path (the reference itself is MATLAB, not runnable here); the
 * product never links or calls this file.  It restates, for the periodic
 * uniform case only (all sides 'per', constant hx, hy), the same arithmetic as
 * the scipy restatement in ins2d_ref.py, from the reference's files:
 *   F / convection / diffusion  spatial/F.m:137-145, convection.m:198-215,
 *                               diffusion.m:22-37 (energy-conserving 2nd order:
 *                               face averages Au_ux, Au_uy, Av_vx, Av_vy;
 *                               fluxes Iu_ux = hy*avg, Iv_uy = (hx/2)(v+v),
 *                               Iu_vx = (hy/2)(u+u), Iv_vy = hx*avg;
 *                               diffusion Dux Su_ux / Re + Duy Su_uy / Re)
 *   divergence / gradient        operator_divergence.m:116-167 (M, G = -M')
 *   FFT pressure solve           pressure_poisson.m:92-104 (dp = real(ifft2(
 *                                -fft2(f)./Ahat)), Ahat = dxdy*4*(sin^2(pi I/Nx)/dx^2
 *                                + sin^2(pi J/Ny)/dy^2), Ahat(1,1) = 1), and the
 *                                early return of pressure_poisson.m:21-32
 *   time_ERK                     unsteady/time_ERK.m:29-168 (shifted tableau,
 *                                steady boundary conditions, first stage with
 *                                dp = pn, additional pressure solve)
 * Layout: u(i,j) at i + j*Nx (u at the left face of cell i), v(i,j) at
 * Nx*Ny + i + j*Nx (v at the lower face of cell j), p(i,j) at i + j*Nx.
 * The FFT is an iterative radix-2 complex transform (power-of-two sizes) over
 * rows and then columns.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  double re, im;
} cplx;

static inline int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

/* R(V) = -conv(V) + Diff V (F.m without the pressure gradient) */
static void rhs(int Nx, int Ny, double hx, double hy, double invRe, const double *V, double *R) {
  const double *u = V, *v = V + (size_t)Nx * Ny;
  double *Ru = R, *Rv = R + (size_t)Nx * Ny;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < Ny; ++j) {
    const int jm = wrap(j - 1, Ny), jp = wrap(j + 1, Ny);
    for (int i = 0; i < Nx; ++i) {
      const int im = wrap(i - 1, Nx), ip = wrap(i + 1, Nx);
#define U(a, b) u[(size_t)(b) * Nx + (a)]
#define W(a, b) v[(size_t)(b) * Nx + (a)]
      /* u-momentum at the face (i, j) */
      {
        const double uxl = 0.5 * (U(im, j) + U(i, j)), uxr = 0.5 * (U(i, j) + U(ip, j));
        const double du2dx = (hy * uxr) * uxr - (hy * uxl) * uxl;
        const double uy0 = 0.5 * (U(i, jm) + U(i, j)), uy1 = 0.5 * (U(i, j) + U(i, jp));
        const double vf0 = 0.5 * hx * (W(im, j) + W(i, j)), vf1 = 0.5 * hx * (W(im, jp) + W(i, jp));
        const double duvdy = vf1 * uy1 - vf0 * uy0;
        const double sxl = (U(i, j) - U(im, j)) / hx, sxr = (U(ip, j) - U(i, j)) / hx;
        const double syl = (U(i, j) - U(i, jm)) / hy, syr = (U(i, jp) - U(i, j)) / hy;
        const double d2u = hy * (invRe * sxr - invRe * sxl) + hx * (invRe * syr - invRe * syl);
        Ru[(size_t)j * Nx + i] = -(du2dx + duvdy) + d2u;
      }
      /* v-momentum at the face (i, j) */
      {
        const double vxl = 0.5 * (W(im, j) + W(i, j)), vxr = 0.5 * (W(i, j) + W(ip, j));
        const double ufl = 0.5 * hy * (U(i, jm) + U(i, j)), ufr = 0.5 * hy * (U(ip, jm) + U(ip, j));
        const double duvdx = ufr * vxr - ufl * vxl;
        const double vy0 = 0.5 * (W(i, jm) + W(i, j)), vy1 = 0.5 * (W(i, j) + W(i, jp));
        const double dv2dy = (hx * vy1) * vy1 - (hx * vy0) * vy0;
        const double sxl = (W(i, j) - W(im, j)) / hx, sxr = (W(ip, j) - W(i, j)) / hx;
        const double syl = (W(i, j) - W(i, jm)) / hy, syr = (W(i, jp) - W(i, j)) / hy;
        const double d2v = hy * (invRe * sxr - invRe * sxl) + hx * (invRe * syr - invRe * syl);
        Rv[(size_t)j * Nx + i] = -(duvdx + dv2dy) + d2v;
      }
#undef U
#undef W
    }
  }
}

/* f = M W * gam   (M: hy (u_{i+1} - u_i) + hx (v_{j+1} - v_j)) */
static void divergence(int Nx, int Ny, double hx, double hy, const double *W, double gam, double *f) {
  const double *u = W, *v = W + (size_t)Nx * Ny;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < Ny; ++j) {
    const int jp = wrap(j + 1, Ny);
    for (int i = 0; i < Nx; ++i) {
      const int ip = wrap(i + 1, Nx);
      f[(size_t)j * Nx + i] = gam * (hy * (u[(size_t)j * Nx + ip] - u[(size_t)j * Nx + i]) +
                                     hx * (v[(size_t)jp * Nx + i] - v[(size_t)j * Nx + i]));
    }
  }
}

/* in-place radix-2 FFT of n points with stride s (sign -1 forward, +1 inverse) */
static void fft1(cplx *a, int n, int s, const cplx *tw, int sign) {
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      cplx t = a[(size_t)i * s];
      a[(size_t)i * s] = a[(size_t)j * s];
      a[(size_t)j * s] = t;
    }
  }
  for (int len = 2; len <= n; len <<= 1) {
    const int step = n / len;
    for (int i = 0; i < n; i += len)
      for (int k = 0; k < len / 2; ++k) {
        cplx w = tw[k * step];
        if (sign > 0) w.im = -w.im;
        cplx *x = &a[(size_t)(i + k) * s], *y = &a[(size_t)(i + k + len / 2) * s];
        const cplx t = {w.re * y->re - w.im * y->im, w.re * y->im + w.im * y->re};
        y->re = x->re - t.re;
        y->im = x->im - t.im;
        x->re += t.re;
        x->im += t.im;
      }
  }
}

/* rows in place; columns in groups of 8 gathered into contiguous buffers
 * (cache-friendly), transformed and scattered back */
static void fft2(cplx *a, int Nx, int Ny, const cplx *twx, const cplx *twy, int sign) {
#pragma omp parallel for schedule(static)
  for (int j = 0; j < Ny; ++j) fft1(a + (size_t)j * Nx, Nx, 1, twx, sign);
  const int G = 8;
#pragma omp parallel
  {
    cplx *tmp = (cplx *)malloc((size_t)G * Ny * sizeof(cplx));
#pragma omp for schedule(static)
    for (int i0 = 0; i0 < Nx; i0 += G) {
      const int g = (Nx - i0) < G ? (Nx - i0) : G;
      for (int j = 0; j < Ny; ++j)
        for (int c = 0; c < g; ++c) tmp[(size_t)c * Ny + j] = a[(size_t)j * Nx + i0 + c];
      for (int c = 0; c < g; ++c) fft1(tmp + (size_t)c * Ny, Ny, 1, twy, sign);
      for (int j = 0; j < Ny; ++j)
        for (int c = 0; c < g; ++c) a[(size_t)j * Nx + i0 + c] = tmp[(size_t)c * Ny + j];
    }
    free(tmp);
  }
}

typedef struct {
  int Nx, Ny;
  double hx, hy, invRe;
  cplx *buf, *twx, *twy;
  double *ahat;
  double *R, *f, *dp, *Vs, *Wt, *kV[4];
} Work;

/* dp = real(ifft2(-fft2(f)./Ahat)); 0 when max|fhat| < 1e-14 */
static void poisson(Work *w, const double *f, double *dp) {
  const int Nx = w->Nx, Ny = w->Ny;
  const size_t n = (size_t)Nx * Ny;
#pragma omp parallel for schedule(static)
  for (size_t k = 0; k < n; ++k) {
    w->buf[k].re = f[k];
    w->buf[k].im = 0.0;
  }
  fft2(w->buf, Nx, Ny, w->twx, w->twy, -1);
  double mx = 0.0;
#pragma omp parallel for reduction(max : mx) schedule(static)
  for (size_t k = 0; k < n; ++k) {
    const double a = hypot(w->buf[k].re, w->buf[k].im);
    if (a > mx) mx = a;
    w->buf[k].re /= -w->ahat[k];
    w->buf[k].im /= -w->ahat[k];
  }
  if (mx < 1e-14) {
    memset(dp, 0, n * sizeof(double));
    return;
  }
  fft2(w->buf, Nx, Ny, w->twx, w->twy, +1);
  const double sc = 1.0 / (double)n;
#pragma omp parallel for schedule(static)
  for (size_t k = 0; k < n; ++k) dp[k] = w->buf[k].re * sc;
}

/* V_out = Vn + dt (Vtemp - c Om^-1 G dp), written as dt (Wt - c Om^-1 G dp) with Wt = Vn/dt + Vtemp */
static void project(const Work *w, const double *Wt, const double *dp, double dt, double c, double *Vo) {
  const int Nx = w->Nx, Ny = w->Ny;
  const double hx = w->hx, hy = w->hy, oi = 1.0 / (hx * hy);
  const size_t n = (size_t)Nx * Ny;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < Ny; ++j) {
    const int jm = wrap(j - 1, Ny);
    for (int i = 0; i < Nx; ++i) {
      const int im = wrap(i - 1, Nx);
      const size_t k = (size_t)j * Nx + i;
      const double gx = hy * (dp[k] - dp[(size_t)j * Nx + im]);
      const double gy = hx * (dp[k] - dp[(size_t)jm * Nx + i]);
      Vo[k] = dt * (Wt[k] - c * oi * gx);
      Vo[n + k] = dt * (Wt[n + k] - c * oi * gy);
    }
  }
}

/* Runs nsteps RK steps (s stages, Butcher A row-major s x s, b, c) on V
 * (2 Nx Ny) and p (Nx Ny) in place; Lx, Ly: domain lengths.  Returns 0, or 1
 * on allocation failure, 2 for sizes that are not powers of two. */
int oracle_erk_periodic(int Nx, int Ny, double Lx, double Ly, double Re, int s, const double *A_, const double *b_,
                        const double *c_, double dt, int nsteps, double *V, double *p, int nthreads) {
  if ((Nx & (Nx - 1)) || (Ny & (Ny - 1)) || s < 1 || s > 4) return 2;
#ifdef _OPENMP
  omp_set_num_threads(nthreads > 0 ? nthreads : omp_get_num_procs());
#else
  (void)nthreads;
#endif
  Work w;
  memset(&w, 0, sizeof w);
  w.Nx = Nx;
  w.Ny = Ny;
  w.hx = Lx / Nx;
  w.hy = Ly / Ny;
  w.invRe = 1.0 / Re;
  const size_t n = (size_t)Nx * Ny, NV = 2 * n;
  w.buf = (cplx *)malloc(n * sizeof(cplx));
  w.twx = (cplx *)malloc((size_t)Nx * sizeof(cplx));
  w.twy = (cplx *)malloc((size_t)Ny * sizeof(cplx));
  w.ahat = (double *)malloc(n * sizeof(double));
  w.R = (double *)malloc(NV * sizeof(double));
  w.f = (double *)malloc(n * sizeof(double));
  w.dp = (double *)malloc(n * sizeof(double));
  w.Vs = (double *)malloc(NV * sizeof(double));
  w.Wt = (double *)malloc(NV * sizeof(double));
  for (int k = 0; k < 4; ++k) w.kV[k] = (double *)malloc(NV * sizeof(double));
  int bad = !w.buf || !w.twx || !w.twy || !w.ahat || !w.R || !w.f || !w.dp || !w.Vs || !w.Wt;
  for (int k = 0; k < 4; ++k) bad |= !w.kV[k];
  if (bad) {
    free(w.buf); free(w.twx); free(w.twy); free(w.ahat); free(w.R); free(w.f); free(w.dp); free(w.Vs); free(w.Wt);
    for (int k = 0; k < 4; ++k) free(w.kV[k]);
    return 1;
  }
  const double pi = acos(-1.0);
  for (int k = 0; k < Nx; ++k) {
    w.twx[k].re = cos(2 * pi * k / Nx);
    w.twx[k].im = -sin(2 * pi * k / Nx);
  }
  for (int k = 0; k < Ny; ++k) {
    w.twy[k].re = cos(2 * pi * k / Ny);
    w.twy[k].im = -sin(2 * pi * k / Ny);
  }
  const double dx = w.hx, dy = w.hy;
  for (int J = 0; J < Ny; ++J)
    for (int I = 0; I < Nx; ++I) {
      const double sx = sin(pi * I / Nx), sy = sin(pi * J / Ny);
      double a = (dx * dy) * 4.0 * (sx * sx / (dx * dx) + sy * sy / (dy * dy));
      if (I == 0 && J == 0) a = 1.0;
      w.ahat[(size_t)J * Nx + I] = a;
    }
  /* shifted tableau (time_ERK.m:29-32) */
  double A[4][4] = {{0}}, c[4] = {0};
  for (int i = 0; i < s; ++i) {
    for (int j = 0; j < s; ++j) A[i][j] = (i < s - 1) ? A_[(i + 1) * s + j] : b_[j];
    c[i] = (i < s - 1) ? c_[i + 1] : 1.0;
  }
  const double oi = 1.0 / (dx * dy);
  for (int step = 0; step < nsteps; ++step) {
    const double *Vi = V;
    const double *dpp = p;
    for (int i = 0; i < s; ++i) {
      rhs(Nx, Ny, dx, dy, w.invRe, Vi, w.R);
      double *kv = w.kV[i];
#pragma omp parallel for schedule(static)
      for (size_t k = 0; k < NV; ++k) {
        kv[k] = oi * w.R[k];
        double vt = 0.0;
        for (int m = 0; m <= i; ++m) vt += A[i][m] * w.kV[m][k];
        w.Wt[k] = V[k] / dt + vt;
      }
      if (i > 0) {
        divergence(Nx, Ny, dx, dy, w.Wt, 1.0 / c[i], w.f);
        poisson(&w, w.f, w.dp);
        dpp = w.dp;
      } else {
        dpp = p; /* time_ERK.m:125-127 */
      }
      project(&w, w.Wt, dpp, dt, c[i], (i == s - 1) ? V : w.Vs);
      Vi = w.Vs;
    }
    /* additional pressure solve (pressure_additional_solve.m:11-13):
     * f = M Om^-1 (R(V) - G p), p += dp */
    rhs(Nx, Ny, dx, dy, w.invRe, V, w.R);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Ny; ++j) {
      const int jm = wrap(j - 1, Ny);
      for (int i = 0; i < Nx; ++i) {
        const int im = wrap(i - 1, Nx);
        const size_t k = (size_t)j * Nx + i;
        w.Wt[k] = oi * (w.R[k] - dy * (p[k] - p[(size_t)j * Nx + im]));
        w.Wt[n + k] = oi * (w.R[n + k] - dx * (p[k] - p[(size_t)jm * Nx + i]));
      }
    }
    divergence(Nx, Ny, dx, dy, w.Wt, 1.0, w.f);
    poisson(&w, w.f, w.dp);
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < n; ++k) p[k] += w.dp[k];
  }
  free(w.buf); free(w.twx); free(w.twy); free(w.ahat); free(w.R); free(w.f); free(w.dp); free(w.Vs); free(w.Wt);
  for (int k = 0; k < 4; ++k) free(w.kV[k]);
  return 0;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
