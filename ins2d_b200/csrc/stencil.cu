// Column-walking evaluation of the momentum right-hand side
//   R = -conv(V) + Diff*V + yDiff - y_p     (F.m:137-145 without G*p)
// for the RK stage kernel (time_ERK.m:90-101) and the residual of the
// additional pressure solve (pressure_additional_solve.m:11-13).
//
// Each thread owns one column i and walks a run of rows j.  Its 1D x-table
// rows (Au_ux, Su_ux, Iv_uy(x), ... at i and i+1) are loaded into registers
// once per run; the y-faces (u at uy, vbar at uy, du/dy, v at vy, dv/dy) are
// computed once per face and slid down the column, so per point only the few
// field values of the stencil are loaded.  Warps with threadIdx.y == 0 walk u
// points, threadIdx.y == 1 walk v points of the same columns, so both share
// their field rows in L1.  Boundary rows of the operators use the same tables
// (the boundary elimination lives in the table entries), so there is one
// code path for every boundary-condition combination.
#include "kernels.cuh"

namespace ins2d {

namespace {

// launch shape (compile-time tunables)
#ifndef INS2D_WALK_RUN
#define INS2D_WALK_RUN 32
#endif
#ifndef INS2D_WALK_MINB
#define INS2D_WALK_MINB 5
#endif
constexpr int WX = 64;               // columns per block (two warps per walker)
constexpr int RUN = INS2D_WALK_RUN;  // rows per column run

template <typename S>
struct XRow {  // one row of an x-table in registers
  int c0, c1, c2;
  S w0, w1, w2, b1, b2;
};
template <typename S>
struct XRowW {  // weights of a second table that shares the columns
  S w0, w1, w2, b1, b2;
};

template <typename S>
__device__ __forceinline__ XRow<S> xrow(const Tab &T, int r) {
  XRow<S> x;
  const int32_t *c = T.c + kT * r;
  const double *w = T.w + kT * r;
  x.c0 = __ldg(c);
  x.c1 = __ldg(c + 1);
  x.c2 = __ldg(c + 2);
  x.w0 = S(__ldg(w));
  x.w1 = S(__ldg(w + 1));
  x.w2 = S(__ldg(w + 2));
  x.b1 = S(__ldg(T.b1 + r));
  x.b2 = S(__ldg(T.b2 + r));
  return x;
}
template <typename S>
__device__ __forceinline__ XRowW<S> xroww(const Tab &T, int r) {
  XRowW<S> x;
  const double *w = T.w + kT * r;
  x.w0 = S(__ldg(w));
  x.w1 = S(__ldg(w + 1));
  x.w2 = S(__ldg(w + 2));
  x.b1 = S(__ldg(T.b1 + r));
  x.b2 = S(__ldg(T.b2 + r));
  return x;
}

// loads the (up to three) entries of a row of f at the columns of x
template <typename S>
struct Trip {
  S a0, a1, a2;
};
template <typename S, typename TV>
__device__ __forceinline__ Trip<S> load3(const TV *__restrict__ row, const XRow<S> &x) {
  Trip<S> t;
  t.a0 = S(__ldg(row + x.c0));
  t.a1 = S(__ldg(row + x.c1));
  t.a2 = (x.w2 != S(0)) ? S(__ldg(row + x.c2)) : S(0);
  return t;
}
template <typename S>
__device__ __forceinline__ S dot3(const XRow<S> &x, const Trip<S> &t) {
  return x.w0 * t.a0 + x.w1 * t.a1 + x.w2 * t.a2;
}
template <typename S>
__device__ __forceinline__ S dot3(const XRowW<S> &x, const Trip<S> &t) {
  return x.w0 * t.a0 + x.w1 * t.a1 + x.w2 * t.a2;
}

// a y-table row (warp-uniform)
template <typename S>
struct YRow {
  int c0, c1, c2;
  S w0, w1, w2, b1, b2;
};
template <typename S>
__device__ __forceinline__ YRow<S> yrow(const Tab &T, int r) {
  YRow<S> y;
  const int32_t *c = T.c + kT * r;
  const double *w = T.w + kT * r;
  y.c0 = __ldg(c);
  y.c1 = __ldg(c + 1);
  y.c2 = __ldg(c + 2);
  y.w0 = S(__ldg(w));
  y.w1 = S(__ldg(w + 1));
  y.w2 = S(__ldg(w + 2));
  y.b1 = S(__ldg(T.b1 + r));
  y.b2 = S(__ldg(T.b2 + r));
  return y;
}

struct Epi {
  // 0: RK stage, FP64 storage (kV, Wt = Vn/dt + Vtemp);
  // 1: residual of the additional solve;
  // 3: F = R - G p into w (walked as mode 1);
  // 2: RK stage, FP32 storage (kV32 and, when the stage combines earlier
  //    stages, Vt32 = Vtemp; Vn and Wt are not touched)
  int mode;
  // stage
  const double *Vn;
  double *kV;
  const double *kprev[kMaxStages];
  double aprev[kMaxStages];
  int nprev;
  double aii, inv_dt;
  double *Wt;
  float *kV32;
  const float *kprev32[kMaxStages];
  float *Vt32;
  // residual
  const double *p;
  double *w;
  double *kV_next;
  float *kV_next32;
};

// NP >= 0: that many earlier stages, unrolled; NP < 0: e.nprev
template <int NP = -1>
__device__ __forceinline__ void epi_stage32(const Epi &e, long long idx, double k) {
  const float kf = (float)k;
  if (e.kV32) e.kV32[idx] = kf;
  if (e.Vt32) {
    double vt = 0.0;
    if constexpr (NP >= 0) {
#pragma unroll
      for (int m = 0; m < NP; ++m) vt += e.aprev[m] * (double)__ldg(e.kprev32[m] + idx);
    } else {
      for (int m = 0; m < e.nprev; ++m) vt += e.aprev[m] * (double)__ldg(e.kprev32[m] + idx);
    }
    vt += e.aii * (double)kf;
    e.Vt32[idx] = (float)vt;
  }
}

__device__ __forceinline__ void epilogue_stage(const Epi &e, long long idx, double oi, double R) {
  const double k = oi * R;
  if (e.mode == 2) {
    epi_stage32(e, idx, k);
    return;
  }
  if (e.kV) e.kV[idx] = k;
  double vt = 0.0;
  for (int m = 0; m < e.nprev; ++m) vt += e.aprev[m] * e.kprev[m][idx];
  vt += e.aii * k;
  e.Wt[idx] = e.Vn[idx] * e.inv_dt + vt;
}

__device__ __forceinline__ void epi_residual(const Epi &e, long long idx, double oi, double R, double g) {
  if (e.mode == 3) {  // F (F.m): the momentum right-hand side with the pressure gradient
    e.w[idx] = R - g;
    return;
  }
  e.w[idx] = oi * (R - g);
  if (e.kV_next) e.kV_next[idx] = oi * R;
  if (e.kV_next32) e.kV_next32[idx] = (float)(oi * R);
}

// ---------------------------------------------------------------------------
// u walker
template <typename S, typename TV>
__device__ void walk_u(const DevOps &P, const TV *__restrict__ u, const TV *__restrict__ v, const Epi &e,
                       int i, int j0, int j1) {
  if (i >= P.Nux) return;
  j1 = min(j1, P.Nuy);
  if (j0 >= j1) return;
  const S ire = S(P.invRe);
  const XRow<S> ax0 = xrow<S>(P.AUX, i), ax1 = xrow<S>(P.AUX, i + 1);
  const XRowW<S> sx0 = xroww<S>(P.SUX, i), sx1 = xroww<S>(P.SUX, i + 1);
  const XRow<S> ix = xrow<S>(P.IVX, i);
  const S gx = S(__ldg(P.gxi + i));
  const S pl = S(__ldg(P.pxl + i)), pr = S(__ldg(P.pxr + i));
  const S uLo = S(__ldg(P.bc.uLo_i + i)), uUp = S(__ldg(P.bc.uUp_i + i));
  const S xvlo = S(__ldg(P.bc.XvLo + i)), xvup = S(__ldg(P.bc.XvUp + i));
  // gradient row (residual mode)
  XRow<double> gt{};
  if (e.mode == 1 || e.mode == 3) gt = xrow<double>(P.MXT, i);
  // face at row r: u_uy, du/dy, vbar_uy
  auto face = [&](int r, S &uy, S &sy, S &vf) {
    const YRow<S> ay = yrow<S>(P.AUY, r);
    const double *__restrict__ sw = P.SUY.w + kT * r;
    const S s0 = S(__ldg(sw)), s1 = S(__ldg(sw + 1)), s2 = S(__ldg(sw + 2));
    const S f0 = S(__ldg(u + (long long)ay.c0 * P.Nux + i));
    const S f1 = S(__ldg(u + (long long)ay.c1 * P.Nux + i));
    const S f2 = (ay.w2 != S(0) || s2 != S(0)) ? S(__ldg(u + (long long)ay.c2 * P.Nux + i)) : S(0);
    uy = ay.w0 * f0 + ay.w1 * f1 + ay.w2 * f2 + ay.b1 * uLo + ay.b2 * uUp;
    sy = s0 * f0 + s1 * f1 + s2 * f2 + S(__ldg(P.SUY.b1 + r)) * uLo + S(__ldg(P.SUY.b2 + r)) * uUp;
    const YRow<S> iy = yrow<S>(P.IVY, r);
    S acc = S(0);
    if (iy.w0 != S(0)) acc += iy.w0 * dot3(ix, load3(v + (long long)iy.c0 * P.Nvx, ix));
    if (iy.w1 != S(0)) acc += iy.w1 * dot3(ix, load3(v + (long long)iy.c1 * P.Nvx, ix));
    if (iy.w2 != S(0)) acc += iy.w2 * dot3(ix, load3(v + (long long)iy.c2 * P.Nvx, ix));
    vf = acc + ix.b1 * S(__ldg(P.bc.vLe + r)) + ix.b2 * S(__ldg(P.bc.vRi + r)) + iy.b1 * xvlo + iy.b2 * xvup;
  };
  S uy0, sy0, vf0;
  face(j0, uy0, sy0, vf0);
  for (int j = j0; j < j1; ++j) {
    S uy1, sy1, vf1;
    face(j + 1, uy1, sy1, vf1);
    const TV *__restrict__ row = u + (long long)j * P.Nux;
    const S ule = S(__ldg(P.bc.uLe_i + j)), uri = S(__ldg(P.bc.uRi_i + j));
    const Trip<S> t0 = load3(row, ax0), t1 = load3(row, ax1);
    const S uxl = dot3(ax0, t0) + ax0.b1 * ule + ax0.b2 * uri;
    const S uxr = dot3(ax1, t1) + ax1.b1 * ule + ax1.b2 * uri;
    const S sxl = dot3(sx0, t0) + sx0.b1 * ule + sx0.b2 * uri;
    const S sxr = dot3(sx1, t1) + sx1.b1 * ule + sx1.b2 * uri;
    const S hy = S(__ldg(P.hy + j));
    const S du2dx = (hy * uxr) * uxr - (hy * uxl) * uxl;
    const S duvdy = vf1 * uy1 - vf0 * uy0;
    const S d2u = hy * (ire * sxr - ire * sxl) + gx * (ire * sy1 - ire * sy0);
    const S ypx = hy * S(__ldg(P.bc.pLe + j)) * pl + hy * S(__ldg(P.bc.pRi + j)) * pr;
    const double R = (double)(-(du2dx + duvdy) + d2u - ypx);
    const long long idx = (long long)j * P.Nux + i;
    const double hyd = __ldg(P.hy + j);
    const double oi = __ldg(P.rhy + j) * __ldg(P.rgxi + i);
    if (e.mode == 0 || e.mode == 2) {
      epilogue_stage(e, idx, oi, R);
    } else {
      const double *prow = e.p + (long long)j * P.Npx;
      const double g = -hyd * (gt.w0 * __ldg(prow + gt.c0) + gt.w1 * __ldg(prow + gt.c1) +
                               (gt.w2 != 0.0 ? gt.w2 * __ldg(prow + gt.c2) : 0.0));
      epi_residual(e, idx, oi, R, g);
    }
    uy0 = uy1;
    sy0 = sy1;
    vf0 = vf1;
  }
}

// ---------------------------------------------------------------------------
// v walker
template <typename S, typename TV>
__device__ void walk_v(const DevOps &P, const TV *__restrict__ u, const TV *__restrict__ v, const Epi &e,
                       int i, int j0, int j1) {
  if (i >= P.Nvx) return;
  j1 = min(j1, P.Nvy);
  if (j0 >= j1) return;
  const S ire = S(P.invRe);
  const XRow<S> vx0 = xrow<S>(P.AVX, i), vx1 = xrow<S>(P.AVX, i + 1);
  const XRowW<S> sv0 = xroww<S>(P.SVX, i), sv1 = xroww<S>(P.SVX, i + 1);
  const XRow<S> ux0 = xrow<S>(P.IUX, i), ux1 = xrow<S>(P.IUX, i + 1);
  const S hx = S(__ldg(P.hx + i));
  const S vLo = S(__ldg(P.bc.vLo_i + i)), vUp = S(__ldg(P.bc.vUp_i + i));
  const S pLo = S(__ldg(P.bc.pLo + i)), pUp = S(__ldg(P.bc.pUp + i));
  const S uLo0 = S(__ldg(P.bc.uLo + i)), uUp0 = S(__ldg(P.bc.uUp + i));
  const S uLo1 = S(__ldg(P.bc.uLo + i + 1)), uUp1 = S(__ldg(P.bc.uUp + i + 1));
  auto face = [&](int r, S &vy, S &sy) {
    const YRow<S> ay = yrow<S>(P.AVY, r);
    const double *__restrict__ sw = P.SVY.w + kT * r;
    const S s0 = S(__ldg(sw)), s1 = S(__ldg(sw + 1)), s2 = S(__ldg(sw + 2));
    const S f0 = S(__ldg(v + (long long)ay.c0 * P.Nvx + i));
    const S f1 = S(__ldg(v + (long long)ay.c1 * P.Nvx + i));
    const S f2 = (ay.w2 != S(0) || s2 != S(0)) ? S(__ldg(v + (long long)ay.c2 * P.Nvx + i)) : S(0);
    vy = ay.w0 * f0 + ay.w1 * f1 + ay.w2 * f2 + ay.b1 * vLo + ay.b2 * vUp;
    sy = s0 * f0 + s1 * f1 + s2 * f2 + S(__ldg(P.SVY.b1 + r)) * vLo + S(__ldg(P.SVY.b2 + r)) * vUp;
  };
  S vy0, sy0;
  face(j0, vy0, sy0);
  for (int j = j0; j < j1; ++j) {
    S vy1, sy1;
    face(j + 1, vy1, sy1);
    const TV *__restrict__ row = v + (long long)j * P.Nvx;
    const S vle = S(__ldg(P.bc.vLe_i + j)), vri = S(__ldg(P.bc.vRi_i + j));
    const Trip<S> t0 = load3(row, vx0), t1 = load3(row, vx1);
    const S vxl = dot3(vx0, t0) + vx0.b1 * vle + vx0.b2 * vri;
    const S vxr = dot3(vx1, t1) + vx1.b1 * vle + vx1.b2 * vri;
    const S svl = dot3(sv0, t0) + sv0.b1 * vle + sv0.b2 * vri;
    const S svr = dot3(sv1, t1) + sv1.b1 * vle + sv1.b2 * vri;
    // ubar at vx faces r = i, i+1 (row j of Iu_vx's y-factor)
    const YRow<S> iy = yrow<S>(P.IUY, j);
    S ufl = S(0), ufr = S(0);
    if (iy.w0 != S(0)) {
      const TV *ur = u + (long long)iy.c0 * P.Nux;
      ufl += iy.w0 * dot3(ux0, load3(ur, ux0));
      ufr += iy.w0 * dot3(ux1, load3(ur, ux1));
    }
    if (iy.w1 != S(0)) {
      const TV *ur = u + (long long)iy.c1 * P.Nux;
      ufl += iy.w1 * dot3(ux0, load3(ur, ux0));
      ufr += iy.w1 * dot3(ux1, load3(ur, ux1));
    }
    if (iy.w2 != S(0)) {
      const TV *ur = u + (long long)iy.c2 * P.Nux;
      ufl += iy.w2 * dot3(ux0, load3(ur, ux0));
      ufr += iy.w2 * dot3(ux1, load3(ur, ux1));
    }
    const S yle = S(__ldg(P.bc.YuLe + j)), yri = S(__ldg(P.bc.YuRi + j));
    ufl += iy.b1 * uLo0 + iy.b2 * uUp0 + ux0.b1 * yle + ux0.b2 * yri;
    ufr += iy.b1 * uLo1 + iy.b2 * uUp1 + ux1.b1 * yle + ux1.b2 * yri;
    const S duvdx = ufr * vxr - ufl * vxl;
    const S dv2dy = (hx * vy1) * vy1 - (hx * vy0) * vy0;
    const S d2v = S(__ldg(P.gyi + j)) * (ire * svr - ire * svl) + hx * (ire * sy1 - ire * sy0);
    const S ypy = hx * pLo * S(__ldg(P.pyl + j)) + hx * pUp * S(__ldg(P.pyu + j));
    const double R = (double)(-(duvdx + dv2dy) + d2v - ypy);
    const long long idx = P.Nu + (long long)j * P.Nvx + i;
    const double oi = __ldg(P.rgyi + j) * __ldg(P.rhx + i);
    if (e.mode == 0 || e.mode == 2) {
      epilogue_stage(e, idx, oi, R);
    } else {
      const YRow<double> gy = yrow<double>(P.MYT, j);
      const double g = -__ldg(P.hx + i) *
                       (gy.w0 * __ldg(e.p + (long long)gy.c0 * P.Npx + i) + gy.w1 * __ldg(e.p + (long long)gy.c1 * P.Npx + i) +
                        (gy.w2 != 0.0 ? gy.w2 * __ldg(e.p + (long long)gy.c2 * P.Npx + i) : 0.0));
      epi_residual(e, idx, oi, R, g);
    }
    vy0 = vy1;
    sy0 = sy1;
  }
}


// ---------------------------------------------------------------------------
// Fast walkers for interior tiles: every table row used by the tile is a
// regular two-point stencil (RegD) without boundary terms, so addresses follow
// from the column/row index and the weights come from the regular weight
// arrays; boundary values do not enter.
template <typename S>
__device__ __forceinline__ S rw(const double *w, int r) {
  return S(__ldg(w + r));
}

// y-direction weights and metrics of one tile's rows, staged in shared
// memory once per block (faces j0..j0+RUN, rows j0..j0+RUN-1): the walkers
// read them per row without a global-memory round trip.
template <int NR>
struct YRowsN {
  double auy0[NR + 1], auy1[NR + 1], suy0[NR + 1], suy1[NR + 1], ivy0[NR + 1], ivy1[NR + 1];
  double avy0[NR + 1], avy1[NR + 1], svy0[NR + 1], svy1[NR + 1];
  double hy[NR], rhy[NR], iuy0[NR], iuy1[NR], gyi[NR], rgyi[NR], myt0[NR], myt1[NR];
};
using YRows = YRowsN<RUN>;

template <int NR>
__device__ __forceinline__ void stage_yrows(const DevOps &P, int j0, YRowsN<NR> &Y) {
  const int t = threadIdx.x + blockDim.x * threadIdx.y;
  if (t <= NR) {
    const int r = j0 + t;
    Y.auy0[t] = __ldg(P.rAUY.w0 + r);
    Y.auy1[t] = __ldg(P.rAUY.w1 + r);
    Y.suy0[t] = __ldg(P.rSUY.w0 + r);
    Y.suy1[t] = __ldg(P.rSUY.w1 + r);
    Y.ivy0[t] = __ldg(P.rIVY.w0 + r);
    Y.ivy1[t] = __ldg(P.rIVY.w1 + r);
    Y.avy0[t] = __ldg(P.rAVY.w0 + r);
    Y.avy1[t] = __ldg(P.rAVY.w1 + r);
    Y.svy0[t] = __ldg(P.rSVY.w0 + r);
    Y.svy1[t] = __ldg(P.rSVY.w1 + r);
  }
  if (t < NR) {
    const int j = j0 + t;
    Y.hy[t] = __ldg(P.hy + j);
    Y.rhy[t] = __ldg(P.rhy + j);
    Y.iuy0[t] = __ldg(P.rIUY.w0 + j);
    Y.iuy1[t] = __ldg(P.rIUY.w1 + j);
    Y.gyi[t] = __ldg(P.gyi + j);
    Y.rgyi[t] = __ldg(P.rgyi + j);
    Y.myt0[t] = __ldg(P.rMYT.w0 + j);
    Y.myt1[t] = __ldg(P.rMYT.w1 + j);
  }
}

// Raw loads of one row of the u walker: the x-face values of row j, the
// field values of the y-face j+1 and the epilogue input; issued one row ahead
// of their use so each warp keeps two rows of loads in flight.
template <typename S>
struct URaw {
  S um, u0, up, f0, f1, va0, va1, vb0, vb1;
  double ep;
};

template <typename S, typename TV>
__device__ void fast_u(const DevOps &P, const TV *__restrict__ u, const TV *__restrict__ v, const Epi &e,
                       int i, int j0, int j1, const YRows &Y) {
  const S ire = S(P.invRe);
  // columns (modulo the row length for periodic wraps)
  const int cA0 = wrapn(i + P.rAUX.s, P.rAUX.n), cA1 = wrapn(cA0 + 1, P.rAUX.n), cA2 = wrapn(cA1 + 1, P.rAUX.n);
  const int cI0 = wrapn(i + P.rIVX.s, P.rIVX.n), cI1 = wrapn(cI0 + 1, P.rIVX.n);
  const S a00 = rw<S>(P.rAUX.w0, i), a01 = rw<S>(P.rAUX.w1, i);
  const S a10 = rw<S>(P.rAUX.w0, i + 1), a11 = rw<S>(P.rAUX.w1, i + 1);
  const S s00 = rw<S>(P.rSUX.w0, i), s01 = rw<S>(P.rSUX.w1, i);
  const S s10 = rw<S>(P.rSUX.w0, i + 1), s11 = rw<S>(P.rSUX.w1, i + 1);
  const S iv0 = rw<S>(P.rIVX.w0, i), iv1 = rw<S>(P.rIVX.w1, i);
  const S gx = S(__ldg(P.gxi + i));
  const double rgx = __ldg(P.rgxi + i);
  const bool twoA = P.rAUX.two, twoAy = P.rAUY.two, twoIx = P.rIVX.two, twoIy = P.rIVY.two;
  const int sAy = P.rAUY.s, sIy = P.rIVY.s;
  const long long Nux = P.Nux, Nvx = P.Nvx;
  // raw values of face r (u column at rows r+sAy, r+sAy+1; v rows r+sIy, r+sIy+1)
  auto load_face = [&](int r, URaw<S> &q) {
    const int ra = wrapn(r + sAy, P.rAUY.n);
    q.f0 = S(__ldg(u + (long long)ra * Nux + i));
    q.f1 = twoAy ? S(__ldg(u + (long long)wrapn(ra + 1, P.rAUY.n) * Nux + i)) : S(0);
    const int rv = wrapn(r + sIy, P.rIVY.n);
    const TV *vr = v + (long long)rv * Nvx;
    q.va0 = S(__ldg(vr + cI0));
    q.va1 = twoIx ? S(__ldg(vr + cI1)) : S(0);
    if (twoIy) {
      const TV *vr1 = v + (long long)wrapn(rv + 1, P.rIVY.n) * Nvx;
      q.vb0 = S(__ldg(vr1 + cI0));
      q.vb1 = twoIx ? S(__ldg(vr1 + cI1)) : S(0);
    } else {
      q.vb0 = q.vb1 = S(0);
    }
  };
  auto face = [&](int r, const URaw<S> &q, S &uy, S &sy, S &vf) {
    const int y = r - j0;
    uy = S(Y.auy0[y]) * q.f0 + S(Y.auy1[y]) * q.f1;
    sy = S(Y.suy0[y]) * q.f0 + S(Y.suy1[y]) * q.f1;
    vf = S(Y.ivy0[y]) * (iv0 * q.va0 + iv1 * q.va1) + S(Y.ivy1[y]) * (iv0 * q.vb0 + iv1 * q.vb1);
  };
  auto load_row = [&](int j, URaw<S> &q) {
    const TV *row = u + (long long)j * Nux;
    q.um = S(__ldg(row + cA0));
    q.u0 = S(__ldg(row + cA1));
    q.up = twoA ? S(__ldg(row + cA2)) : S(0);
    load_face(j + 1, q);
    const long long idx = (long long)j * Nux + i;
    q.ep = (e.mode == 0) ? __ldg(e.Vn + idx) : 0.0;
  };
  S uy0, sy0, vf0;
  {
    URaw<S> q0;
    load_face(j0, q0);
    face(j0, q0, uy0, sy0, vf0);
  }
  URaw<S> cur;
  load_row(j0, cur);
  for (int j = j0; j < j1; ++j) {
    URaw<S> nxt;
    if (j + 1 < j1) load_row(j + 1, nxt);
    S uy1, sy1, vf1;
    face(j + 1, cur, uy1, sy1, vf1);
    const S uxl = a00 * cur.um + a01 * cur.u0, uxr = a10 * cur.u0 + a11 * cur.up;
    const S sxl = s00 * cur.um + s01 * cur.u0, sxr = s10 * cur.u0 + s11 * cur.up;
    const double hyd = Y.hy[j - j0];
    const S hy = S(hyd);
    const S du2dx = (hy * uxr) * uxr - (hy * uxl) * uxl;
    const S duvdy = vf1 * uy1 - vf0 * uy0;
    const S d2u = hy * (ire * sxr - ire * sxl) + gx * (ire * sy1 - ire * sy0);
    const double R = (double)(-(du2dx + duvdy) + d2u);
    const long long idx = (long long)j * Nux + i;
    const double oi = Y.rhy[j - j0] * rgx;
    if (e.mode == 0) {
      const double k = oi * R;
      if (e.kV) e.kV[idx] = k;
      double vt = 0.0;
      for (int m = 0; m < e.nprev; ++m) vt += e.aprev[m] * __ldg(e.kprev[m] + idx);
      vt += e.aii * k;
      e.Wt[idx] = cur.ep * e.inv_dt + vt;
    } else if (e.mode == 2) {
      epi_stage32(e, idx, oi * R);
    } else {
      const double g = -hyd * reg_x(P.rMXT, i, e.p, (long long)j * P.Npx);
      epi_residual(e, idx, oi, R, g);
    }
    uy0 = uy1;
    sy0 = sy1;
    vf0 = vf1;
    cur = nxt;
  }
}

template <typename S>
struct VRaw {
  S vm, v0, vp, f0, f1, ua0, ua1, ua2, ub0, ub1, ub2;
  double ep;
};

template <typename S, typename TV>
__device__ void fast_v(const DevOps &P, const TV *__restrict__ u, const TV *__restrict__ v, const Epi &e,
                       int i, int j0, int j1, const YRows &Y) {
  const S ire = S(P.invRe);
  const int cV0 = wrapn(i + P.rAVX.s, P.rAVX.n), cV1 = wrapn(cV0 + 1, P.rAVX.n), cV2 = wrapn(cV1 + 1, P.rAVX.n);
  const int cU0 = wrapn(i + P.rIUX.s, P.rIUX.n), cU1 = wrapn(cU0 + 1, P.rIUX.n), cU2 = wrapn(cU1 + 1, P.rIUX.n);
  const S v00 = rw<S>(P.rAVX.w0, i), v01 = rw<S>(P.rAVX.w1, i);
  const S v10 = rw<S>(P.rAVX.w0, i + 1), v11 = rw<S>(P.rAVX.w1, i + 1);
  const S s00 = rw<S>(P.rSVX.w0, i), s01 = rw<S>(P.rSVX.w1, i);
  const S s10 = rw<S>(P.rSVX.w0, i + 1), s11 = rw<S>(P.rSVX.w1, i + 1);
  const S wu00 = rw<S>(P.rIUX.w0, i), wu01 = rw<S>(P.rIUX.w1, i);
  const S wu10 = rw<S>(P.rIUX.w0, i + 1), wu11 = rw<S>(P.rIUX.w1, i + 1);
  const double hxd = __ldg(P.hx + i);
  const double rhx = __ldg(P.rhx + i);
  const S hx = S(hxd);
  const bool twoV = P.rAVX.two, twoVy = P.rAVY.two, twoUx = P.rIUX.two, twoUy = P.rIUY.two;
  const int sVy = P.rAVY.s, sUy = P.rIUY.s;
  const long long Nux = P.Nux, Nvx = P.Nvx;
  auto load_face = [&](int r, VRaw<S> &q) {
    const int ra = wrapn(r + sVy, P.rAVY.n);
    q.f0 = S(__ldg(v + (long long)ra * Nvx + i));
    q.f1 = twoVy ? S(__ldg(v + (long long)wrapn(ra + 1, P.rAVY.n) * Nvx + i)) : S(0);
  };
  auto face = [&](int r, const VRaw<S> &q, S &vy, S &sy) {
    const int y = r - j0;
    vy = S(Y.avy0[y]) * q.f0 + S(Y.avy1[y]) * q.f1;
    sy = S(Y.svy0[y]) * q.f0 + S(Y.svy1[y]) * q.f1;
  };
  auto load_row = [&](int j, VRaw<S> &q) {
    const TV *row = v + (long long)j * Nvx;
    q.vm = S(__ldg(row + cV0));
    q.v0 = S(__ldg(row + cV1));
    q.vp = twoV ? S(__ldg(row + cV2)) : S(0);
    const int ru = wrapn(j + sUy, P.rIUY.n);
    const TV *ur = u + (long long)ru * Nux;
    q.ua0 = S(__ldg(ur + cU0));
    q.ua1 = S(__ldg(ur + cU1));
    q.ua2 = twoUx ? S(__ldg(ur + cU2)) : S(0);
    if (twoUy) {
      const TV *ur1 = u + (long long)wrapn(ru + 1, P.rIUY.n) * Nux;
      q.ub0 = S(__ldg(ur1 + cU0));
      q.ub1 = S(__ldg(ur1 + cU1));
      q.ub2 = twoUx ? S(__ldg(ur1 + cU2)) : S(0);
    } else {
      q.ub0 = q.ub1 = q.ub2 = S(0);
    }
    load_face(j + 1, q);
    const long long idx = P.Nu + (long long)j * Nvx + i;
    q.ep = (e.mode == 0) ? __ldg(e.Vn + idx) : 0.0;
  };
  S vy0, sy0;
  {
    VRaw<S> q0;
    load_face(j0, q0);
    face(j0, q0, vy0, sy0);
  }
  VRaw<S> cur;
  load_row(j0, cur);
  for (int j = j0; j < j1; ++j) {
    VRaw<S> nxt;
    if (j + 1 < j1) load_row(j + 1, nxt);
    S vy1, sy1;
    face(j + 1, cur, vy1, sy1);
    const S vxl = v00 * cur.vm + v01 * cur.v0, vxr = v10 * cur.v0 + v11 * cur.vp;
    const S svl = s00 * cur.vm + s01 * cur.v0, svr = s10 * cur.v0 + s11 * cur.vp;
    // ubar at vx faces i, i+1: IUY row j times IUX rows i, i+1
    const S la = wu00 * cur.ua0 + wu01 * cur.ua1, ra = wu10 * cur.ua1 + wu11 * cur.ua2;
    const S lb = wu00 * cur.ub0 + wu01 * cur.ub1, rb = wu10 * cur.ub1 + wu11 * cur.ub2;
    const S wy0 = S(Y.iuy0[j - j0]), wy1 = S(Y.iuy1[j - j0]);
    const S ufl = wy0 * la + wy1 * lb, ufr = wy0 * ra + wy1 * rb;
    const S duvdx = ufr * vxr - ufl * vxl;
    const S dv2dy = (hx * vy1) * vy1 - (hx * vy0) * vy0;
    const double gyd = Y.gyi[j - j0];
    const S d2v = S(gyd) * (ire * svr - ire * svl) + hx * (ire * sy1 - ire * sy0);
    const double R = (double)(-(duvdx + dv2dy) + d2v);
    const long long idx = P.Nu + (long long)j * Nvx + i;
    const double oi = Y.rgyi[j - j0] * rhx;
    if (e.mode == 0) {
      const double k = oi * R;
      if (e.kV) e.kV[idx] = k;
      double vt = 0.0;
      for (int m = 0; m < e.nprev; ++m) vt += e.aprev[m] * __ldg(e.kprev[m] + idx);
      vt += e.aii * k;
      e.Wt[idx] = cur.ep * e.inv_dt + vt;
    } else if (e.mode == 2) {
      epi_stage32(e, idx, oi * R);
    } else {
      // (G p)_v = -hx MYT p with the row's weights from shared memory
      const int c0 = wrapn(j + P.rMYT.s, P.rMYT.n);
      double gy = Y.myt0[j - j0] * __ldg(e.p + (long long)c0 * P.Npx + i);
      if (P.rMYT.two) gy += Y.myt1[j - j0] * __ldg(e.p + (long long)wrapn(c0 + 1, P.rMYT.n) * P.Npx + i);
      const double g = -hxd * gy;
      epi_residual(e, idx, oi, R, g);
    }
    vy0 = vy1;
    sy0 = sy1;
    cur = nxt;
  }
}

// ---------------------------------------------------------------------------
// Tiled walkers for the interior tiles of single contexts.  A block of 256
// threads takes one WX x RUN tile: the u and v rows it reads (the tile with a
// halo of at least two points on each side, three on the right) are copied
// into shared memory first with cp.async in 16-byte chunks -- every chunk a
// separate asynchronous copy, so a block has its whole tile in flight at
// once, and a periodic wrap is only a different source address per chunk --
// then each thread walks RUN/2 rows of one column (warps 0-3: u, 4-7: v; two
// row segments per column) with the arithmetic of fast_u / fast_v, reading
// its stencil values from shared memory.  Requirements (checked on the
// host): every shift of the regular rows in [-2, 1], and rows of u and v
// that start on 16-byte boundaries (Nux, Nvx, Nu multiples of 16 bytes /
// sizeof(TV)).
constexpr int kTileThreads = 256;
constexpr int kTileSeg = RUN / 2;   // rows per thread
constexpr int kTileRows = RUN + 5;  // staged rows j0-2 .. j0+RUN+2

// staged columns i0-HL .. : HL = one 16-byte chunk of halo on the left,
// at least WX+3-... on the right, a whole number of chunks per row
template <typename TV>
struct TileGeo {
  static constexpr int EPC = 16 / (int)sizeof(TV);            // elements per chunk
  static constexpr int HL = EPC;                              // left halo (>= 2)
  static constexpr int COLS = ((HL + WX + 3 + EPC - 1) / EPC) * EPC;
  static constexpr int CHUNKS = COLS / EPC;
};

template <typename TV>
struct TileSm {
  TV u[kTileRows][TileGeo<TV>::COLS];
  TV v[kTileRows][TileGeo<TV>::COLS];
};

__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Global operands of one row's epilogue, loaded a row ahead: the walker
// issues row j+1's loads before row j's stencil and stores, so their latency
// overlaps that work (issued after the stores, they would wait on them as
// possible aliases).  MODE 0: Vn and, for NP > 0, the earlier stages' kV;
// MODE 1: the two pressure values of the gradient.
// The earlier stages' kV are prefetched for NP <= INS2D_TILE_AHEAD_K only:
// with more, the two rows' operands exceed the 80-register budget of three
// blocks per SM and spill; those stages read them in place.
#ifndef INS2D_TILE_AHEAD_K
#define INS2D_TILE_AHEAD_K 1
#endif
template <int MODE, int NP>
struct EpiAhead {
  static constexpr bool K = MODE == 0 && NP > 0 && NP <= INS2D_TILE_AHEAD_K;
  double a, b;
  double kp[K ? NP : 1];
};
template <int MODE, int NP>
__device__ __forceinline__ void stage_ahead(const Epi &e, long long idx, EpiAhead<MODE, NP> &x) {
  x.a = __ldg(e.Vn + idx);
  if constexpr (EpiAhead<MODE, NP>::K) {
#pragma unroll
    for (int m = 0; m < NP; ++m) x.kp[m] = __ldg(e.kprev[m] + idx);
  }
}
// the FP64 stage epilogue from prefetched operands: kV = k and
// Wt = Vn/dt + (sum over the earlier stages a_m kV_m + aii k) (time_ERK.m:96-101);
// NP >= 0: that many earlier stages, unrolled; NP < 0: e.nprev
template <int NP>
__device__ __forceinline__ void stage_store(const Epi &e, long long idx, double k, const EpiAhead<0, NP> &x) {
  if (e.kV) e.kV[idx] = k;
  double vt = 0.0;
  if constexpr (EpiAhead<0, NP>::K) {
#pragma unroll
    for (int m = 0; m < NP; ++m) vt += e.aprev[m] * x.kp[m];
  } else if constexpr (NP >= 0) {
#pragma unroll
    for (int m = 0; m < NP; ++m) vt += e.aprev[m] * __ldg(e.kprev[m] + idx);
  } else {
    for (int m = 0; m < e.nprev; ++m) vt += e.aprev[m] * __ldg(e.kprev[m] + idx);
  }
  e.Wt[idx] = x.a * e.inv_dt + (vt + e.aii * k);
}

// MODE 0: FP64-storage stage, 1: residual, 2: FP32-storage stage
template <typename S, int MODE, typename TV, int NP>
__device__ void tile_u(const DevOps &P, const TileSm<TV> &T, const Epi &e, int i, int i0, int j0, int ja, int jb,
                       const YRowsN<RUN> &Y) {
  const S ire = S(P.invRe);
  const int ci = i - i0 + TileGeo<TV>::HL;  // shared-memory column of u(i, .)
  const int cA0 = ci + P.rAUX.s, cA1 = cA0 + 1, cA2 = cA1 + 1;
  const int cI0 = ci + P.rIVX.s, cI1 = cI0 + 1;
  const S a00 = rw<S>(P.rAUX.w0, i), a01 = rw<S>(P.rAUX.w1, i);
  const S a10 = rw<S>(P.rAUX.w0, i + 1), a11 = rw<S>(P.rAUX.w1, i + 1);
  const S s00 = rw<S>(P.rSUX.w0, i), s01 = rw<S>(P.rSUX.w1, i);
  const S s10 = rw<S>(P.rSUX.w0, i + 1), s11 = rw<S>(P.rSUX.w1, i + 1);
  const S iv0 = rw<S>(P.rIVX.w0, i), iv1 = rw<S>(P.rIVX.w1, i);
  const S gx = S(__ldg(P.gxi + i));
  const double rgx = __ldg(P.rgxi + i);
  const bool twoA = P.rAUX.two, twoAy = P.rAUY.two, twoIx = P.rIVX.two, twoIy = P.rIVY.two;
  const int sAy = P.rAUY.s - j0 + 2, sIy = P.rIVY.s - j0 + 2;  // shared-memory row of field row r: r + s
  auto face = [&](int r, S &uy, S &sy, S &vf) {
    const int y = r - j0;
    const int ra = r + sAy, rv = r + sIy;
    const S f0 = S(T.u[ra][ci]);
    const S f1 = twoAy ? S(T.u[ra + 1][ci]) : S(0);
    const S va0 = S(T.v[rv][cI0]);
    const S va1 = twoIx ? S(T.v[rv][cI1]) : S(0);
    S vb0 = S(0), vb1 = S(0);
    if (twoIy) {
      vb0 = S(T.v[rv + 1][cI0]);
      vb1 = twoIx ? S(T.v[rv + 1][cI1]) : S(0);
    }
    uy = S(Y.auy0[y]) * f0 + S(Y.auy1[y]) * f1;
    sy = S(Y.suy0[y]) * f0 + S(Y.suy1[y]) * f1;
    vf = S(Y.ivy0[y]) * (iv0 * va0 + iv1 * va1) + S(Y.ivy1[y]) * (iv0 * vb0 + iv1 * vb1);
  };
  // pressure gradient columns and weights (residual mode)
  const int pc0 = MODE == 1 ? wrapn(i + P.rMXT.s, P.rMXT.n) : 0, pc1 = MODE == 1 ? wrapn(pc0 + 1, P.rMXT.n) : 0;
  const bool twoG = MODE == 1 && P.rMXT.two;
  const double gw0 = MODE == 1 ? __ldg(P.rMXT.w0 + i) : 0.0, gw1 = twoG ? __ldg(P.rMXT.w1 + i) : 0.0;
  auto ahead = [&](int j, EpiAhead<MODE, NP> &x) {
    if constexpr (MODE == 0) {
      stage_ahead<MODE, NP>(e, (long long)j * P.Nux + i, x);
    } else if constexpr (MODE == 1) {
      const double *pr = e.p + (long long)j * P.Npx;
      x.a = __ldg(pr + pc0);
      x.b = twoG ? __ldg(pr + pc1) : 0.0;
    }
  };
  EpiAhead<MODE, NP> nxt;
  if constexpr (MODE != 2) ahead(ja, nxt);
  S uy0, sy0, vf0;
  face(ja, uy0, sy0, vf0);
#pragma unroll 2
  for (int j = ja; j < jb; ++j) {
    const EpiAhead<MODE, NP> cur = nxt;
    if constexpr (MODE != 2)
      if (j + 1 < jb) ahead(j + 1, nxt);
    S uy1, sy1, vf1;
    face(j + 1, uy1, sy1, vf1);
    const int rr = j - j0 + 2;
    const S um = S(T.u[rr][cA0]), u0 = S(T.u[rr][cA1]), up = twoA ? S(T.u[rr][cA2]) : S(0);
    const S uxl = a00 * um + a01 * u0, uxr = a10 * u0 + a11 * up;
    const S sxl = s00 * um + s01 * u0, sxr = s10 * u0 + s11 * up;
    const double hyd = Y.hy[j - j0];
    const S hy = S(hyd);
    const S du2dx = (hy * uxr) * uxr - (hy * uxl) * uxl;
    const S duvdy = vf1 * uy1 - vf0 * uy0;
    const S d2u = hy * (ire * sxr - ire * sxl) + gx * (ire * sy1 - ire * sy0);
    const double R = (double)(-(du2dx + duvdy) + d2u);
    const long long idx = (long long)j * P.Nux + i;
    const double oi = Y.rhy[j - j0] * rgx;
    if constexpr (MODE == 0) {
      stage_store<NP>(e, idx, oi * R, cur);
    } else if constexpr (MODE == 2) {
      epi_stage32<NP>(e, idx, oi * R);
    } else {
      double gp = gw0 * cur.a;
      if (twoG) gp += gw1 * cur.b;
      epi_residual(e, idx, oi, R, -hyd * gp);
    }
    uy0 = uy1;
    sy0 = sy1;
    vf0 = vf1;
  }
}

template <typename S, int MODE, typename TV, int NP>
__device__ void tile_v(const DevOps &P, const TileSm<TV> &T, const Epi &e, int i, int i0, int j0, int ja, int jb,
                       const YRowsN<RUN> &Y) {
  const S ire = S(P.invRe);
  const int ci = i - i0 + TileGeo<TV>::HL;
  const int cV0 = ci + P.rAVX.s, cV1 = cV0 + 1, cV2 = cV1 + 1;
  const int cU0 = ci + P.rIUX.s, cU1 = cU0 + 1, cU2 = cU1 + 1;
  const S v00 = rw<S>(P.rAVX.w0, i), v01 = rw<S>(P.rAVX.w1, i);
  const S v10 = rw<S>(P.rAVX.w0, i + 1), v11 = rw<S>(P.rAVX.w1, i + 1);
  const S s00 = rw<S>(P.rSVX.w0, i), s01 = rw<S>(P.rSVX.w1, i);
  const S s10 = rw<S>(P.rSVX.w0, i + 1), s11 = rw<S>(P.rSVX.w1, i + 1);
  const S wu00 = rw<S>(P.rIUX.w0, i), wu01 = rw<S>(P.rIUX.w1, i);
  const S wu10 = rw<S>(P.rIUX.w0, i + 1), wu11 = rw<S>(P.rIUX.w1, i + 1);
  const double hxd = __ldg(P.hx + i);
  const double rhx = __ldg(P.rhx + i);
  const S hx = S(hxd);
  const bool twoV = P.rAVX.two, twoVy = P.rAVY.two, twoUx = P.rIUX.two, twoUy = P.rIUY.two;
  const int sVy = P.rAVY.s - j0 + 2, sUy = P.rIUY.s - j0 + 2;
  auto face = [&](int r, S &vy, S &sy) {
    const int y = r - j0;
    const int ra = r + sVy;
    const S f0 = S(T.v[ra][ci]);
    const S f1 = twoVy ? S(T.v[ra + 1][ci]) : S(0);
    vy = S(Y.avy0[y]) * f0 + S(Y.avy1[y]) * f1;
    sy = S(Y.svy0[y]) * f0 + S(Y.svy1[y]) * f1;
  };
  const bool twoG = MODE == 1 && P.rMYT.two;
  auto ahead = [&](int j, EpiAhead<MODE, NP> &x) {
    if constexpr (MODE == 0) {
      stage_ahead<MODE, NP>(e, P.Nu + (long long)j * P.Nvx + i, x);
    } else if constexpr (MODE == 1) {
      const int c0 = wrapn(j + P.rMYT.s, P.rMYT.n);
      x.a = __ldg(e.p + (long long)c0 * P.Npx + i);
      x.b = twoG ? __ldg(e.p + (long long)wrapn(c0 + 1, P.rMYT.n) * P.Npx + i) : 0.0;
    }
  };
  EpiAhead<MODE, NP> nxt;
  if constexpr (MODE != 2) ahead(ja, nxt);
  S vy0, sy0;
  face(ja, vy0, sy0);
#pragma unroll 2
  for (int j = ja; j < jb; ++j) {
    const EpiAhead<MODE, NP> cur = nxt;
    if constexpr (MODE != 2)
      if (j + 1 < jb) ahead(j + 1, nxt);
    S vy1, sy1;
    face(j + 1, vy1, sy1);
    const int rr = j - j0 + 2;
    const S vm = S(T.v[rr][cV0]), v0 = S(T.v[rr][cV1]), vp = twoV ? S(T.v[rr][cV2]) : S(0);
    const int ru = j + sUy;
    const S ua0 = S(T.u[ru][cU0]), ua1 = S(T.u[ru][cU1]), ua2 = twoUx ? S(T.u[ru][cU2]) : S(0);
    S ub0 = S(0), ub1 = S(0), ub2 = S(0);
    if (twoUy) {
      ub0 = S(T.u[ru + 1][cU0]);
      ub1 = S(T.u[ru + 1][cU1]);
      ub2 = twoUx ? S(T.u[ru + 1][cU2]) : S(0);
    }
    const S vxl = v00 * vm + v01 * v0, vxr = v10 * v0 + v11 * vp;
    const S svl = s00 * vm + s01 * v0, svr = s10 * v0 + s11 * vp;
    const S la = wu00 * ua0 + wu01 * ua1, ra = wu10 * ua1 + wu11 * ua2;
    const S lb = wu00 * ub0 + wu01 * ub1, rb = wu10 * ub1 + wu11 * ub2;
    const S wy0 = S(Y.iuy0[j - j0]), wy1 = S(Y.iuy1[j - j0]);
    const S ufl = wy0 * la + wy1 * lb, ufr = wy0 * ra + wy1 * rb;
    const S duvdx = ufr * vxr - ufl * vxl;
    const S dv2dy = (hx * vy1) * vy1 - (hx * vy0) * vy0;
    const double gyd = Y.gyi[j - j0];
    const S d2v = S(gyd) * (ire * svr - ire * svl) + hx * (ire * sy1 - ire * sy0);
    const double R = (double)(-(duvdx + dv2dy) + d2v);
    const long long idx = P.Nu + (long long)j * P.Nvx + i;
    const double oi = Y.rgyi[j - j0] * rhx;
    if constexpr (MODE == 0) {
      stage_store<NP>(e, idx, oi * R, cur);
    } else if constexpr (MODE == 2) {
      epi_stage32<NP>(e, idx, oi * R);
    } else {
      double gy = Y.myt0[j - j0] * cur.a;
      if (twoG) gy += Y.myt1[j - j0] * cur.b;
      epi_residual(e, idx, oi, R, -hxd * gy);
    }
    vy0 = vy1;
    sy0 = sy1;
  }
}

// Copies the u and v rows j0-2 .. j0+RUN+2, columns i0-HL .. (wrapped) of
// the velocity-sized field V into T with cp.async: a thread keeps one 16-byte
// chunk column of one field and walks its rows RSTEP apart (tiles are whole,
// so a staged coordinate wraps once at most).
template <typename TV>
__device__ __forceinline__ void stage_tile_fields(const DevOps &P, const TV *__restrict__ V, TileSm<TV> &T, int i0,
                                                  int j0, int tid) {
  using G = TileGeo<TV>;
  constexpr int CH2 = 2 * G::CHUNKS, RSTEP = kTileThreads / CH2;
  if (tid >= RSTEP * CH2) return;
  const int q = tid % CH2, f = q >= G::CHUNKS, ch = q - f * G::CHUNKS;
  const int nx = f ? P.Nvx : P.Nux, ny = f ? P.Nvy : P.Nuy;
  const TV *src = V + (f ? P.Nu : 0LL) + wrapn(i0 - G::HL + G::EPC * ch, nx);
  TV *dst = (f ? &T.v[0][0] : &T.u[0][0]) + G::EPC * ch;
  int r = tid / CH2;
  int gr = wrapn(j0 - 2 + r, ny);
  for (; r < kTileRows; r += RSTEP) {
    cp_async16(dst + r * G::COLS, src + (long long)gr * nx);
    gr += RSTEP;
    if (gr >= ny) gr -= ny;
  }
}

#ifndef INS2D_TILE_MINB
#define INS2D_TILE_MINB 3
#endif
// MODE 0-2 as tile_u / tile_v
template <typename S, int MODE, typename TV, int NP>
__global__ void __launch_bounds__(kTileThreads, INS2D_TILE_MINB)
    k_walk_tile(const __grid_constant__ DevOps P, const TV *__restrict__ V, const __grid_constant__ Epi e) {
  __shared__ __align__(16) TileSm<TV> T;
  __shared__ YRowsN<RUN> Y;
  pdl_wait();
  pdl_trigger();
  const int bx = P.fbx0 + blockIdx.x, by = P.fby0 + blockIdx.y;
  const int i0 = bx * WX, j0 = by * RUN;
  const int tid = threadIdx.x + WX * threadIdx.y;
  stage_tile_fields<TV>(P, V, T, i0, j0, tid);
  stage_yrows(P, j0, Y);
  cp_async_wait_all();
  __syncthreads();
  const int i = i0 + threadIdx.x;
  const int seg = threadIdx.y & 1;
  const int ja = j0 + seg * kTileSeg, jb = ja + kTileSeg;
  if (threadIdx.y < 2)
    tile_u<S, MODE, TV, NP>(P, T, e, i, i0, j0, ja, jb, Y);
  else
    tile_v<S, MODE, TV, NP>(P, T, e, i, i0, j0, ja, jb, Y);
}

// one WX x RUN tile (bx, by): u walkers in warps with threadIdx.y == 0, v in 1
template <typename S, typename TV>
__device__ __forceinline__ void tile_fast(const DevOps &P, const TV *__restrict__ V, const Epi &e, int bx, int by) {
  __shared__ YRows Y;
  const int i = bx * WX + threadIdx.x;
  const int j0 = by * RUN, j1 = j0 + RUN;
  const TV *u = V, *v = V + P.Nu;
  stage_yrows(P, j0, Y);
  __syncthreads();
  if (threadIdx.y == 0)
    fast_u<S, TV>(P, u, v, e, i, j0, j1, Y);
  else
    fast_v<S, TV>(P, u, v, e, i, j0, j1, Y);
}
template <typename S, typename TV>
__device__ __forceinline__ void tile_generic(const DevOps &P, const TV *__restrict__ V, const Epi &e, int bx,
                                             int by) {
  const int i = bx * WX + threadIdx.x;
  const int j0 = by * RUN, j1 = j0 + RUN;
  const TV *u = V, *v = V + P.Nu;
  if (threadIdx.y == 0)
    walk_u<S, TV>(P, u, v, e, i, j0, j1);
  else
    walk_v<S, TV>(P, u, v, e, i, j0, j1);
}

template <typename S, typename TV>
__global__ void __launch_bounds__(WX * 2, INS2D_WALK_MINB) k_walk_fast(const __grid_constant__ DevOps P, const TV *__restrict__ V,
                                                      const __grid_constant__ Epi e) {
  tile_fast<S, TV>(P, V, e, P.fbx0 + blockIdx.x, P.fby0 + blockIdx.y);
}

template <typename S, typename TV>
__global__ void __launch_bounds__(WX * 2) k_walk(const __grid_constant__ DevOps P, const TV *__restrict__ V,
                                                 const __grid_constant__ Epi e) {
  if ((int)blockIdx.x >= P.fbx0 && (int)blockIdx.x < P.fbx1 && (int)blockIdx.y >= P.fby0 &&
      (int)blockIdx.y < P.fby1)
    return;  // interior tile: handled by k_walk_fast / k_walk_tile
  tile_generic<S, TV>(P, V, e, blockIdx.x, blockIdx.y);
}

// --- ensembles: one launch over the tiles of all member grids ------------------
// The member's descriptor is copied to shared memory; the stage's pointers
// come from the member's arrays.
__device__ __forceinline__ void copy_words(void *dst, const void *src, int bytes) {
  const int tid = threadIdx.x + blockDim.x * threadIdx.y, nt = blockDim.x * blockDim.y;
  for (int k = tid; k < bytes / 8; k += nt) ((long long *)dst)[k] = ((const long long *)src)[k];
}

__device__ __forceinline__ const double *ens_epi(const EnsMemberD &M, const EnsWalk &w, Epi &e) {
  e = Epi{};
  e.mode = w.mode;
  if (w.mode == 0) {
    e.Vn = M.V;
    e.kV = w.store ? M.kV[w.stage] : nullptr;
    for (int q = 0; q < w.nprev; ++q) {
      e.kprev[q] = M.kV[w.kidx[q]];
      e.aprev[q] = w.aprev[q];
    }
    e.nprev = w.nprev;
    e.aii = w.aii;
    e.inv_dt = 1.0 / M.dt;
    e.Wt = M.Wt;
    return w.use_vs ? M.Vs : M.V;
  }
  e.p = M.p;
  e.w = M.wres;
  e.kV_next = w.cache ? M.kV[0] : nullptr;
  return M.V;
}

template <typename S, bool FAST>
__device__ __forceinline__ void walk_ens_body(const EnsMemberD *__restrict__ mem, const int4 *__restrict__ work,
                                              const EnsWalk &w) {
  __shared__ __align__(16) DevOps sP;
  __shared__ __align__(16) Epi sE;
  __shared__ const double *sV;
  const int4 it = work[blockIdx.x];
  const EnsMemberD &M = mem[it.x];
  copy_words(&sP, &M.P, (int)sizeof(DevOps));
  if (threadIdx.x == 0 && threadIdx.y == 0) sV = ens_epi(M, w, sE);
  __syncthreads();
  if (FAST)
    tile_fast<S, double>(sP, sV, sE, it.y, it.z);
  else
    tile_generic<S, double>(sP, sV, sE, it.y, it.z);
}

template <typename S>
__global__ void __launch_bounds__(WX * 2, INS2D_WALK_MINB) k_walk_ens_fast(const EnsMemberD *__restrict__ mem,
                                                                          const int4 *__restrict__ work,
                                                                          const __grid_constant__ EnsWalk w) {
  walk_ens_body<S, true>(mem, work, w);
}
template <typename S>
__global__ void __launch_bounds__(WX * 2) k_walk_ens_gen(const EnsMemberD *__restrict__ mem,
                                                         const int4 *__restrict__ work,
                                                         const __grid_constant__ EnsWalk w) {
  walk_ens_body<S, false>(mem, work, w);
}

// MODE 0 and 2 with the count of earlier stages as a template argument (0..3
// unrolled, more at run time)
template <typename S, int MODE, typename TV>
void launch_tile(const DevOps &P, const TV *V, const Epi &e, cudaStream_t s) {
  const dim3 gf(P.fbx1 - P.fbx0, P.fby1 - P.fby0), tb(WX, kTileThreads / WX);
  if constexpr (MODE == 0 || MODE == 2) {
    switch (e.nprev) {
      case 0: launch_k(k_walk_tile<S, MODE, TV, 0>, gf, tb, 0, s, P, V, e); break;
      case 1: launch_k(k_walk_tile<S, MODE, TV, 1>, gf, tb, 0, s, P, V, e); break;
      case 2: launch_k(k_walk_tile<S, MODE, TV, 2>, gf, tb, 0, s, P, V, e); break;
      case 3: launch_k(k_walk_tile<S, MODE, TV, 3>, gf, tb, 0, s, P, V, e); break;
      default: launch_k(k_walk_tile<S, MODE, TV, -1>, gf, tb, 0, s, P, V, e); break;
    }
  } else {
    launch_k(k_walk_tile<S, MODE, TV, -1>, gf, tb, 0, s, P, V, e);
  }
}

template <typename S, typename TV>
void launch_walk_t(const DevOps &P, const TV *V, const Epi &e, cudaStream_t s) {
  const int nx = P.Nux > P.Nvx ? P.Nux : P.Nvx;
  const int ny = P.Nuy > P.Nvy ? P.Nuy : P.Nvy;
  dim3 g((nx + WX - 1) / WX, (ny + RUN - 1) / RUN);
  const bool has_fast = P.fbx1 > P.fbx0 && P.fby1 > P.fby0;
  const bool tiled = (sizeof(TV) == 8 ? P.tile_ok : P.tile_ok32) && (((uintptr_t)V & 15) == 0);
  if (has_fast) {
    const dim3 gf(P.fbx1 - P.fbx0, P.fby1 - P.fby0);
    if (tiled) {
      if (e.mode == 0)
        launch_tile<S, 0, TV>(P, V, e, s);
      else if (e.mode == 2)
        launch_tile<S, 2, TV>(P, V, e, s);
      else
        launch_tile<S, 1, TV>(P, V, e, s);  // residual and F
    } else {
      k_walk_fast<S, TV><<<gf, dim3(WX, 2), 0, s>>>(P, V, e);
    }
  }
  if (!P.all_fast) k_walk<S, TV><<<g, dim3(WX, 2), 0, s>>>(P, V, e);
}

// FP64 contexts: FP64 fields, FP64 arithmetic; FP32-stencil contexts: FP32
// arithmetic on FP64 fields (V32 == nullptr) or on the FP32 stage velocity
void launch_walk(const DevOps &P, const double *V, const float *V32, const Epi &e, bool fp32, cudaStream_t s) {
  if (V32)
    launch_walk_t<float, float>(P, V32, e, s);
  else if (fp32)
    launch_walk_t<float, double>(P, V, e, s);
  else
    launch_walk_t<double, double>(P, V, e, s);
}

}  // namespace

// The tiled walkers' shared memory is static (below 48 KB per block): no
// opt-in is needed; kept so the context's set-up has one place to prepare the
// walkers on its device.
cudaError_t walker_prepare() { return cudaSuccess; }

// The rectangle of tiles whose every column and row lies in the regular
// ranges the fast walkers need (both walkers of a block must qualify).
void walker_rectangle(DevOps &P) {
  auto in = [](const RegD &r, int a, int b) { return a >= r.lo && b < r.hi; };  // rows a..b inclusive
  const int nx = P.Nux > P.Nvx ? P.Nux : P.Nvx;
  const int ny = P.Nuy > P.Nvy ? P.Nuy : P.Nvy;
  const int nbx = (nx + WX - 1) / WX, nby = (ny + RUN - 1) / RUN;
  int bx0 = -1, bx1 = -1, by0 = -1, by1 = -1;
  for (int bx = 0; bx < nbx; ++bx) {
    const int i0 = bx * WX, i1 = i0 + WX;  // columns i0..i1-1
    const bool ok = i1 <= P.Nux && i1 <= P.Nvx && in(P.rAUX, i0, i1) && in(P.rIVX, i0, i1 - 1) &&
                    in(P.rMXT, i0, i1 - 1) && in(P.rAVX, i0, i1) && in(P.rIUX, i0, i1);
    if (ok) {
      if (bx0 < 0) bx0 = bx;
      bx1 = bx + 1;
    }
  }
  for (int by = 0; by < nby; ++by) {
    const int j0 = by * RUN, j1 = j0 + RUN;  // rows j0..j1-1
    const bool ok = j1 <= P.Nuy && j1 <= P.Nvy && in(P.rAUY, j0, j1) && in(P.rIVY, j0, j1) && in(P.rAVY, j0, j1) &&
                    in(P.rIUY, j0, j1 - 1) && in(P.rMYT, j0, j1 - 1);
    if (ok) {
      if (by0 < 0) by0 = by;
      by1 = by + 1;
    }
  }
  if (bx0 < 0 || by0 < 0) bx0 = bx1 = by0 = by1 = 0;
  P.all_fast = bx0 == 0 && bx1 == nbx && by0 == 0 && by1 == nby && bx1 > bx0 && by1 > by0;
  // the tiled walkers stage columns i0-2 .. i0+WX+3 and rows j0-2 .. j0+RUN+2
  // in 16-byte chunks: every shift must keep the stencil inside that halo
  auto shift_ok = [](const RegD &r) { return r.s >= -2 && r.s <= 1; };
  P.tile_ok = shift_ok(P.rAUX) && shift_ok(P.rAUY) && shift_ok(P.rIVX) && shift_ok(P.rIVY) && shift_ok(P.rAVX) &&
              shift_ok(P.rAVY) && shift_ok(P.rIUX) && shift_ok(P.rIUY) && P.Nux % 2 == 0 && P.Nvx % 2 == 0 &&
              P.Nu % 2 == 0;
  P.tile_ok32 = P.tile_ok && P.Nux % 4 == 0 && P.Nvx % 4 == 0 && P.Nu % 4 == 0;
  P.fbx0 = bx0;
  P.fbx1 = bx1;
  P.fby0 = by0;
  P.fby1 = by1;
}

void walk_tiles(const DevOps &P, int member, std::vector<int4> &fast, std::vector<int4> &gen) {
  const int nx = P.Nux > P.Nvx ? P.Nux : P.Nvx;
  const int ny = P.Nuy > P.Nvy ? P.Nuy : P.Nvy;
  const int nbx = (nx + WX - 1) / WX, nby = (ny + RUN - 1) / RUN;
  for (int by = 0; by < nby; ++by)
    for (int bx = 0; bx < nbx; ++bx) {
      const bool f = bx >= P.fbx0 && bx < P.fbx1 && by >= P.fby0 && by < P.fby1;
      (f ? fast : gen).push_back(make_int4(member, bx, by, 0));
    }
}

void launch_walk_ens(const EnsMemberD *mem, const int4 *fast, int nfast, const int4 *gen, int ngen, const EnsWalk &w,
                     bool fp32, cudaStream_t s) {
  if (nfast > 0) {
    if (fp32)
      k_walk_ens_fast<float><<<nfast, dim3(WX, 2), 0, s>>>(mem, fast, w);
    else
      k_walk_ens_fast<double><<<nfast, dim3(WX, 2), 0, s>>>(mem, fast, w);
  }
  if (ngen > 0) {
    if (fp32)
      k_walk_ens_gen<float><<<ngen, dim3(WX, 2), 0, s>>>(mem, gen, w);
    else
      k_walk_ens_gen<double><<<ngen, dim3(WX, 2), 0, s>>>(mem, gen, w);
  }
}

void launch_stage(const DevOps &P, const StageArgs &a, bool fp32, cudaStream_t s) {
  Epi e{};
  e.mode = a.store32 ? 2 : 0;
  e.Vn = a.Vn;
  e.kV = a.kV;
  for (int m = 0; m < a.nprev; ++m) {
    e.kprev[m] = a.kprev[m];
    e.kprev32[m] = a.kprev32[m];
    e.aprev[m] = a.aprev[m];
  }
  e.nprev = a.nprev;
  e.aii = a.aii;
  e.inv_dt = a.inv_dt;
  e.Wt = a.Wt;
  e.kV32 = a.kV32;
  e.Vt32 = a.Vt32;
  launch_walk(P, a.V, a.V32, e, fp32, s);
}

void launch_F_walk(const DevOps &P, const double *V, const double *p, double *F_out, cudaStream_t s) {
  Epi e{};
  e.mode = 3;
  e.p = p;
  e.w = F_out;
  launch_walk(P, V, nullptr, e, false, s);
}

void launch_residual(const DevOps &P, const double *V, const double *p, double *w, double *kV_next,
                     float *kV_next32, bool fp32, cudaStream_t s) {
  Epi e{};
  e.mode = 1;
  e.p = p;
  e.w = w;
  e.kV_next = kV_next;
  e.kV_next32 = kV_next32;
  launch_walk(P, V, nullptr, e, fp32, s);
}

}  // namespace ins2d
