// Device descriptor and per-point stencil functions of the INS2D operators.
//
// Each operator of the reference is a Kronecker product of 1D operators; the
// 1D factors arrive as row tables (kTab entries per row, see setup.hpp) and
// the boundary-condition vectors as sums of outer products of 1D vectors
// (set_bc_vectors.m evaluated factor-wise).  Fields are stored as in the
// reference: u(i,j) at i + j*Nux, v(i,j) at i + j*Nvx, p(i,j) at i + j*Npx.
#pragma once

#include <cstdint>

namespace ins2d {

constexpr int kT = 3;

struct Tab {
  const int32_t *c;   // nrows*kT column indices
  const double *w;    // nrows*kT weights (0 for padding)
  const double *b1;   // nrows, boundary coefficient of the first BC value
  const double *b2;   // nrows, boundary coefficient of the second BC value
};

// Boundary values at the current time (set_bc_vectors.m:52-85 samples) and
// derived 1D products (see ctx.cu upload_bc).
struct BcVals {
  const double *uLo, *uUp;        // Nx+1
  const double *uLo_i, *uUp_i;    // Nux
  const double *uLe_i, *uRi_i;    // Ny
  const double *vLe, *vRi;        // Ny+1
  const double *vLo_i, *vUp_i;    // Nx
  const double *vLe_i, *vRi_i;    // Nvy
  const double *XvLo, *XvUp;      // Nux: (Iv_uy x-factor) * vLo_i / vUp_i
  const double *YuLe, *YuRi;      // Nvy: (Iu_vx y-factor) * uLe_i / uRi_i
  const double *pLe, *pRi;        // Ny
  const double *pLo, *pUp;        // Nx
  const double *dudtLe_i, *dudtRi_i;  // Ny
  const double *dvdtLo_i, *dvdtUp_i;  // Nx
};

// Regular interior of a 1D table: rows [lo,hi) are w0[r]*f[r+s] + w1[r]*f[r+s+1]
// without boundary terms (two = 0: w1 is zero in the whole range).
struct RegD {
  int s, lo, hi, two, n;  // n: column count (indices wrap modulo n)
  const double *w0, *w1;
};
__device__ __forceinline__ int wrapn(int c, int n) { return c < 0 ? c + n : (c >= n ? c - n : c); }

// Programmatic dependent launch (kernels started by launch_k with the
// attribute set): pdl_wait returns once the previous kernel in the stream has
// completed and its writes are visible; it is a no-op for a plain launch.  A
// kernel that calls it touches no global memory before it.  pdl_trigger,
// after the wait, lets the next kernel's blocks be scheduled while this
// kernel's last blocks run (they wait in their own pdl_wait).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

struct DevOps {
  int Nx, Ny, Nux, Nuy, Nvx, Nvy, Npx, Npy;
  long long Nu, Nv, Np;
  double invRe;
  Tab AUX, SUX, AUY, SUY, IVX, IVY, MX, MXT;
  Tab AVX, SVX, AVY, SVY, IUX, IUY, MY, MYT;
  Tab TX, TY;
  const double *TXd, *TYd;
  const double *hx, *hy, *gxi, *gyi;
  const double *rhx, *rhy, *rgxi, *rgyi;  // reciprocals (Om^-1 = 1/(hy gxi) as (1/hy)(1/gxi))
  const double *pxl, *pxr, *pyl, *pyu;
  const double *fft_ax, *fft_ay;
  double fft_dxdy;
  BcVals bc;
  // fast-walker data: regular ranges (pairs share ranges) and the block
  // rectangle [fbx0,fbx1) x [fby0,fby1) whose tiles lie inside all of them
  RegD rAUX, rSUX, rAUY, rSUY, rIVX, rIVY, rMXT, rAVX, rSVX, rAVY, rSVY, rIUX, rIUY, rMYT, rMX, rMY;
  int fbx0, fbx1, fby0, fby1;
  int tile_ok;    // the interior tiles may use the shared-memory tiled walkers (FP64 fields)
  int tile_ok32;  // ... on FP32 fields
  int all_fast;   // the rectangle holds every tile of the grid (no table-walker tiles)
  int nsm;        // multiprocessors of the device (persistent launches)
};

// --- 1D table application ---------------------------------------------------
// x-direction: sum_k w(r,k) f[base + c(r,k)]
template <typename S>
__device__ __forceinline__ S tab_x(const Tab &T, int r, const double *__restrict__ f, long long base) {
  const int32_t *c = T.c + kT * r;
  const double *w = T.w + kT * r;
  return S(__ldg(w)) * S(__ldg(f + base + __ldg(c))) + S(__ldg(w + 1)) * S(__ldg(f + base + __ldg(c + 1))) +
         S(__ldg(w + 2)) * S(__ldg(f + base + __ldg(c + 2)));
}
// y-direction: sum_k w(r,k) f[c(r,k)*stride + i]
template <typename S>
__device__ __forceinline__ S tab_y(const Tab &T, int r, const double *__restrict__ f, int stride, int i) {
  const int32_t *c = T.c + kT * r;
  const double *w = T.w + kT * r;
  return S(__ldg(w)) * S(__ldg(f + (long long)__ldg(c) * stride + i)) +
         S(__ldg(w + 1)) * S(__ldg(f + (long long)__ldg(c + 1) * stride + i)) +
         S(__ldg(w + 2)) * S(__ldg(f + (long long)__ldg(c + 2) * stride + i));
}
template <typename S>
__device__ __forceinline__ S bcx(const Tab &T, int r, const double *v1, const double *v2, int j) {
  return S(__ldg(T.b1 + r)) * S(__ldg(v1 + j)) + S(__ldg(T.b2 + r)) * S(__ldg(v2 + j));
}

// vbar at uy point (row r in 0..Ny, u column i): Iv_uy*v + yIv_uy
// (operator_interpolation.m:237-271, set_bc_vectors.m:443-452)
template <typename S>
__device__ __forceinline__ S vf_uy(const DevOps &P, const double *__restrict__ cv, int r, int i) {
  const int32_t *c = P.IVY.c + kT * r;
  const double *w = P.IVY.w + kT * r;
  S s = S(0);
#pragma unroll
  for (int k = 0; k < kT; ++k) {
    double wk = __ldg(w + k);
    if (wk != 0.0) s += S(wk) * tab_x<S>(P.IVX, i, cv, (long long)__ldg(c + k) * P.Nvx);
  }
  s += bcx<S>(P.IVX, i, P.bc.vLe, P.bc.vRi, r);
  s += S(__ldg(P.IVY.b1 + r)) * S(__ldg(P.bc.XvLo + i)) + S(__ldg(P.IVY.b2 + r)) * S(__ldg(P.bc.XvUp + i));
  return s;
}

// ubar at vx point (v row j, column r in 0..Nx): Iu_vx*u + yIu_vx
// (operator_interpolation.m:277-308, set_bc_vectors.m:485-494)
template <typename S>
__device__ __forceinline__ S uf_vx(const DevOps &P, const double *__restrict__ cu, int j, int r) {
  const int32_t *c = P.IUY.c + kT * j;
  const double *w = P.IUY.w + kT * j;
  S s = S(0);
#pragma unroll
  for (int k = 0; k < kT; ++k) {
    double wk = __ldg(w + k);
    if (wk != 0.0) s += S(wk) * tab_x<S>(P.IUX, r, cu, (long long)__ldg(c + k) * P.Nux);
  }
  s += S(__ldg(P.IUY.b1 + j)) * S(__ldg(P.bc.uLo + r)) + S(__ldg(P.IUY.b2 + j)) * S(__ldg(P.bc.uUp + r));
  s += bcx<S>(P.IUX, r, P.bc.YuLe, P.bc.YuRi, j);
  return s;
}

// u-momentum residual without the pressure gradient:
// -convu + Diffu*u + yDiffu - y_px   (F.m:137-145, convection.m:198-204,
// diffusion.m:29), at u point (i,j).  C = (cu,cv) is the convecting field.
template <typename S, bool SAMEC>
__device__ __forceinline__ S rhs_u(const DevOps &P, const double *__restrict__ u, const double *__restrict__ v,
                                   const double *__restrict__ cu, const double *__restrict__ cv, int i, int j,
                                   double ypfac = 1.0) {
  const long long bu = (long long)j * P.Nux;
  const S hy = S(__ldg(P.hy + j));
  // u at ux faces (Au_ux*u + yAu_ux) and ubar there (Iu_ux = diag(hy) Au_ux)
  S uxl = tab_x<S>(P.AUX, i, u, bu) + bcx<S>(P.AUX, i, P.bc.uLe_i, P.bc.uRi_i, j);
  S uxr = tab_x<S>(P.AUX, i + 1, u, bu) + bcx<S>(P.AUX, i + 1, P.bc.uLe_i, P.bc.uRi_i, j);
  S cxl = uxl, cxr = uxr;
  if (!SAMEC) {
    cxl = tab_x<S>(P.AUX, i, cu, bu) + bcx<S>(P.AUX, i, P.bc.uLe_i, P.bc.uRi_i, j);
    cxr = tab_x<S>(P.AUX, i + 1, cu, bu) + bcx<S>(P.AUX, i + 1, P.bc.uLe_i, P.bc.uRi_i, j);
  }
  const S du2dx = (hy * cxr) * uxr - (hy * cxl) * uxl;
  // u at uy faces and vbar there
  S uyl = tab_y<S>(P.AUY, j, u, P.Nux, i) + bcx<S>(P.AUY, j, P.bc.uLo_i, P.bc.uUp_i, i);
  S uyr = tab_y<S>(P.AUY, j + 1, u, P.Nux, i) + bcx<S>(P.AUY, j + 1, P.bc.uLo_i, P.bc.uUp_i, i);
  S vfl = vf_uy<S>(P, cv, j, i);
  S vfr = vf_uy<S>(P, cv, j + 1, i);
  const S duvdy = vfr * uyr - vfl * uyl;
  // diffusion: Dux (1/Re) Su_ux + Duy (1/Re) Su_uy (operator_convection_diffusion.m:460)
  const S ire = S(P.invRe);
  S sxl = tab_x<S>(P.SUX, i, u, bu) + bcx<S>(P.SUX, i, P.bc.uLe_i, P.bc.uRi_i, j);
  S sxr = tab_x<S>(P.SUX, i + 1, u, bu) + bcx<S>(P.SUX, i + 1, P.bc.uLe_i, P.bc.uRi_i, j);
  S syl = tab_y<S>(P.SUY, j, u, P.Nux, i) + bcx<S>(P.SUY, j, P.bc.uLo_i, P.bc.uUp_i, i);
  S syr = tab_y<S>(P.SUY, j + 1, u, P.Nux, i) + bcx<S>(P.SUY, j + 1, P.bc.uLo_i, P.bc.uUp_i, i);
  const S d2u = hy * (ire * sxr - ire * sxl) + S(__ldg(P.gxi + i)) * (ire * syr - ire * syl);
  // y_px = kron(hy.*pLe, y1D_le) + kron(hy.*pRi, y1D_ri)
  const S ypx = hy * S(__ldg(P.bc.pLe + j)) * S(__ldg(P.pxl + i)) + hy * S(__ldg(P.bc.pRi + j)) * S(__ldg(P.pxr + i));
  return -(du2dx + duvdy) + d2u - S(ypfac) * ypx;
}

// v-momentum residual without the pressure gradient, at v point (i,j)
// (convection.m:206-212).
template <typename S, bool SAMEC>
__device__ __forceinline__ S rhs_v(const DevOps &P, const double *__restrict__ u, const double *__restrict__ v,
                                   const double *__restrict__ cu, const double *__restrict__ cv, int i, int j,
                                   double ypfac = 1.0) {
  const long long bv = (long long)j * P.Nvx;
  const S hx = S(__ldg(P.hx + i));
  S vxl = tab_x<S>(P.AVX, i, v, bv) + bcx<S>(P.AVX, i, P.bc.vLe_i, P.bc.vRi_i, j);
  S vxr = tab_x<S>(P.AVX, i + 1, v, bv) + bcx<S>(P.AVX, i + 1, P.bc.vLe_i, P.bc.vRi_i, j);
  S ufl = uf_vx<S>(P, cu, j, i);
  S ufr = uf_vx<S>(P, cu, j, i + 1);
  const S duvdx = ufr * vxr - ufl * vxl;
  S vyl = tab_y<S>(P.AVY, j, v, P.Nvx, i) + bcx<S>(P.AVY, j, P.bc.vLo_i, P.bc.vUp_i, i);
  S vyr = tab_y<S>(P.AVY, j + 1, v, P.Nvx, i) + bcx<S>(P.AVY, j + 1, P.bc.vLo_i, P.bc.vUp_i, i);
  S cyl = vyl, cyr = vyr;
  if (!SAMEC) {
    cyl = tab_y<S>(P.AVY, j, cv, P.Nvx, i) + bcx<S>(P.AVY, j, P.bc.vLo_i, P.bc.vUp_i, i);
    cyr = tab_y<S>(P.AVY, j + 1, cv, P.Nvx, i) + bcx<S>(P.AVY, j + 1, P.bc.vLo_i, P.bc.vUp_i, i);
  }
  const S dv2dy = (hx * cyr) * vyr - (hx * cyl) * vyl;
  const S ire = S(P.invRe);
  S sxl = tab_x<S>(P.SVX, i, v, bv) + bcx<S>(P.SVX, i, P.bc.vLe_i, P.bc.vRi_i, j);
  S sxr = tab_x<S>(P.SVX, i + 1, v, bv) + bcx<S>(P.SVX, i + 1, P.bc.vLe_i, P.bc.vRi_i, j);
  S syl = tab_y<S>(P.SVY, j, v, P.Nvx, i) + bcx<S>(P.SVY, j, P.bc.vLo_i, P.bc.vUp_i, i);
  S syr = tab_y<S>(P.SVY, j + 1, v, P.Nvx, i) + bcx<S>(P.SVY, j + 1, P.bc.vLo_i, P.bc.vUp_i, i);
  const S d2v = S(__ldg(P.gyi + j)) * (ire * sxr - ire * sxl) + hx * (ire * syr - ire * syl);
  const S ypy = hx * S(__ldg(P.bc.pLo + i)) * S(__ldg(P.pyl + j)) + hx * S(__ldg(P.bc.pUp + i)) * S(__ldg(P.pyu + j));
  return -(duvdx + dv2dy) + d2v - S(ypfac) * ypy;
}

// (Gx p)(i,j) = -(Mx' p) (operator_divergence.m:164)
__device__ __forceinline__ double grad_x(const DevOps &P, const double *__restrict__ p, int i, int j) {
  return -__ldg(P.hy + j) * tab_x<double>(P.MXT, i, p, (long long)j * P.Npx);
}
__device__ __forceinline__ double grad_y(const DevOps &P, const double *__restrict__ p, int i, int j) {
  return -__ldg(P.hx + i) * tab_y<double>(P.MYT, j, p, P.Npx, i);
}
// (M*V)(i,j) without BC vector (operator_divergence.m:89,135)
__device__ __forceinline__ double div_in(const DevOps &P, const double *__restrict__ u, const double *__restrict__ v,
                                         int i, int j) {
  return __ldg(P.hy + j) * tab_x<double>(P.MX, i, u, (long long)j * P.Nux) +
         __ldg(P.hx + i) * tab_y<double>(P.MY, j, v, P.Nvx, i);
}
// yM(i,j) (set_bc_vectors.m:99-117) from the given boundary arrays
__device__ __forceinline__ double div_bc(const DevOps &P, const double *uLe, const double *uRi, const double *vLo,
                                         const double *vUp, int i, int j) {
  return __ldg(P.hy + j) * (__ldg(P.MX.b1 + i) * __ldg(uLe + j) + __ldg(P.MX.b2 + i) * __ldg(uRi + j)) +
         __ldg(P.hx + i) * (__ldg(P.MY.b1 + j) * __ldg(vLo + i) + __ldg(P.MY.b2 + j) * __ldg(vUp + i));
}
// (A p)(i,j), A = M Om^-1 G = -(hy_j TX + hx_i TY)
__device__ __forceinline__ bool in_reg(const RegD &r, int row) { return row >= r.lo && row < r.hi; }
// regular-row versions (no tables, no boundary terms)
__device__ __forceinline__ double reg_x(const RegD &r, int row, const double *__restrict__ f, long long base) {
  const int c0 = wrapn(row + r.s, r.n);
  double a = __ldg(r.w0 + row) * __ldg(f + base + c0);
  if (r.two) a += __ldg(r.w1 + row) * __ldg(f + base + wrapn(c0 + 1, r.n));
  return a;
}
__device__ __forceinline__ double reg_y(const RegD &r, int row, const double *__restrict__ f, int stride, int i) {
  const int c0 = wrapn(row + r.s, r.n);
  double a = __ldg(r.w0 + row) * __ldg(f + (long long)c0 * stride + i);
  if (r.two) a += __ldg(r.w1 + row) * __ldg(f + (long long)wrapn(c0 + 1, r.n) * stride + i);
  return a;
}
__device__ __forceinline__ double grad_x_fast(const DevOps &P, const double *__restrict__ p, int i, int j) {
  if (in_reg(P.rMXT, i)) return -__ldg(P.hy + j) * reg_x(P.rMXT, i, p, (long long)j * P.Npx);
  return grad_x(P, p, i, j);
}
__device__ __forceinline__ double grad_y_fast(const DevOps &P, const double *__restrict__ p, int i, int j) {
  if (in_reg(P.rMYT, j)) return -__ldg(P.hx + i) * reg_y(P.rMYT, j, p, P.Npx, i);
  return grad_y(P, p, i, j);
}

// Sources of the velocity-sized field W whose divergence a solve takes:
// W itself (FP64), or W = Vn * sv + sa * T with T stored in FP32 (the
// FP32-storage stages: Vn/dt + Vtemp, evaluated in FP64).
struct WPlain {
  const double *W;
  __device__ __forceinline__ double operator()(long long k) const { return __ldg(W + k); }
};
struct WSplit {
  const double *Vn;
  const float *T;
  double sv, sa;
  __device__ __forceinline__ double operator()(long long k) const {
    return __ldg(Vn + k) * sv + sa * (double)__ldg(T + k);
  }
};
template <class F>
__device__ __forceinline__ double reg_x_f(const RegD &r, int row, const F &f, long long base) {
  const int c0 = wrapn(row + r.s, r.n);
  double a = __ldg(r.w0 + row) * f(base + c0);
  if (r.two) a += __ldg(r.w1 + row) * f(base + wrapn(c0 + 1, r.n));
  return a;
}
template <class F>
__device__ __forceinline__ double reg_y_f(const RegD &r, int row, const F &f, long long base, int stride, int i) {
  const int c0 = wrapn(row + r.s, r.n);
  double a = __ldg(r.w0 + row) * f(base + (long long)c0 * stride + i);
  if (r.two) a += __ldg(r.w1 + row) * f(base + (long long)wrapn(c0 + 1, r.n) * stride + i);
  return a;
}
template <class F>
__device__ __forceinline__ double tab_x_f(const Tab &T, int r, const F &f, long long base) {
  const int32_t *c = T.c + kT * r;
  const double *w = T.w + kT * r;
  return __ldg(w) * f(base + __ldg(c)) + __ldg(w + 1) * f(base + __ldg(c + 1)) + __ldg(w + 2) * f(base + __ldg(c + 2));
}
template <class F>
__device__ __forceinline__ double tab_y_f(const Tab &T, int r, const F &f, long long base, int stride, int i) {
  const int32_t *c = T.c + kT * r;
  const double *w = T.w + kT * r;
  return __ldg(w) * f(base + (long long)__ldg(c) * stride + i) + __ldg(w + 1) * f(base + (long long)__ldg(c + 1) * stride + i) +
         __ldg(w + 2) * f(base + (long long)__ldg(c + 2) * stride + i);
}

// f(i,j) = (M W + alpha yM + beta ydM)(i,j) * gamma
template <class F>
__device__ __forceinline__ double div_cell_f(const DevOps &P, const F &W, double alpha, double beta, double gamma,
                                             int i, int j) {
  double d;
  if (in_reg(P.rMX, i) && in_reg(P.rMY, j)) {
    // interior cell: regular rows of Mx and My, no boundary contribution
    d = __ldg(P.hy + j) * reg_x_f(P.rMX, i, W, (long long)j * P.Nux) +
        __ldg(P.hx + i) * reg_y_f(P.rMY, j, W, P.Nu, P.Nvx, i);
  } else {
    d = __ldg(P.hy + j) * tab_x_f(P.MX, i, W, (long long)j * P.Nux) +
        __ldg(P.hx + i) * tab_y_f(P.MY, j, W, P.Nu, P.Nvx, i);
    if (alpha != 0.0) d += alpha * div_bc(P, P.bc.uLe_i, P.bc.uRi_i, P.bc.vLo_i, P.bc.vUp_i, i, j);
    if (beta != 0.0) d += beta * div_bc(P, P.bc.dudtLe_i, P.bc.dudtRi_i, P.bc.dvdtLo_i, P.bc.dvdtUp_i, i, j);
  }
  return d * gamma;
}
__device__ __forceinline__ double div_cell(const DevOps &P, const double *__restrict__ W, double alpha, double beta,
                                           double gamma, int i, int j) {
  return div_cell_f(P, WPlain{W}, alpha, beta, gamma, i, j);
}

__device__ __forceinline__ double lap(const DevOps &P, const double *__restrict__ p, int i, int j) {
  return -(__ldg(P.hy + j) * tab_x<double>(P.TX, i, p, (long long)j * P.Npx) +
           __ldg(P.hx + i) * tab_y<double>(P.TY, j, p, P.Npx, i));
}
__device__ __forceinline__ double lap_diag(const DevOps &P, int i, int j) {
  return -(__ldg(P.hy + j) * __ldg(P.TXd + i) + __ldg(P.hx + i) * __ldg(P.TYd + j));
}
// Om_inv (operator_mesh.m:335,342) as a product of 1D reciprocals (within
// one rounding of 1/(hy*gxi))
__device__ __forceinline__ double om_inv_u(const DevOps &P, int i, int j) {
  return __ldg(P.rhy + j) * __ldg(P.rgxi + i);
}
__device__ __forceinline__ double om_inv_v(const DevOps &P, int i, int j) {
  return __ldg(P.rgyi + j) * __ldg(P.rhx + i);
}

}  // namespace ins2d
