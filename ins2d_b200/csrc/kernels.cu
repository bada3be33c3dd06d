// Stencil kernels of the INS2D hot path: RK stage right-hand side, residual,
// F, divergence, projection, Laplacian and conservation diagnostics.
//
// Thread mapping: one thread per (i,j) of the union of the u, v and p index
// spaces, 32x8 thread blocks (x fastest, coalesced along rows).  Stencil
// neighbours are served from L1/L2; each field is read from DRAM once per
// kernel.  Reductions are deterministic: per-block partials reduced in block
// order by the last block to finish.
#include <algorithm>
#include <cfloat>
#include <cstdlib>

#include "kernels.cuh"
#include "reduce.cuh"

namespace ins2d {

bool pdl_enabled() {
  static const bool on = [] {
    const char *v = std::getenv("INS2D_PDL");
    return v && v[0] == '1';
  }();
  return on;
}

namespace {

constexpr int BX = 32, BY = 8;

inline dim3 grid_for(int nx, int ny) { return dim3((nx + BX - 1) / BX, (ny + BY - 1) / BY); }

template <bool SAMEC>
__global__ void __launch_bounds__(256) k_F(const __grid_constant__ DevOps P, const double *__restrict__ V,
                                          const double *__restrict__ C, const double *__restrict__ p,
                                          double *__restrict__ Fo, const RedScratch red) {
  const int i = blockIdx.x * BX + threadIdx.x;
  const int j = blockIdx.y * BY + threadIdx.y;
  const double *u = V, *v = V + P.Nu, *cu = C, *cv = C + P.Nu;
  const double ypfac = p ? 1.0 : 0.0;
  double mx[1] = {0.0};
  const int ops[1] = {R_MAX};
  if (i < P.Nux && j < P.Nuy) {
    const long long idx = (long long)j * P.Nux + i;
    double R = rhs_u<double, SAMEC>(P, u, v, cu, cv, i, j, ypfac);
    if (p) R -= grad_x(P, p, i, j);
    Fo[idx] = R;
    mx[0] = fmax(mx[0], fabs(R));
  }
  if (i < P.Nvx && j < P.Nvy) {
    const long long idx = P.Nu + (long long)j * P.Nvx + i;
    double R = rhs_v<double, SAMEC>(P, u, v, cu, cv, i, j, ypfac);
    if (p) R -= grad_y(P, p, i, j);
    Fo[idx] = R;
    mx[0] = fmax(mx[0], fabs(R));
  }
  grid_reduce<1>(mx, ops, red);
}

template <bool WANTMAX, class F>
__global__ void __launch_bounds__(256) k_div(const __grid_constant__ DevOps P, const F W, double alpha, double beta,
                                            double gamma, double *__restrict__ f, const RedScratch red) {
  const int i = blockIdx.x * BX + threadIdx.x;
  const int j = blockIdx.y * BY + threadIdx.y;
  double mx[1] = {0.0};
  const int ops[1] = {R_MAX};
  if (i < P.Npx && j < P.Npy) {
    const double d = div_cell_f(P, W, alpha, beta, gamma, i, j);
    f[(long long)j * P.Npx + i] = d;
    mx[0] = fabs(d);
  }
  if (WANTMAX) grid_reduce<1>(mx, ops, red);
}

// V_out(i,j) = dt (Wt - c Om^-1 G dp) at the u and v points of (i,j)
__device__ __forceinline__ void project_cell(const DevOps &P, const double *__restrict__ Wt,
                                             const double *__restrict__ dp, double dt, double c,
                                             double *__restrict__ Vo, int i, int j) {
  if (i < P.Nux && j < P.Nuy) {
    const long long idx = (long long)j * P.Nux + i;
    Vo[idx] = dt * (Wt[idx] - c * om_inv_u(P, i, j) * grad_x_fast(P, dp, i, j));
  }
  if (i < P.Nvx && j < P.Nvy) {
    const long long idx = P.Nu + (long long)j * P.Nvx + i;
    Vo[idx] = dt * (Wt[idx] - c * om_inv_v(P, i, j) * grad_y_fast(P, dp, i, j));
  }
}

// Each thread projects kProjRows rows (BY apart) of one column, so a warp
// has that many independent rows of loads in flight and the column's x
// weights are read once.
#ifndef INS2D_PROJ_ROWS
#define INS2D_PROJ_ROWS 4
#endif
constexpr int kProjRows = INS2D_PROJ_ROWS;
__global__ void __launch_bounds__(256) k_project(const __grid_constant__ DevOps P, const double *__restrict__ Wt,
                                                const double *__restrict__ dp, double dt, double c,
                                                double *__restrict__ Vo) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * BX + threadIdx.x;
  const int j0 = blockIdx.y * (BY * kProjRows) + threadIdx.y;
#pragma unroll
  for (int r = 0; r < kProjRows; ++r) project_cell(P, Wt, dp, dt, c, Vo, i, j0 + r * BY);
}

// the first stage from the cached residual fused into its projection:
// Wt = Vn/dt + aii kV0 (k_stage_cached's expression) formed in registers, so
// Wt is neither written nor read again (the first stage solves no Poisson
// equation when the boundary conditions are steady: dp = p)
__global__ void __launch_bounds__(256) k_project_cached(const __grid_constant__ DevOps P,
                                                       const double *__restrict__ Vn,
                                                       const double *__restrict__ kV0, double aii, double inv_dt,
                                                       const double *__restrict__ dp, double dt, double c,
                                                       double *__restrict__ Vo) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * BX + threadIdx.x;
  const int j0 = blockIdx.y * (BY * kProjRows) + threadIdx.y;
#pragma unroll
  for (int r = 0; r < kProjRows; ++r) {
    const int j = j0 + r * BY;
    if (i < P.Nux && j < P.Nuy) {
      const long long idx = (long long)j * P.Nux + i;
      const double w = Vn[idx] * inv_dt + aii * kV0[idx];
      Vo[idx] = dt * (w - c * om_inv_u(P, i, j) * grad_x_fast(P, dp, i, j));
    }
    if (i < P.Nvx && j < P.Nvy) {
      const long long idx = P.Nu + (long long)j * P.Nvx + i;
      const double w = Vn[idx] * inv_dt + aii * kV0[idx];
      Vo[idx] = dt * (w - c * om_inv_v(P, i, j) * grad_y_fast(P, dp, i, j));
    }
  }
}

// FP32-storage stages: V_out = Vn + dt (a T - c Om^-1 G dp) in FP64 (T = the
// stage's Vtemp / a), stored as TO: float for the next stage's stencils, double
// for the new state (then V_out may be Vn itself: each point is read before it
// is written by the same thread)
template <typename TO>
__global__ void __launch_bounds__(256) k_project32(const __grid_constant__ DevOps P, const double *Vn,
                                                  const float *__restrict__ T, double a, const double *__restrict__ dp,
                                                  double dt, double c, TO *Vo) {
  const int i = blockIdx.x * BX + threadIdx.x;
  const int j0 = blockIdx.y * (BY * kProjRows) + threadIdx.y;
#pragma unroll
  for (int r = 0; r < kProjRows; ++r) {
    const int j = j0 + r * BY;
    if (i < P.Nux && j < P.Nuy) {
      const long long idx = (long long)j * P.Nux + i;
      Vo[idx] = (TO)(Vn[idx] + dt * (a * (double)T[idx] - c * om_inv_u(P, i, j) * grad_x_fast(P, dp, i, j)));
    }
    if (i < P.Nvx && j < P.Nvy) {
      const long long idx = P.Nu + (long long)j * P.Nvx + i;
      Vo[idx] = (TO)(Vn[idx] + dt * (a * (double)T[idx] - c * om_inv_v(P, i, j) * grad_y_fast(P, dp, i, j)));
    }
  }
}

__global__ void __launch_bounds__(256) k_correct(const __grid_constant__ DevOps P, const double *__restrict__ Vi,
                                                const double *__restrict__ dp, double *__restrict__ Vo) {
  const int i = blockIdx.x * BX + threadIdx.x;
  const int j = blockIdx.y * BY + threadIdx.y;
  if (i < P.Nux && j < P.Nuy) {
    const long long idx = (long long)j * P.Nux + i;
    Vo[idx] = Vi[idx] - om_inv_u(P, i, j) * grad_x(P, dp, i, j);
  }
  if (i < P.Nvx && j < P.Nvy) {
    const long long idx = P.Nu + (long long)j * P.Nvx + i;
    Vo[idx] = Vi[idx] - om_inv_v(P, i, j) * grad_y(P, dp, i, j);
  }
}

__global__ void __launch_bounds__(256) k_lap(const __grid_constant__ DevOps P, const double *__restrict__ p,
                                            double *__restrict__ Ap) {
  const int i = blockIdx.x * BX + threadIdx.x;
  const int j = blockIdx.y * BY + threadIdx.y;
  if (i < P.Npx && j < P.Npy) Ap[(long long)j * P.Npx + i] = lap(P, p, i, j);
}

// each thread takes kConsRows rows (BY apart) of one column, so the grid has
// kConsRows times fewer blocks (and block partials to reduce)
constexpr int kConsRows = 16;
__global__ void __launch_bounds__(256) k_conservation(const __grid_constant__ DevOps P, const double *__restrict__ V,
                                                     const RedScratch red) {
  const int i = blockIdx.x * BX + threadIdx.x;
  const int jb = blockIdx.y * (BY * kConsRows) + threadIdx.y;
  const double *u = V, *v = V + P.Nu;
  double q[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const int ops[5] = {R_MAX, R_SUM, R_SUM, R_SUM, R_SUM};
#pragma unroll 4
  for (int r = 0; r < kConsRows; ++r) {
    const int j = jb + r * BY;
    if (i < P.Npx && j < P.Npy)  // M V + yM; interior cells by their regular two-point rows
      q[0] = fmax(q[0], fabs(div_cell_f(P, WPlain{V}, 1.0, 0.0, 1.0, i, j)));
    if (i < P.Nux && j < P.Nuy) {
      const double om = __ldg(P.hy + j) * __ldg(P.gxi + i);
      const double x = u[(long long)j * P.Nux + i];
      q[1] += om * x;
      q[3] += om * x * x;
    }
    if (i < P.Nvx && j < P.Nvy) {
      const double om = __ldg(P.gyi + j) * __ldg(P.hx + i);
      const double x = v[(long long)j * P.Nvx + i];
      q[2] += om * x;
      q[4] += om * x * x;
    }
  }
  grid_reduce<5>(q, ops, red);
}

__global__ void k_stage_cached(const double *__restrict__ kV0, const double *__restrict__ Vn, double aii,
                               double inv_dt, double *__restrict__ Wt, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    Wt[k] = Vn[k] * inv_dt + aii * kV0[k];
}

__global__ void k_add(const double *__restrict__ x, double *__restrict__ y, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    y[k] += x[k];
}

// --- ensembles ---------------------------------------------------------------------
__device__ __forceinline__ void copy_ops(DevOps *dst, const DevOps *src) {
  const int tid = threadIdx.x + blockDim.x * threadIdx.y, nt = blockDim.x * blockDim.y;
  for (int k = tid; k < (int)(sizeof(DevOps) / 8); k += nt) ((long long *)dst)[k] = ((const long long *)src)[k];
}

__global__ void __launch_bounds__(256) k_div_ens(const EnsMemberD *__restrict__ mem, const int4 *__restrict__ tiles,
                                                int mode, double gamma) {
  __shared__ __align__(16) DevOps sP;
  const int4 t = tiles[blockIdx.x];
  const EnsMemberD &M = mem[t.x];
  copy_ops(&sP, &M.P);
  __syncthreads();
  const int i = t.y * BX + threadIdx.x, j = t.z * BY + threadIdx.y;
  if (i < sP.Npx && j < sP.Npy)
    M.f[(long long)j * sP.Npx + i] =
        mode == 0 ? div_cell(sP, M.Wt, 1.0 / M.dt, 0.0, gamma, i, j) : div_cell(sP, M.wres, 0.0, 0.0, 1.0, i, j);
}

__global__ void __launch_bounds__(256) k_project_ens(const EnsMemberD *__restrict__ mem,
                                                    const int4 *__restrict__ tiles, double c, int from_p,
                                                    int last) {
  __shared__ __align__(16) DevOps sP;
  const int4 t = tiles[blockIdx.x];
  const EnsMemberD &M = mem[t.x];
  copy_ops(&sP, &M.P);
  __syncthreads();
  project_cell(sP, M.Wt, from_p ? M.p : M.dp, M.dt, c, last ? M.V : M.Vs, t.y * BX + threadIdx.x,
               t.z * BY + threadIdx.y);
}

__global__ void __launch_bounds__(256) k_stage_cached_ens(const EnsMemberD *__restrict__ mem,
                                                         const int4 *__restrict__ tiles, double aii) {
  const int4 t = tiles[blockIdx.x];
  const EnsMemberD &M = mem[t.x];
  const double inv_dt = 1.0 / M.dt;
  const int i = t.y * BX + threadIdx.x, j = t.z * BY + threadIdx.y;
  const DevOps &P = M.P;
  if (i < P.Nux && j < P.Nuy) {
    const long long idx = (long long)j * P.Nux + i;
    M.Wt[idx] = M.V[idx] * inv_dt + aii * M.kV[0][idx];
  }
  if (i < P.Nvx && j < P.Nvy) {
    const long long idx = P.Nu + (long long)j * P.Nvx + i;
    M.Wt[idx] = M.V[idx] * inv_dt + aii * M.kV[0][idx];
  }
}

}  // namespace

namespace {
// VEC: x is 16-byte aligned and read two values at a time
template <bool VEC>
__global__ void __launch_bounds__(256) k_maxabs(const double *__restrict__ x, long long n, const RedScratch red) {
  double m[1] = {0.0};
  const int ops[1] = {R_MAX};
  constexpr int W = VEC ? 2 : 1;
  const long long stride = (long long)gridDim.x * blockDim.x * W;
  for (long long k = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * W; k < n; k += stride) {
    if (VEC && k + 1 < n) {
      const double2 v = __ldg(reinterpret_cast<const double2 *>(x + k));
      m[0] = fmax(m[0], fmax(fabs(v.x), fabs(v.y)));
    } else {
      m[0] = fmax(m[0], fabs(__ldg(x + k)));
    }
  }
  grid_reduce<1>(m, ops, red);
}
}  // namespace

void launch_maxabs(const double *x, long long n, const RedScratch &red, cudaStream_t s) {
  const bool vec = ((uintptr_t)x & 15) == 0;
  long long b = ((vec ? n / 2 : n) + 255) / 256;
  if (b > 148LL * 8) b = 148LL * 8;
  if (b > red.max_blocks) b = red.max_blocks;
  if (b < 1) b = 1;
  if (vec)
    k_maxabs<true><<<(unsigned)b, 256, 0, s>>>(x, n, red);
  else
    k_maxabs<false><<<(unsigned)b, 256, 0, s>>>(x, n, red);
}

void launch_F(const DevOps &P, const double *V, const double *C, const double *p, double *F_out,
              const RedScratch &red, cudaStream_t s) {
  dim3 g = grid_for(P.Nux > P.Nvx ? P.Nux : P.Nvx, P.Nuy > P.Nvy ? P.Nuy : P.Nvy);
  if (C == nullptr || C == V)
    k_F<true><<<g, dim3(BX, BY), 0, s>>>(P, V, V, p, F_out, red);
  else
    k_F<false><<<g, dim3(BX, BY), 0, s>>>(P, V, C, p, F_out, red);
}

void launch_div(const DevOps &P, const double *W, double alpha, double beta, double gamma, double *f,
                bool want_max, const RedScratch &red, cudaStream_t s) {
  dim3 g = grid_for(P.Npx, P.Npy);
  if (want_max)
    k_div<true><<<g, dim3(BX, BY), 0, s>>>(P, WPlain{W}, alpha, beta, gamma, f, red);
  else
    k_div<false><<<g, dim3(BX, BY), 0, s>>>(P, WPlain{W}, alpha, beta, gamma, f, red);
}

void launch_div_split(const DevOps &P, const double *Vn, const float *T, double sv, double sa, double alpha,
                      double beta, double gamma, double *f, cudaStream_t s) {
  k_div<false><<<grid_for(P.Npx, P.Npy), dim3(BX, BY), 0, s>>>(P, WSplit{Vn, T, sv, sa}, alpha, beta, gamma, f,
                                                                RedScratch{});
}

void launch_project(const DevOps &P, const double *Wt, const double *dp, double dt, double c, double *V_out,
                    cudaStream_t s) {
  const int nx = P.Nux > P.Nvx ? P.Nux : P.Nvx, ny = P.Nuy > P.Nvy ? P.Nuy : P.Nvy;
  const dim3 g((nx + BX - 1) / BX, (ny + BY * kProjRows - 1) / (BY * kProjRows));
  launch_k(k_project, g, dim3(BX, BY), 0, s, P, Wt, dp, dt, c, V_out);
}

template <typename TO>
void launch_project32_t(const DevOps &P, const double *Vn, const float *T, double a, const double *dp, double dt,
                        double c, TO *V_out, cudaStream_t s) {
  const int nx = P.Nux > P.Nvx ? P.Nux : P.Nvx, ny = P.Nuy > P.Nvy ? P.Nuy : P.Nvy;
  const dim3 g((nx + BX - 1) / BX, (ny + BY * kProjRows - 1) / (BY * kProjRows));
  k_project32<TO><<<g, dim3(BX, BY), 0, s>>>(P, Vn, T, a, dp, dt, c, V_out);
}
void launch_project32(const DevOps &P, const double *Vn, const float *T, double a, const double *dp, double dt,
                      double c, float *V_out, cudaStream_t s) {
  launch_project32_t(P, Vn, T, a, dp, dt, c, V_out, s);
}
void launch_project32(const DevOps &P, const double *Vn, const float *T, double a, const double *dp, double dt,
                      double c, double *V_out, cudaStream_t s) {
  launch_project32_t(P, Vn, T, a, dp, dt, c, V_out, s);
}

void launch_project_cached(const DevOps &P, const double *Vn, const double *kV0, double aii, double inv_dt,
                           const double *dp, double dt, double c, double *V_out, cudaStream_t s) {
  const int nx = P.Nux > P.Nvx ? P.Nux : P.Nvx, ny = P.Nuy > P.Nvy ? P.Nuy : P.Nvy;
  const dim3 g((nx + BX - 1) / BX, (ny + BY * kProjRows - 1) / (BY * kProjRows));
  launch_k(k_project_cached, g, dim3(BX, BY), 0, s, P, Vn, kV0, aii, inv_dt, dp, dt, c, V_out);
}

void launch_correct(const DevOps &P, const double *V_in, const double *dp, double *V_out, cudaStream_t s) {
  dim3 g = grid_for(P.Nux > P.Nvx ? P.Nux : P.Nvx, P.Nuy > P.Nvy ? P.Nuy : P.Nvy);
  k_correct<<<g, dim3(BX, BY), 0, s>>>(P, V_in, dp, V_out);
}

void launch_lap(const DevOps &P, const double *p, double *Ap, cudaStream_t s) {
  k_lap<<<grid_for(P.Npx, P.Npy), dim3(BX, BY), 0, s>>>(P, p, Ap);
}

void launch_conservation(const DevOps &P, const double *V, const RedScratch &red, cudaStream_t s) {
  int nx = P.Nux > P.Nvx ? P.Nux : P.Nvx;
  int ny = P.Nuy > P.Nvy ? P.Nuy : P.Nvy;
  const dim3 g((nx + BX - 1) / BX, (ny + BY * kConsRows - 1) / (BY * kConsRows));
  k_conservation<<<g, dim3(BX, BY), 0, s>>>(P, V, red);
}

void launch_stage_cached(const double *kV0, const double *Vn, double aii, double inv_dt, double *Wt, long long n,
                         cudaStream_t s) {
  long long b = (n + 255) / 256;
  if (b > 148 * 32) b = 148 * 32;
  k_stage_cached<<<(unsigned)b, 256, 0, s>>>(kV0, Vn, aii, inv_dt, Wt, n);
}

void launch_add(const double *x, double *y, long long n, cudaStream_t s) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  k_add<<<(unsigned)b, 256, 0, s>>>(x, y, n);
}

}  // namespace ins2d

namespace ins2d {

void cell_tiles(const DevOps &P, int member, std::vector<int4> &out) {
  const int nx = std::max(P.Npx, std::max(P.Nux, P.Nvx)), ny = std::max(P.Npy, std::max(P.Nuy, P.Nvy));
  for (int by = 0; by < (ny + BY - 1) / BY; ++by)
    for (int bx = 0; bx < (nx + BX - 1) / BX; ++bx) out.push_back(make_int4(member, bx, by, 0));
}

void launch_div_ens(const EnsMemberD *mem, const int4 *tiles, int n, int mode, double gamma, cudaStream_t s) {
  if (n > 0) k_div_ens<<<n, dim3(BX, BY), 0, s>>>(mem, tiles, mode, gamma);
}

void launch_project_ens(const EnsMemberD *mem, const int4 *tiles, int n, double c, int from_p, int last,
                        cudaStream_t s) {
  if (n > 0) k_project_ens<<<n, dim3(BX, BY), 0, s>>>(mem, tiles, c, from_p, last);
}

void launch_stage_cached_ens(const EnsMemberD *mem, const int4 *tiles, int n, double aii, cudaStream_t s) {
  if (n > 0) k_stage_cached_ens<<<n, dim3(BX, BY), 0, s>>>(mem, tiles, aii);
}

}  // namespace ins2d
