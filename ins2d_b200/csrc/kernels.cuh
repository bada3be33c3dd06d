// Launch wrappers of the INS2D device kernels (kernels.cu, fft.cu, pcg.cu).
#pragma once

#include <cuda_runtime.h>

#include "device.cuh"

namespace ins2d {

constexpr int kMaxStages = 8;

// Deterministic reduction scratch: per-block partials, a completion counter
// and the final values (written by the last block to finish).
struct RedScratch {
  double *partials = nullptr;    // capacity >= max_blocks * kRedQ
  unsigned int *counter = nullptr;
  double *result = nullptr;      // kRedQ values
  int max_blocks = 0;
};
constexpr int kRedQ = 6;

struct StageArgs {
  const double *V;       // velocity of this stage, V = [u; v]
  const double *Vn;      // velocity at t_n
  double *kV;            // out: Om^-1 R(V) of this stage (may be null)
  const double *kprev[kMaxStages];
  double aprev[kMaxStages];
  int nprev;
  double aii;            // Butcher coefficient of this stage's own kV
  double inv_dt;
  double *Wt;            // out: Vn/dt + Vtemp
};

// One RK stage right-hand side: kV = Om^-1 (-conv + Diff V + yDiff - y_p),
// Vtemp = sum_m A(i,m) kV_m, Wt = Vn/dt + Vtemp   (time_ERK.m:90-101,117)
void launch_stage(const DevOps &P, const StageArgs &a, bool fp32, cudaStream_t s);
// computes P.fbx0.. (the interior tile rectangle of the stencil walkers)
void walker_rectangle(DevOps &P);
// w = Om^-1 (R(V) - G p) (pressure_additional_solve.m:11-13); when kV_next is
// non-null also stores Om^-1 R(V) there.
void launch_residual(const DevOps &P, const double *V, const double *p, double *w, double *kV_next, bool fp32,
                     cudaStream_t s);
// F_out = -conv(V;C) + Diff V + yDiff - (G p + y_p) (F.m); maxres into red.result[0]
void launch_F(const DevOps &P, const double *V, const double *C, const double *p, double *F_out,
              const RedScratch &red, cudaStream_t s);
// f = (M W + alpha*yM + beta*ydM) * gamma over the pressure cells; max|f|
// into red.result[0] when want_max.
void launch_div(const DevOps &P, const double *W, double alpha, double beta, double gamma, double *f,
                bool want_max, const RedScratch &red, cudaStream_t s);
// V_out = dt*(Wt - c*Om^-1*G*dp)   (time_ERK.m:132 with Vn/dt folded into Wt)
void launch_project(const DevOps &P, const double *Wt, const double *dp, double dt, double c, double *V_out,
                    cudaStream_t s);
// V_out = V_in - Om^-1 G dp   (input_check.m:107)
void launch_correct(const DevOps &P, const double *V_in, const double *dp, double *V_out, cudaStream_t s);
void launch_lap(const DevOps &P, const double *p, double *Ap, cudaStream_t s);
// red.result = {max|M V + yM|, sum Omu u, sum Omv v, sum Omu u^2, sum Omv v^2}
void launch_conservation(const DevOps &P, const double *V, const RedScratch &red, cudaStream_t s);
// first RK stage when kV0 = Om^-1 R(Vn) is already known (it is the residual
// of the previous step's additional pressure solve): Wt = Vn/dt + aii*kV0
void launch_stage_cached(const double *kV0, const double *Vn, double aii, double inv_dt, double *Wt, long long n,
                         cudaStream_t s);
// y += x
void launch_add(const double *x, double *y, long long n, cudaStream_t s);

// --- FFT Poisson (fft.cu) -------------------------------------------------------
struct FftPlan {
  int Nx = 0, Ny = 0, logx = -1, logy = -1;  // log2 when a power of two, else -1
  double2 *twx = nullptr, *twy = nullptr;    // twiddles e^{-2 pi i k/N}
  double2 *spec = nullptr;                   // (Nx/2+1) x Ny complex spectrum
  double *maxabs = nullptr;                  // max |fhat| of the last solve
};
bool fft_supported(int Nx, int Ny);
// dp = real(ifft2(-fft2(f)./Ahat)) (pressure_poisson.m:92-104); dp += result when
// accumulate.  Returns 0 (dp untouched / zero) when max|fhat| < 1e-14 (:21-32).
void launch_fft_poisson(const DevOps &P, const FftPlan &plan, const double *f, double *dp, bool accumulate,
                        cudaStream_t s);

// --- PCG (pcg.cu) ---------------------------------------------------------------
struct PcgScalars {
  double rz, pq, rr0, rr, alpha, beta, tol2, maxx, minx, maxres;
  long long it, maxit;
  int done, status;
  unsigned int counter;
  int pad;
};
struct PcgWork {
  double *x, *r, *p, *q;
  PcgScalars *sc;      // device
  double *partials;    // >= blocks * 4
  int blocks;
};
void pcg_init(const DevOps &P, const PcgWork &W, const double *f, double tol, long long maxit, cudaStream_t s);
void pcg_iterations(const DevOps &P, const PcgWork &W, int n, cudaStream_t s);
void pcg_finish(const DevOps &P, const PcgWork &W, double *dp, bool accumulate, cudaStream_t s);
int pcg_blocks(const DevOps &P);
// Small grids: the whole solve in one thread block (dp written or accumulated
// when converged; status/iterations in W.sc)
constexpr long long kPcgBlockMaxCells = 16384;
bool pcg_use_block(const DevOps &P);
void pcg_solve_block(const DevOps &P, const PcgWork &W, const double *f, double *dp, double tol, long long maxit,
                     bool accumulate, cudaStream_t s);

}  // namespace ins2d
