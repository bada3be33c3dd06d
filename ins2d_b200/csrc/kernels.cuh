// Launch wrappers of the INS2D device kernels (kernels.cu, fft.cu, pcg.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "device.cuh"
#include "mg.cuh"

namespace ins2d {

constexpr int kMaxStages = 8;

// Programmatic dependent launch of the explicit step's kernels (the stage and
// residual walkers, the FFT passes, the projections): off unless INS2D_PDL=1
// in the environment of the process.  Measured on B200 in the step graphs it
// did not pay: 0.863 against 0.859 ms per RK4 step at 2048^2, 0.164 against
// 0.140 ms at 512^2.
bool pdl_enabled();

// k<<<g, b, sm, s>>>(args...) for a kernel that begins with pdl_wait(); with
// programmatic serialisation allowed when pdl_enabled().  Launch errors are
// left for cudaGetLastError, as with <<< >>>.
template <typename... KArgs, typename... Args>
inline void launch_k(void (*k)(KArgs...), dim3 g, dim3 b, size_t sm, cudaStream_t s, Args &&...args) {
  if (!pdl_enabled()) {
    k<<<g, b, sm, s>>>(static_cast<KArgs>(args)...);
    return;
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = g;
  cfg.blockDim = b;
  cfg.dynamicSmemBytes = sm;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
}

// Makes `dev` the calling thread's current device for the lifetime of the
// guard and restores the device that was current before (every C-ABI entry
// point leaves the caller's current device as it found it).
struct DeviceGuard {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) err = cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard &) = delete;
  DeviceGuard &operator=(const DeviceGuard &) = delete;
};

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
  const double *V;       // velocity of this stage, V = [u; v] (FP64), or null
  const float *V32;      // the stage velocity in FP32 (FP32-storage contexts), or null
  const double *Vn;      // velocity at t_n
  double *kV;            // out: Om^-1 R(V) of this stage (may be null)
  const double *kprev[kMaxStages];
  double aprev[kMaxStages];
  int nprev;
  double aii;            // Butcher coefficient of this stage's own kV
  double inv_dt;
  double *Wt;            // out: Vn/dt + Vtemp
  // FP32 storage (store32): kV32 (may be null) instead of kV, the earlier
  // stages from kprev32, and Vtemp into Vt32 (only when nprev > 0; otherwise
  // Vtemp = aii kV32); Vn and Wt are not used
  bool store32;
  float *kV32;
  const float *kprev32[kMaxStages];
  float *Vt32;
};

// One RK stage right-hand side: kV = Om^-1 (-conv + Diff V + yDiff - y_p),
// Vtemp = sum_m A(i,m) kV_m, Wt = Vn/dt + Vtemp   (time_ERK.m:90-101,117)
void launch_stage(const DevOps &P, const StageArgs &a, bool fp32, cudaStream_t s);
// computes P.fbx0.. (the interior tile rectangle of the stencil walkers)
void walker_rectangle(DevOps &P);
// opts the tiled walkers in to their dynamic shared memory on the current
// device (once per context); returns the first failure
cudaError_t walker_prepare();
// w = Om^-1 (R(V) - G p) (pressure_additional_solve.m:11-13); when kV_next
// (kV_next32) is non-null also stores Om^-1 R(V) there (rounded to FP32).
void launch_residual(const DevOps &P, const double *V, const double *p, double *w, double *kV_next,
                     float *kV_next32, bool fp32, cudaStream_t s);
// F_out = -conv(V) + Diff V + yDiff - (G p + y_p) (F.m:137-145 with C = V and
// the pressure) by the stencil walkers, FP64 fields and arithmetic
void launch_F_walk(const DevOps &P, const double *V, const double *p, double *F_out, cudaStream_t s);
// red.result[0] = max |x| over n values (deterministic)
void launch_maxabs(const double *x, long long n, const RedScratch &red, cudaStream_t s);
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
// FP32-storage contexts: f = (M (Vn sv + sa T) + alpha yM + beta ydM) gamma
// with T in FP32 (the stage's Vtemp or kV), evaluated in FP64
void launch_div_split(const DevOps &P, const double *Vn, const float *T, double sv, double sa, double alpha,
                      double beta, double gamma, double *f, cudaStream_t s);
// FP32-storage contexts: V_out = Vn + dt (a T - c Om^-1 G dp) (time_ERK.m:132),
// into the FP32 stage velocity or the FP64 new state (V_out may be Vn)
void launch_project32(const DevOps &P, const double *Vn, const float *T, double a, const double *dp, double dt,
                      double c, float *V_out, cudaStream_t s);
void launch_project32(const DevOps &P, const double *Vn, const float *T, double a, const double *dp, double dt,
                      double c, double *V_out, cudaStream_t s);
// the first stage from the cached residual and its projection in one pass:
// V_out = dt (Vn/dt + aii kV0 - c Om^-1 G dp)
void launch_project_cached(const DevOps &P, const double *Vn, const double *kV0, double aii, double inv_dt,
                           const double *dp, double dt, double c, double *V_out, cudaStream_t s);
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

// --- ensembles: many independent member grids per launch -----------------------
// Member descriptor in device memory: operator tables, state and work arrays.
struct PcgWork;
struct EnsMemberD;
// Stage (mode 0) or additional-solve residual (mode 1) walker arguments shared
// by all members (same Butcher tableau; each member's dt is in its descriptor).
struct EnsWalk {
  int mode, stage, store, use_vs, nprev, cache;
  int kidx[kMaxStages];
  double aprev[kMaxStages];
  double aii;
};
// Host: the walker tiles {member, bx, by, 0} of one member, split into fast
// (interior) and generic tiles.
void walk_tiles(const DevOps &P, int member, std::vector<int4> &fast, std::vector<int4> &gen);
void launch_walk_ens(const EnsMemberD *mem, const int4 *fast, int nfast, const int4 *gen, int ngen, const EnsWalk &w,
                     bool fp32, cudaStream_t s);
// Host: the 32x8 cell tiles {member, bx, by, 0} covering a member's u, v and p
// index spaces.
void cell_tiles(const DevOps &P, int member, std::vector<int4> &out);
// f = (M Wt + yM/dt) gamma (mode 0, stage) or f = M wres (mode 1, residual)
void launch_div_ens(const EnsMemberD *mem, const int4 *tiles, int n, int mode, double gamma, cudaStream_t s);
// V_out = dt (Wt - c Om^-1 G dp_src); dp_src = p (from_p) or dp; V_out = V
// (last stage) or Vs
void launch_project_ens(const EnsMemberD *mem, const int4 *tiles, int n, double c, int from_p, int last,
                        cudaStream_t s);
// Wt = V/dt + aii kV[0] (first stage from the cached residual)
void launch_stage_cached_ens(const EnsMemberD *mem, const int4 *tiles, int n, double aii, cudaStream_t s);

// --- FFT Poisson (fft.cu) -------------------------------------------------------
struct FftPlan {
  int Nx = 0, Ny = 0, logx = -1, logy = -1;  // log2 when a power of two, else -1
  double2 *twx = nullptr, *twy = nullptr;    // 2N entries each: fft_twiddle_table(N)
  double2 *spec = nullptr;                   // (Nx/2+1) x Ny complex spectrum
  double *maxabs = nullptr;                  // max |fhat| of the last solve
};
bool fft_supported(int Nx, int Ny);
// Twiddles of a length-n transform as 2n complex values (4n doubles): entries
// [0, n) hold e^{-2 pi i k/n}; for power-of-two n, entry n + Lt/2 + k holds
// e^{-2 pi i k/Lt} for every power of two 2 <= Lt <= n and k < Lt/2.
std::vector<double> fft_twiddle_table(int n);
// dp = real(ifft2(-fft2(f)./Ahat)) (pressure_poisson.m:92-104); dp += result when
// accumulate.  Returns 0 (dp untouched / zero) when max|fhat| < 1e-14 (:21-32).
// The return value is the error of the enqueued memset (kernel launch errors
// are left to cudaGetLastError as for every launch).
cudaError_t launch_fft_poisson(const DevOps &P, const FftPlan &plan, const double *f, double *dp, bool accumulate,
                               cudaStream_t s);
// Same with the right-hand side f = (M W + alpha yM + beta ydM) gamma computed
// inside the first pass (only when fft_fuses_div(plan): power-of-two rows >= 64).
bool fft_fuses_div(const FftPlan &plan);
// kernel launches of one solve (the column transform takes one or three)
int fft_kernels(const FftPlan &plan);
cudaError_t launch_fft_poisson_div(const DevOps &P, const FftPlan &plan, const double *W, double alpha,
                                   double beta, double gamma, double *dp, bool accumulate, cudaStream_t s);
// z = A^+ r by the same transform (the exact inverse of a periodic uniform
// grid, as a PCG preconditioner): the early return is read from *gate
// instead of the spectrum (a word holding a large value disables it); every
// pass returns at once while *skip is non-zero (a converged CG)
cudaError_t launch_fft_precond(const DevOps &P, const FftPlan &plan, const double *r, double *z,
                               const unsigned long long *gate, const int *skip, cudaStream_t s);
// Same with W = Vn sv + sa T, T in FP32 (FP32-storage stages)
cudaError_t launch_fft_poisson_div_split(const DevOps &P, const FftPlan &plan, const double *Vn, const float *T,
                                         double sv, double sa, double alpha, double beta, double gamma, double *dp,
                                         bool accumulate, cudaStream_t s);
// Opts the transform kernels in to large dynamic shared memory on the current
// device; returns the first failure.
cudaError_t fft_prepare();

// --- fast-diagonalization preconditioner (fdm.cu) -----------------------------------
// Generalized eigenbases of the pressure matrix's 1D factors (fdm_host.cpp)
// and the work arrays of one application.
struct FdmD {
  int nx = 0, ny = 0;
  const double *Qx = nullptr, *Qy = nullptr;  // nx x nx, ny x ny row-major (Q[i*n + a])
  const double *lx = nullptr, *ly = nullptr;  // eigenvalues
  double thr = 0.0;                           // lx + ly <= thr: the null mode (left out)
  double *t1 = nullptr, *t2 = nullptr;        // nx*ny each
  double *z = nullptr;                        // the preconditioned residual
  // periodic uniform grids: the Fourier basis, applied by the FFT solve
  bool spectral = false;
  const FftPlan *fft = nullptr;
  const unsigned long long *gate = nullptr;  // device word holding 1.0 (no early return)
};
// z = A^+ r (four dense products); no work once *done is set (done may be null)
void fdm_apply(const FdmD &F, const double *r, double *z, const int *done, cudaStream_t s);
// one ensemble member's fast-diagonalization data (device copy): z = A^+ r
struct EnsFdmD {
  int nx, ny;
  const double *Qx, *Qy, *lx, *ly;
  double thr;
  const double *r;  // the member's CG residual
  double *t1, *t2, *z;
};
struct EnsCg;
// Host: the 64x64 output tiles {member, tile row, tile column, 0} of a member
// with an ny x nx pressure grid
void fdm_tiles(int member, int nx, int ny, std::vector<int4> &out);
// z = A^+ r for every member not yet converged (cg[m].done == 0): the four
// products, one launch each over all members' tiles
void fdm_apply_ens(const EnsFdmD *F, const int4 *tiles, int ntiles, const EnsCg *cg, cudaStream_t s);

// --- PCG (pcg.cu) ---------------------------------------------------------------
struct PcgScalars {
  double rz, pq, rr0, rr, alpha, beta, tol2, maxx, minx, maxres;
  long long it, maxit;
  int done, status;
  unsigned int counter;
  int loops;  // passes of a device-side iteration loop (graph form)
};
// Solve statistics accumulated on the device by the solves of a captured
// step graph (the host reads them after the graph launches).
struct SolveAccum {
  long long n_solves, iters_total, iters_max;
  double norm1_max;
  int status;  // first non-zero solve status (INS2D_E*), 0 if none
  int pad;
  double fail_rr;
  long long fail_maxit;
};
// Graph form of the PCG loop: sets the WHILE condition h to "not done and
// fewer than limit passes" (count: this launch ends a pass of the body)
void launch_pcg_cond(PcgScalars *sc, cudaGraphConditionalHandle h, int limit, int count, cudaStream_t s);
// adds a finished solve's iterations, residual and status to *acc (a loop
// that stopped at its pass limit before convergence counts as INS2D_ETIMEOUT)
void launch_solve_accum(const PcgScalars *sc, SolveAccum *acc, cudaStream_t s);
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
// Multi-block PCG with the multigrid preconditioner: k_init + one V-cycle,
// then n iterations of SpMV, update, V-cycle, r'z, p update (mg.cu launches).
void pcg_init_mg(const DevOps &P, const MgD &M, const PcgWork &W, const double *f, double tol, long long maxit,
                 cudaStream_t s);
void pcg_iterations_mg(const DevOps &P, const MgD &M, const PcgWork &W, int n, cudaStream_t s);
// The same with the fast-diagonalization preconditioner
void pcg_init_fdm(const DevOps &P, const FdmD &F, const PcgWork &W, const double *f, double tol, long long maxit,
                  cudaStream_t s);
void pcg_iterations_fdm(const DevOps &P, const FdmD &F, const PcgWork &W, int n, cudaStream_t s);
// small grids (at most 128 cells per direction, not the spectral form): the
// whole fast-diagonalization PCG solve in one thread block
bool pcg_use_block_fdm(const FdmD &F);
void pcg_solve_block_fdm(const DevOps &P, const FdmD &F, const PcgWork &W, const double *f, double *dp, double tol,
                         long long maxit, bool accumulate, cudaStream_t s);

struct EnsMemberD {
  DevOps P;
  double dt;  // this member's time step
  double *V, *p, *Vs, *Wt, *kV[kMaxStages], *f, *dp, *wres;
  PcgWork W;
  const MgD *mg;  // device copy of the member's hierarchy, or null (Jacobi)
  const double *zf;  // batched solves with fast diagonalization: the preconditioned residual
};
// per-member solve statistics, accumulated over a run
struct EnsStats {
  long long n_solves, iters_total, iters_max;
  double norm1_max;
  int status, pad;
};
// --- batched ensemble solves (ens_pcg.cu) ----------------------------------
// columns per thread block of the batched y-line solves (32, or 16: two row
// segments per warp)
#ifndef INS2D_ENS_YCW
#define INS2D_ENS_YCW 16
#endif
constexpr int kEnsYcols = INS2D_ENS_YCW;
// per-member CG scalars and accumulators
struct EnsCg {
  double acc_pq, acc_rr, acc_rz, maxf;
  double rz, rr0, rr, alpha, beta, tol2;
  long long it, maxit;
  int done, status;
};
// members' multigrid levels: lev[m * kMgMaxLevels + l]
struct EnsMgD {
  const MgLevelD *lev;
  const int *nlev;
  const double *const *cinv;
  const int *ncoarse;
};
// work of one phase over members: member mem[s] owns global work indices
// [start[s], start[s+1]); total = start[n]
struct EnsSeg {
  const int *mem;
  const long long *start;
  int n;
  long long total;
};
struct EnsMgPlan {
  int lmax = 0;
  int ltail = 0;              // levels >= ltail: one thread block per member (k_emg_tail)
  const MgD *const *mgs = nullptr;  // device: each member's hierarchy
  EnsSeg xl[kMgMaxLevels], yl[kMgMaxLevels], rs[kMgMaxLevels], pr[kMgMaxLevels];
  EnsSeg yg[kMgMaxLevels];  // groups of 32 columns (one thread block each)
  EnsSeg co{};
};
void ens_vcycle(const EnsMemberD *mem, const EnsMgD &G, const EnsCg *cg, const EnsMgPlan &pl, double omega,
                double alpha, cudaStream_t s);
// op 0 init (x = 0, r = f), 1 q = A p, 2 x/r update, 3 r'z, 4 r'z with p = z, 5 p update
void ens_cg_vec(const EnsMemberD *mem, const EnsMgD &G, const int2 *tiles, int ntiles, EnsCg *cg, int op,
                cudaStream_t s);
// op 0 after init, 1 first r'z, 2 alpha, 3 convergence, 4 beta; *active = members still iterating
// WHILE condition of the batched solve's graph form (some member iterating,
// fewer than limit passes; count 0 resets the pass counter *loops)
void ens_loop_cond(const EnsCg *cg, int n, int *loops, int limit, int count, cudaGraphConditionalHandle h,
                   cudaStream_t s);
void ens_cg_scalar(EnsCg *cg, int n, int op, int *active, cudaStream_t s);
void ens_cg_finish(const EnsMemberD *mem, const int2 *tiles, int ntiles, EnsCg *cg, int n, int which,
                   EnsStats *stats, cudaStream_t s);

// Poisson solves of all members in one persistent launch: each thread block
// takes the next member of `order` from a device queue and runs the whole
// PCG (pcg_block_body).  which = 0: f -> dp; which = 1: p += solve(f)
// (additional solve).  queue: two zeroed counters, left zeroed on exit.
void launch_pcg_members(const EnsMemberD *mem, const int *order, int n, int which, double tol2, long long maxit,
                        unsigned *queue, EnsStats *stats, int threads, int blocks, cudaStream_t s);
// Small grids: the whole solve in one thread block (dp written or accumulated
// when converged; status/iterations in W.sc)
constexpr long long kPcgBlockMaxCells = 16384;
bool pcg_use_block(const DevOps &P);
void pcg_solve_block(const DevOps &P, const PcgWork &W, const double *f, double *dp, double tol, long long maxit,
                     bool accumulate, cudaStream_t s);
// Same with a multigrid V-cycle as the preconditioner (mg.cuh); one thread
// block, for grids up to kPcgBlockMgMaxCells cells.
constexpr long long kPcgBlockMgMaxCells = 65536;
void pcg_solve_block_mg(const DevOps &P, const MgD &M, const PcgWork &W, const double *f, double *dp, double tol,
                        long long maxit, bool accumulate, cudaStream_t s);

}  // namespace ins2d
