/* ins2d.h -- C-ABI of the B200 INS2D hot path (libins2d.so).
 *
 * The hot path is the explicit Runge-Kutta stage loop of the energy-conserving
 * staggered finite-volume incompressible Navier-Stokes solver INS2D, with its
 * right-hand side F and the pressure-Poisson projection.  The entry points
 * below replace, one for one, the MATLAB functions a case calls through main():
 *
 *   ins2d_ctx_create        operators.m:1-18 + operator_*.m   (the options struct)
 *   ins2d_set_bc_values     set_bc_vectors.m:1-706            (BC vectors at t)
 *   ins2d_F                 spatial/F.m:1                     ([maxres,F] = F(V,C,p,T,t,options))
 *   ins2d_divergence        check_conservation.m:37           (M*V + yM)
 *   ins2d_pressure_poisson  solvers/pressure/pressure_poisson.m:1 (dp = pressure_poisson(f,t,options))
 *   ins2d_pressure_additional_solve solvers/pressure/pressure_additional_solve.m:1
 *   ins2d_erk_step          unsteady/time_ERK.m:1             ([Vnew,pnew] = time_ERK(Vn,pn,Tn,tn,dt,options))
 *   ins2d_conservation      spatial/check_conservation.m:1    ([maxdiv,umom,vmom,k])
 *   ins2d_laplacian         A*p with A = M*Om_inv*G           (operator_divergence.m:208)
 * and the Fortran MEX gateway cg.F:31 ([x,iter,norm1,norm2]=cg(...)) whose role
 * ins2d_pressure_poisson takes over with a device PCG.
 *
 * Conventions
 *  - Vectors use the reference's ordering: x fastest, V = [u; v],
 *    u(i,j) -> i + j*Nux_in, v(i,j) -> i + j*Nvx_in, p(i,j) -> i + j*Npx.
 *  - All arithmetic is IEEE binary64 unless the context was created with
 *    precision = INS2D_PREC_FP32_STENCIL (FP32 convection/diffusion stencils
 *    and stage combination; divergence, Poisson solve and projection stay FP64).
 *  - `mem` selects where array arguments live: INS2D_MEM_HOST (the call copies
 *    in and out, host buffers owned by the caller) or INS2D_MEM_DEVICE (device
 *    pointers on the context's device, used in place).
 *  - Every function returns an int status (INS2D_OK = 0); the text of the last
 *    error is ins2d_last_error(ctx).
 *  - A context is used by one host thread at a time; distinct contexts are
 *    independent.  Work is issued on the context's stream (ins2d_set_stream),
 *    and each call returns after that stream has finished the call's work.
 */
#ifndef INS2D_H
#define INS2D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (failure modes of cg.F:262, pressure_poisson.m:58-63,
 * boundary_conditions.m:17-40) */
#define INS2D_OK 0
#define INS2D_EINVAL 1      /* invalid argument / unsupported BC combination */
#define INS2D_ENOTCONV 2    /* PCG did not reach CG_acc within CG_maxit */
#define INS2D_EBREAKDOWN 3  /* PCG breakdown (p'Ap = 0) */
#define INS2D_ENONFINITE 4  /* NaN/Inf met in a solve or step */
#define INS2D_ETIMEOUT 5    /* a bounded device wait gave up */
#define INS2D_ECUDA 6       /* CUDA runtime error */
#define INS2D_ENOMEM 7      /* device allocation failed */

/* boundary-condition types (options.BC.{u,v}.{left,right,low,up}) */
#define INS2D_BC_DIR 0
#define INS2D_BC_PRES 1
#define INS2D_BC_PER 2
#define INS2D_BC_SYM 3

/* options.solversettings.poisson: 1 direct, 2 pcg+ILU, 3 cg MEX, 4 CG+DIC,
 * 5 PETSc -> all served by the device PCG; 6 -> FFT (periodic, uniform). */
#define INS2D_POISSON_DIRECT 1
#define INS2D_POISSON_CG_MEX 3
#define INS2D_POISSON_CG 4
#define INS2D_POISSON_FFT 6

/* preconditioner of the device PCG (poisson 1-5).  The reference's cg.F uses
 * a diagonal incomplete Cholesky factor (sequential sweeps, cg.F:317-390);
 * the device offers fast diagonalization, a multigrid V-cycle or the Jacobi
 * diagonal.  Either way CG iterates to the same relative residual CG_acc. */
#define INS2D_PRECOND_DEFAULT 0 /* fast diagonalization where it applies, else multigrid, else Jacobi;
                                   ensemble members: multigrid */
#define INS2D_PRECOND_JACOBI 1
#define INS2D_PRECOND_MG 2
/* fast diagonalization: A is separable, A = -(diag(hy) (x) TX + TY (x)
 * diag(hx)), so the generalized eigenbases of the 1D factors TX, TY give its
 * inverse on the range of A as four dense transforms (periodic uniform grids:
 * the Fourier basis, i.e. the FFT solve).  CG then converges in one or two
 * iterations.  Grids up to 1024 cells per direction (set-up O(n^3) on the
 * host), or any periodic uniform grid the FFT solver takes. */
#define INS2D_PRECOND_FDM 3

#define INS2D_PREC_FP64 0
#define INS2D_PREC_FP32_STENCIL 1

#define INS2D_MEM_HOST 0
#define INS2D_MEM_DEVICE 1

#define INS2D_MAX_STAGES 8

typedef struct ins2d_ctx ins2d_ctx;

/* options.grid.{Nx,Ny,x,y} (mesh_generation.m:17-49): grid-line coordinates */
typedef struct {
  int32_t Nx, Ny;
  const double *x; /* Nx+1 */
  const double *y; /* Ny+1 */
} ins2d_grid_desc;

/* options.BC (boundary_conditions.m:1-40) */
typedef struct {
  int32_t u_left, u_right, u_low, u_up;
  int32_t v_left, v_right, v_low, v_up;
  int32_t bc_unsteady; /* options.BC.BC_unsteady */
} ins2d_bc_desc;

/* options.{fluid,solversettings,time} */
typedef struct {
  double Re;            /* options.fluid.Re */
  int32_t poisson;      /* options.solversettings.poisson */
  double CG_acc;        /* options.solversettings.CG_acc  (relative: ||r||/||f||) */
  int32_t CG_maxit;     /* options.solversettings.CG_maxit */
  int32_t p_add_solve;  /* options.solversettings.p_add_solve */
  int32_t rk_stages;    /* s of the Butcher tableau (getRKmethod.m) */
  double rk_A[INS2D_MAX_STAGES * INS2D_MAX_STAGES]; /* s x s, row-major */
  double rk_b[INS2D_MAX_STAGES];
  double rk_c[INS2D_MAX_STAGES];
  int32_t precision;    /* INS2D_PREC_* */
  int32_t device;       /* CUDA device ordinal */
  int32_t precond;      /* INS2D_PRECOND_* (0 = default) */
} ins2d_opts;

/* Boundary values sampled by the caller from the case's uBC/vBC handles at
 * time t, exactly the samples set_bc_vectors.m:52-79 takes.  NULL pressure
 * arrays mean 0 (boundary_conditions.m:107-116); NULL time derivatives mean 0. */
typedef struct {
  const double *uLo, *uUp;     /* Nx+1   uBC(x, y(1)), uBC(x, y(end)) */
  const double *uLo_i, *uUp_i; /* Nux_in uBC(xin, y(1|end)) */
  const double *uLe_i, *uRi_i; /* Ny     uBC(x(1|end), yp) */
  const double *vLe, *vRi;     /* Ny+1   vBC(x(1|end), y) */
  const double *vLo_i, *vUp_i; /* Nx     vBC(xp, y(1|end)) */
  const double *vLe_i, *vRi_i; /* Nvy_in vBC(x(1|end), yin) */
  const double *pLe, *pRi;     /* Ny     options.BC.pLe/pRi */
  const double *pLo, *pUp;     /* Nx     options.BC.pLo/pUp */
  const double *dudtLe_i, *dudtRi_i; /* Ny  dudtBC(x(1|end), yp)  (BC_unsteady) */
  const double *dvdtLo_i, *dvdtUp_i; /* Nx  dvdtBC(xp, y(1|end))  (BC_unsteady) */
} ins2d_bc_values;

/* options.grid counts (operator_mesh.m:25-110) */
typedef struct {
  int32_t Nx, Ny;
  int32_t Nux_in, Nuy_in, Nvx_in, Nvy_in;
  int32_t Npx, Npy;
  int32_t Nu, Nv, NV, Np;
} ins2d_sizes;

/* [iter, norm1, norm2] of cg.F:15-17 (iters = 0 for the FFT path) */
typedef struct {
  int32_t iters;
  double norm1; /* sqrt(||r||^2/||f||^2) */
  double norm2; /* max|r| / (max x - min x) */
} ins2d_solve_stats;

typedef struct {
  int32_t n_solves;
  int32_t iters_total;
  int32_t iters_max;
  double norm1_max;
} ins2d_step_stats;

/* --- context (the `options` struct) ------------------------------------- */
int ins2d_ctx_create(const ins2d_grid_desc *grid, const ins2d_bc_desc *bc,
                     const ins2d_opts *opts, ins2d_ctx **out);
int ins2d_ctx_destroy(ins2d_ctx *ctx);
const char *ins2d_last_error(const ins2d_ctx *ctx);
int ins2d_get_sizes(const ins2d_ctx *ctx, ins2d_sizes *out);
/* stream: a cudaStream_t (NULL = the context's own stream) */
int ins2d_set_stream(ins2d_ctx *ctx, void *stream);
/* Orders the context's later work after all work queued so far on the
 * cudaStream_t `stream` (an event recorded there, waited on by the context's
 * stream).  For device inputs produced on another stream, e.g. by a torch
 * kernel that may still be running: the context's own stream does not wait
 * for other streams by itself.  No-op when `stream` is the context's stream. */
int ins2d_wait_stream(ins2d_ctx *ctx, void *stream);
/* Grids whose PCG runs one launch per phase (more than 65536 cells with the
 * multigrid preconditioner, or the fast-diagonalization preconditioner) are
 * driven by the host, which polls a device convergence flag between chunks
 * of iterations.  This bounds the iterations the host launches while the
 * flag stays unset; past it the solve returns INS2D_ETIMEOUT.  iterations < 0
 * restores the default, CG_maxit + 1024.  Inside the CUDA graphs of
 * ins2d_erk_run (runs of two or more steps with steady boundary conditions)
 * the same solves loop on the device, in a conditional WHILE node; the
 * value bounds its passes (default CG_maxit / iterations per pass + 4) and
 * the run reports INS2D_ETIMEOUT when a loop stopped there unconverged.
 * Changing the value drops the captured graphs. */
int ins2d_set_poll_limit(ins2d_ctx *ctx, int64_t iterations);
/* set_bc_vectors.m:1 -- boundary values at time t (steady cases call it once) */
int ins2d_set_bc_values(ins2d_ctx *ctx, double t, const ins2d_bc_values *vals);
/* Unsteady boundary conditions (options.BC.BC_unsteady = 1): the context calls
 * fn(user, t, ctx) whenever the reference would call set_bc_vectors(t,options)
 * (time_ERK.m:62,106-109, F.m:97-99, pressure_additional_solve.m:11-13); fn
 * samples the case's uBC/vBC/dudtBC/dvdtBC at t and calls ins2d_set_bc_values.
 * A MEX gateway implements fn with mexCallMATLAB on the case's handles. */
typedef int (*ins2d_bc_sampler_fn)(void *user, double t, ins2d_ctx *ctx);
int ins2d_set_bc_sampler(ins2d_ctx *ctx, ins2d_bc_sampler_fn fn, void *user);

/* --- measurement ------------------------------------------------------------
 * Kernel families of a time step.  ins2d_profile(ctx, 1) starts bracketing
 * each family's launches with CUDA events on the context stream (and resets
 * the counters); ins2d_profile_read returns the accumulated device time (ms)
 * and the number of kernel launches per family since the last read, and
 * resets them.  Launches are counted whether or not profiling is on. */
#define INS2D_PROF_STAGE 0    /* RK stage right-hand side + combination */
#define INS2D_PROF_DIV 1      /* divergence right-hand side of the Poisson solve */
#define INS2D_PROF_POISSON 2  /* FFT passes or PCG kernels */
#define INS2D_PROF_PROJECT 3  /* projection V = Vn + dt (Vtemp - c Om^-1 G dp) */
#define INS2D_PROF_RESIDUAL 4 /* residual of the additional pressure solve */
#define INS2D_PROF_OTHER 5    /* F, divergence, Laplacian, conservation entry points */
#define INS2D_PROF_N 6
int ins2d_profile(ins2d_ctx *ctx, int enable);
int ins2d_profile_read(ins2d_ctx *ctx, double ms[INS2D_PROF_N], int64_t launches[INS2D_PROF_N]);

/* --- the hot path ---------------------------------------------------------- */
/* F.m:1 with getJacobian=0, T=0: F_out = -conv(V;C) + Diff*V + yDiff - (G*p + y_p);
 * C = NULL means C = V; p = NULL with nopressure=1 drops the pressure terms.
 * maxres (may be NULL) = max|F| (F.m:187). */
int ins2d_F(ins2d_ctx *ctx, const double *V, const double *C, const double *p,
            double t, int nopressure, double *F_out, double *maxres, int mem);
/* f_out = M*V + yM (check_conservation.m:37); maxdiv (may be NULL) = max|f_out| */
int ins2d_divergence(ins2d_ctx *ctx, const double *V, double *f_out, double *maxdiv, int mem);
/* Ap = A*p, A = M*diag(Om_inv)*G (operator_divergence.m:208) */
int ins2d_laplacian(ins2d_ctx *ctx, const double *p, double *Ap, int mem);
/* dp = pressure_poisson(f,t,options) (pressure_poisson.m:1-106): initial
 * guess 0; returns 0 when max|A*0 - f| < 1e-14 (:33-38); PCG to the relative
 * residual CG_acc (cg.F:240-247) or the FFT solve (:92-104). */
int ins2d_pressure_poisson(ins2d_ctx *ctx, const double *f, double *dp,
                           ins2d_solve_stats *stats, int mem);
/* p = pressure_additional_solve(V,p,T,t,options) (in place on p) */
int ins2d_pressure_additional_solve(ins2d_ctx *ctx, const double *V, double *p, double t,
                                    ins2d_solve_stats *stats, int mem);
/* [V,p] = time_ERK(V,p,T,t,dt,options), in place on V and p.  After an error
 * status the contents of V and p are unspecified, as with device memory: with
 * INS2D_MEM_HOST, V's copy out starts after the last projection, so V may
 * already hold the step's velocity when the additional solve fails. */
int ins2d_erk_step(ins2d_ctx *ctx, double *V, double *p, double t, double dt,
                   ins2d_step_stats *stats, int mem);
/* nsteps consecutive time_ERK steps from t with a fixed dt (solver_unsteady.m:72-102
 * without process_iteration); V, p device pointers updated in place.  With
 * steady boundary conditions and nsteps >= 2 each step is captured once as
 * a CUDA graph and replayed (PCG iteration loops as conditional WHILE
 * nodes); a PCG error is then reported after the step that raised it at the
 * latest 32 steps later, or at the end of the run. */
int ins2d_erk_run(ins2d_ctx *ctx, double *V, double *p, double t, double dt, int32_t nsteps,
                  ins2d_step_stats *stats, int mem);
/* The initial projection of input_check.m:95-111: when max|M V + yM| (also
 * returned in *maxdiv, may be NULL) exceeds 1e-12, V -= Om_inv .* (G dp) with
 * dp = pressure_poisson(M V + yM, t); V in place. */
int ins2d_initial_projection(ins2d_ctx *ctx, double *V, double t, double *maxdiv, int mem);
/* out[4] = {maxdiv, umom, vmom, k} (check_conservation.m:1-76) */
int ins2d_conservation(ins2d_ctx *ctx, const double *V, double t, double out[4], int mem);

/* --- allocation-free FFT solve ---------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (an application that gives the whole GPU to its own memory pool, a
 * plugin inside a host that owns the allocator, a real-time loop where
 * cudaMalloc must not run): dp = real(ifft2(-fft2(f)./Ahat)) on a periodic
 * uniform Nx x Ny grid with spacings dx, dy -- the FFT branch of
 * pressure_poisson.m:92-104 with its early return -- for device arrays f, dp
 * on the current device and a cudaStream_t stream (NULL = default stream).
 * Allocates nothing: the scratch lives in one static device array of
 * about 8.8 MB that every GPU loading the library keeps until exit.
 * Limits: 2 <= Nx, Ny <= INS2D_NOALLOC_MAX_N, Nx*Ny <= INS2D_NOALLOC_MAX_CELLS,
 * and sizes the FFT path supports; other sizes return INS2D_EINVAL.
 * The first call on a device looks up the array's device address and sets
 * kernel attributes.  A call whose (Nx, Ny, dx, dy) differ from the previous
 * call's on that device builds the twiddle and symbol tables on the host and
 * copies them in from pageable memory, waiting for the copies; a call with
 * the same values reuses the tables already on the device.  Every call
 * blocks until the stream has finished its work, so no call can be captured
 * into a CUDA graph.
 * All calls share the array: calls that overlap on the GPU (other streams,
 * other host threads) race and must be serialised by the caller.  An error
 * already pending on the calling thread (cudaGetLastError) is left to the
 * caller, neither cleared nor reported as this call's failure. */
#define INS2D_NOALLOC_MAX_N 4096
#define INS2D_NOALLOC_MAX_CELLS (1 << 20)
int ins2d_fft_poisson_noalloc(const double *f, double *dp, int32_t Nx, int32_t Ny, double dx, double dy,
                              void *stream);

/* --- one grid over several GPUs: FFT solve in y-slabs ---------------------
 * The reference's only distributed path is the PETSc-MPI Poisson solve
 * (solvers/pressure/petsc_poisson_par.c:38-52).  Here the FFT branch of
 * pressure_poisson.m:92-104 is split at the transposes for a periodic
 * uniform Nx x Ny grid whose rows are split over processes (one per GPU):
 * each rank transforms its rows, an all-to-all between the calls (done by
 * the caller, e.g. over NCCL) gives each rank whole columns of a range of
 * wave numbers, the column transforms apply -1/Ahat, and the inverse goes
 * back the same way.  Arrays are device arrays of the given device: spec
 * rows nrows x (Nx/2+1) complex (interleaved doubles), cols Ny x width
 * complex holding wave numbers I0 .. I0+width-1 (those >= Nx/2+1 are
 * padding).  Nx, Ny powers of two from 64 to 8192.  Every call returns after
 * the stream has finished its work. */
typedef struct ins2d_slab_fft ins2d_slab_fft;
int ins2d_slab_fft_create(int32_t Nx, int32_t Ny, double dx, double dy, int32_t device, ins2d_slab_fft **out);
int ins2d_slab_fft_destroy(ins2d_slab_fft *s);
const char *ins2d_slab_fft_last_error(const ins2d_slab_fft *s);
/* spec = forward transforms of the rows of f (nrows x Nx, real) */
int ins2d_slab_fft_rows_forward(ins2d_slab_fft *s, const double *f, int32_t nrows, double *spec, void *stream);
/* in place on cols: forward column transforms, -1/Ahat (Ahat(0,0) = 1),
 * inverse column transforms; *maxabs = max |fhat| of these columns (the
 * caller takes the maximum over the ranks for the early return) */
int ins2d_slab_fft_columns(ins2d_slab_fft *s, double *cols, int32_t width, int32_t I0, double *maxabs, void *stream);
/* dp rows (nrows x Nx) = inverse row transforms of spec, scaled 1/(Nx Ny);
 * all zero when maxabs (the maximum over all ranks) < 1e-14
 * (pressure_poisson.m:21-32) */
int ins2d_slab_fft_rows_inverse(ins2d_slab_fft *s, const double *spec, int32_t nrows, double maxabs, double *dp,
                                void *stream);

/* --- ensembles ------------------------------------------------------------
 * No single counterpart in the reference: the reference runs one case per
 * MATLAB process (main.m); ensembles of independent flows (different grids,
 * boundary conditions and Re, e.g. snapshot generation for reduced-order
 * models, process_iteration.m:79-87) are many such runs.  Here the members
 * are advanced together: each phase of a time step is one launch over all
 * members, and the Poisson solves are one persistent launch whose thread
 * blocks take members from a queue.  Members are full contexts (their
 * operators, boundary values, F, conservation, ... are reached through
 * ins2d_ens_member); the ensemble owns each member's state V, p.
 * Restrictions: steady boundary conditions, the PCG pressure solver
 * (poisson 1-5), the same device, precision, CG_acc, CG_maxit and RK method
 * for all members, at most 262144 pressure cells per member.
 * Preconditioner: when every member's opts.precond is INS2D_PRECOND_DEFAULT
 * or INS2D_PRECOND_FDM and every member has at most 1024 pressure cells per
 * direction, the solves are batched across members with fast
 * diagonalization; otherwise the members use multigrid (or Jacobi when
 * asked for) in the form the tuner picks.  Each time step is captured once as
 * a CUDA graph. */
typedef struct ins2d_ens ins2d_ens;
int ins2d_ens_create(int32_t n, const ins2d_grid_desc *grids, const ins2d_bc_desc *bcs,
                     const ins2d_opts *opts, ins2d_ens **out);
int ins2d_ens_destroy(ins2d_ens *e);
const char *ins2d_ens_last_error(const ins2d_ens *e);
int32_t ins2d_ens_size(const ins2d_ens *e);
/* member context (owned by the ensemble; NULL when m is out of range) */
ins2d_ctx *ins2d_ens_member(ins2d_ens *e, int32_t m);
int ins2d_ens_set_stream(ins2d_ens *e, void *stream);
/* as ins2d_wait_stream, for the ensemble's stream */
int ins2d_ens_wait_stream(ins2d_ens *e, void *stream);
/* member state V (NV values), p (Np values) in or out */
int ins2d_ens_set_state(ins2d_ens *e, int32_t m, const double *V, const double *p, int mem);
int ins2d_ens_get_state(ins2d_ens *e, int32_t m, double *V, double *p, int mem);
/* a member's own time step (dt > 0; 0 = the dt of ins2d_ens_erk_run), e.g. a
 * member whose explicit stability limit is below the ensemble's dt */
int ins2d_ens_set_member_dt(ins2d_ens *e, int32_t m, double dt);
/* device pointers of a member's state (valid for the ensemble's lifetime) */
int ins2d_ens_state_ptr(ins2d_ens *e, int32_t m, double **V, double **p);
/* nsteps of time_ERK for every member (time step dt, or the member's own);
 * stats: n entries
 * (per member, accumulated over the run) or NULL.  A member whose solve fails
 * makes the call return that status, naming the member. */
int ins2d_ens_erk_run(ins2d_ens *e, double t, double dt, int32_t nsteps, ins2d_step_stats *stats);
/* form of the member solves: -1 = chosen by the tuner on the first run
 * (default), 0 = batched across members, 256 or 512 = persistent launch with
 * that many threads per member (multigrid ensembles only: a
 * fast-diagonalization ensemble returns INS2D_EINVAL) */
int ins2d_ens_set_solver(ins2d_ens *e, int32_t threads);
/* form of the member solves chosen by the tuner on the first run: threads
 * per member of the persistent solve (512 or 256; 0 = solves batched across
 * members, one launch per phase), its resident blocks, and the tuner's
 * timings (ms of one solve phase for 512, 256 threads and batched) */
int ins2d_ens_solve_shape(const ins2d_ens *e, int32_t *threads, int32_t *blocks, double tuned_ms[3]);

/* --- learned initial guess of the PCG ---------------------------------------
 * No counterpart in the reference: its solves start from zero
 * (pressure_poisson.m:61-70, cg.F:207-229 with x_in = 0).  A small
 * convolutional network (six 3x3 convolutions, 1 -> 32 -> 32 -> 32 -> 32 -> 32
 * -> 1 channels, ReLU between, no biases, zero padding; BF16 tensor-core
 * layers accumulating in FP32) maps the Jacobi-scaled right-hand side to an
 * approximation of the solution.  The solver uses the network's odd part
 * (N(v) - N(-v))/2 (one forward pass over the pair v, -v), since A^-1 is
 * linear.  The PCG starts from that guess (scaled by the Rayleigh-Ritz factor
 * (x0'f)/(x0'A x0)) and still stops on the reference's rule
 * ||r|| <= CG_acc ||f||, so a solution changes only within the tolerance.
 * One network serves one context at a time (its activation buffers are
 * shared).  Parameters (INS2D_CNN_NPARAM floats): W1 [32][9],
 * W2..W5 [32][9][32] ([out][tap][in]), W6 [9][32]; tap t = (dy+1)*3 + (dx+1).
 * Inputs, targets and outputs of the network are fp32 device arrays of B
 * fields of H x W (x fastest). */
#define INS2D_CNN_NPARAM 37440
typedef struct ins2d_cnn ins2d_cnn;
/* He-normal weights from the seed; out_scale 1 */
int ins2d_cnn_create(int32_t device, uint64_t seed, ins2d_cnn **out);
int ins2d_cnn_destroy(ins2d_cnn *net);
const char *ins2d_cnn_last_error(const ins2d_cnn *net);
int ins2d_cnn_set_stream(ins2d_cnn *net, void *stream);
/* tensor-core instructions of the 32 -> 32 layers (forward and
 * backward-data): tcgen05.mma with TMEM accumulators (default) or the
 * warp-level mma.sync m16n8k16; both BF16 x BF16 -> FP32 */
#define INS2D_CNN_PATH_TCGEN05 0
#define INS2D_CNN_PATH_MMA_SYNC 1
int ins2d_cnn_set_path(ins2d_cnn *net, int32_t path);
/* host copies of the FP32 master weights (w may be NULL) and the output scale */
int ins2d_cnn_get_params(ins2d_cnn *net, float *w, float *out_scale);
int ins2d_cnn_set_params(ins2d_cnn *net, const float *w, float out_scale);
/* y = out_scale * net(in) */
int ins2d_cnn_forward(ins2d_cnn *net, const float *in, float *y, int32_t B, int32_t H, int32_t W);
/* host copy of the BF16 output of layer 1..5 (NHWC, 32 channels per pixel)
 * of the last forward pass over `pixels` = B*H*W pixels */
int ins2d_cnn_get_activations(ins2d_cnn *net, int32_t layer, int64_t pixels, uint16_t *out);
/* loss = mean((net(in) - tgt)^2) and its gradient (host array of
 * INS2D_CNN_NPARAM floats, may be NULL); no update */
int ins2d_cnn_loss_grad(ins2d_cnn *net, const float *in, const float *tgt, int32_t B, int32_t H, int32_t W,
                        double *loss, float *grad);
/* one Adam step (beta 0.9/0.999, eps 1e-8) on that loss */
int ins2d_cnn_train_step(ins2d_cnn *net, const float *in, const float *tgt, int32_t B, int32_t H, int32_t W,
                         float lr, double *loss);
/* The residual loss on a context's grid: mean((A y - diag(A) in)^2) with
 * y = net(in) and A = M Om^-1 G the context's pressure operator (for inputs
 * from ins2d_cnn_prepare_pairs, diag(A) in = f / s, so this is the scaled
 * residual of y as a solution); it rewards what a local network can learn, an
 * approximate inverse of A on the short wavelengths.  in: B fields of the
 * context's Npy x Npx pressure grid.  loss_grad returns the loss and the
 * gradient (host array, may be NULL); train_step takes one Adam step. */
int ins2d_cnn_loss_grad_residual(ins2d_ctx *ctx, ins2d_cnn *net, const float *in, int32_t B, double *loss,
                                 float *grad);
int ins2d_cnn_train_step_residual(ins2d_ctx *ctx, ins2d_cnn *net, const float *in, int32_t B, float lr,
                                  double *loss);
/* Training pairs of a context's grid: for npairs right-hand sides f and
 * solutions p (device, Np each, one after another) writes the network input
 * in = (f / diag A) / s and target tgt = (p - center * mean(p)) / s, with
 * s = rms(f / diag A) per pair (fp32 device arrays, Np each). */
int ins2d_cnn_prepare_pairs(ins2d_ctx *ctx, const double *f, const double *p, int32_t npairs, int32_t center,
                            float *in, float *tgt);
/* attach (net != NULL) or detach the learned initial guess of ctx's PCG
 * solves (poisson 1-5; the FFT path is direct and ignores it).  The context
 * borrows the network: keep it alive while attached. */
int ins2d_set_learned_guess(ins2d_ctx *ctx, ins2d_cnn *net);
/* role of the attached network: INS2D_LEARNED_GUESS (default: the PCG with
 * the context's preconditioner starts from the network's guess) or
 * INS2D_LEARNED_PRECOND (flexible CG, FCG(1), from the guess with the network
 * as the preconditioner, z = M(r); after 200 iterations without convergence
 * or on a breakdown the plain PCG finishes from the current iterate).  Both
 * stop on ||r|| <= CG_acc ||f||. */
#define INS2D_LEARNED_GUESS 0
#define INS2D_LEARNED_PRECOND 1
int ins2d_set_learned_mode(ins2d_ctx *ctx, int32_t mode);
/* Recording of the solver's own (f, dp) pairs: each later PCG solve without
 * a learned guess copies its right-hand side and solution into the device
 * buffers f_buf, p_buf (capacity pairs of Np doubles) until they are full;
 * capacity 0 stops recording.  ins2d_recorded_pairs gives the count. */
int ins2d_record_pairs(ins2d_ctx *ctx, double *f_buf, double *p_buf, int32_t capacity);
int32_t ins2d_recorded_pairs(const ins2d_ctx *ctx);
/* The whole training recipe in one call, for callers without device buffers
 * of their own (a MATLAB gateway): from the state (V, p) at time t (host or
 * device arrays per mem; not modified) the context runs record_steps time
 * steps of dt, recording up to max_pairs (f, dp) pairs of its PCG solves
 * (the attached network, if any, is not used meanwhile), then trains net
 * for train_steps Adam steps on the residual loss: batches of `batch`
 * recorded inputs and `noise` white-noise fields, each with its negation,
 * rate cosine-decayed from lr to lr/20, batch draws seeded by `seed`.
 * loss_first / loss_last (may be NULL): the loss of the first and last step.
 * Allocates its work arrays for the duration of the call. */
int ins2d_learned_train(ins2d_ctx *ctx, ins2d_cnn *net, const double *V, const double *p, double t, double dt,
                        int32_t record_steps, int32_t max_pairs, int32_t train_steps, int32_t batch, float lr,
                        int32_t noise, uint64_t seed, int mem, double *loss_first, double *loss_last);

#ifdef __cplusplus
}
#endif
#endif /* INS2D_H */
