// Context and C-ABI of libins2d.so (include/ins2d.h).
//
// The context plays the role of the reference's `options` struct: it holds
// the device-resident operator tables (derived once, setup.cpp), the boundary
// values of the current time, the Butcher tableau and the solver settings.
// time_ERK's stage loop (unsteady/time_ERK.m:78-168) is orchestrated here on
// the host; all arithmetic runs in the device kernels on the context stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "cnn.cuh"
#include "ins2d.h"
#include "kernels.cuh"
#include "setup.hpp"
#include "mg_host.hpp"
#include "fdm_host.hpp"

using namespace ins2d;

// a captured time step (erk_run: FFT solves, or PCG solves whose iteration
// loops are conditional WHILE nodes of the graph)
struct StepGraph {
  cudaGraphExec_t exec = nullptr;
  const double *V = nullptr, *p = nullptr;
  double dt = 0.0;
  long long launches[INS2D_PROF_N] = {};
};

struct ins2d_ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  HostOps H;
  DevOps P{};
  ins2d_opts opts{};
  ins2d_bc_desc bcd{};
  bool fp32 = false;
  int poisson = 4;
  std::string err;
  std::vector<void *> allocs;
  // RK tableau shifted as in time_ERK.m:29-32
  int s = 0;
  double A[kMaxStages][kMaxStages] = {};
  double c[kMaxStages] = {};
  bool need_store[kMaxStages] = {};
  // device work arrays
  double *Vs = nullptr, *Wt = nullptr, *kV[kMaxStages] = {};
  // FP32 storage of the stage quantities (FP32-stencil contexts): the stage
  // velocity, each stage's kV and the combined Vtemp
  bool store32 = false;
  float *Vs32 = nullptr, *kV32[kMaxStages] = {}, *Vt32 = nullptr;
  double *f = nullptr, *dp = nullptr, *wres = nullptr;
  double *stV = nullptr, *stC = nullptr, *stO = nullptr, *stP = nullptr, *stQ = nullptr;  // host-mode staging
  double *bcblob = nullptr;
  size_t bc_count = 0;
  RedScratch red;
  FftPlan fft;
  PcgWork pcg{};
  bool use_mg = false;
  MgD mg{};
  // fast-diagonalization preconditioner (INS2D_PRECOND_FDM)
  bool use_fdm = false;
  FdmD fdm{};
  FftPlan fdm_fft;
  PcgScalars *h_sc = nullptr;   // pinned
  // PCG solves inside a step graph: the iteration loop is a WHILE node whose
  // body is captured on body_stream; their statistics accumulate on the device
  bool dev_loop = false;
  cudaStream_t body_stream = nullptr;
  SolveAccum *accum = nullptr;    // device
  SolveAccum *h_accum = nullptr;  // pinned
  // steps on host memory: p's copy in runs on copy_stream while the first
  // stage's right-hand side is computed (the step waits on ev_p before it
  // reads p), and V's copy out starts on copy_stream after the last
  // projection, while the additional pressure solve runs
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_p = nullptr, ev_v = nullptr;
  bool p_pending = false;
  double *v_out_host = nullptr;  // erk_step copies V there after its last projection
  bool v_out_done = false;
  double *h_red = nullptr;      // pinned
  // host copies of boundary samples (check_conservation.m boundary terms)
  std::vector<double> uLe_i, uRi_i, vLo_i, vUp_i;
  ins2d_bc_sampler_fn sampler = nullptr;
  void *sampler_user = nullptr;
  double bc_time = 0.0;
  // launch counts and optional device-time profile per kernel family
  long long launches[INS2D_PROF_N] = {};
  bool prof = false;
  struct Rec {
    int fam;
    cudaEvent_t a, b;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t order_ev = nullptr;  // ins2d_wait_stream
  long long poll_limit = -1;       // ins2d_set_poll_limit (-1: CG_maxit + 1024)
  StepGraph step_graph[2];
  // learned initial guess of the PCG (borrowed network) and its work arrays
  ins2d_cnn *cnn = nullptr;
  int lg_mode = INS2D_LEARNED_GUESS;
  double *lg_x0 = nullptr, *lg_q = nullptr, *lg_r0 = nullptr, *lg_red = nullptr, *lg_p = nullptr, *lg_z = nullptr;
  // recording of (f, dp) pairs of the plain PCG solves
  double *rec_f = nullptr, *rec_p = nullptr;
  int rec_cap = 0, rec_n = 0;
};

namespace {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define CK(x)                                                                                   \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess) throw CudaError(std::string(#x) + ": " + cudaGetErrorString(e_));   \
  } while (0)

template <typename T>
T *dalloc(ins2d_ctx *c, size_t n) {
  void *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T));
  if (e != cudaSuccess) throw std::bad_alloc();
  c->allocs.push_back(p);
  return (T *)p;
}

Tab upload_tab(ins2d_ctx *c, const Table &t) {
  Tab d;
  int32_t *cc = dalloc<int32_t>(c, t.col.size());
  double *w = dalloc<double>(c, t.w.size());
  double *b1 = dalloc<double>(c, t.b1.size());
  double *b2 = dalloc<double>(c, t.b2.size());
  CK(cudaMemcpy(cc, t.col.data(), t.col.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(w, t.w.data(), t.w.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b1, t.b1.data(), t.b1.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b2, t.b2.data(), t.b2.size() * sizeof(double), cudaMemcpyHostToDevice));
  d.c = cc;
  d.w = w;
  d.b1 = b1;
  d.b2 = b2;
  return d;
}

const double *upload_vec(ins2d_ctx *c, const std::vector<double> &v) {
  double *d = dalloc<double>(c, v.size());
  if (!v.empty()) CK(cudaMemcpy(d, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
  return d;
}

// Layout of the boundary-value blob: {name, length}.
struct BcSlot {
  const double **dst;
  int n;
};

std::vector<BcSlot> bc_slots(ins2d_ctx *c) {
  HostOps &H = c->H;
  BcVals &b = c->P.bc;
  return {{&b.uLo, H.Nx + 1},   {&b.uUp, H.Nx + 1},   {&b.uLo_i, H.Nux},   {&b.uUp_i, H.Nux},
          {&b.uLe_i, H.Ny},     {&b.uRi_i, H.Ny},     {&b.vLe, H.Ny + 1},  {&b.vRi, H.Ny + 1},
          {&b.vLo_i, H.Nx},     {&b.vUp_i, H.Nx},     {&b.vLe_i, H.Nvy},   {&b.vRi_i, H.Nvy},
          {&b.XvLo, H.Nux},     {&b.XvUp, H.Nux},     {&b.YuLe, H.Nvy},    {&b.YuRi, H.Nvy},
          {&b.pLe, H.Ny},       {&b.pRi, H.Ny},       {&b.pLo, H.Nx},      {&b.pUp, H.Nx},
          {&b.dudtLe_i, H.Ny},  {&b.dudtRi_i, H.Ny},  {&b.dvdtLo_i, H.Nx}, {&b.dvdtUp_i, H.Nx}};
}

cudaEvent_t take_event(ins2d_ctx *c) {
  if (!c->pool.empty()) {
    cudaEvent_t e = c->pool.back();
    c->pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  CK(cudaEventCreate(&e));
  return e;
}

// Brackets the launches of one kernel family with CUDA events on the
// context stream when profiling is on; counts the launches always.
struct Prof {
  ins2d_ctx *c;
  int fam;
  cudaEvent_t b = nullptr;
  Prof(ins2d_ctx *c_, int fam_, int nlaunch) : c(c_), fam(fam_) {
    c->launches[fam] += nlaunch;
    if (c->prof) {
      b = take_event(c);
      CK(cudaEventRecord(b, c->stream));
    }
  }
  ~Prof() {
    if (c->prof && b) {
      cudaEvent_t e = take_event(c);
      cudaEventRecord(e, c->stream);
      c->recs.push_back({fam, b, e});
    }
  }
};

int fail(ins2d_ctx *c, int code, const std::string &msg) {
  if (c) c->err = msg;
  return code;
}

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

void setup_rk(ins2d_ctx *c) {
  // default: classical RK44 (getRKmethod.m:313-316)
  int s = c->opts.rk_stages;
  double A0[kMaxStages][kMaxStages] = {}, b0[kMaxStages] = {}, c0[kMaxStages] = {};
  if (s <= 0) {
    s = 4;
    A0[1][0] = 0.5;
    A0[2][1] = 0.5;
    A0[3][2] = 1.0;
    b0[0] = 1.0 / 6;
    b0[1] = 1.0 / 3;
    b0[2] = 1.0 / 3;
    b0[3] = 1.0 / 6;
    c0[1] = 0.5;
    c0[2] = 0.5;
    c0[3] = 1.0;
  } else {
    for (int i = 0; i < s; ++i) {
      for (int j = 0; j < s; ++j) A0[i][j] = c->opts.rk_A[i * s + j];
      b0[i] = c->opts.rk_b[i];
      c0[i] = c->opts.rk_c[i];
    }
  }
  c->s = s;
  // shifted tableau (time_ERK.m:29-32): rows 2..s of A then b'; c = [c(2:end); 1]
  for (int i = 0; i < s; ++i)
    for (int j = 0; j < s; ++j) c->A[i][j] = (i < s - 1) ? A0[i + 1][j] : b0[j];
  for (int i = 0; i < s; ++i) c->c[i] = (i < s - 1) ? c0[i + 1] : 1.0;
  for (int m = 0; m < s; ++m) {
    c->need_store[m] = false;
    for (int i = m + 1; i < s; ++i)
      if (c->A[i][m] != 0.0) c->need_store[m] = true;
  }
}

// ---------------------------------------------------------------------------
// Poisson solve: dp = pressure_poisson(f) (or dp += ... when accumulate)

// Adds a conditional WHILE node to the graph being captured on stream s.
// pre(h) is captured on s before the node and sets the condition's first
// value; body(bs, h) is captured on body_stream (a second stream of the same
// device) into the node's body graph, and its last kernel sets the condition
// again.  Throws CudaError when s is not capturing.
template <class Pre, class Body>
void capture_while(cudaStream_t s, cudaStream_t body_stream, Pre pre, Body body) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
  if (cs != cudaStreamCaptureStatusActive) throw CudaError("device-side loop outside a stream capture");
  cudaGraphConditionalHandle h;
  CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
  pre(h);
  CK(cudaGetLastError());
  CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, g, deps, nd, &np));
  CK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  CK(cudaStreamBeginCaptureToGraph(body_stream, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                   cudaStreamCaptureModeThreadLocal));
  try {
    body(body_stream, h);
  } catch (...) {
    cudaGraph_t junk = nullptr;
    cudaStreamEndCapture(body_stream, &junk);
    throw;
  }
  const cudaError_t le = cudaGetLastError();
  cudaGraph_t body_out = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(body_stream, &body_out);
  CK(le);
  CK(ee);
}

// The PCG solve inside a step being captured as a CUDA graph (c->dev_loop):
// no host round trip.  The iterations are the body of a conditional WHILE
// node, captured on the context's second stream into the node's body graph;
// a one-thread kernel after the initialisation and at the end of each pass
// sets the condition to "not converged and fewer passes than the limit", so
// the loop ends by itself.  The solve's iterations, residual and status are
// added to c->accum, which the host reads after the graph launches (cg.F's
// errors are reported then).
int solve_pcg_graph(ins2d_ctx *c, const double *f, double *dp, bool accumulate, double tol) {
  const bool block = c->use_fdm ? pcg_use_block_fdm(c->fdm)
                                : (c->use_mg ? (c->P.Np <= kPcgBlockMgMaxCells) : pcg_use_block(c->P));
  Prof pr(c, INS2D_PROF_POISSON, block ? 1 : 2);
  if (block) {
    if (c->use_fdm)
      pcg_solve_block_fdm(c->P, c->fdm, c->pcg, f, dp, tol, c->opts.CG_maxit, accumulate, c->stream);
    else if (c->use_mg)
      pcg_solve_block_mg(c->P, c->mg, c->pcg, f, dp, tol, c->opts.CG_maxit, accumulate, c->stream);
    else
      pcg_solve_block(c->P, c->pcg, f, dp, tol, c->opts.CG_maxit, accumulate, c->stream);
    CK(cudaGetLastError());
    launch_solve_accum(c->pcg.sc, c->accum, c->stream);
    CK(cudaGetLastError());
    return INS2D_OK;
  }
  if (c->use_fdm)
    pcg_init_fdm(c->P, c->fdm, c->pcg, f, tol, c->opts.CG_maxit, c->stream);
  else if (c->use_mg)
    pcg_init_mg(c->P, c->mg, c->pcg, f, tol, c->opts.CG_maxit, c->stream);
  else
    pcg_init(c->P, c->pcg, f, tol, c->opts.CG_maxit, c->stream);
  CK(cudaGetLastError());
  const int chunk = (c->use_fdm || c->use_mg) ? 1 : 4;
  const long long lim = c->poll_limit >= 0 ? c->poll_limit : (long long)c->opts.CG_maxit / chunk + 4;
  const int limit = (int)std::min<long long>(lim, 1 << 30);
  capture_while(
      c->stream, c->body_stream,
      [&](cudaGraphConditionalHandle h) { launch_pcg_cond(c->pcg.sc, h, limit, 0, c->stream); },
      [&](cudaStream_t bs, cudaGraphConditionalHandle h) {
        if (c->use_fdm) {
          pcg_iterations_fdm(c->P, c->fdm, c->pcg, chunk, bs);
          c->launches[INS2D_PROF_POISSON] += (c->fdm.spectral ? 4LL + fft_kernels(c->fdm_fft) : 8LL) * chunk;
        } else if (c->use_mg) {
          pcg_iterations_mg(c->P, c->mg, c->pcg, chunk, bs);
          c->launches[INS2D_PROF_POISSON] += (long long)(4 + 6 * mg_tail_level(c->mg) + 1) * chunk;
        } else {
          pcg_iterations(c->P, c->pcg, chunk, bs);
          c->launches[INS2D_PROF_POISSON] += 3LL * chunk;
        }
        launch_pcg_cond(c->pcg.sc, h, limit, 1, bs);
      });
  pcg_finish(c->P, c->pcg, dp, accumulate, c->stream);
  launch_solve_accum(c->pcg.sc, c->accum, c->stream);
  c->launches[INS2D_PROF_POISSON] += 3;
  CK(cudaGetLastError());
  return INS2D_OK;
}

// PCG to the relative residual tol (cg.F's rule ||r|| <= tol ||f||)
int solve_pcg(ins2d_ctx *c, const double *f, double *dp, bool accumulate, ins2d_solve_stats *st, double tol) {
  if (c->dev_loop) {
    if (st) *st = ins2d_solve_stats{0, 0.0, 0.0};
    return solve_pcg_graph(c, f, dp, accumulate, tol);
  }
  const bool block = c->use_fdm ? pcg_use_block_fdm(c->fdm)
                                : (c->use_mg ? (c->P.Np <= kPcgBlockMgMaxCells) : pcg_use_block(c->P));
  Prof pr(c, INS2D_PROF_POISSON, block ? 1 : 2);
  if (block) {
    if (c->use_fdm)
      pcg_solve_block_fdm(c->P, c->fdm, c->pcg, f, dp, tol, c->opts.CG_maxit, accumulate, c->stream);
    else if (c->use_mg)
      pcg_solve_block_mg(c->P, c->mg, c->pcg, f, dp, tol, c->opts.CG_maxit, accumulate, c->stream);
    else
      pcg_solve_block(c->P, c->pcg, f, dp, tol, c->opts.CG_maxit, accumulate, c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_sc, c->pcg.sc, sizeof(PcgScalars), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const PcgScalars &h = *c->h_sc;
    if (st) {
      st->iters = (int32_t)h.it;
      st->norm1 = std::sqrt(h.rr);
      st->norm2 = (h.maxx - h.minx) != 0.0 ? h.maxres / (h.maxx - h.minx) : 0.0;
    }
    if (h.status == INS2D_ENOTCONV) {
      char buf[160];
      snprintf(buf, sizeof buf, "CG didn't converge in %d iterations; residual= %g", c->opts.CG_maxit,
               std::sqrt(h.rr));
      return fail(c, INS2D_ENOTCONV, buf);
    }
    if (h.status == INS2D_EBREAKDOWN) return fail(c, INS2D_EBREAKDOWN, "PCG breakdown: p'Ap = 0");
    if (h.status == INS2D_ENONFINITE) return fail(c, INS2D_ENONFINITE, "PCG: non-finite residual");
    return INS2D_OK;
  }
  if (c->use_fdm)
    pcg_init_fdm(c->P, c->fdm, c->pcg, f, tol, c->opts.CG_maxit, c->stream);
  else if (c->use_mg)
    pcg_init_mg(c->P, c->mg, c->pcg, f, tol, c->opts.CG_maxit, c->stream);
  else
    pcg_init(c->P, c->pcg, f, tol, c->opts.CG_maxit, c->stream);
  CK(cudaGetLastError());
  // the fast-diagonalization preconditioner is exact up to rounding: one
  // iteration at a time between the polls
  int chunk = c->use_fdm ? 1 : (c->use_mg ? 2 : 4);
  long long launched = 0;
  for (;;) {
    CK(cudaMemcpyAsync(c->h_sc, c->pcg.sc, sizeof(PcgScalars), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (c->h_sc->done) break;
    const long long limit = c->poll_limit >= 0 ? c->poll_limit : (long long)c->opts.CG_maxit + 1024;
    if (launched >= limit)
      return fail(c, INS2D_ETIMEOUT, "PCG: device convergence flag not set within the host's iteration limit");
    if (c->use_fdm) {
      pcg_iterations_fdm(c->P, c->fdm, c->pcg, chunk, c->stream);
      c->launches[INS2D_PROF_POISSON] += (c->fdm.spectral ? 4LL + fft_kernels(c->fdm_fft) : 8LL) * chunk;
    } else if (c->use_mg) {
      pcg_iterations_mg(c->P, c->mg, c->pcg, chunk, c->stream);
      c->launches[INS2D_PROF_POISSON] += (long long)(4 + 6 * mg_tail_level(c->mg) + 1) * chunk;
    } else {
      pcg_iterations(c->P, c->pcg, chunk, c->stream);
      c->launches[INS2D_PROF_POISSON] += 3LL * chunk;
    }
    CK(cudaGetLastError());
    launched += chunk;
    chunk = c->use_fdm ? 1 : (c->use_mg ? 4 : std::min(chunk * 2, 128));
  }
  const PcgScalars &h = *c->h_sc;
  if (st) {
    st->iters = (int32_t)h.it;
    st->norm1 = std::sqrt(h.rr);
    st->norm2 = (h.maxx - h.minx) != 0.0 ? h.maxres / (h.maxx - h.minx) : 0.0;
  }
  if (h.status == INS2D_ENOTCONV) {
    char buf[160];
    snprintf(buf, sizeof buf, "CG didn't converge in %d iterations; residual= %g", c->opts.CG_maxit,
             std::sqrt(h.rr));
    return fail(c, INS2D_ENOTCONV, buf);
  }
  if (h.status == INS2D_EBREAKDOWN) return fail(c, INS2D_EBREAKDOWN, "PCG breakdown: p'Ap = 0");
  if (h.status == INS2D_ENONFINITE) return fail(c, INS2D_ENONFINITE, "PCG: non-finite residual");
  pcg_finish(c->P, c->pcg, dp, accumulate, c->stream);
  c->launches[INS2D_PROF_POISSON] += 1;
  CK(cudaGetLastError());
  return INS2D_OK;
}

// PCG from the learned initial guess: x0 = a * net(f) with the Rayleigh-Ritz
// factor a = (x0'f)/(x0'A x0) (the best multiple of the network's output in
// the energy norm), then CG on A e = r0 = f - A x0 to ||r|| <= CG_acc ||f||
// (the inner tolerance is rescaled to ||r0||), dp = x0 + e.  Right-hand
// sides with max|f| < 1e-14 take the plain path (pressure_poisson.m:33-38).
// Flexible CG with the network as the preconditioner, from x = lg_x0 with
// residual r = lg_r0 (FCG(1): each new direction z = M(r) is A-orthogonalised
// against the previous one, beta = -(z'Ap)/(p'Ap), which keeps CG's short
// recurrence meaningful for a nonlinear M).  Same stopping rule as cg.F.  If
// it has not converged after kFcgMaxit iterations or breaks down, the plain
// PCG finishes the solve from the current iterate.
constexpr int kFcgMaxit = 200;
int fcg_learned(ins2d_ctx *c, double *dp, bool accumulate, ins2d_solve_stats *st, double ff) {
  const long long n = c->P.Np;
  const double tol = c->opts.CG_acc;
  double *x = c->lg_x0, *r = c->lg_r0, *q = c->lg_q, *p = c->lg_p, *z = c->lg_z;
  const int maxit = std::min(c->opts.CG_maxit, kFcgMaxit);
  bool conv = false;
  double rr = 0.0;
  int it = 0;
  {
    Prof pr(c, INS2D_PROF_POISSON, 12);
    cnn::precond(c->cnn, c->P, r, z, c->stream);
    CK(cudaMemcpyAsync(p, z, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  }
  while (it < maxit) {
    Prof pr(c, INS2D_PROF_POISSON, 20);
    launch_lap(c->P, p, q, c->stream);
    CK(cudaGetLastError());
    double d[2], u[2];
    cnn::fcg_pq(n, p, q, r, c->lg_red, d, c->stream);
    if (!std::isfinite(d[0]) || !std::isfinite(d[1]) || d[0] == 0.0) break;
    cnn::fcg_update(n, d[1] / d[0], x, r, p, q, c->lg_red, u, c->stream);
    ++it;
    rr = u[0];
    if (!std::isfinite(rr)) return fail(c, INS2D_ENONFINITE, "FCG: non-finite residual");
    if (rr <= tol * tol * ff || u[1] < 1e-300) {
      conv = true;
      break;
    }
    cnn::precond(c->cnn, c->P, r, z, c->stream);
    cnn::fcg_p(n, -cnn::fcg_zq(n, z, q, c->lg_red, c->stream) / d[0], z, p, c->stream);
  }
  cnn::check(c->cnn, c->stream);
  if (conv) {
    Prof pr(c, INS2D_PROF_POISSON, 1);
    if (accumulate)
      launch_add(x, dp, n, c->stream);
    else
      CK(cudaMemcpyAsync(dp, x, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaGetLastError());
    if (st) *st = ins2d_solve_stats{it, std::sqrt(rr / ff), 0.0};
    return INS2D_OK;
  }
  double d[2];
  cnn::fcg_pq(n, r, r, r, c->lg_red, d, c->stream);
  const double scale = std::sqrt(d[0] / ff);
  int rc = solve_pcg(c, r, dp, accumulate, st, tol / scale);
  if (rc) return rc;
  if (st) {
    st->norm1 *= scale;
    st->iters += it;
  }
  Prof pr(c, INS2D_PROF_POISSON, 1);
  launch_add(x, dp, n, c->stream);
  CK(cudaGetLastError());
  return INS2D_OK;
}

int solve_learned(ins2d_ctx *c, const double *f, double *dp, bool accumulate, ins2d_solve_stats *st) {
  const long long n = c->P.Np;
  const double tol = c->opts.CG_acc;
  double d[4], rd[2];
  {
    Prof pr(c, INS2D_PROF_POISSON, 13);
    cnn::guess(c->cnn, c->P, f, c->lg_x0, c->stream);
    launch_lap(c->P, c->lg_x0, c->lg_q, c->stream);
    CK(cudaGetLastError());
    cnn::dots(n, c->lg_x0, f, c->lg_q, c->lg_red, d, c->stream);
  }
  if (!(d[3] >= 1e-14) || !std::isfinite(d[0]) || !std::isfinite(d[1]) || d[1] == 0.0)
    return solve_pcg(c, f, dp, accumulate, st, tol);
  {
    Prof pr(c, INS2D_PROF_POISSON, 2);
    cnn::residual(n, f, c->lg_q, d[0] / d[1], c->lg_x0, c->lg_r0, c->lg_red, rd, c->stream);
  }
  const double ff = d[2], rr0 = rd[0];
  if (rr0 <= tol * tol * ff || rd[1] < 1e-14) {
    Prof pr(c, INS2D_PROF_POISSON, 1);
    if (accumulate)
      launch_add(c->lg_x0, dp, n, c->stream);
    else
      CK(cudaMemcpyAsync(dp, c->lg_x0, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaGetLastError());
    if (st) *st = ins2d_solve_stats{0, std::sqrt(rr0 / ff), 0.0};
    return INS2D_OK;
  }
  if (c->lg_mode == INS2D_LEARNED_PRECOND) return fcg_learned(c, dp, accumulate, st, ff);
  const double scale = std::sqrt(rr0 / ff);
  int rc = solve_pcg(c, c->lg_r0, dp, accumulate, st, tol / scale);
  if (rc) return rc;
  if (st) st->norm1 *= scale;
  Prof pr(c, INS2D_PROF_POISSON, 1);
  launch_add(c->lg_x0, dp, n, c->stream);
  CK(cudaGetLastError());
  return INS2D_OK;
}

int solve(ins2d_ctx *c, const double *f, double *dp, bool accumulate, ins2d_solve_stats *st) {
  if (st) *st = ins2d_solve_stats{0, 0.0, 0.0};
  if (c->poisson == INS2D_POISSON_FFT) {
    Prof pr(c, INS2D_PROF_POISSON, fft_kernels(c->fft));
    CK(launch_fft_poisson(c->P, c->fft, f, dp, accumulate, c->stream));
    CK(cudaGetLastError());
    return INS2D_OK;
  }
  if (c->cnn) return solve_learned(c, f, dp, accumulate, st);
  int rc = solve_pcg(c, f, dp, accumulate, st, c->opts.CG_acc);
  if (rc == INS2D_OK && c->rec_n < c->rec_cap) {
    // the solution stays in the PCG iterate x after the solve
    const size_t nb = (size_t)c->P.Np * sizeof(double);
    CK(cudaMemcpyAsync(c->rec_f + (size_t)c->rec_n * c->P.Np, f, nb, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->rec_p + (size_t)c->rec_n * c->P.Np, c->pcg.x, nb, cudaMemcpyDeviceToDevice, c->stream));
    c->rec_n += 1;
  }
  return rc;
}

// dp = pressure_poisson(f) with f = (M W + alpha yM + beta ydM) gamma: on the
// FFT path the divergence is computed inside the first transform pass;
// otherwise by its own kernel before the solve.
int solve_div(ins2d_ctx *c, const double *W, double alpha, double beta, double gamma, double *dp, bool accumulate,
              ins2d_solve_stats *st) {
  if (c->poisson == INS2D_POISSON_FFT && fft_fuses_div(c->fft)) {
    if (st) *st = ins2d_solve_stats{0, 0.0, 0.0};
    Prof pr(c, INS2D_PROF_POISSON, fft_kernels(c->fft));
    CK(launch_fft_poisson_div(c->P, c->fft, W, alpha, beta, gamma, dp, accumulate, c->stream));
    CK(cudaGetLastError());
    return INS2D_OK;
  }
  {
    Prof pr(c, INS2D_PROF_DIV, 1);
    launch_div(c->P, W, alpha, beta, gamma, c->f, false, c->red, c->stream);
  }
  CK(cudaGetLastError());
  return solve(c, c->f, dp, accumulate, st);
}

// the same with W = Vn sv + sa T, T in FP32 (FP32-storage stages)
int solve_div_split(ins2d_ctx *c, const double *Vn, const float *T, double sv, double sa, double alpha, double beta,
                    double gamma, double *dp, bool accumulate, ins2d_solve_stats *st) {
  if (c->poisson == INS2D_POISSON_FFT && fft_fuses_div(c->fft)) {
    if (st) *st = ins2d_solve_stats{0, 0.0, 0.0};
    Prof pr(c, INS2D_PROF_POISSON, fft_kernels(c->fft));
    CK(launch_fft_poisson_div_split(c->P, c->fft, Vn, T, sv, sa, alpha, beta, gamma, dp, accumulate, c->stream));
    CK(cudaGetLastError());
    return INS2D_OK;
  }
  {
    Prof pr(c, INS2D_PROF_DIV, 1);
    launch_div_split(c->P, Vn, T, sv, sa, alpha, beta, gamma, c->f, c->stream);
  }
  CK(cudaGetLastError());
  return solve(c, c->f, dp, accumulate, st);
}

void stats_add(ins2d_step_stats *s, const ins2d_solve_stats &o) {
  if (!s) return;
  s->n_solves += 1;
  s->iters_total += o.iters;
  s->iters_max = std::max(s->iters_max, o.iters);
  s->norm1_max = std::max(s->norm1_max, o.norm1);
}

int sample_bc(ins2d_ctx *c, double t) {
  if (!c->bcd.bc_unsteady) return INS2D_OK;
  if (!c->sampler) return fail(c, INS2D_EINVAL, "unsteady boundary conditions need a sampler (ins2d_set_bc_sampler)");
  int rc = c->sampler(c->sampler_user, t, c);
  if (rc != INS2D_OK && c->err.empty()) c->err = "boundary sampler failed";
  return rc;
}

// p = pressure_additional_solve(V,p,T,t,options)   (device pointers); when
// kV_next is given it also receives Om^-1 R(V) (the next step's first-stage
// right-hand side).
int additional_solve(ins2d_ctx *c, const double *V, double *p, double t, ins2d_solve_stats *st,
                     bool cache = false) {
  int rc = sample_bc(c, t);
  if (rc) return rc;
  {
    Prof pr(c, INS2D_PROF_RESIDUAL, 1);
    double *kn = (cache && !c->store32) ? c->kV[0] : nullptr;
    float *kn32 = (cache && c->store32) ? c->kV32[0] : nullptr;
    launch_residual(c->P, V, p, c->wres, kn, kn32, c->fp32, c->stream);
  }
  return solve_div(c, c->wres, 0.0, c->bcd.bc_unsteady ? 1.0 : 0.0, 1.0, p, true, st);
}

// The step reads or writes p only after wait_p: on host memory p is still
// being copied in on copy_stream while the first stage's right-hand side runs.
void wait_p(ins2d_ctx *c) {
  if (!c->p_pending) return;
  CK(cudaStreamWaitEvent(c->stream, c->ev_p, 0));
  c->p_pending = false;
}
// after the step's last projection: V is final, so its copy to the host
// (when requested) starts on copy_stream beside the additional solve
void copy_v_out(ins2d_ctx *c, const double *V) {
  if (!c->v_out_host) return;
  CK(cudaEventRecord(c->ev_v, c->stream));
  CK(cudaStreamWaitEvent(c->copy_stream, c->ev_v, 0));
  CK(cudaMemcpyAsync(c->v_out_host, V, (size_t)(c->P.Nu + c->P.Nv) * sizeof(double), cudaMemcpyDeviceToHost,
                     c->copy_stream));
  c->v_out_host = nullptr;
  c->v_out_done = true;
}

// [V,p] = time_ERK(V,p,T,t,dt,options) on device pointers, in place.
// k0_cached: kV[0] already holds Om^-1 R(V) (steady BCs, the previous step of
// the same run computed it in its additional solve); on return *cache_next
// says whether kV[0] holds it for the next step.
// time_ERK with FP32 storage of the stage quantities (FP32-stencil contexts):
// the stage velocity, kV and Vtemp in FP32; Vn, p, the divergence (f =
// (M (Vn/dt + Vtemp) + yM/dt)/c evaluated in FP64), the Poisson solve and the
// projection (V = Vn + dt (Vtemp - c Om^-1 G dp) in FP64) as in the FP64 path.
int erk_step32(ins2d_ctx *c, double *V, double *p, double t, double dt, ins2d_step_stats *stats, bool k0_cached,
               bool *cache_next) {
  const DevOps &P = c->P;
  if (cache_next) *cache_next = false;
  int rc = sample_bc(c, t);
  if (rc) return rc;
  const double *dpp = nullptr;
  for (int i = 0; i < c->s; ++i) {
    const float *Ti = nullptr;  // Vtemp_i = ai * Ti
    double ai = 1.0;
    if (i == 0 && k0_cached && !c->bcd.bc_unsteady) {
      Ti = c->kV32[0];  // the previous step's residual: kV of this step's first stage
      ai = c->A[0][0];
    } else {
      StageArgs a{};
      a.V = (i == 0) ? V : nullptr;
      a.V32 = (i == 0) ? nullptr : c->Vs32;
      a.store32 = true;
      a.nprev = 0;
      for (int m = 0; m < i; ++m)
        if (c->A[i][m] != 0.0) {
          a.kprev32[a.nprev] = c->kV32[m];
          a.aprev[a.nprev] = c->A[i][m];
          ++a.nprev;
        }
      a.aii = c->A[i][i];
      a.inv_dt = 1.0 / dt;
      a.kV32 = (c->need_store[i] || a.nprev == 0) ? c->kV32[i] : nullptr;
      a.Vt32 = a.nprev > 0 ? c->Vt32 : nullptr;
      Prof pr(c, INS2D_PROF_STAGE, 1);
      launch_stage(P, a, true, c->stream);
      if (a.nprev > 0) {
        Ti = c->Vt32;
        ai = 1.0;
      } else {
        Ti = c->kV32[i];
        ai = c->A[i][i];
      }
    }
    const double ti = t + c->c[i] * dt;
    if (c->bcd.bc_unsteady) {
      rc = sample_bc(c, ti);
      if (rc) return rc;
    }
    if (c->bcd.bc_unsteady || i > 0) {
      // f = (M*(Vn/dt + Vtemp) + yM/dt)/c_i   (time_ERK.m:117)
      ins2d_solve_stats st;
      rc = solve_div_split(c, V, Ti, 1.0 / dt, ai, 1.0 / dt, 0.0, 1.0 / c->c[i], c->dp, false, &st);
      if (rc) return rc;
      stats_add(stats, st);
      dpp = c->dp;
    } else {
      dpp = p;  // time_ERK.m:125-127
    }
    wait_p(c);
    {
      Prof pr(c, INS2D_PROF_PROJECT, 1);
      if (i == c->s - 1)
        launch_project32(P, V, Ti, ai, dpp, dt, c->c[i], V, c->stream);
      else
        launch_project32(P, V, Ti, ai, dpp, dt, c->c[i], c->Vs32, c->stream);
    }
    CK(cudaGetLastError());
    if (i == c->s - 1) copy_v_out(c, V);
  }
  wait_p(c);
  if (c->bcd.bc_unsteady && !c->opts.p_add_solve) {
    CK(cudaMemcpyAsync(p, dpp, P.Np * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));  // p = kp(:,end)
  } else {
    ins2d_solve_stats st;
    const bool cache = cache_next && !c->bcd.bc_unsteady;
    rc = additional_solve(c, V, p, t + dt, &st, cache);
    if (rc) return rc;
    stats_add(stats, st);
    if (cache) *cache_next = true;
  }
  return INS2D_OK;
}

int erk_step(ins2d_ctx *c, double *V, double *p, double t, double dt, ins2d_step_stats *stats, bool k0_cached,
             bool *cache_next) {
  if (c->store32) return erk_step32(c, V, p, t, dt, stats, k0_cached, cache_next);
  const DevOps &P = c->P;
  if (cache_next) *cache_next = false;
  int rc = sample_bc(c, t);
  if (rc) return rc;
  const double *dpp = nullptr;
  for (int i = 0; i < c->s; ++i) {
    if (i == 0 && k0_cached && !c->bcd.bc_unsteady && c->s > 1) {
      // first stage from the cached residual fused into its projection
      // (dp = p: time_ERK.m:125-127); Wt is not formed
      wait_p(c);
      Prof pr(c, INS2D_PROF_PROJECT, 1);
      launch_project_cached(P, V, c->kV[0], c->A[0][0], 1.0 / dt, p, dt, c->c[0], c->Vs, c->stream);
      CK(cudaGetLastError());
      continue;
    }
    if (i == 0 && k0_cached && !c->bcd.bc_unsteady) {
      Prof pr(c, INS2D_PROF_STAGE, 1);
      launch_stage_cached(c->kV[0], V, c->A[0][0], 1.0 / dt, c->Wt, P.Nu + P.Nv, c->stream);
    } else {
      StageArgs a{};
      a.V = (i == 0) ? V : c->Vs;
      a.Vn = V;
      a.kV = (c->need_store[i] || i == 0) ? c->kV[i] : nullptr;
      a.nprev = 0;
      for (int m = 0; m < i; ++m)
        if (c->A[i][m] != 0.0) {
          a.kprev[a.nprev] = c->kV[m];
          a.aprev[a.nprev] = c->A[i][m];
          ++a.nprev;
        }
      a.aii = c->A[i][i];
      a.inv_dt = 1.0 / dt;
      a.Wt = c->Wt;
      Prof pr(c, INS2D_PROF_STAGE, 1);
      launch_stage(P, a, c->fp32, c->stream);
    }
    const double ti = t + c->c[i] * dt;
    if (c->bcd.bc_unsteady) {
      rc = sample_bc(c, ti);
      if (rc) return rc;
    }
    if (c->bcd.bc_unsteady || i > 0) {
      // f = (M*(Vn/dt + Vtemp) + yM/dt)/c_i   (time_ERK.m:117)
      ins2d_solve_stats st;
      rc = solve_div(c, c->Wt, 1.0 / dt, 0.0, 1.0 / c->c[i], c->dp, false, &st);
      if (rc) return rc;
      stats_add(stats, st);
      dpp = c->dp;
    } else {
      dpp = p;  // time_ERK.m:125-127
    }
    wait_p(c);
    {
      Prof pr(c, INS2D_PROF_PROJECT, 1);
      launch_project(P, c->Wt, dpp, dt, c->c[i], (i == c->s - 1) ? V : c->Vs, c->stream);
    }
    CK(cudaGetLastError());
    if (i == c->s - 1) copy_v_out(c, V);
  }
  wait_p(c);
  if (c->bcd.bc_unsteady && !c->opts.p_add_solve) {
    CK(cudaMemcpyAsync(p, dpp, P.Np * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));  // p = kp(:,end)
  } else {
    ins2d_solve_stats st;
    const bool cache = cache_next && !c->bcd.bc_unsteady;
    rc = additional_solve(c, V, p, t + dt, &st, cache);
    if (rc) return rc;
    stats_add(stats, st);
    if (cache) *cache_next = true;
  }
  return INS2D_OK;
}

// device pointer or host staging copy
const double *in_dev(ins2d_ctx *c, const double *src, double *stage, size_t n, int mem) {
  if (!src) return nullptr;
  if (mem == INS2D_MEM_DEVICE) return src;
  CK(cudaMemcpyAsync(stage, src, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  return stage;
}

int check_mem(ins2d_ctx *c, int mem) {
  if (mem != INS2D_MEM_HOST && mem != INS2D_MEM_DEVICE) return fail(c, INS2D_EINVAL, "mem must be INS2D_MEM_HOST or INS2D_MEM_DEVICE");
  return INS2D_OK;
}

#define API_BEGIN                \
  if (!ctx) return INS2D_EINVAL; \
  ctx->err.clear();              \
  DeviceGuard dguard_(ctx->device); \
  try {                          \
    CK(dguard_.err);
#define API_END                                                  \
  }                                                              \
  catch (const CudaError &e) {                                   \
    return fail(ctx, INS2D_ECUDA, e.what());                     \
  }                                                              \
  catch (const cnn::CudaError &e) {                              \
    return fail(ctx, INS2D_ECUDA, e.what());                     \
  }                                                              \
  catch (const std::bad_alloc &) {                               \
    return fail(ctx, INS2D_ENOMEM, "device allocation failed");  \
  }                                                              \
  catch (const std::exception &e) {                              \
    return fail(ctx, INS2D_EINVAL, e.what());                    \
  }

}  // namespace

extern "C" {

int ins2d_ctx_create(const ins2d_grid_desc *grid, const ins2d_bc_desc *bc, const ins2d_opts *opts, ins2d_ctx **out) {
  if (!grid || !bc || !opts || !out || !grid->x || !grid->y) return INS2D_EINVAL;
  *out = nullptr;
  ins2d_ctx *c = new (std::nothrow) ins2d_ctx();
  if (!c) return INS2D_ENOMEM;
  c->opts = *opts;
  c->bcd = *bc;
  c->device = opts->device;
  c->fp32 = opts->precision == INS2D_PREC_FP32_STENCIL;
  c->poisson = opts->poisson;
  DeviceGuard dg(c->device);
  int rc = INS2D_OK;
  try {
    if (!(opts->Re > 0)) throw std::invalid_argument("Re must be positive");
    if (opts->precision != INS2D_PREC_FP64 && opts->precision != INS2D_PREC_FP32_STENCIL)
      throw std::invalid_argument("unknown precision");
    if (opts->poisson < 1 || opts->poisson > 6) throw std::invalid_argument("wrong poisson method");
    if (opts->poisson != INS2D_POISSON_FFT && !(opts->CG_acc > 0)) throw std::invalid_argument("CG_acc must be positive");
    if (opts->poisson != INS2D_POISSON_FFT && opts->CG_maxit < 1) throw std::invalid_argument("CG_maxit must be >= 1");
    if (opts->precond < INS2D_PRECOND_DEFAULT || opts->precond > INS2D_PRECOND_FDM)
      throw std::invalid_argument("wrong preconditioner");
    if (opts->rk_stages < 0 || opts->rk_stages > kMaxStages) throw std::invalid_argument("rk_stages out of range");
    for (int i = 0; i < opts->rk_stages; ++i)
      for (int j = i; j < opts->rk_stages; ++j)
        if (opts->rk_A[i * opts->rk_stages + j] != 0.0) throw std::invalid_argument("Butcher tableau is not explicit");
    CK(dg.err);
    int bcs[8] = {bc->u_left, bc->u_right, bc->u_low, bc->u_up, bc->v_left, bc->v_right, bc->v_low, bc->v_up};
    build_host_ops(c->H, grid->Nx, grid->Ny, grid->x, grid->y, bcs, opts->Re);
    if (c->poisson == INS2D_POISSON_FFT) {
      if (!c->H.fft_ok)
        throw std::invalid_argument(
            "Fourier transform for pressure Poisson needs periodic boundary conditions and a uniform grid");
      if (!fft_supported(grid->Nx, grid->Ny)) throw std::invalid_argument("grid size not supported by the FFT solver");
    }
    setup_rk(c);
    HostOps &H = c->H;
    DevOps &P = c->P;
    P.Nx = H.Nx; P.Ny = H.Ny; P.Nux = H.Nux; P.Nuy = H.Nuy; P.Nvx = H.Nvx; P.Nvy = H.Nvy;
    P.Npx = H.Npx; P.Npy = H.Npy;
    P.Nu = H.Nu(); P.Nv = H.Nv(); P.Np = H.Np();
    P.invRe = 1.0 / H.Re;
    P.AUX = upload_tab(c, H.AUX); P.SUX = upload_tab(c, H.SUX); P.AUY = upload_tab(c, H.AUY);
    P.SUY = upload_tab(c, H.SUY); P.IVX = upload_tab(c, H.IVX); P.IVY = upload_tab(c, H.IVY);
    P.MX = upload_tab(c, H.MX); P.MXT = upload_tab(c, H.MXT);
    P.AVX = upload_tab(c, H.AVX); P.SVX = upload_tab(c, H.SVX); P.AVY = upload_tab(c, H.AVY);
    P.SVY = upload_tab(c, H.SVY); P.IUX = upload_tab(c, H.IUX); P.IUY = upload_tab(c, H.IUY);
    P.MY = upload_tab(c, H.MY); P.MYT = upload_tab(c, H.MYT);
    P.TX = upload_tab(c, H.TX); P.TY = upload_tab(c, H.TY);
    P.TXd = upload_vec(c, H.TXd); P.TYd = upload_vec(c, H.TYd);
    P.hx = upload_vec(c, H.hx); P.hy = upload_vec(c, H.hy);
    P.gxi = upload_vec(c, H.gxi); P.gyi = upload_vec(c, H.gyi);
    {
      auto rec = [](const std::vector<double> &v) {
        std::vector<double> r(v.size());
        for (size_t k = 0; k < v.size(); ++k) r[k] = 1.0 / v[k];
        return r;
      };
      P.rhx = upload_vec(c, rec(H.hx)); P.rhy = upload_vec(c, rec(H.hy));
      P.rgxi = upload_vec(c, rec(H.gxi)); P.rgyi = upload_vec(c, rec(H.gyi));
    }
    P.pxl = upload_vec(c, H.pxl); P.pxr = upload_vec(c, H.pxr);
    P.pyl = upload_vec(c, H.pyl); P.pyu = upload_vec(c, H.pyu);
    auto reg = [&](const Regular &r, const Table &t) {
      RegD d;
      d.s = r.s;
      d.lo = r.lo;
      d.hi = r.hi;
      d.two = r.two;
      d.n = t.ncols;
      d.w0 = upload_vec(c, t.rw0);
      d.w1 = upload_vec(c, t.rw1);
      return d;
    };
    P.rAUX = reg(H.rAUX, H.AUX); P.rSUX = reg(H.rAUX, H.SUX);
    P.rAUY = reg(H.rAUY, H.AUY); P.rSUY = reg(H.rAUY, H.SUY);
    P.rIVX = reg(H.rIVX, H.IVX); P.rIVY = reg(H.rIVY, H.IVY); P.rMXT = reg(H.rMXT, H.MXT);
    P.rAVX = reg(H.rAVX, H.AVX); P.rSVX = reg(H.rAVX, H.SVX);
    P.rAVY = reg(H.rAVY, H.AVY); P.rSVY = reg(H.rAVY, H.SVY);
    P.rIUX = reg(H.rIUX, H.IUX); P.rIUY = reg(H.rIUY, H.IUY); P.rMYT = reg(H.rMYT, H.MYT);
    P.rMX = reg(H.rMX, H.MX); P.rMY = reg(H.rMY, H.MY);
    walker_rectangle(P);
    CK(walker_prepare());
    CK(cudaDeviceGetAttribute(&P.nsm, cudaDevAttrMultiProcessorCount, c->device));
    if (H.fft_ok) {
      P.fft_ax = upload_vec(c, H.fft_ax);
      P.fft_ay = upload_vec(c, H.fft_ay);
      P.fft_dxdy = H.fft_dxdy;
    } else {
      P.fft_ax = P.fft_ay = nullptr;
      P.fft_dxdy = 0.0;
    }
    // boundary values (zero until ins2d_set_bc_values)
    auto slots = bc_slots(c);
    size_t tot = 0;
    for (auto &s : slots) tot += (size_t)s.n;
    c->bc_count = tot;
    c->bcblob = dalloc<double>(c, tot);
    CK(cudaMemset(c->bcblob, 0, tot * sizeof(double)));
    size_t off = 0;
    for (auto &s : slots) {
      *s.dst = c->bcblob + off;
      off += (size_t)s.n;
    }
    c->uLe_i.assign(H.Ny, 0.0); c->uRi_i.assign(H.Ny, 0.0);
    c->vLo_i.assign(H.Nx, 0.0); c->vUp_i.assign(H.Nx, 0.0);
    // work arrays
    const size_t NV = (size_t)(P.Nu + P.Nv), Np = (size_t)P.Np;
    c->Vs = dalloc<double>(c, NV);
    c->Wt = dalloc<double>(c, NV);
    for (int m = 0; m < c->s; ++m) c->kV[m] = (c->need_store[m] || m == 0) ? dalloc<double>(c, NV) : nullptr;
    if (c->fp32) {
      c->store32 = true;
      c->Vs32 = dalloc<float>(c, NV);
      c->Vt32 = dalloc<float>(c, NV);
      for (int m = 0; m < c->s; ++m) c->kV32[m] = dalloc<float>(c, NV);
    }
    c->wres = dalloc<double>(c, NV);
    c->f = dalloc<double>(c, Np);
    c->dp = dalloc<double>(c, Np);
    c->stV = dalloc<double>(c, NV);
    c->stC = dalloc<double>(c, NV);
    c->stO = dalloc<double>(c, NV);
    c->stP = dalloc<double>(c, Np);
    c->stQ = dalloc<double>(c, Np);
    const int nx = std::max(P.Nux, P.Nvx), ny = std::max(P.Nuy, P.Nvy);
    const int maxb = ((nx + 31) / 32) * ((ny + 7) / 8) + 64;
    c->red.partials = dalloc<double>(c, (size_t)maxb * kRedQ);
    c->red.counter = dalloc<unsigned int>(c, 1);
    c->red.result = dalloc<double>(c, kRedQ);
    c->red.max_blocks = maxb;
    CK(cudaMemset(c->red.counter, 0, sizeof(unsigned int)));
    if (c->poisson == INS2D_POISSON_FFT) {
      CK(fft_prepare());
      FftPlan &F = c->fft;
      F.Nx = H.Nx;
      F.Ny = H.Ny;
      F.logx = is_pow2(H.Nx) ? (int)std::lround(std::log2((double)H.Nx)) : -1;
      F.logy = is_pow2(H.Ny) ? (int)std::lround(std::log2((double)H.Ny)) : -1;
      const std::vector<double> tx = fft_twiddle_table(H.Nx), ty = fft_twiddle_table(H.Ny);
      F.twx = dalloc<double2>(c, 2 * (size_t)H.Nx);
      F.twy = dalloc<double2>(c, 2 * (size_t)H.Ny);
      CK(cudaMemcpy(F.twx, tx.data(), tx.size() * sizeof(double), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(F.twy, ty.data(), ty.size() * sizeof(double), cudaMemcpyHostToDevice));
      F.spec = dalloc<double2>(c, (size_t)(H.Nx / 2 + 1) * H.Ny);
      F.maxabs = dalloc<double>(c, 1);
    } else {
      PcgWork &W = c->pcg;
      W.x = dalloc<double>(c, Np);
      W.r = dalloc<double>(c, Np);
      W.p = dalloc<double>(c, Np);
      W.q = dalloc<double>(c, Np);
      W.sc = dalloc<PcgScalars>(c, 1);
      W.blocks = pcg_blocks(P);
      W.partials = dalloc<double>(c, (size_t)W.blocks * 8 + 16);
      CK(cudaMemset(W.sc, 0, sizeof(PcgScalars)));
      // the default: fast diagonalization where it applies (periodic uniform
      // grids the FFT takes, or up to kFdmMaxN cells per direction), else
      // multigrid, else Jacobi
      const bool fdm_fits = (H.fft_ok && fft_supported(H.Nx, H.Ny)) || std::max(H.Npx, H.Npy) <= kFdmMaxN;
      if (opts->precond == INS2D_PRECOND_FDM || (opts->precond == INS2D_PRECOND_DEFAULT && fdm_fits)) {
        FdmD &D = c->fdm;
        D.nx = H.Npx;
        D.ny = H.Npy;
        D.z = dalloc<double>(c, Np);
        if (H.fft_ok && fft_supported(H.Nx, H.Ny)) {
          // periodic uniform grid: the Fourier basis, i.e. the FFT solve
          CK(fft_prepare());
          FftPlan &F = c->fdm_fft;
          F.Nx = H.Nx;
          F.Ny = H.Ny;
          F.logx = is_pow2(H.Nx) ? (int)std::lround(std::log2((double)H.Nx)) : -1;
          F.logy = is_pow2(H.Ny) ? (int)std::lround(std::log2((double)H.Ny)) : -1;
          const std::vector<double> tx = fft_twiddle_table(H.Nx), ty = fft_twiddle_table(H.Ny);
          F.twx = dalloc<double2>(c, 2 * (size_t)H.Nx);
          F.twy = dalloc<double2>(c, 2 * (size_t)H.Ny);
          CK(cudaMemcpy(F.twx, tx.data(), tx.size() * sizeof(double), cudaMemcpyHostToDevice));
          CK(cudaMemcpy(F.twy, ty.data(), ty.size() * sizeof(double), cudaMemcpyHostToDevice));
          F.spec = dalloc<double2>(c, (size_t)(H.Nx / 2 + 1) * H.Ny);
          F.maxabs = dalloc<double>(c, 1);  // the symbol factors P.fft_ax, fft_ay are set above
          double *gate = dalloc<double>(c, 1);
          const double one = 1.0;
          CK(cudaMemcpy(gate, &one, sizeof one, cudaMemcpyHostToDevice));
          D.spectral = true;
          D.fft = &c->fdm_fft;
          D.gate = (const unsigned long long *)gate;
        } else {
          if (std::max(H.Npx, H.Npy) > kFdmMaxN)
            throw std::invalid_argument("fast-diagonalization preconditioner: grid larger than " +
                                        std::to_string(kFdmMaxN) + " cells in a direction");
          const FdmHost1D fx = fdm_1d(H.TX, H.hx), fy = fdm_1d(H.TY, H.hy);
          D.Qx = upload_vec(c, fx.Q);
          D.Qy = upload_vec(c, fy.Q);
          D.lx = upload_vec(c, fx.lam);
          D.ly = upload_vec(c, fy.lam);
          D.thr = 1e-12 * (fx.lam.back() + fy.lam.back());
          D.t1 = dalloc<double>(c, Np);
          D.t2 = dalloc<double>(c, Np);
        }
        c->use_fdm = true;
      } else if (opts->precond != INS2D_PRECOND_JACOBI) {
        std::vector<MgHostLevel> lv;
        try {
          lv = mg_build_levels(H);
        } catch (const std::runtime_error &e) {
          if (opts->precond == INS2D_PRECOND_MG) throw std::invalid_argument(e.what());
        }
        if (!lv.empty()) {
          mg_setup_device(lv, c->mg, [c](size_t n) { return dalloc<double>(c, n); }, nullptr);
          c->use_mg = true;
        }
      }
    }
    CK(cudaMallocHost((void **)&c->h_sc, sizeof(PcgScalars)));
    CK(cudaMallocHost((void **)&c->h_red, sizeof(double) * kRedQ));
    CK(cudaMallocHost((void **)&c->h_accum, sizeof(SolveAccum)));
    c->accum = dalloc<SolveAccum>(c, 1);
    CK(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->body_stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->ev_p, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_v, cudaEventDisableTiming));
    c->stream = c->own_stream;
    CK(cudaDeviceSynchronize());
  } catch (const CudaError &e) {
    c->err = e.what();
    rc = INS2D_ECUDA;
  } catch (const std::bad_alloc &) {
    c->err = "device allocation failed";
    rc = INS2D_ENOMEM;
  } catch (const std::exception &e) {
    c->err = e.what();
    rc = INS2D_EINVAL;
  }
  if (rc != INS2D_OK) {
    // keep the context so the caller can read ins2d_last_error, but free memory
    for (void *p : c->allocs) cudaFree(p);
    c->allocs.clear();
    *out = c;
    return rc;
  }
  *out = c;
  return INS2D_OK;
}

int ins2d_ctx_destroy(ins2d_ctx *ctx) {
  if (!ctx) return INS2D_OK;
  DeviceGuard dg(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  for (auto &g : ctx->step_graph)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  for (void *p : ctx->allocs) cudaFree(p);
  for (auto &r : ctx->recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : ctx->pool) cudaEventDestroy(e);
  if (ctx->order_ev) cudaEventDestroy(ctx->order_ev);
  if (ctx->h_sc) cudaFreeHost(ctx->h_sc);
  if (ctx->h_red) cudaFreeHost(ctx->h_red);
  if (ctx->h_accum) cudaFreeHost(ctx->h_accum);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  if (ctx->body_stream) cudaStreamDestroy(ctx->body_stream);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->ev_p) cudaEventDestroy(ctx->ev_p);
  if (ctx->ev_v) cudaEventDestroy(ctx->ev_v);
  delete ctx;
  return INS2D_OK;
}

const char *ins2d_last_error(const ins2d_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int ins2d_get_sizes(const ins2d_ctx *ctx, ins2d_sizes *o) {
  if (!ctx || !o) return INS2D_EINVAL;
  const HostOps &H = ctx->H;
  o->Nx = H.Nx; o->Ny = H.Ny;
  o->Nux_in = H.Nux; o->Nuy_in = H.Nuy; o->Nvx_in = H.Nvx; o->Nvy_in = H.Nvy;
  o->Npx = H.Npx; o->Npy = H.Npy;
  o->Nu = (int32_t)H.Nu(); o->Nv = (int32_t)H.Nv(); o->NV = (int32_t)(H.Nu() + H.Nv()); o->Np = (int32_t)H.Np();
  return INS2D_OK;
}

int ins2d_set_stream(ins2d_ctx *ctx, void *stream) {
  if (!ctx) return INS2D_EINVAL;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return INS2D_OK;
}

int ins2d_set_poll_limit(ins2d_ctx *ctx, int64_t iterations) {
  API_BEGIN
  const long long v = iterations < 0 ? -1 : (long long)iterations;
  if (v != ctx->poll_limit) {
    // captured step graphs hold the loop limit: capture again
    CK(cudaStreamSynchronize(ctx->stream));
    for (auto &g : ctx->step_graph)
      if (g.exec) {
        CK(cudaGraphExecDestroy(g.exec));
        g.exec = nullptr;
      }
  }
  ctx->poll_limit = v;
  return INS2D_OK;
  API_END
}

int ins2d_wait_stream(ins2d_ctx *ctx, void *stream) {
  API_BEGIN
  const cudaStream_t other = (cudaStream_t)stream;
  if (other == ctx->stream) return INS2D_OK;
  if (!ctx->order_ev) CK(cudaEventCreateWithFlags(&ctx->order_ev, cudaEventDisableTiming));
  CK(cudaEventRecord(ctx->order_ev, other));
  CK(cudaStreamWaitEvent(ctx->stream, ctx->order_ev, 0));
  return INS2D_OK;
  API_END
}

int ins2d_profile(ins2d_ctx *ctx, int enable) {
  if (!ctx) return INS2D_EINVAL;
  DeviceGuard dg(ctx->device);
  for (auto &r : ctx->recs) {
    ctx->pool.push_back(r.a);
    ctx->pool.push_back(r.b);
  }
  ctx->recs.clear();
  for (auto &l : ctx->launches) l = 0;
  ctx->prof = enable != 0;
  return INS2D_OK;
}

int ins2d_profile_read(ins2d_ctx *ctx, double ms[INS2D_PROF_N], int64_t launches[INS2D_PROF_N]) {
  API_BEGIN
  CK(cudaStreamSynchronize(ctx->stream));
  double acc[INS2D_PROF_N] = {};
  for (auto &r : ctx->recs) {
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, r.a, r.b));
    acc[r.fam] += t;
    ctx->pool.push_back(r.a);
    ctx->pool.push_back(r.b);
  }
  ctx->recs.clear();
  for (int k = 0; k < INS2D_PROF_N; ++k) {
    if (ms) ms[k] = acc[k];
    if (launches) launches[k] = ctx->launches[k];
    ctx->launches[k] = 0;
  }
  return INS2D_OK;
  API_END
}

int ins2d_set_bc_sampler(ins2d_ctx *ctx, ins2d_bc_sampler_fn fn, void *user) {
  if (!ctx) return INS2D_EINVAL;
  ctx->sampler = fn;
  ctx->sampler_user = user;
  return INS2D_OK;
}

int ins2d_set_bc_values(ins2d_ctx *ctx, double t, const ins2d_bc_values *v) {
  if (!v) return fail(ctx, INS2D_EINVAL, "null boundary values");
  API_BEGIN
  HostOps &H = ctx->H;
  auto get = [](const double *p, int n) {
    return p ? std::vector<double>(p, p + n) : std::vector<double>((size_t)n, 0.0);
  };
  std::vector<double> uLo = get(v->uLo, H.Nx + 1), uUp = get(v->uUp, H.Nx + 1);
  std::vector<double> uLo_i = get(v->uLo_i, H.Nux), uUp_i = get(v->uUp_i, H.Nux);
  std::vector<double> uLe_i = get(v->uLe_i, H.Ny), uRi_i = get(v->uRi_i, H.Ny);
  std::vector<double> vLe = get(v->vLe, H.Ny + 1), vRi = get(v->vRi, H.Ny + 1);
  std::vector<double> vLo_i = get(v->vLo_i, H.Nx), vUp_i = get(v->vUp_i, H.Nx);
  std::vector<double> vLe_i = get(v->vLe_i, H.Nvy), vRi_i = get(v->vRi_i, H.Nvy);
  // products with the interpolation factors (set_bc_vectors.m:450-451, 492-493)
  std::vector<double> XvLo = matvec(H.IVX.T, vLo_i), XvUp = matvec(H.IVX.T, vUp_i);
  std::vector<double> YuLe = matvec(H.IUY.T, uLe_i), YuRi = matvec(H.IUY.T, uRi_i);
  std::vector<double> all;
  all.reserve(ctx->bc_count);
  for (const auto *vec : {&uLo, &uUp, &uLo_i, &uUp_i, &uLe_i, &uRi_i, &vLe, &vRi, &vLo_i, &vUp_i, &vLe_i, &vRi_i,
                          &XvLo, &XvUp, &YuLe, &YuRi})
    all.insert(all.end(), vec->begin(), vec->end());
  for (auto pr : {std::make_pair(v->pLe, H.Ny), std::make_pair(v->pRi, H.Ny), std::make_pair(v->pLo, H.Nx),
                  std::make_pair(v->pUp, H.Nx), std::make_pair(v->dudtLe_i, H.Ny), std::make_pair(v->dudtRi_i, H.Ny),
                  std::make_pair(v->dvdtLo_i, H.Nx), std::make_pair(v->dvdtUp_i, H.Nx)}) {
    auto g = get(pr.first, pr.second);
    all.insert(all.end(), g.begin(), g.end());
  }
  if (all.size() != ctx->bc_count) return fail(ctx, INS2D_EINVAL, "internal: boundary blob size mismatch");
  // the blob is read by kernels queued earlier on the stream: order the update after them
  CK(cudaMemcpyAsync(ctx->bcblob, all.data(), all.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->uLe_i = uLe_i;
  ctx->uRi_i = uRi_i;
  ctx->vLo_i = vLo_i;
  ctx->vUp_i = vUp_i;
  ctx->bc_time = t;
  return INS2D_OK;
  API_END
}

int ins2d_F(ins2d_ctx *ctx, const double *V, const double *C, const double *p, double t, int nopressure,
            double *F_out, double *maxres, int mem) {
  API_BEGIN
  if (check_mem(ctx, mem)) return INS2D_EINVAL;
  if (!V || !F_out || (!nopressure && !p)) return fail(ctx, INS2D_EINVAL, "F: null argument");
  int rc = sample_bc(ctx, t);
  if (rc) return rc;
  const size_t NV = (size_t)(ctx->P.Nu + ctx->P.Nv);
  const double *dV = in_dev(ctx, V, ctx->stV, NV, mem);
  const double *dC = (C && C != V) ? in_dev(ctx, C, ctx->stC, NV, mem) : dV;
  const double *dP = nopressure ? nullptr : in_dev(ctx, p, ctx->stP, (size_t)ctx->P.Np, mem);
  double *dO = mem == INS2D_MEM_DEVICE ? F_out : ctx->stO;
  if (dP && dC == dV && !ctx->fp32) {
    // the stencil walkers (the stage kernels' F) and a max|F| reduction
    Prof pr(ctx, INS2D_PROF_OTHER, 2);
    launch_F_walk(ctx->P, dV, dP, dO, ctx->stream);
    launch_maxabs(dO, (long long)NV, ctx->red, ctx->stream);
  } else {
    // C != V (F.m's linearisation point), nopressure, or FP32-stencil
    // contexts (diagnostics stay FP64): one thread per point
    Prof pr(ctx, INS2D_PROF_OTHER, 1);
    launch_F(ctx->P, dV, dC, dP, dO, ctx->red, ctx->stream);
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(ctx->h_red, ctx->red.result, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (mem == INS2D_MEM_HOST) CK(cudaMemcpyAsync(F_out, dO, NV * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (maxres) *maxres = ctx->h_red[0];
  return INS2D_OK;
  API_END
}

int ins2d_divergence(ins2d_ctx *ctx, const double *V, double *f_out, double *maxdiv, int mem) {
  API_BEGIN
  if (check_mem(ctx, mem)) return INS2D_EINVAL;
  if (!V || !f_out) return fail(ctx, INS2D_EINVAL, "divergence: null argument");
  const size_t NV = (size_t)(ctx->P.Nu + ctx->P.Nv);
  const double *dV = in_dev(ctx, V, ctx->stV, NV, mem);
  double *dO = mem == INS2D_MEM_DEVICE ? f_out : ctx->stP;
  Prof pr(ctx, INS2D_PROF_OTHER, 1);
  launch_div(ctx->P, dV, 1.0, 0.0, 1.0, dO, true, ctx->red, ctx->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(ctx->h_red, ctx->red.result, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (mem == INS2D_MEM_HOST)
    CK(cudaMemcpyAsync(f_out, dO, (size_t)ctx->P.Np * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (maxdiv) *maxdiv = ctx->h_red[0];
  return INS2D_OK;
  API_END
}

int ins2d_laplacian(ins2d_ctx *ctx, const double *p, double *Ap, int mem) {
  API_BEGIN
  if (check_mem(ctx, mem)) return INS2D_EINVAL;
  if (!p || !Ap) return fail(ctx, INS2D_EINVAL, "laplacian: null argument");
  const size_t Np = (size_t)ctx->P.Np;
  const double *dp = in_dev(ctx, p, ctx->stP, Np, mem);
  double *dO = mem == INS2D_MEM_DEVICE ? Ap : ctx->stQ;
  Prof pr(ctx, INS2D_PROF_OTHER, 1);
  launch_lap(ctx->P, dp, dO, ctx->stream);
  CK(cudaGetLastError());
  if (mem == INS2D_MEM_HOST) CK(cudaMemcpyAsync(Ap, dO, Np * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return INS2D_OK;
  API_END
}

int ins2d_pressure_poisson(ins2d_ctx *ctx, const double *f, double *dp, ins2d_solve_stats *stats, int mem) {
  API_BEGIN
  if (check_mem(ctx, mem)) return INS2D_EINVAL;
  if (!f || !dp) return fail(ctx, INS2D_EINVAL, "pressure_poisson: null argument");
  const size_t Np = (size_t)ctx->P.Np;
  const double *df = in_dev(ctx, f, ctx->stP, Np, mem);
  double *dO = mem == INS2D_MEM_DEVICE ? dp : ctx->stQ;
  int rc = solve(ctx, df, dO, false, stats);
  if (rc) return rc;
  if (mem == INS2D_MEM_HOST) CK(cudaMemcpyAsync(dp, dO, Np * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return INS2D_OK;
  API_END
}

int ins2d_pressure_additional_solve(ins2d_ctx *ctx, const double *V, double *p, double t, ins2d_solve_stats *stats,
                                    int mem) {
  API_BEGIN
  if (check_mem(ctx, mem)) return INS2D_EINVAL;
  if (!V || !p) return fail(ctx, INS2D_EINVAL, "pressure_additional_solve: null argument");
  const size_t NV = (size_t)(ctx->P.Nu + ctx->P.Nv), Np = (size_t)ctx->P.Np;
  const double *dV = in_dev(ctx, V, ctx->stV, NV, mem);
  double *dP = p;
  if (mem == INS2D_MEM_HOST) {
    CK(cudaMemcpyAsync(ctx->stP, p, Np * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    dP = ctx->stP;
  }
  int rc = additional_solve(ctx, dV, dP, t, stats);
  if (rc) return rc;
  if (mem == INS2D_MEM_HOST) CK(cudaMemcpyAsync(p, dP, Np * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return INS2D_OK;
  API_END
}

int ins2d_erk_run(ins2d_ctx *ctx, double *V, double *p, double t, double dt, int32_t nsteps, ins2d_step_stats *stats,
                  int mem) {
  API_BEGIN
  if (check_mem(ctx, mem)) return INS2D_EINVAL;
  if (!V || !p || nsteps < 0) return fail(ctx, INS2D_EINVAL, "erk: bad argument");
  if (!(dt > 0)) return fail(ctx, INS2D_EINVAL, "dt must be positive");
  if (stats) *stats = ins2d_step_stats{0, 0, 0, 0.0};
  const size_t NV = (size_t)(ctx->P.Nu + ctx->P.Nv), Np = (size_t)ctx->P.Np;
  // every return leaves copy_stream idle (no copy into the caller's memory
  // outlives the call)
  struct CopyGuard {
    ins2d_ctx *c;
    ~CopyGuard() {
      cudaStreamSynchronize(c->copy_stream);
      c->p_pending = false;
      c->v_out_host = nullptr;
      c->v_out_done = false;
    }
  } copy_guard{ctx};
  double *dV = V, *dP = p;
  if (mem == INS2D_MEM_HOST) {
    CK(cudaMemcpyAsync(ctx->stV, V, NV * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    // p after V on the copy stream, beside the first stage (wait_p)
    CK(cudaEventRecord(ctx->ev_p, ctx->stream));
    CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_p, 0));
    CK(cudaMemcpyAsync(ctx->stP, p, Np * sizeof(double), cudaMemcpyHostToDevice, ctx->copy_stream));
    CK(cudaEventRecord(ctx->ev_p, ctx->copy_stream));
    ctx->p_pending = true;
    dV = ctx->stV;
    dP = ctx->stP;
  }
  // With steady boundary conditions a step is a launch sequence without host
  // round trips -- FFT solves, or PCG solves whose iteration loops run on the
  // device as conditional WHILE nodes -- so it is captured once as a CUDA
  // graph (first step, and steps whose first stage comes from the cache) and
  // replayed; the graphs are keyed by the state pointers and dt.  The PCG
  // solves' statistics and errors accumulate on the device and are read
  // every kAccumCheck steps and at the end of the run.
  const bool pcg_graphs = ctx->poisson != INS2D_POISSON_FFT && !ctx->cnn && ctx->rec_n >= ctx->rec_cap;
  const bool graphs = (ctx->poisson == INS2D_POISSON_FFT || pcg_graphs) && !ctx->bcd.bc_unsteady && !ctx->prof &&
                      nsteps >= 2;
  const bool dev_stats = graphs && pcg_graphs;
  constexpr int kAccumCheck = 32;
  auto read_accum = [&]() -> int {
    CK(cudaMemcpyAsync(ctx->h_accum, ctx->accum, sizeof(SolveAccum), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const SolveAccum &a = *ctx->h_accum;
    if (a.status == INS2D_ENOTCONV) {
      char buf[160];
      snprintf(buf, sizeof buf, "CG didn't converge in %lld iterations; residual= %g", a.fail_maxit,
               std::sqrt(a.fail_rr));
      return fail(ctx, INS2D_ENOTCONV, buf);
    }
    if (a.status == INS2D_EBREAKDOWN) return fail(ctx, INS2D_EBREAKDOWN, "PCG breakdown: p'Ap = 0");
    if (a.status == INS2D_ENONFINITE) return fail(ctx, INS2D_ENONFINITE, "PCG: non-finite residual");
    if (a.status == INS2D_ETIMEOUT)
      return fail(ctx, INS2D_ETIMEOUT, "PCG: device convergence flag not set within the iteration-loop limit");
    if (a.status != 0) return fail(ctx, a.status, "PCG failed");
    return INS2D_OK;
  };
  if (dev_stats) CK(cudaMemsetAsync(ctx->accum, 0, sizeof(SolveAccum), ctx->stream));
  if (graphs) wait_p(ctx);  // before any capture: the graphs read p
  bool cached = false;
  for (int n = 0; n < nsteps; ++n) {
    if (graphs) {
      const int g = cached ? 1 : 0;
      StepGraph &G = ctx->step_graph[g];
      if (!G.exec || G.V != dV || G.p != dP || G.dt != dt) {
        if (G.exec) cudaGraphExecDestroy(G.exec);
        G.exec = nullptr;
        long long before[INS2D_PROF_N];
        std::memcpy(before, ctx->launches, sizeof before);
        cudaGraph_t gr;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        bool next = false;
        ctx->dev_loop = pcg_graphs;
        int rc;
        try {
          rc = erk_step(ctx, dV, dP, t + n * dt, dt, nullptr, cached, &next);
        } catch (...) {
          ctx->dev_loop = false;
          cudaGraph_t junk = nullptr;
          if (cudaStreamEndCapture(ctx->stream, &junk) == cudaSuccess && junk) cudaGraphDestroy(junk);
          throw;
        }
        ctx->dev_loop = false;
        cudaError_t ce = cudaStreamEndCapture(ctx->stream, &gr);
        if (rc) {
          if (ce == cudaSuccess) cudaGraphDestroy(gr);
          return rc;
        }
        CK(ce);
        cudaError_t ie = cudaGraphInstantiate(&G.exec, gr, 0);
        cudaGraphDestroy(gr);
        CK(ie);
        for (int k = 0; k < INS2D_PROF_N; ++k) {
          G.launches[k] = ctx->launches[k] - before[k];
          ctx->launches[k] = before[k];
        }
        G.V = dV;
        G.p = dP;
        G.dt = dt;
      }
      CK(cudaGraphLaunch(G.exec, ctx->stream));
      for (int k = 0; k < INS2D_PROF_N; ++k) ctx->launches[k] += G.launches[k];
      if (!dev_stats) {
        // s FFT solves per step (stages 2..s and the additional solve), no iterations
        for (int k = 0; k < ctx->s; ++k) stats_add(stats, ins2d_solve_stats{0, 0.0, 0.0});
      } else if ((n + 1) % kAccumCheck == 0 && n + 1 < nsteps) {
        const int rc = read_accum();
        if (rc) return rc;
      }
      cached = true;
      continue;
    }
    bool next = false;
    if (mem == INS2D_MEM_HOST && n + 1 == nsteps) ctx->v_out_host = V;
    int rc = erk_step(ctx, dV, dP, t + n * dt, dt, stats, cached, n + 1 < nsteps ? &next : nullptr);
    if (rc) return rc;
    cached = next;
  }
  if (dev_stats && nsteps > 0) {
    const int rc = read_accum();
    if (rc) return rc;
    if (stats) {
      const SolveAccum &a = *ctx->h_accum;
      stats->n_solves = (int32_t)a.n_solves;
      stats->iters_total = (int32_t)a.iters_total;
      stats->iters_max = (int32_t)a.iters_max;
      stats->norm1_max = a.norm1_max;
    }
  }
  wait_p(ctx);
  if (mem == INS2D_MEM_HOST) {
    if (!ctx->v_out_done) CK(cudaMemcpyAsync(V, dV, NV * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(p, dP, Np * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaStreamSynchronize(ctx->copy_stream));
  return INS2D_OK;
  API_END
}

int ins2d_erk_step(ins2d_ctx *ctx, double *V, double *p, double t, double dt, ins2d_step_stats *stats, int mem) {
  return ins2d_erk_run(ctx, V, p, t, dt, 1, stats, mem);
}

// input_check.m:95-111: when max|M V + yM| > 1e-12, V -= Om_inv .* (G dp)
// with dp = pressure_poisson(M V + yM); V in place.
int ins2d_initial_projection(ins2d_ctx *ctx, double *V, double t, double *maxdiv, int mem) {
  API_BEGIN
  if (check_mem(ctx, mem)) return INS2D_EINVAL;
  if (!V) return fail(ctx, INS2D_EINVAL, "initial_projection: null argument");
  int rc = sample_bc(ctx, t);
  if (rc) return rc;
  const size_t NV = (size_t)(ctx->P.Nu + ctx->P.Nv);
  const double *dV = in_dev(ctx, V, ctx->stV, NV, mem);
  {
    Prof pr(ctx, INS2D_PROF_OTHER, 1);
    launch_div(ctx->P, dV, 1.0, 0.0, 1.0, ctx->f, true, ctx->red, ctx->stream);
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(ctx->h_red, ctx->red.result, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const double md = ctx->h_red[0];
  if (maxdiv) *maxdiv = md;
  if (!(md > 1e-12)) return INS2D_OK;
  ins2d_solve_stats st;
  rc = solve(ctx, ctx->f, ctx->dp, false, &st);
  if (rc) return rc;
  {
    Prof pr(ctx, INS2D_PROF_OTHER, 1);
    launch_correct(ctx->P, dV, ctx->dp, ctx->stO, ctx->stream);
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(V, ctx->stO, NV * sizeof(double),
                     mem == INS2D_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return INS2D_OK;
  API_END
}

int ins2d_conservation(ins2d_ctx *ctx, const double *V, double t, double out[4], int mem) {
  API_BEGIN
  if (check_mem(ctx, mem)) return INS2D_EINVAL;
  if (!V || !out) return fail(ctx, INS2D_EINVAL, "conservation: null argument");
  int rc = sample_bc(ctx, t);
  if (rc) return rc;
  const size_t NV = (size_t)(ctx->P.Nu + ctx->P.Nv);
  const double *dV = in_dev(ctx, V, ctx->stV, NV, mem);
  Prof pr(ctx, INS2D_PROF_OTHER, 1);
  launch_conservation(ctx->P, dV, ctx->red, ctx->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(ctx->h_red, ctx->red.result, 5 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const HostOps &H = ctx->H;
  const double *r = ctx->h_red;
  double umom = r[1], vmom = r[2], k = 0.5 * r[3] + 0.5 * r[4];
  // Dirichlet boundary contributions (check_conservation.m:45-76)
  auto dot = [](const std::vector<double> &a, const std::vector<double> &b, bool sq) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += (sq ? a[i] * a[i] : a[i]) * b[i];
    return s;
  };
  const int *bc = H.bc;
  if (bc[0] == BC_DIR) { umom += dot(ctx->uLe_i, H.hy, false) * H.gx[0]; k += 0.5 * dot(ctx->uLe_i, H.hy, true) * H.gx[0]; }
  if (bc[1] == BC_DIR) { umom += dot(ctx->uRi_i, H.hy, false) * H.gx[H.Nx]; k += 0.5 * dot(ctx->uRi_i, H.hy, true) * H.gx[H.Nx]; }
  if (bc[6] == BC_DIR) { vmom += dot(ctx->vLo_i, H.hx, false) * H.gy[0]; k += 0.5 * dot(ctx->vLo_i, H.hx, true) * H.gy[0]; }
  if (bc[7] == BC_DIR) { vmom += dot(ctx->vUp_i, H.hx, false) * H.gy[H.Ny]; k += 0.5 * dot(ctx->vUp_i, H.hx, true) * H.gy[H.Ny]; }
  out[0] = r[0];
  out[1] = umom;
  out[2] = vmom;
  out[3] = k;
  return INS2D_OK;
  API_END
}


int ins2d_cnn_prepare_pairs(ins2d_ctx *ctx, const double *f, const double *p, int32_t npairs, int32_t center,
                            float *in, float *tgt) {
  API_BEGIN
  if (npairs < 0 || (npairs > 0 && (!f || !p || !in || !tgt)))
    return fail(ctx, INS2D_EINVAL, "cnn_prepare_pairs: null argument or negative count");
  const long long Np = ctx->P.Np;
  if (!ctx->lg_red) ctx->lg_red = dalloc<double>(ctx, cnn::red_doubles());
  for (int32_t k = 0; k < npairs; ++k)
    cnn::prepare(ctx->P, f + k * Np, p + k * Np, center ? 1 : 0, in + k * Np, tgt + k * Np, ctx->lg_red,
                 ctx->stream);
  CK(cudaStreamSynchronize(ctx->stream));
  return INS2D_OK;
  API_END
}

namespace {
int cnn_residual_call(ins2d_ctx *ctx, ins2d_cnn *net, const float *in, int32_t B, float lr, double *loss,
                      float *grad) {
  if (!net || !in || B < 1) return fail(ctx, INS2D_EINVAL, "cnn residual loss: null network/input or B < 1");
  if (net->device != ctx->device) return fail(ctx, INS2D_EINVAL, "cnn residual loss: network on another device");
  if ((long long)B * ctx->P.Np > (1LL << 26)) return fail(ctx, INS2D_EINVAL, "cnn residual loss: B*Np > 2^26");
  if (lr < 0.0f || !std::isfinite(lr)) return fail(ctx, INS2D_EINVAL, "cnn residual loss: lr must be >= 0");
  const double l = cnn::loss_grad(net, in, nullptr, B, ctx->P.Npy, ctx->P.Npx, net->stream, &ctx->P);
  if (!std::isfinite(l)) return fail(ctx, INS2D_ENONFINITE, "cnn residual loss: non-finite loss");
  if (loss) *loss = l;
  if (grad) {
    CK(cudaMemcpyAsync(grad, net->g, cnn::kNParam * sizeof(float), cudaMemcpyDeviceToHost, net->stream));
    CK(cudaStreamSynchronize(net->stream));
  }
  if (lr > 0.0f) cnn::adam(net, lr, net->stream);
  return INS2D_OK;
}
}  // namespace

int ins2d_cnn_loss_grad_residual(ins2d_ctx *ctx, ins2d_cnn *net, const float *in, int32_t B, double *loss,
                                 float *grad) {
  API_BEGIN
  return cnn_residual_call(ctx, net, in, B, 0.0f, loss, grad);
  API_END
}

int ins2d_cnn_train_step_residual(ins2d_ctx *ctx, ins2d_cnn *net, const float *in, int32_t B, float lr,
                                  double *loss) {
  API_BEGIN
  if (!(lr > 0.0f)) return fail(ctx, INS2D_EINVAL, "cnn_train_step_residual: lr must be > 0");
  return cnn_residual_call(ctx, net, in, B, lr, loss, nullptr);
  API_END
}

int ins2d_set_learned_guess(ins2d_ctx *ctx, ins2d_cnn *net) {
  API_BEGIN
  if (net && net->device != ctx->device)
    return fail(ctx, INS2D_EINVAL, "set_learned_guess: network and context on different devices");
  if (net && !ctx->lg_x0) {
    const size_t Np = (size_t)ctx->P.Np;
    ctx->lg_x0 = dalloc<double>(ctx, Np);
    ctx->lg_q = dalloc<double>(ctx, Np);
    ctx->lg_r0 = dalloc<double>(ctx, Np);
    ctx->lg_p = dalloc<double>(ctx, Np);
    ctx->lg_z = dalloc<double>(ctx, Np);
    if (!ctx->lg_red) ctx->lg_red = dalloc<double>(ctx, cnn::red_doubles());
  }
  if (net) cnn::reserve(net, 2 * ctx->P.Np);
  ctx->cnn = net;
  return INS2D_OK;
  API_END
}

int ins2d_set_learned_mode(ins2d_ctx *ctx, int32_t mode) {
  if (!ctx) return INS2D_EINVAL;
  if (mode != INS2D_LEARNED_GUESS && mode != INS2D_LEARNED_PRECOND)
    return fail(ctx, INS2D_EINVAL, "set_learned_mode: unknown mode");
  ctx->lg_mode = mode;
  return INS2D_OK;
}

// The training recipe of the learned guess in one call, for callers without
// device buffers of their own (a MATLAB gateway): record the solver's pairs
// over record_steps time steps from (V, p) (the caller's arrays are not
// modified), prepare them, and train with the residual loss.
int ins2d_learned_train(ins2d_ctx *ctx, ins2d_cnn *net, const double *V, const double *p, double t, double dt,
                        int32_t record_steps, int32_t max_pairs, int32_t train_steps, int32_t batch, float lr,
                        int32_t noise, uint64_t seed, int mem, double *loss_first, double *loss_last) {
  API_BEGIN
  if (check_mem(ctx, mem)) return INS2D_EINVAL;
  if (!net || !V || !p || record_steps < 1 || max_pairs < 1 || train_steps < 1 || batch < 1 || noise < 0 ||
      !(lr > 0.0f) || !(dt > 0.0))
    return fail(ctx, INS2D_EINVAL, "learned_train: bad argument");
  if (net->device != ctx->device) return fail(ctx, INS2D_EINVAL, "learned_train: network on another device");
  const long long Np = ctx->P.Np;
  const size_t NV = (size_t)(ctx->P.Nu + ctx->P.Nv);
  const int fields = 2 * (batch + noise);
  if ((long long)fields * Np > (1LL << 26)) return fail(ctx, INS2D_EINVAL, "learned_train: batch too large");
  cudaStream_t s = ctx->stream;
  std::vector<void *> tmp;
  auto talloc = [&](size_t bytes) {
    void *q = nullptr;
    if (cudaMalloc(&q, bytes) != cudaSuccess) throw std::bad_alloc();
    tmp.push_back(q);
    return q;
  };
  struct Free {
    std::vector<void *> &v;
    ~Free() {
      for (void *q : v) cudaFree(q);
    }
  } guard{tmp};
  double *dV = (double *)talloc(NV * sizeof(double)), *dP = (double *)talloc(Np * sizeof(double));
  const cudaMemcpyKind kind = mem == INS2D_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  CK(cudaMemcpyAsync(dV, V, NV * sizeof(double), kind, s));
  CK(cudaMemcpyAsync(dP, p, Np * sizeof(double), kind, s));
  double *fb = (double *)talloc((size_t)max_pairs * Np * sizeof(double));
  double *pb = (double *)talloc((size_t)max_pairs * Np * sizeof(double));
  ins2d_cnn *saved = ctx->cnn;
  ctx->cnn = nullptr;  // record the plain solver's pairs
  ctx->rec_f = fb;
  ctx->rec_p = pb;
  ctx->rec_cap = max_pairs;
  ctx->rec_n = 0;
  int rc = ins2d_erk_run(ctx, dV, dP, t, dt, record_steps, nullptr, INS2D_MEM_DEVICE);
  const int n = ctx->rec_n;
  ctx->rec_f = ctx->rec_p = nullptr;
  ctx->rec_cap = ctx->rec_n = 0;
  ctx->cnn = saved;
  if (rc) return rc;
  if (n < 1) return fail(ctx, INS2D_EINVAL, "learned_train: no PCG solves to record (FFT path?)");
  if (!ctx->lg_red) ctx->lg_red = dalloc<double>(ctx, cnn::red_doubles());
  float *in = (float *)talloc((size_t)n * Np * sizeof(float));
  for (int k = 0; k < n; ++k)
    cnn::prepare(ctx->P, fb + (size_t)k * Np, nullptr, 0, in + (size_t)k * Np, nullptr, ctx->lg_red, s);
  float *xb = (float *)talloc((size_t)fields * Np * sizeof(float));
  CK(cudaStreamSynchronize(s));
  // output scale: the inputs' rms over the network's at out_scale 1
  net->out_scale = 1.0f;
  const int b0 = std::min(batch, n);
  cnn::forward(net, in, b0, ctx->P.Npy, ctx->P.Npx, s);
  const double sx = cnn::sumsq(in, (long long)b0 * Np, ctx->lg_red, s);
  const double sy = cnn::sumsq(net->y, (long long)b0 * Np, ctx->lg_red, s);
  net->out_scale = (float)(sy > 0.0 ? std::sqrt(sx / sy) : 1.0);
  // Adam on random batches (splitmix64 from the seed), cosine-decayed rate
  uint64_t st = seed;
  auto next = [&]() {
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  const double lr_final = 0.05 * lr;
  for (int it = 0; it < train_steps; ++it) {
    for (int j = 0; j < batch; ++j) {
      const int k = (int)(next() % (uint64_t)n);
      CK(cudaMemcpyAsync(xb + (size_t)j * Np, in + (size_t)k * Np, Np * sizeof(float), cudaMemcpyDeviceToDevice, s));
    }
    if (noise) cnn::gaussian(xb + (size_t)batch * Np, (long long)noise * Np, next(), s);
    cnn::negate_tail(xb, (long long)(batch + noise) * Np, s);
    const double l = cnn::loss_grad(net, xb, nullptr, fields, ctx->P.Npy, ctx->P.Npx, s, &ctx->P);
    if (!std::isfinite(l)) return fail(ctx, INS2D_ENONFINITE, "learned_train: non-finite loss");
    if (it == 0 && loss_first) *loss_first = l;
    if (loss_last) *loss_last = l;
    const double rate =
        lr_final + 0.5 * (lr - lr_final) * (1.0 + std::cos(3.141592653589793 * it / std::max(train_steps - 1, 1)));
    cnn::adam(net, (float)rate, s);
  }
  CK(cudaStreamSynchronize(s));
  return INS2D_OK;
  API_END
}

int ins2d_record_pairs(ins2d_ctx *ctx, double *f_buf, double *p_buf, int32_t capacity) {
  API_BEGIN
  if (capacity < 0 || (capacity > 0 && (!f_buf || !p_buf)))
    return fail(ctx, INS2D_EINVAL, "record_pairs: null buffer or negative capacity");
  ctx->rec_f = capacity ? f_buf : nullptr;
  ctx->rec_p = capacity ? p_buf : nullptr;
  ctx->rec_cap = capacity;
  ctx->rec_n = 0;
  return INS2D_OK;
  API_END
}

int32_t ins2d_recorded_pairs(const ins2d_ctx *ctx) { return ctx ? ctx->rec_n : 0; }

}  // extern "C"

// ===========================================================================
// Ensembles: many independent flows (different grids, boundary conditions,
// Re) advanced together.  Each member is a full context (its operator
// tables, multigrid hierarchy, work arrays); the ensemble adds the members'
// state (V, p), a device table of member descriptors and the tile work lists,
// so every phase of a time step is ONE launch over all members: the stage
// and residual walkers over the members' tiles, the divergence and
// projection over their cells, and the Poisson solves as a persistent launch
// whose thread blocks take members from a queue (largest first) and run each
// member's whole PCG.  A step is captured once as a CUDA graph and replayed.
// The solve launch shape (threads per member) is chosen by timing the
// candidates on the first run.
struct ins2d_ens {
  int device = 0;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  cudaEvent_t order_ev = nullptr;  // ins2d_ens_wait_stream
  std::vector<ins2d_ctx *> mem;
  std::vector<double *> V, p;  // member state (owned by the member contexts' allocations)
  std::vector<double> dt_member;  // per-member time step (0: the run's dt)
  double dt_uploaded = -1.0;
  std::string err;
  bool fp32 = false;
  double tol2 = 0.0;
  long long maxit = 0;
  // device tables
  EnsMemberD *d_mem = nullptr;
  std::vector<MgD *> d_mg;
  int4 *d_fast = nullptr, *d_gen = nullptr, *d_cells = nullptr;
  int n_fast = 0, n_gen = 0, n_cells = 0;
  int *d_order = nullptr;
  unsigned *d_queue = nullptr;
  EnsStats *d_stats = nullptr;
  std::vector<void *> allocs;
  bool uploaded = false;
  // batched solver (ens_pcg.cu): member levels, work segments, CG scalars
  bool can_batch = false;
  EnsMgD mgd{};
  EnsMgPlan plan{};
  int2 *d_ctiles = nullptr;
  int n_ctiles = 0;
  EnsCg *d_cg = nullptr;
  int *d_active = nullptr, *h_active = nullptr;
  // launch shape of the member solves (autotuned: 512 or 256 threads per
  // member in the persistent solve, or 0 = batched solve) and the step graphs
  int solve_threads = 0, solve_blocks = 0;
  int forced = -1;  // -1: tune on the first run
  bool tuned = false;
  double tuned_ms[3] = {0.0, 0.0, 0.0};
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t chunk_graph = nullptr;  // a chunk of batched PCG iterations
  // fast-diagonalization preconditioner of the batched solves (every member
  // at most kFdmMaxN cells per direction, default or fdm preconditioner)
  bool use_fdm = false;
  // batched solves inside a step graph: the iteration loop is a WHILE node
  bool dev_loop = false;
  cudaStream_t body_stream = nullptr;
  int *d_loops = nullptr;
  EnsFdmD *d_fdm = nullptr;
  std::vector<double *> fdm_z;
  int4 *d_ftiles = nullptr;
  int n_ftiles = 0;
};

namespace {

int ens_fail(ins2d_ens *e, int code, const std::string &msg) {
  if (e) e->err = msg;
  return code;
}

template <typename T>
T *ens_alloc(ins2d_ens *e, size_t n) {
  void *p = nullptr;
  if (cudaMalloc(&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) throw std::bad_alloc();
  e->allocs.push_back(p);
  return (T *)p;
}

void ens_release_graphs(ins2d_ens *e) {
  for (auto &g : e->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  if (e->chunk_graph) {
    cudaGraphExecDestroy(e->chunk_graph);
    e->chunk_graph = nullptr;
  }
}

#ifndef INS2D_ENS_TAIL_LEVEL
#define INS2D_ENS_TAIL_LEVEL 2
#endif
// Work segments, member level tables and CG scalars of the batched solver.
void ens_build_batch(ins2d_ens *e, const std::vector<int> &order) {
  const int n = (int)e->mem.size();
  std::vector<MgLevelD> lev((size_t)n * kMgMaxLevels);
  std::vector<int> nlev(n), ncoarse(n);
  std::vector<const double *> cinv(n);
  int lmax = 0;
  for (int m = 0; m < n; ++m) {
    const MgD &M = e->mem[m]->mg;
    for (int l = 0; l < M.nlev; ++l) lev[(size_t)m * kMgMaxLevels + l] = M.L[l];
    nlev[m] = M.nlev;
    ncoarse[m] = M.ncoarse;
    cinv[m] = M.cinv;
    lmax = std::max(lmax, M.nlev);
  }
  MgLevelD *d_lev = ens_alloc<MgLevelD>(e, lev.size());
  int *d_nlev = ens_alloc<int>(e, n), *d_nco = ens_alloc<int>(e, n);
  const double **d_ci = ens_alloc<const double *>(e, n);
  CK(cudaMemcpy(d_lev, lev.data(), lev.size() * sizeof(MgLevelD), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_nlev, nlev.data(), n * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_nco, ncoarse.data(), n * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_ci, cinv.data(), n * sizeof(const double *), cudaMemcpyHostToDevice));
  e->mgd = EnsMgD{d_lev, d_nlev, d_ci, d_nco};
  // segments: members in solve order (largest first), counts per phase
  auto make_seg = [&](auto count) {
    std::vector<int> mm;
    std::vector<long long> st{0};
    for (int m : order) {
      const long long c = count(m);
      if (c <= 0) continue;
      mm.push_back(m);
      st.push_back(st.back() + c);
    }
    EnsSeg sg{};
    sg.n = (int)mm.size();
    sg.total = st.back();
    if (sg.n > 0) {
      int *dm = ens_alloc<int>(e, mm.size());
      long long *ds = ens_alloc<long long>(e, st.size());
      CK(cudaMemcpy(dm, mm.data(), mm.size() * sizeof(int), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(ds, st.data(), st.size() * sizeof(long long), cudaMemcpyHostToDevice));
      sg.mem = dm;
      sg.start = ds;
    }
    return sg;
  };
  EnsMgPlan &pl = e->plan;
  pl.lmax = lmax;
  for (int l = 0; l < lmax - 1; ++l) {
    auto L = [&](int m) -> const MgLevelD & { return lev[(size_t)m * kMgMaxLevels + l]; };
    auto C = [&](int m) -> const MgLevelD & { return lev[(size_t)m * kMgMaxLevels + l + 1]; };
    pl.xl[l] = make_seg([&](int m) { return nlev[m] - 1 > l ? (long long)L(m).ny : 0LL; });
    pl.yl[l] = make_seg([&](int m) { return nlev[m] - 1 > l ? (long long)L(m).nx : 0LL; });
    pl.yg[l] = make_seg([&](int m) {
      return nlev[m] - 1 > l ? (long long)(L(m).nx + kEnsYcols - 1) / kEnsYcols : 0LL;
    });
    pl.rs[l] = make_seg([&](int m) { return nlev[m] - 1 > l ? (long long)C(m).nx * C(m).ny : 0LL; });
    pl.pr[l] = make_seg([&](int m) { return nlev[m] - 1 > l ? (long long)L(m).nx * L(m).ny : 0LL; });
  }
  pl.co = make_seg([&](int m) { return (long long)ncoarse[m]; });
  // levels from INS2D_ENS_TAIL_LEVEL down run in one block per member
  pl.ltail = std::min(INS2D_ENS_TAIL_LEVEL, std::max(lmax - 1, 0));
  const MgD **d_mgs = ens_alloc<const MgD *>(e, n);
  std::vector<const MgD *> hm(e->d_mg.begin(), e->d_mg.end());
  CK(cudaMemcpy(d_mgs, hm.data(), n * sizeof(const MgD *), cudaMemcpyHostToDevice));
  pl.mgs = d_mgs;
  std::vector<int2> ct;
  for (int m : order)
    for (long long k = 0; k < e->mem[m]->P.Np; k += 256) ct.push_back(make_int2(m, (int)k));
  e->d_ctiles = ens_alloc<int2>(e, ct.size());
  CK(cudaMemcpy(e->d_ctiles, ct.data(), ct.size() * sizeof(int2), cudaMemcpyHostToDevice));
  e->n_ctiles = (int)ct.size();
  if (e->use_fdm) {
    std::vector<int4> ft;
    for (int m : order) fdm_tiles(m, e->mem[m]->P.Npx, e->mem[m]->P.Npy, ft);
    e->d_ftiles = ens_alloc<int4>(e, ft.size());
    CK(cudaMemcpy(e->d_ftiles, ft.data(), ft.size() * sizeof(int4), cudaMemcpyHostToDevice));
    e->n_ftiles = (int)ft.size();
  }
  std::vector<EnsCg> cg(n);
  for (int m = 0; m < n; ++m) {
    cg[m] = EnsCg{};
    cg[m].tol2 = e->tol2;
    cg[m].maxit = e->maxit;
  }
  e->d_cg = ens_alloc<EnsCg>(e, n);
  CK(cudaMemcpy(e->d_cg, cg.data(), n * sizeof(EnsCg), cudaMemcpyHostToDevice));
  e->d_active = ens_alloc<int>(e, 1);
  CK(cudaMallocHost((void **)&e->h_active, sizeof(int)));
}

// All members' Poisson solves, batched across members (one launch per phase;
// the host checks every few iterations whether any member still iterates).
void ens_solve_batched(ins2d_ens *e, int which) {
  const int n = (int)e->mem.size();
  const MgD &M0 = e->mem[0]->mg;
  const double om = M0.omega, al = M0.alpha;
  cudaStream_t s = e->stream;
  // the preconditioner: fast diagonalization (four products over all
  // members' tiles) or the members' V-cycles
  auto precond_on = [&](cudaStream_t st) {
    if (e->use_fdm)
      fdm_apply_ens(e->d_fdm, e->d_ftiles, e->n_ftiles, e->d_cg, st);
    else
      ens_vcycle(e->d_mem, e->mgd, e->d_cg, e->plan, om, al, st);
  };
  auto precond = [&]() { precond_on(s); };
  ens_cg_vec(e->d_mem, e->mgd, e->d_ctiles, e->n_ctiles, e->d_cg, 0, s);
  ens_cg_scalar(e->d_cg, n, 0, nullptr, s);
  precond();
  ens_cg_vec(e->d_mem, e->mgd, e->d_ctiles, e->n_ctiles, e->d_cg, 4, s);
  ens_cg_scalar(e->d_cg, n, 1, nullptr, s);
  const int chunk = e->use_fdm ? (e->dev_loop ? 1 : 2) : 4;
  auto iterations_on = [&](cudaStream_t st) {
    for (int k = 0; k < chunk; ++k) {
      ens_cg_vec(e->d_mem, e->mgd, e->d_ctiles, e->n_ctiles, e->d_cg, 1, st);
      ens_cg_scalar(e->d_cg, n, 2, nullptr, st);
      ens_cg_vec(e->d_mem, e->mgd, e->d_ctiles, e->n_ctiles, e->d_cg, 2, st);
      ens_cg_scalar(e->d_cg, n, 3, e->d_active, st);
      precond_on(st);
      ens_cg_vec(e->d_mem, e->mgd, e->d_ctiles, e->n_ctiles, e->d_cg, 3, st);
      ens_cg_scalar(e->d_cg, n, 4, nullptr, st);
      ens_cg_vec(e->d_mem, e->mgd, e->d_ctiles, e->n_ctiles, e->d_cg, 5, st);
    }
  };
  auto iterations = [&]() { iterations_on(s); };
  if (e->dev_loop) {
    // inside a step graph: the loop is a WHILE node that ends when no member
    // iterates or after CG_maxit / chunk + 4 passes
    const int limit = (int)std::min<long long>(e->maxit / chunk + 4, 1 << 30);
    capture_while(
        s, e->body_stream, [&](cudaGraphConditionalHandle h) { ens_loop_cond(e->d_cg, n, e->d_loops, limit, 0, h, s); },
        [&](cudaStream_t bs, cudaGraphConditionalHandle h) {
          iterations_on(bs);
          ens_loop_cond(e->d_cg, n, e->d_loops, limit, 1, h, bs);
        });
    ens_cg_finish(e->d_mem, e->d_ctiles, e->n_ctiles, e->d_cg, n, which, e->d_stats, s);
    return;
  }
  // the chunk of iterations is one CUDA graph (its launches depend only on
  // the ensemble's device tables), replayed until no member iterates
  if (!e->chunk_graph) {
    cudaGraph_t gr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    iterations();
    CK(cudaStreamEndCapture(s, &gr));
    cudaError_t ie = cudaGraphInstantiate(&e->chunk_graph, gr, 0);
    cudaGraphDestroy(gr);
    CK(ie);
  }
  for (long long done_it = 0;; done_it += chunk) {
    CK(cudaGraphLaunch(e->chunk_graph, s));
    CK(cudaMemcpyAsync(e->h_active, e->d_active, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (*e->h_active == 0) break;
    if (done_it > e->maxit + 2 * chunk) throw CudaError("ensemble PCG: members still active after CG_maxit");
  }
  ens_cg_finish(e->d_mem, e->d_ctiles, e->n_ctiles, e->d_cg, n, which, e->d_stats, s);
}

// descriptor table, work lists and member order (largest first)
void ens_upload(ins2d_ens *e, double dt) {
  const int n = (int)e->mem.size();
  std::vector<EnsMemberD> h(n);
  std::vector<int4> fast, gen, cells;
  for (int m = 0; m < n; ++m) {
    ins2d_ctx *c = e->mem[m];
    EnsMemberD &d = h[m];
    d = EnsMemberD{};
    d.P = c->P;
    d.dt = e->dt_member[m] > 0.0 ? e->dt_member[m] : dt;
    d.V = e->V[m];
    d.p = e->p[m];
    d.Vs = c->Vs;
    d.Wt = c->Wt;
    for (int k = 0; k < kMaxStages; ++k) d.kV[k] = c->kV[k];
    d.f = c->f;
    d.dp = c->dp;
    d.wres = c->wres;
    d.W = c->pcg;
    d.mg = c->use_mg ? e->d_mg[m] : nullptr;
    d.zf = e->use_fdm ? e->fdm_z[m] : nullptr;
    walk_tiles(c->P, m, fast, gen);
    cell_tiles(c->P, m, cells);
  }
  std::vector<int> order(n);
  for (int m = 0; m < n; ++m) order[m] = m;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return e->mem[a]->P.Np > e->mem[b]->P.Np; });
  if (!e->d_mem) {
    e->d_mem = ens_alloc<EnsMemberD>(e, n);
    e->d_order = ens_alloc<int>(e, n);
    e->d_queue = ens_alloc<unsigned>(e, 2);
    e->d_stats = ens_alloc<EnsStats>(e, n);
    e->d_fast = ens_alloc<int4>(e, fast.size());
    e->d_gen = ens_alloc<int4>(e, gen.size());
    e->d_cells = ens_alloc<int4>(e, cells.size());
    CK(cudaMemset(e->d_queue, 0, 2 * sizeof(unsigned)));
  }
  CK(cudaMemcpy(e->d_mem, h.data(), n * sizeof(EnsMemberD), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(e->d_order, order.data(), n * sizeof(int), cudaMemcpyHostToDevice));
  if (!fast.empty()) CK(cudaMemcpy(e->d_fast, fast.data(), fast.size() * sizeof(int4), cudaMemcpyHostToDevice));
  if (!gen.empty()) CK(cudaMemcpy(e->d_gen, gen.data(), gen.size() * sizeof(int4), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(e->d_cells, cells.data(), cells.size() * sizeof(int4), cudaMemcpyHostToDevice));
  e->n_fast = (int)fast.size();
  e->n_gen = (int)gen.size();
  e->n_cells = (int)cells.size();
  if (e->can_batch && !e->d_cg) ens_build_batch(e, order);
  e->uploaded = true;
  e->dt_uploaded = dt;
}

int sm_count(int device) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
  return v > 0 ? v : 1;
}

void ens_solve(ins2d_ens *e, int which) {
  if (e->solve_threads == 0 && e->can_batch) {
    ens_solve_batched(e, which);
    return;
  }
  launch_pcg_members(e->d_mem, e->d_order, (int)e->mem.size(), which, e->tol2, e->maxit, e->d_queue, e->d_stats,
                     e->solve_threads, e->solve_blocks, e->stream);
}

// one time step of every member (time_ERK.m with steady boundary conditions;
// each member's dt is in its descriptor)
void ens_step(ins2d_ens *e, bool k0_cached) {
  const ins2d_ctx *c0 = e->mem[0];
  const int s = c0->s;
  for (int i = 0; i < s; ++i) {
    if (i == 0 && k0_cached) {
      launch_stage_cached_ens(e->d_mem, e->d_cells, e->n_cells, c0->A[0][0], e->stream);
    } else {
      EnsWalk w{};
      w.mode = 0;
      w.stage = i;
      w.store = (c0->need_store[i] || i == 0) ? 1 : 0;
      w.use_vs = i > 0;
      for (int m = 0; m < i; ++m)
        if (c0->A[i][m] != 0.0) {
          w.kidx[w.nprev] = m;
          w.aprev[w.nprev] = c0->A[i][m];
          ++w.nprev;
        }
      w.aii = c0->A[i][i];
      launch_walk_ens(e->d_mem, e->d_fast, e->n_fast, e->d_gen, e->n_gen, w, e->fp32, e->stream);
    }
    if (i > 0) {
      launch_div_ens(e->d_mem, e->d_cells, e->n_cells, 0, 1.0 / c0->c[i], e->stream);
      ens_solve(e, 0);
    }
    launch_project_ens(e->d_mem, e->d_cells, e->n_cells, c0->c[i], i == 0 ? 1 : 0, i == s - 1 ? 1 : 0, e->stream);
  }
  // additional pressure solve; its residual is the next step's first stage
  EnsWalk w{};
  w.mode = 1;
  w.cache = 1;
  launch_walk_ens(e->d_mem, e->d_fast, e->n_fast, e->d_gen, e->n_gen, w, e->fp32, e->stream);
  launch_div_ens(e->d_mem, e->d_cells, e->n_cells, 1, 1.0, e->stream);
  ens_solve(e, 1);
}

// Times the member solve with each candidate launch shape on the current
// right-hand sides (the solves are repeatable: x0 = 0, deterministic
// reductions) and keeps the fastest.
void ens_autotune(ins2d_ens *e) {
  const int sms = sm_count(e->device), n = (int)e->mem.size();
  // 0: batched across members; fast-diagonalization ensembles solve batched
  const int cand[3] = {e->use_fdm ? 0 : 512, 256, 0};
  const int ncand = e->use_fdm ? 1 : (e->can_batch ? 3 : 2);
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  int best = -1;
  float best_ms = 0.f;
  for (int k = 0; k < ncand; ++k) {
    e->solve_threads = cand[k];
    e->solve_blocks = cand[k] ? std::min(n, sms * (512 / cand[k])) : 0;
    ens_solve(e, 0);  // warm-up
    CK(cudaEventRecord(a, e->stream));
    ens_solve(e, 0);
    CK(cudaEventRecord(b, e->stream));
    CK(cudaEventSynchronize(b));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, a, b));
    e->tuned_ms[k] = ms;
    if (best < 0 || ms < best_ms) {
      best = k;
      best_ms = ms;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  e->solve_threads = cand[best];
  e->solve_blocks = cand[best] ? std::min(n, sms * (512 / cand[best])) : 0;
}

#define ENS_BEGIN                 \
  if (!e) return INS2D_EINVAL;    \
  e->err.clear();                 \
  DeviceGuard dguard_(e->device); \
  try {                           \
    CK(dguard_.err);
#define ENS_END                                                     \
  }                                                                 \
  catch (const CudaError &x) {                                      \
    return ens_fail(e, INS2D_ECUDA, x.what());                      \
  }                                                                 \
  catch (const std::bad_alloc &) {                                  \
    return ens_fail(e, INS2D_ENOMEM, "device allocation failed");   \
  }                                                                 \
  catch (const std::exception &x) {                                 \
    return ens_fail(e, INS2D_EINVAL, x.what());                     \
  }

}  // namespace

extern "C" {

int ins2d_ens_create(int32_t n, const ins2d_grid_desc *grids, const ins2d_bc_desc *bcs, const ins2d_opts *opts,
                     ins2d_ens **out) {
  if (!out || n < 1 || !grids || !bcs || !opts) return INS2D_EINVAL;
  *out = nullptr;
  ins2d_ens *e = new (std::nothrow) ins2d_ens();
  if (!e) return INS2D_ENOMEM;
  int rc = INS2D_OK;
  std::string msg;
  for (int m = 0; m < n && rc == INS2D_OK; ++m) {
    const ins2d_opts &o = opts[m];
    if (bcs[m].bc_unsteady) {
      rc = INS2D_EINVAL;
      msg = "ensemble members need steady boundary conditions";
    } else if (o.poisson == INS2D_POISSON_FFT) {
      rc = INS2D_EINVAL;
      msg = "ensemble members use the PCG pressure solver (poisson 1-5)";
    } else if (o.device != opts[0].device || o.precision != opts[0].precision || o.CG_acc != opts[0].CG_acc ||
               o.CG_maxit != opts[0].CG_maxit || o.rk_stages != opts[0].rk_stages ||
               std::memcmp(o.rk_A, opts[0].rk_A, sizeof(o.rk_A)) != 0 ||
               std::memcmp(o.rk_c, opts[0].rk_c, sizeof(o.rk_c)) != 0 ||
               std::memcmp(o.rk_b, opts[0].rk_b, sizeof(o.rk_b)) != 0) {
      rc = INS2D_EINVAL;
      msg = "ensemble members must share device, precision, CG_acc, CG_maxit and the RK method";
    }
    if (rc) break;
    ins2d_ctx *c = nullptr;
    // the ensemble's solvers (persistent per member, or batched) run the
    // multigrid V-cycle: members take it unless Jacobi is asked for
    ins2d_opts om = o;
    if (om.precond != INS2D_PRECOND_JACOBI) om.precond = INS2D_PRECOND_MG;
    rc = ins2d_ctx_create(&grids[m], &bcs[m], &om, &c);
    if (rc) {
      msg = std::string("member ") + std::to_string(m) + ": " + (c ? c->err : std::string("create failed"));
      if (c) ins2d_ctx_destroy(c);
      break;
    }
    e->mem.push_back(c);
    if ((long long)c->P.Np > 262144) {
      rc = INS2D_EINVAL;
      msg = "ensemble members are limited to 262144 pressure cells";
    }
  }
  if (rc == INS2D_OK) {
    try {
      e->device = opts[0].device;
      DeviceGuard dg(e->device);
      CK(dg.err);
      e->fp32 = e->mem[0]->fp32;
      e->tol2 = opts[0].CG_acc * opts[0].CG_acc;
      e->maxit = opts[0].CG_maxit;
      for (ins2d_ctx *c : e->mem) {
        e->V.push_back(dalloc<double>(c, (size_t)(c->P.Nu + c->P.Nv)));
        e->p.push_back(dalloc<double>(c, (size_t)c->P.Np));
        CK(cudaMemset(e->V.back(), 0, (size_t)(c->P.Nu + c->P.Nv) * sizeof(double)));
        CK(cudaMemset(e->p.back(), 0, (size_t)c->P.Np * sizeof(double)));
        MgD *dm = nullptr;
        if (c->use_mg) {
          dm = ens_alloc<MgD>(e, 1);
          CK(cudaMemcpy(dm, &c->mg, sizeof(MgD), cudaMemcpyHostToDevice));
        }
        e->d_mg.push_back(dm);
        e->dt_member.push_back(0.0);
      }
      e->can_batch = true;
      for (ins2d_ctx *c : e->mem) e->can_batch = e->can_batch && c->use_mg;
      // fast diagonalization for the batched solves when every member takes
      // the default (or fdm) preconditioner and is small enough for dense bases
      bool fdm = e->can_batch;
      for (int m = 0; m < n && fdm; ++m) {
        const ins2d_ctx *c = e->mem[m];
        fdm = (opts[m].precond == INS2D_PRECOND_DEFAULT || opts[m].precond == INS2D_PRECOND_FDM) &&
              std::max(c->H.Npx, c->H.Npy) <= kFdmMaxN;
      }
      if (fdm) {
        std::vector<EnsFdmD> hf(n);
        for (int m = 0; m < n; ++m) {
          ins2d_ctx *c = e->mem[m];
          const HostOps &H = c->H;
          const FdmHost1D fx = fdm_1d(H.TX, H.hx), fy = fdm_1d(H.TY, H.hy);
          EnsFdmD &D = hf[m];
          D.nx = H.Npx;
          D.ny = H.Npy;
          D.Qx = upload_vec(c, fx.Q);
          D.Qy = upload_vec(c, fy.Q);
          D.lx = upload_vec(c, fx.lam);
          D.ly = upload_vec(c, fy.lam);
          D.thr = 1e-12 * (fx.lam.back() + fy.lam.back());
          D.r = c->pcg.r;
          const size_t Np = (size_t)c->P.Np;
          D.t1 = dalloc<double>(c, Np);
          D.t2 = dalloc<double>(c, Np);
          D.z = dalloc<double>(c, Np);
          e->fdm_z.push_back(D.z);
        }
        e->d_fdm = ens_alloc<EnsFdmD>(e, n);
        CK(cudaMemcpy(e->d_fdm, hf.data(), n * sizeof(EnsFdmD), cudaMemcpyHostToDevice));
        e->use_fdm = true;
      }
      CK(cudaStreamCreateWithFlags(&e->own_stream, cudaStreamNonBlocking));
      CK(cudaStreamCreateWithFlags(&e->body_stream, cudaStreamNonBlocking));
      e->d_loops = ens_alloc<int>(e, 1);
      e->stream = e->own_stream;
      CK(cudaDeviceSynchronize());
    } catch (const CudaError &x) {
      rc = INS2D_ECUDA;
      msg = x.what();
    } catch (const std::bad_alloc &) {
      rc = INS2D_ENOMEM;
      msg = "device allocation failed";
    }
  }
  if (rc != INS2D_OK) {
    e->err = msg;
    *out = e;  // the caller reads the message, then destroys
    return rc;
  }
  *out = e;
  return INS2D_OK;
}

int ins2d_ens_destroy(ins2d_ens *e) {
  if (!e) return INS2D_OK;
  DeviceGuard dg(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  ens_release_graphs(e);
  if (e->order_ev) cudaEventDestroy(e->order_ev);
  if (e->h_active) cudaFreeHost(e->h_active);
  for (void *p : e->allocs) cudaFree(p);
  for (ins2d_ctx *c : e->mem) ins2d_ctx_destroy(c);
  if (e->own_stream) cudaStreamDestroy(e->own_stream);
  if (e->body_stream) cudaStreamDestroy(e->body_stream);
  delete e;
  return INS2D_OK;
}

const char *ins2d_ens_last_error(const ins2d_ens *e) { return e ? e->err.c_str() : "null ensemble"; }

int32_t ins2d_ens_size(const ins2d_ens *e) { return e ? (int32_t)e->mem.size() : 0; }

ins2d_ctx *ins2d_ens_member(ins2d_ens *e, int32_t m) {
  if (!e || m < 0 || m >= (int32_t)e->mem.size()) return nullptr;
  return e->mem[m];
}

int ins2d_ens_set_stream(ins2d_ens *e, void *stream) {
  if (!e) return INS2D_EINVAL;
  e->stream = stream ? (cudaStream_t)stream : e->own_stream;
  ens_release_graphs(e);
  return INS2D_OK;
}

int ins2d_ens_wait_stream(ins2d_ens *e, void *stream) {
  ENS_BEGIN
  const cudaStream_t other = (cudaStream_t)stream;
  if (other == e->stream) return INS2D_OK;
  if (!e->order_ev) CK(cudaEventCreateWithFlags(&e->order_ev, cudaEventDisableTiming));
  CK(cudaEventRecord(e->order_ev, other));
  CK(cudaStreamWaitEvent(e->stream, e->order_ev, 0));
  return INS2D_OK;
  ENS_END
}

int ins2d_ens_set_state(ins2d_ens *e, int32_t m, const double *V, const double *p, int mem) {
  ENS_BEGIN
  if (m < 0 || m >= (int32_t)e->mem.size() || !V || !p) return ens_fail(e, INS2D_EINVAL, "set_state: bad argument");
  if (mem != INS2D_MEM_HOST && mem != INS2D_MEM_DEVICE) return ens_fail(e, INS2D_EINVAL, "bad mem");
  const ins2d_ctx *c = e->mem[m];
  const cudaMemcpyKind k = mem == INS2D_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  CK(cudaMemcpyAsync(e->V[m], V, (size_t)(c->P.Nu + c->P.Nv) * sizeof(double), k, e->stream));
  CK(cudaMemcpyAsync(e->p[m], p, (size_t)c->P.Np * sizeof(double), k, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return INS2D_OK;
  ENS_END
}

int ins2d_ens_get_state(ins2d_ens *e, int32_t m, double *V, double *p, int mem) {
  ENS_BEGIN
  if (m < 0 || m >= (int32_t)e->mem.size() || !V || !p) return ens_fail(e, INS2D_EINVAL, "get_state: bad argument");
  if (mem != INS2D_MEM_HOST && mem != INS2D_MEM_DEVICE) return ens_fail(e, INS2D_EINVAL, "bad mem");
  const ins2d_ctx *c = e->mem[m];
  const cudaMemcpyKind k = mem == INS2D_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  CK(cudaMemcpyAsync(V, e->V[m], (size_t)(c->P.Nu + c->P.Nv) * sizeof(double), k, e->stream));
  CK(cudaMemcpyAsync(p, e->p[m], (size_t)c->P.Np * sizeof(double), k, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  return INS2D_OK;
  ENS_END
}

int ins2d_ens_set_member_dt(ins2d_ens *e, int32_t m, double dt) {
  if (!e || m < 0 || m >= (int32_t)e->mem.size() || !(dt >= 0.0)) return INS2D_EINVAL;
  e->dt_member[m] = dt;
  e->uploaded = false;
  return INS2D_OK;
}

int ins2d_ens_state_ptr(ins2d_ens *e, int32_t m, double **V, double **p) {
  if (!e || m < 0 || m >= (int32_t)e->mem.size() || !V || !p) return INS2D_EINVAL;
  *V = e->V[m];
  *p = e->p[m];
  return INS2D_OK;
}

int ins2d_ens_erk_run(ins2d_ens *e, double t, double dt, int32_t nsteps, ins2d_step_stats *stats) {
  ENS_BEGIN
  (void)t;  // steady boundary conditions: the step does not depend on t
  if (nsteps < 0 || !(dt > 0)) return ens_fail(e, INS2D_EINVAL, "erk_run: bad argument");
  const int n = (int)e->mem.size();
  if (!e->uploaded || e->dt_uploaded != dt) ens_upload(e, dt);
  CK(cudaMemsetAsync(e->d_stats, 0, n * sizeof(EnsStats), e->stream));
  for (int k = 0; k < nsteps; ++k) {
    const int g = k > 0 ? 1 : 0;  // graph 1: first stage from the cached residual
    if (e->forced < 0 && !e->tuned) {
      // first use: one direct step, then tune the solve launch on the
      // right-hand side it left behind (re-solving it changes no state: the
      // tuner writes dp, which every stage overwrites); the step's
      // statistics are kept
      e->solve_threads = e->use_fdm ? 0 : 512;
      e->solve_blocks = e->use_fdm ? 0 : std::min(n, sm_count(e->device));
      ens_step(e, g == 1);
      std::vector<EnsStats> keep(n);
      CK(cudaMemcpyAsync(keep.data(), e->d_stats, n * sizeof(EnsStats), cudaMemcpyDeviceToHost, e->stream));
      CK(cudaStreamSynchronize(e->stream));
      ens_autotune(e);
      e->tuned = true;
      CK(cudaMemcpyAsync(e->d_stats, keep.data(), n * sizeof(EnsStats), cudaMemcpyHostToDevice, e->stream));
      CK(cudaStreamSynchronize(e->stream));
      continue;
    }
    if (!e->graph[g]) {
      // batched solves: their iteration loops become WHILE nodes of the graph
      cudaGraph_t gr;
      CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
      e->dev_loop = e->solve_threads == 0;
      try {
        ens_step(e, g == 1);
      } catch (...) {
        e->dev_loop = false;
        cudaGraph_t junk = nullptr;
        if (cudaStreamEndCapture(e->stream, &junk) == cudaSuccess && junk) cudaGraphDestroy(junk);
        throw;
      }
      e->dev_loop = false;
      CK(cudaStreamEndCapture(e->stream, &gr));
      cudaError_t ie = cudaGraphInstantiate(&e->graph[g], gr, 0);
      cudaGraphDestroy(gr);
      CK(ie);
    }
    CK(cudaGraphLaunch(e->graph[g], e->stream));
  }
  std::vector<EnsStats> hs(n);
  CK(cudaMemcpyAsync(hs.data(), e->d_stats, n * sizeof(EnsStats), cudaMemcpyDeviceToHost, e->stream));
  CK(cudaStreamSynchronize(e->stream));
  int first_bad = -1;
  for (int m = 0; m < n; ++m) {
    if (stats) {
      stats[m].n_solves = (int32_t)hs[m].n_solves;
      stats[m].iters_total = (int32_t)hs[m].iters_total;
      stats[m].iters_max = (int32_t)hs[m].iters_max;
      stats[m].norm1_max = hs[m].norm1_max;
    }
    if (hs[m].status != 0 && first_bad < 0) first_bad = m;
  }
  if (first_bad >= 0) {
    const int st = hs[first_bad].status;
    return ens_fail(e, st, std::string("member ") + std::to_string(first_bad) +
                               (st == INS2D_ENOTCONV ? ": CG didn't converge" : ": solve failed"));
  }
  return INS2D_OK;
  ENS_END
}

int ins2d_ens_set_solver(ins2d_ens *e, int32_t threads) {
  if (!e || !(threads == -1 || threads == 0 || threads == 256 || threads == 512)) return INS2D_EINVAL;
  if (threads == 0 && !e->can_batch) return ens_fail(e, INS2D_EINVAL, "batched solves need the multigrid preconditioner");
  if (threads > 0 && e->use_fdm)
    return ens_fail(e, INS2D_EINVAL, "fast-diagonalization ensembles solve batched (threads 0 or -1)");
  e->forced = threads;
  if (threads >= 0) {
    e->solve_threads = threads;
    e->solve_blocks = threads ? std::min((int)e->mem.size(), sm_count(e->device) * (512 / threads)) : 0;
  } else {
    e->solve_threads = 0;
    e->solve_blocks = 0;
  }
  ens_release_graphs(e);
  return INS2D_OK;
}

int ins2d_ens_solve_shape(const ins2d_ens *e, int32_t *threads, int32_t *blocks, double tuned_ms[3]) {
  if (!e) return INS2D_EINVAL;
  if (threads) *threads = e->solve_threads;
  if (blocks) *blocks = e->solve_blocks;
  if (tuned_ms)
    for (int k = 0; k < 3; ++k) tuned_ms[k] = e->tuned_ms[k];
  return INS2D_OK;
}

}  // extern "C"
