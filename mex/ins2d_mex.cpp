// MATLAB/Octave MEX gateway for libins2d.so: lets a reference case call the
// B200 hot path through the reference's own function names.
//
//   h = ins2d_mex('create', options)                    % after operators.m
//   [maxres,F] = ins2d_mex('F', h, V, C, p, t, nopressure)       % F.m:1
//   [dp,iter,norm1,norm2] = ins2d_mex('pressure_poisson', h, f, t)  % pressure_poisson.m:1, cg.F:15-17
//   p = ins2d_mex('pressure_additional_solve', h, V, p, t)
//   [V,p] = ins2d_mex('time_ERK', h, V, p, t, dt)       % time_ERK.m:1
//   [maxdiv,umom,vmom,k] = ins2d_mex('check_conservation', h, V, t)
//   [l0,l1] = ins2d_mex('learned_train', h, V, p, t, dt, record_steps, train_steps, mode)
//       % no counterpart in the reference: trains the learned initial guess on
//       % the pairs of the first record_steps steps and attaches it to the
//       % PCG solves; mode 'guess' (default) or 'precond' (flexible CG)
//   ins2d_mex('learned_detach', h)
//   ins2d_mex('destroy', h)
//
// The gateway flattens the options struct (grid x/y, BC types, fluid.Re,
// solversettings.{poisson,CG_acc,CG_maxit,p_add_solve}, time.RK tableau)
// into the C structs of include/ins2d.h, samples options' uBC/vBC handles via
// mexCallMATLAB (set_bc_vectors.m:52-79) whenever the context asks for BC
// values, and maps a non-zero status to mexErrMsgIdAndTxt (the reference
// errors the same way, cg.F:262).  It follows the conventions of the
// reference's only MEX file, solvers/pressure/cg.F:31-150: inputs borrowed
// read-only, outputs allocated with mxCreateDoubleMatrix.
//
// Needs mex.h (MATLAB or Octave); build with
//   mex -I../include ins2d_mex.cpp -L../ins2d_b200 -lins2d
// It is not compiled in this repository's test environment (no MATLAB/Octave).
#include <mex.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "ins2d.h"

namespace {

int bc_code(const mxArray *bc, const char *comp, const char *side) {
  const mxArray *c = mxGetField(bc, 0, comp);
  const mxArray *s = c ? mxGetField(c, 0, side) : nullptr;
  if (!s || !mxIsChar(s)) mexErrMsgIdAndTxt("ins2d:bc", "options.BC.%s.%s missing", comp, side);
  char buf[8];
  mxGetString(s, buf, sizeof buf);
  if (!strcmp(buf, "dir")) return INS2D_BC_DIR;
  if (!strcmp(buf, "pres")) return INS2D_BC_PRES;
  if (!strcmp(buf, "per")) return INS2D_BC_PER;
  if (!strcmp(buf, "sym")) return INS2D_BC_SYM;
  mexErrMsgIdAndTxt("ins2d:bc", "wrong BC for %s-%s", comp, side);
  return -1;
}

double field_d(const mxArray *s, const char *a, const char *b, double dflt) {
  const mxArray *x = mxGetField(s, 0, a);
  if (x && b) x = mxGetField(x, 0, b);
  return (x && mxIsNumeric(x)) ? mxGetScalar(x) : dflt;
}

struct Handle {
  ins2d_ctx *ctx = nullptr;
  mxArray *options = nullptr;  // persistent copy (uBC/vBC handles, grid)
  ins2d_cnn *net = nullptr;    // learned initial guess / preconditioner, if trained
};

void check(Handle *h, int rc) {
  if (rc != INS2D_OK) mexErrMsgIdAndTxt("ins2d:status", "%s", ins2d_last_error(h->ctx));
}

// calls options' uBC/vBC (globals uBC vBC in the reference, main.m:37)
std::vector<double> call_bc(const char *fn, const std::vector<double> &x, const std::vector<double> &y, double t,
                            const mxArray *options) {
  mxArray *in[5];
  in[0] = mxCreateString(fn);
  in[1] = mxCreateDoubleMatrix(x.size(), 1, mxREAL);
  std::memcpy(mxGetPr(in[1]), x.data(), x.size() * sizeof(double));
  in[2] = mxCreateDoubleMatrix(y.size(), 1, mxREAL);
  std::memcpy(mxGetPr(in[2]), y.data(), y.size() * sizeof(double));
  in[3] = mxCreateDoubleScalar(t);
  in[4] = const_cast<mxArray *>(options);
  mxArray *out = nullptr;
  mexCallMATLAB(1, &out, 5, in, "feval");
  std::vector<double> r(mxGetPr(out), mxGetPr(out) + mxGetNumberOfElements(out));
  mxDestroyArray(out);
  for (int k = 0; k < 4; ++k) mxDestroyArray(in[k]);
  return r;
}

int sampler(void *user, double t, ins2d_ctx *ctx) {
  Handle *h = (Handle *)user;
  const mxArray *grid = mxGetField(h->options, 0, "grid");
  auto vec = [&](const char *name) {
    const mxArray *a = mxGetField(grid, 0, name);
    return std::vector<double>(mxGetPr(a), mxGetPr(a) + mxGetNumberOfElements(a));
  };
  std::vector<double> x = vec("x"), y = vec("y"), xp = vec("xp"), yp = vec("yp"), xin = vec("xin"), yin = vec("yin");
  std::vector<double> x1{x.front()}, xN{x.back()}, y1{y.front()}, yN{y.back()};
  char ub[64], vb[64];
  mxGetString(mxGetField(mxGetField(h->options, 0, "case"), 0, "uBC_name"), ub, sizeof ub);
  mxGetString(mxGetField(mxGetField(h->options, 0, "case"), 0, "vBC_name"), vb, sizeof vb);
  auto uLo = call_bc(ub, x, y1, t, h->options), uUp = call_bc(ub, x, yN, t, h->options);
  auto uLo_i = call_bc(ub, xin, y1, t, h->options), uUp_i = call_bc(ub, xin, yN, t, h->options);
  auto uLe_i = call_bc(ub, x1, yp, t, h->options), uRi_i = call_bc(ub, xN, yp, t, h->options);
  auto vLe = call_bc(vb, x1, y, t, h->options), vRi = call_bc(vb, xN, y, t, h->options);
  auto vLo_i = call_bc(vb, xp, y1, t, h->options), vUp_i = call_bc(vb, xp, yN, t, h->options);
  auto vLe_i = call_bc(vb, x1, yin, t, h->options), vRi_i = call_bc(vb, xN, yin, t, h->options);
  ins2d_bc_values v{};
  v.uLo = uLo.data(); v.uUp = uUp.data(); v.uLo_i = uLo_i.data(); v.uUp_i = uUp_i.data();
  v.uLe_i = uLe_i.data(); v.uRi_i = uRi_i.data(); v.vLe = vLe.data(); v.vRi = vRi.data();
  v.vLo_i = vLo_i.data(); v.vUp_i = vUp_i.data(); v.vLe_i = vLe_i.data(); v.vRi_i = vRi_i.data();
  return ins2d_set_bc_values(ctx, t, &v);
}

Handle *get_handle(const mxArray *a) {
  if (!mxIsUint64(a)) mexErrMsgIdAndTxt("ins2d:handle", "invalid handle");
  return (Handle *)(uintptr_t)(*(uint64_t *)mxGetData(a));
}

mxArray *col(const double *p, size_t n) {
  mxArray *m = mxCreateDoubleMatrix(n, 1, mxREAL);
  std::memcpy(mxGetPr(m), p, n * sizeof(double));
  return m;
}

}  // namespace

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  if (nrhs < 1 || !mxIsChar(prhs[0])) mexErrMsgIdAndTxt("ins2d:args", "first argument: command string");
  char cmd[48];
  mxGetString(prhs[0], cmd, sizeof cmd);
  if (!strcmp(cmd, "create")) {
    const mxArray *o = prhs[1];
    const mxArray *grid = mxGetField(o, 0, "grid");
    const mxArray *x = mxGetField(grid, 0, "x"), *y = mxGetField(grid, 0, "y");
    ins2d_grid_desc g{(int32_t)mxGetNumberOfElements(x) - 1, (int32_t)mxGetNumberOfElements(y) - 1, mxGetPr(x),
                      mxGetPr(y)};
    const mxArray *bc = mxGetField(o, 0, "BC");
    ins2d_bc_desc b{bc_code(bc, "u", "left"), bc_code(bc, "u", "right"), bc_code(bc, "u", "low"),
                    bc_code(bc, "u", "up"),   bc_code(bc, "v", "left"), bc_code(bc, "v", "right"),
                    bc_code(bc, "v", "low"),  bc_code(bc, "v", "up"),   (int32_t)field_d(o, "BC", "BC_unsteady", 0)};
    ins2d_opts op{};
    op.Re = field_d(o, "fluid", "Re", 1.0);
    op.poisson = (int32_t)field_d(o, "solversettings", "poisson", 4);
    op.CG_acc = field_d(o, "solversettings", "CG_acc", 1e-8);
    op.CG_maxit = (int32_t)field_d(o, "solversettings", "CG_maxit", 1000);
    op.p_add_solve = (int32_t)field_d(o, "solversettings", "p_add_solve", 1);
    op.rk_stages = 0;  // RK44 unless the caller passes a tableau in options.time.{A,b,c}
    const mxArray *tm = mxGetField(o, 0, "time");
    const mxArray *A = tm ? mxGetField(tm, 0, "A_RK") : nullptr;
    if (A) {
      int s = (int)mxGetM(A);
      op.rk_stages = s;
      for (int i = 0; i < s; ++i)
        for (int j = 0; j < s; ++j) op.rk_A[i * s + j] = mxGetPr(A)[i + j * s];  // column-major
      for (int i = 0; i < s; ++i) {
        op.rk_b[i] = mxGetPr(mxGetField(tm, 0, "b_RK"))[i];
        op.rk_c[i] = mxGetPr(mxGetField(tm, 0, "c_RK"))[i];
      }
    }
    Handle *h = new Handle();
    int rc = ins2d_ctx_create(&g, &b, &op, &h->ctx);
    if (rc != INS2D_OK) {
      std::string msg = ins2d_last_error(h->ctx);
      ins2d_ctx_destroy(h->ctx);
      delete h;
      mexErrMsgIdAndTxt("ins2d:create", "%s", msg.c_str());
    }
    h->options = mxDuplicateArray(o);
    mexMakeArrayPersistent(h->options);
    if (b.bc_unsteady) ins2d_set_bc_sampler(h->ctx, sampler, h);
    check(h, sampler(h, 0.0, h->ctx));
    plhs[0] = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
    *(uint64_t *)mxGetData(plhs[0]) = (uint64_t)(uintptr_t)h;
    return;
  }
  Handle *h = get_handle(prhs[1]);
  ins2d_sizes sz;
  ins2d_get_sizes(h->ctx, &sz);
  if (!strcmp(cmd, "destroy")) {
    ins2d_ctx_destroy(h->ctx);
    if (h->net) ins2d_cnn_destroy(h->net);
    mxDestroyArray(h->options);
    delete h;
  } else if (!strcmp(cmd, "learned_train")) {
    if (nrhs < 6) mexErrMsgIdAndTxt("ins2d:args", "learned_train: h, V, p, t, dt[, record_steps, train_steps, mode]");
    const int rec = nrhs > 6 ? (int)mxGetScalar(prhs[6]) : 24;
    const int steps = nrhs > 7 ? (int)mxGetScalar(prhs[7]) : 300;
    char mode[16] = "guess";
    if (nrhs > 8 && mxIsChar(prhs[8])) mxGetString(prhs[8], mode, sizeof mode);
    if (!h->net) {
      int32_t dev = 0;
      const mxArray *dv = mxGetField(h->options, 0, "device");
      if (dv && mxIsNumeric(dv)) dev = (int32_t)mxGetScalar(dv);
      if (ins2d_cnn_create(dev, 0, &h->net) != INS2D_OK) mexErrMsgIdAndTxt("ins2d:cnn", "cnn_create failed");
    }
    double l0 = 0.0, l1 = 0.0;
    check(h, ins2d_learned_train(h->ctx, h->net, mxGetPr(prhs[2]), mxGetPr(prhs[3]), mxGetScalar(prhs[4]),
                                 mxGetScalar(prhs[5]), rec, 4 * rec + 8, steps, 4, 2e-3f, 4, 0, INS2D_MEM_HOST, &l0,
                                 &l1));
    check(h, ins2d_set_learned_guess(h->ctx, h->net));
    check(h, ins2d_set_learned_mode(h->ctx, strcmp(mode, "precond") ? INS2D_LEARNED_GUESS : INS2D_LEARNED_PRECOND));
    plhs[0] = mxCreateDoubleScalar(l0);
    if (nlhs > 1) plhs[1] = mxCreateDoubleScalar(l1);
  } else if (!strcmp(cmd, "learned_detach")) {
    check(h, ins2d_set_learned_guess(h->ctx, nullptr));
  } else if (!strcmp(cmd, "F")) {
    std::vector<double> F(sz.NV);
    double maxres = 0;
    const double *C = (nrhs > 3 && !mxIsEmpty(prhs[3])) ? mxGetPr(prhs[3]) : nullptr;
    int nop = nrhs > 6 ? (int)mxGetScalar(prhs[6]) : 0;
    check(h, ins2d_F(h->ctx, mxGetPr(prhs[2]), C, nop ? nullptr : mxGetPr(prhs[4]), mxGetScalar(prhs[5]), nop,
                     F.data(), &maxres, INS2D_MEM_HOST));
    plhs[0] = mxCreateDoubleScalar(maxres);
    if (nlhs > 1) plhs[1] = col(F.data(), F.size());
  } else if (!strcmp(cmd, "pressure_poisson")) {
    std::vector<double> dp(sz.Np);
    ins2d_solve_stats st{};
    check(h, ins2d_pressure_poisson(h->ctx, mxGetPr(prhs[2]), dp.data(), &st, INS2D_MEM_HOST));
    plhs[0] = col(dp.data(), dp.size());
    if (nlhs > 1) plhs[1] = mxCreateDoubleScalar(st.iters);
    if (nlhs > 2) plhs[2] = mxCreateDoubleScalar(st.norm1);
    if (nlhs > 3) plhs[3] = mxCreateDoubleScalar(st.norm2);
  } else if (!strcmp(cmd, "pressure_additional_solve")) {
    std::vector<double> p(mxGetPr(prhs[3]), mxGetPr(prhs[3]) + sz.Np);
    check(h, ins2d_pressure_additional_solve(h->ctx, mxGetPr(prhs[2]), p.data(), mxGetScalar(prhs[4]), nullptr,
                                             INS2D_MEM_HOST));
    plhs[0] = col(p.data(), p.size());
  } else if (!strcmp(cmd, "time_ERK")) {
    std::vector<double> V(mxGetPr(prhs[2]), mxGetPr(prhs[2]) + sz.NV);
    std::vector<double> p(mxGetPr(prhs[3]), mxGetPr(prhs[3]) + sz.Np);
    check(h, ins2d_erk_step(h->ctx, V.data(), p.data(), mxGetScalar(prhs[4]), mxGetScalar(prhs[5]), nullptr,
                            INS2D_MEM_HOST));
    plhs[0] = col(V.data(), V.size());
    if (nlhs > 1) plhs[1] = col(p.data(), p.size());
  } else if (!strcmp(cmd, "check_conservation")) {
    double out[4];
    check(h, ins2d_conservation(h->ctx, mxGetPr(prhs[2]), mxGetScalar(prhs[3]), out, INS2D_MEM_HOST));
    for (int k = 0; k < 4 && k < (nlhs > 0 ? nlhs : 1); ++k) plhs[k] = mxCreateDoubleScalar(out[k]);
  } else {
    mexErrMsgIdAndTxt("ins2d:args", "unknown command %s", cmd);
  }
}
