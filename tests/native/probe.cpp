// Test-only probe: exposes the host-side operator tables of setup.cpp to the
// CPU tests (no CUDA), so the derivation can be checked against the oracle's
// assembled sparse matrices.
#include <cstring>
#include <string>

#include "setup.hpp"

using namespace ins2d;

static std::string g_err;

extern "C" const char *probe_error() { return g_err.c_str(); }

extern "C" void *probe_build(int Nx, int Ny, const double *x, const double *y, const int *bc, double Re) {
  HostOps *H = new HostOps();
  try {
    build_host_ops(*H, Nx, Ny, x, y, bc, Re);
  } catch (const std::exception &e) {
    g_err = e.what();
    delete H;
    return nullptr;
  }
  return H;
}

extern "C" void probe_free(void *h) { delete (HostOps *)h; }

extern "C" int probe_sizes(void *h, int *out) {
  HostOps *H = (HostOps *)h;
  out[0] = H->Nux; out[1] = H->Nuy; out[2] = H->Nvx; out[3] = H->Nvy; out[4] = H->Npx; out[5] = H->Npy;
  return 0;
}

extern "C" int probe_table(void *h, const char *name, int *nrows, int *ncols, const int **col, const double **w,
                           const double **b1, const double **b2) {
  HostOps *H = (HostOps *)h;
  const Table *t = nullptr;
  struct { const char *n; const Table *t; } all[] = {
      {"AUX", &H->AUX}, {"SUX", &H->SUX}, {"AUY", &H->AUY}, {"SUY", &H->SUY}, {"IVX", &H->IVX}, {"IVY", &H->IVY},
      {"MX", &H->MX},   {"MXT", &H->MXT}, {"AVX", &H->AVX}, {"SVX", &H->SVX}, {"AVY", &H->AVY}, {"SVY", &H->SVY},
      {"IUX", &H->IUX}, {"IUY", &H->IUY}, {"MY", &H->MY},   {"MYT", &H->MYT}, {"TX", &H->TX},   {"TY", &H->TY}};
  for (auto &a : all)
    if (std::strcmp(a.n, name) == 0) t = a.t;
  if (!t) return 1;
  *nrows = t->nrows;
  *ncols = t->ncols;
  *col = t->col.data();
  *w = t->w.data();
  *b1 = t->b1.data();
  *b2 = t->b2.data();
  return 0;
}

// --- multigrid hierarchy (mg_host.cpp) ---------------------------------------
#include <vector>

#include "mg_host.hpp"

struct ProbeMg {
  std::vector<MgHostLevel> lv;
  std::vector<double> pinv;
};

extern "C" void *probe_mg_build(void *h) {
  ProbeMg *m = new ProbeMg();
  try {
    m->lv = mg_build_levels(*(HostOps *)h);
    const MgHostLevel &c = m->lv.back();
    m->pinv = mg_pinv(mg_dense(c), c.nx * c.ny);
  } catch (const std::exception &e) {
    g_err = e.what();
    delete m;
    return nullptr;
  }
  return m;
}
extern "C" void probe_mg_free(void *m) { delete (ProbeMg *)m; }
extern "C" int probe_mg_nlev(void *m) { return (int)((ProbeMg *)m)->lv.size(); }
// dims = {nx, ny, perx, pery, cx, cy}; vec: 0..7 = xm, x0, xp, hx, ym, y0, yp, hy
extern "C" int probe_mg_level(void *m, int l, int *dims, int which, const double **v) {
  const MgHostLevel &L = ((ProbeMg *)m)->lv.at(l);
  dims[0] = L.nx; dims[1] = L.ny; dims[2] = L.perx; dims[3] = L.pery; dims[4] = L.cx; dims[5] = L.cy;
  const std::vector<double> *all[8] = {&L.xm, &L.x0, &L.xp, &L.hx, &L.ym, &L.y0, &L.yp, &L.hy};
  if (which < 0 || which > 7) return 1;
  *v = all[which]->data();
  return 0;
}
extern "C" const double *probe_mg_pinv(void *m) { return ((ProbeMg *)m)->pinv.data(); }

// generalized eigen-decomposition of TX (dir 0) or TY (dir 1) against the
// cell widths hx / hy (the fast-diagonalization preconditioner's factors)
#include "fdm_host.hpp"
extern "C" int probe_fdm(void *h, int dir, double *Q, double *lam) {
  HostOps *H = (HostOps *)h;
  try {
    FdmHost1D F = dir == 0 ? fdm_1d(H->TX, H->hx) : fdm_1d(H->TY, H->hy);
    std::memcpy(Q, F.Q.data(), F.Q.size() * sizeof(double));
    std::memcpy(lam, F.lam.data(), F.lam.size() * sizeof(double));
    return F.n;
  } catch (const std::exception &e) {
    g_err = e.what();
    return -1;
  }
}
