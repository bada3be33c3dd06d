// Host-side operator derivation; see setup.hpp.  Each function cites the
// reference file it restates (bsanderse/INS2D, MATLAB).
#include "setup.hpp"

#include <cmath>
#include <sstream>
#include <stdexcept>

namespace ins2d {

namespace {
[[noreturn]] void fail(const std::string &msg) { throw std::runtime_error(msg); }
const char *bcname(int t) {
  switch (t) {
    case BC_DIR: return "dir";
    case BC_PRES: return "pres";
    case BC_PER: return "per";
    case BC_SYM: return "sym";
  }
  return "?";
}
std::vector<double> ones(int n) { return std::vector<double>((size_t)n, 1.0); }
std::vector<double> slice(const std::vector<double> &v, int a, int b) {  // [a,b)
  return std::vector<double>(v.begin() + a, v.begin() + b);
}
std::vector<double> cat(std::initializer_list<std::vector<double>> parts) {
  std::vector<double> r;
  for (auto &p : parts) r.insert(r.end(), p.begin(), p.end());
  return r;
}
}  // namespace

void Sp::set(int i, int j, double v) {
  if (i < 0 || i >= m || j < 0 || j >= n) fail("Sp::set out of range");
  if (v == 0.0)
    rows[i].erase(j);
  else
    rows[i][j] = v;
}

Sp Sp::eye(int n) {
  Sp A(n, n);
  for (int i = 0; i < n; ++i) A.rows[i][i] = 1.0;
  return A;
}

Sp Sp::diag(const std::vector<double> &d) {
  Sp A((int)d.size(), (int)d.size());
  for (size_t i = 0; i < d.size(); ++i)
    if (d[i] != 0.0) A.rows[i][(int)i] = d[i];
  return A;
}

Sp mul(const Sp &A, const Sp &B) {
  if (A.n != B.m) fail("mul: inner dimensions differ");
  Sp C(A.m, B.n);
  for (int i = 0; i < A.m; ++i) {
    auto &ci = C.rows[i];
    for (auto &ka : A.rows[i])
      for (auto &jb : B.rows[ka.first]) ci[jb.first] += ka.second * jb.second;
    for (auto it = ci.begin(); it != ci.end();) it = (it->second == 0.0) ? ci.erase(it) : std::next(it);
  }
  return C;
}

Sp sub(const Sp &A, const Sp &B) {
  if (A.m != B.m || A.n != B.n) fail("sub: dimensions differ");
  Sp C = A;
  for (int i = 0; i < B.m; ++i) {
    auto &ci = C.rows[i];
    for (auto &jb : B.rows[i]) ci[jb.first] -= jb.second;
    for (auto it = ci.begin(); it != ci.end();) it = (it->second == 0.0) ? ci.erase(it) : std::next(it);
  }
  return C;
}

Sp transpose(const Sp &A) {
  Sp T(A.n, A.m);
  for (int i = 0; i < A.m; ++i)
    for (auto &jv : A.rows[i]) T.rows[jv.first][i] = jv.second;
  return T;
}

Sp scale_rows(const Sp &A, int row, double s) {
  Sp C = A;
  for (auto &jv : C.rows[row]) jv.second *= s;
  return C;
}

Sp spdiags(const std::vector<std::vector<double>> &Bcols, const std::vector<int> &d, int m, int n) {
  Sp A(m, n);
  for (size_t k = 0; k < d.size(); ++k) {
    int dk = d[k];
    int lo = std::max(1, 1 - dk), hi = std::min(m, n - dk);
    for (int i = lo; i <= hi; ++i) {  // 1-based row i, column i+dk
      int idx = i + (m >= n ? dk : 0);
      if (idx < 1 || idx > (int)Bcols[k].size()) fail("spdiags: diagonal data too short");
      double v = Bcols[k][idx - 1];
      if (v != 0.0) A.rows[i - 1][i + dk - 1] += v;
    }
  }
  return A;
}

std::vector<double> matvec(const Sp &A, const std::vector<double> &x) {
  if ((int)x.size() != A.n) fail("matvec: size mismatch");
  std::vector<double> y((size_t)A.m, 0.0);
  for (int i = 0; i < A.m; ++i) {
    double s = 0.0;
    for (auto &jv : A.rows[i]) s += jv.second * x[jv.first];
    y[i] = s;
  }
  return y;
}

// u = B1D*u_in + Btemp*ybc with Btemp = Bb*(Bbc*Bb)^-1 (BC_general.m:124-125).
static BC1 finish_bc(const Sp &Bin, const Sp &Bb, const Sp &Bbc, std::vector<double> y1,
                     std::vector<double> y2, int Nb) {
  Sp small = mul(Bbc, Bb);  // Nb x Nb
  double a[2][2] = {{0, 0}, {0, 0}};
  for (int i = 0; i < Nb; ++i)
    for (auto &jv : small.rows[i]) a[i][jv.first] = jv.second;
  Sp inv(Nb, Nb);
  if (Nb == 1) {
    if (a[0][0] == 0.0) fail("singular boundary system");
    inv.set(0, 0, 1.0 / a[0][0]);
  } else {
    double det = a[0][0] * a[1][1] - a[0][1] * a[1][0];
    if (det == 0.0) fail("singular boundary system");
    inv.set(0, 0, a[1][1] / det);
    inv.set(0, 1, -a[0][1] / det);
    inv.set(1, 0, -a[1][0] / det);
    inv.set(1, 1, a[0][0] / det);
  }
  BC1 r;
  r.Btemp = mul(Bb, inv);
  r.B1D = sub(Bin, mul(r.Btemp, mul(Bbc, Bin)));
  r.ybc1 = std::move(y1);
  r.ybc2 = std::move(y2);
  return r;
}

static BC1 no_boundary(int Nt) {
  BC1 r;
  r.B1D = Sp::eye(Nt);
  r.Btemp = Sp(Nt, 2);
  r.ybc1 = {0.0, 0.0};
  r.ybc2 = {0.0, 0.0};
  return r;
}

// spatial/boundaryconditions/proposed/BC_general.m:1-130 (grid lines)
BC1 bc_general(int Nt, int Nin, int Nb, int t1, int t2, double h1, double h2) {
  if (Nt != Nin + Nb) fail("BC_general: inner + boundary points != total points");
  if (Nb == 0) return no_boundary(Nt);
  Sp Bbc(Nb, Nt), Bb(Nt, Nb), Bin;
  std::vector<double> y1((size_t)Nb, 0.0), y2((size_t)Nb, 0.0);
  if (Nb == 2) {
    Bin = spdiags({ones(Nt)}, {-1}, Nt, Nin);
    Bb.set(0, 0, 1);
    Bb.set(Nt - 1, Nb - 1, 1);
    switch (t1) {
      case BC_DIR: Bbc.set(0, 0, 1); y1[0] = 1; break;
      case BC_PRES: Bbc.set(0, 0, -1); Bbc.set(0, 1, 1); y1[0] = 2 * h1; break;
      case BC_PER:
        Bbc.set(0, 0, -1); Bbc.set(0, Nt - 2, 1); Bbc.set(Nb - 1, 1, -1); Bbc.set(Nb - 1, Nt - 1, 1);
        break;
      default: fail(std::string("BC_general: not implemented: ") + bcname(t1));
    }
    switch (t2) {
      case BC_DIR: Bbc.set(Nb - 1, Nt - 1, 1); y2[1] = 1; break;
      case BC_PRES: Bbc.set(Nb - 1, Nt - 2, -1); Bbc.set(Nb - 1, Nt - 1, 1); y2[1] = 2 * h2; break;
      case BC_PER:
        Bbc.set(0, 0, -1); Bbc.set(0, Nt - 2, 1); Bbc.set(Nb - 1, 1, -1); Bbc.set(Nb - 1, Nt - 1, 1);
        break;
      default: fail(std::string("BC_general: not implemented: ") + bcname(t2));
    }
  } else if (Nb == 1) {
    int diagpos = -1;
    switch (t1) {
      case BC_DIR: Bbc.set(0, 0, 1); y1[0] = 1; Bb.set(0, 0, 1); break;
      case BC_PRES: diagpos = 0; break;
      case BC_PER: diagpos = 0; Bbc.set(0, 0, -1); Bbc.set(0, Nt - 1, 1); Bb.set(Nt - 1, 0, 1); break;
      default: fail(std::string("BC_general: not implemented: ") + bcname(t1));
    }
    switch (t2) {
      case BC_DIR: Bbc.set(Nb - 1, Nt - 1, 1); y2[0] = 1; Bb.set(Nt - 1, Nb - 1, 1); break;
      case BC_PRES: break;
      case BC_PER: diagpos = 0; Bbc.set(0, 0, -1); Bbc.set(0, Nt - 1, 1); Bb.set(Nt - 1, 0, 1); break;
      default: fail(std::string("BC_general: not implemented: ") + bcname(t2));
    }
    Bin = spdiags({ones(Nt)}, {diagpos}, Nt, Nin);
  } else {
    fail("BC_general: Nb must be 0, 1 or 2");
  }
  return finish_bc(Bin, Bb, Bbc, y1, y2, Nb);
}

// spatial/boundaryconditions/proposed/BC_general_stag.m:1-138 (staggered
// lines); with Nb=2 this is also BC_diff_stag.m (zeroth-order mirror).
BC1 bc_general_stag(int Nt, int Nin, int Nb, int t1, int t2, double h1, double h2) {
  if (Nt != Nin + Nb) fail("BC_general_stag: inner + boundary points != total points");
  if (Nb == 0) return no_boundary(Nt);
  Sp Bbc(Nb, Nt), Bb(Nt, Nb), Bin;
  std::vector<double> y1((size_t)Nb, 0.0), y2((size_t)Nb, 0.0);
  if (Nb == 2) {
    Bin = spdiags({ones(Nt)}, {-1}, Nt, Nin);
    Bb.set(0, 0, 1);
    Bb.set(Nt - 1, Nb - 1, 1);
    switch (t1) {
      case BC_DIR: Bbc.set(0, 0, 0.5); Bbc.set(0, 1, 0.5); y1[0] = 1; break;
      case BC_SYM: Bbc.set(0, 0, -1); Bbc.set(0, 1, 1); y1[0] = h1; break;
      case BC_PER:
        Bbc.set(0, 0, -1); Bbc.set(0, Nt - 2, 1); Bbc.set(1, 1, -1); Bbc.set(1, Nt - 1, 1);
        break;
      default: fail(std::string("BC_general_stag: not implemented: ") + bcname(t1));
    }
    switch (t2) {
      case BC_DIR: Bbc.set(Nb - 1, Nt - 2, 0.5); Bbc.set(Nb - 1, Nt - 1, 0.5); y2[1] = 1; break;
      case BC_SYM: Bbc.set(1, Nt - 2, -1); Bbc.set(1, Nt - 1, 1); y2[1] = h2; break;
      case BC_PER:
        Bbc.set(0, 0, -1); Bbc.set(0, Nt - 2, 1); Bbc.set(1, 1, -1); Bbc.set(1, Nt - 1, 1);
        break;
      default: fail(std::string("BC_general_stag: not implemented: ") + bcname(t2));
    }
  } else if (Nb == 1) {
    switch (t1) {
      case BC_DIR: Bbc.set(0, 0, 0.5); Bbc.set(0, 1, 0.5); y1[0] = 1; Bb.set(0, 0, 1); break;
      case BC_SYM: Bbc.set(0, 0, -1); Bbc.set(0, 1, 1); y1[0] = h1; break;
      case BC_PER: Bbc.set(0, 0, -1); Bbc.set(0, Nt - 1, 1); Bb.set(0, 0, 1); break;
      default: fail(std::string("BC_general_stag: not implemented: ") + bcname(t1));
    }
    switch (t2) {
      case BC_DIR: Bbc.set(0, Nt - 2, 0.5); Bbc.set(0, Nt - 1, 0.5); y2[0] = 1; Bb.set(Nt - 1, 0, 1); break;
      case BC_SYM: Bbc.set(0, Nt - 2, -1); Bbc.set(0, Nt - 1, 1); y2[0] = h2; break;
      case BC_PER: Bbc.set(0, 0, -1); Bbc.set(0, Nt - 1, 1); Bb.set(0, 0, 1); break;
      default: fail(std::string("BC_general_stag: not implemented: ") + bcname(t2));
    }
    Bin = spdiags({ones(Nt)}, {-1}, Nt, Nin);
  } else {
    fail("BC_general_stag: Nb must be 0, 1 or 2");
  }
  return finish_bc(Bin, Bb, Bbc, y1, y2, Nb);
}

Table make_table(const Sp &T, const std::string &name) {
  Table t;
  t.T = T;
  t.nrows = T.m;
  t.ncols = T.n;
  t.col.assign((size_t)T.m * kTab, 0);
  t.w.assign((size_t)T.m * kTab, 0.0);
  t.b1.assign((size_t)T.m, 0.0);
  t.b2.assign((size_t)T.m, 0.0);
  for (int i = 0; i < T.m; ++i) {
    if ((int)T.rows[i].size() > kTab) {
      std::ostringstream os;
      os << "operator " << name << " row " << i << " has " << T.rows[i].size()
         << " entries (grid too small for this boundary combination)";
      fail(os.str());
    }
    int k = 0, first = T.rows[i].empty() ? 0 : T.rows[i].begin()->first;
    for (auto &jv : T.rows[i]) {
      t.col[(size_t)i * kTab + k] = jv.first;
      t.w[(size_t)i * kTab + k] = jv.second;
      ++k;
    }
    for (; k < kTab; ++k) t.col[(size_t)i * kTab + k] = first;  // zero weight
  }
  return t;
}

Table make_table(const Sp &Pre, const BC1 &bc, const std::string &name) {
  Table t = make_table(mul(Pre, bc.B1D), name);
  t.b1 = matvec(Pre, matvec(bc.Btemp, bc.ybc1));
  t.b2 = matvec(Pre, matvec(bc.Btemp, bc.ybc2));
  return t;
}

Regular find_regular(Table &T) {
  // Rows r whose entries sit at columns (r+s) and (r+s+1) taken modulo the
  // column count (periodic wrap rows qualify), without boundary terms.
  Regular R;
  const int n = T.nrows, nc = T.ncols;
  T.rw0.assign((size_t)n, 0.0);
  T.rw1.assign((size_t)n, 0.0);
  if (n == 0 || nc < 3) return R;
  auto md = [nc](int c) { return ((c % nc) + nc) % nc; };
  auto is_reg = [&](int r, int s) {
    if (T.b1[r] != 0.0 || T.b2[r] != 0.0) return false;
    if (T.T.rows[r].empty()) return false;
    for (auto &jv : T.T.rows[r])
      if (jv.first != md(r + s) && jv.first != md(r + s + 1)) return false;
    return true;
  };
  const int mid = n / 2;
  if (T.T.rows[mid].empty()) return R;
  const int s = T.T.rows[mid].begin()->first - mid;
  if (!is_reg(mid, s)) return R;
  int lo = mid, hi = mid + 1;
  while (lo > 0 && is_reg(lo - 1, s)) --lo;
  while (hi < n && is_reg(hi, s)) ++hi;
  R.s = s;
  R.lo = lo;
  R.hi = hi;
  R.two = 0;
  for (int r = lo; r < hi; ++r)
    for (auto &jv : T.T.rows[r]) {
      if (jv.first == md(r + s + 1)) {
        R.two = 1;
        T.rw1[r] = jv.second;
      } else {
        T.rw0[r] = jv.second;
      }
    }
  return R;
}

Regular intersect(const Regular &a, const Regular &b) {
  Regular r = a;
  if (a.s != b.s) {
    r.lo = r.hi = 0;
    return r;
  }
  r.lo = std::max(a.lo, b.lo);
  r.hi = std::min(a.hi, b.hi);
  r.two = a.two | b.two;
  if (r.hi < r.lo) r.hi = r.lo;
  return r;
}

void align_pair(Table &A, Table &B, const std::string &name) {
  if (A.nrows != B.nrows) fail("align_pair: row counts differ for " + name);
  for (int i = 0; i < A.nrows; ++i) {
    std::map<int, std::pair<double, double>> u;
    for (auto &jv : A.T.rows[i]) u[jv.first].first = jv.second;
    for (auto &jv : B.T.rows[i]) u[jv.first].second = jv.second;
    if ((int)u.size() > kTab) fail("align_pair: too many columns in a row of " + name);
    int k = 0, first = u.empty() ? 0 : u.begin()->first;
    for (auto &e : u) {
      A.col[(size_t)i * kTab + k] = B.col[(size_t)i * kTab + k] = e.first;
      A.w[(size_t)i * kTab + k] = e.second.first;
      B.w[(size_t)i * kTab + k] = e.second.second;
      ++k;
    }
    for (; k < kTab; ++k) {
      A.col[(size_t)i * kTab + k] = B.col[(size_t)i * kTab + k] = first;
      A.w[(size_t)i * kTab + k] = B.w[(size_t)i * kTab + k] = 0.0;
    }
  }
}

static bool valid_pair(int a, int b, std::initializer_list<int> allowed) {
  bool oka = false, okb = false;
  for (int t : allowed) {
    oka |= (a == t);
    okb |= (b == t);
  }
  return oka && okb && ((a == BC_PER) == (b == BC_PER));
}

void build_host_ops(HostOps &H, int Nx, int Ny, const double *x, const double *y,
                    const int bc[8], double Re) {
  if (Nx < 2 || Ny < 2) fail("grid needs at least 2 cells per direction");
  for (int k = 0; k < 8; ++k) H.bc[k] = bc[k];
  const int uL = bc[0], uR = bc[1], uLo = bc[2], uUp = bc[3];
  const int vL = bc[4], vR = bc[5], vLo = bc[6], vUp = bc[7];
  // boundary_conditions.m:17-40
  if (!valid_pair(uL, uR, {BC_DIR, BC_PER, BC_PRES})) fail("wrong BC for u-left/u-right");
  if (!valid_pair(uLo, uUp, {BC_DIR, BC_PER, BC_SYM})) fail("wrong BC for u-low/u-up");
  if (!valid_pair(vL, vR, {BC_DIR, BC_PER, BC_SYM})) fail("wrong BC for v-left/v-right");
  if (!valid_pair(vLo, vUp, {BC_DIR, BC_PER, BC_PRES})) fail("wrong BC for v-low/v-up");
  H.Re = Re;
  H.Nx = Nx;
  H.Ny = Ny;
  H.x.assign(x, x + Nx + 1);
  H.y.assign(y, y + Ny + 1);
  // mesh_generation.m:17-39
  H.xp.resize(Nx); H.hx.resize(Nx); H.gx.assign(Nx + 1, 0.0);
  H.yp.resize(Ny); H.hy.resize(Ny); H.gy.assign(Ny + 1, 0.0);
  for (int i = 0; i < Nx; ++i) {
    H.xp[i] = (H.x[i] + H.x[i + 1]) / 2;
    H.hx[i] = H.x[i + 1] - H.x[i];
    if (!(H.hx[i] > 0)) fail("x must be strictly increasing");
  }
  for (int j = 0; j < Ny; ++j) {
    H.yp[j] = (H.y[j] + H.y[j + 1]) / 2;
    H.hy[j] = H.y[j + 1] - H.y[j];
    if (!(H.hy[j] > 0)) fail("y must be strictly increasing");
  }
  H.gx[0] = H.hx[0] / 2;
  for (int i = 1; i < Nx; ++i) H.gx[i] = (H.hx[i - 1] + H.hx[i]) / 2;
  H.gx[Nx] = H.hx[Nx - 1] / 2;
  H.gy[0] = H.hy[0] / 2;
  for (int j = 1; j < Ny; ++j) H.gy[j] = (H.hy[j - 1] + H.hy[j]) / 2;
  H.gy[Ny] = H.hy[Ny - 1] / 2;
  const auto &hx = H.hx, &hy = H.hy, &gx = H.gx, &gy = H.gy;

  // operator_mesh.m:25-104 counts
  int Nux_in = Nx + 1;
  if (uL == BC_DIR || uL == BC_SYM) --Nux_in;
  if (uR == BC_DIR || uR == BC_SYM) --Nux_in;
  if (uL == BC_PER && uR == BC_PER) --Nux_in;
  const int Nux_t = Nux_in + 2, Nuy_in = Ny, Nuy_t = Ny + 2;
  const int Nvx_in = Nx, Nvx_t = Nx + 2;
  int Nvy_in = Ny + 1;
  if (vLo == BC_DIR || vLo == BC_SYM) --Nvy_in;
  if (vUp == BC_DIR || vUp == BC_SYM) --Nvy_in;
  if (vLo == BC_PER && vUp == BC_PER) --Nvy_in;
  const int Nvy_t = Nvy_in + 2;
  H.Nux = Nux_in; H.Nuy = Nuy_in; H.Nvx = Nvx_in; H.Nvy = Nvy_in; H.Npx = Nx; H.Npy = Ny;

  // operator_mesh.m:173-249 (x) and 260-327 (y)
  H.gxd = gx;
  H.gxd[0] = hx[0];
  H.gxd[Nx] = hx[Nx - 1];
  int diagpos_x = 0;
  if (uL == BC_DIR && uR == BC_DIR) {
    H.xin = slice(H.x, 1, Nx); H.hxd = hx; H.gxi = slice(gx, 1, Nx); diagpos_x = 1;
  } else if (uL == BC_DIR && uR == BC_PRES) {
    H.xin = slice(H.x, 1, Nx + 1); H.hxd = cat({hx, {hx[Nx - 1]}}); H.gxi = slice(gx, 1, Nx + 1); diagpos_x = 1;
  } else if (uL == BC_PRES && uR == BC_DIR) {
    H.xin = slice(H.x, 0, Nx); H.hxd = cat({{hx[0]}, hx}); H.gxi = slice(gx, 0, Nx); diagpos_x = 0;
  } else if (uL == BC_PRES && uR == BC_PRES) {
    H.xin = H.x; H.hxd = cat({{hx[0]}, hx, {hx[Nx - 1]}}); H.gxi = gx; diagpos_x = 0;
  } else if (uL == BC_PER && uR == BC_PER) {
    H.xin = slice(H.x, 0, Nx);
    H.hxd = cat({{hx[Nx - 1]}, hx});
    H.gxi = cat({{gx[0] + gx[Nx]}, slice(gx, 1, Nx)});
    H.gxd[0] = (hx[0] + hx[Nx - 1]) / 2;
    H.gxd[Nx] = (hx[0] + hx[Nx - 1]) / 2;
    diagpos_x = 0;
  } else {
    fail("unsupported u-left/u-right combination");
  }
  H.gyd = gy;
  H.gyd[0] = hy[0];
  H.gyd[Ny] = hy[Ny - 1];
  int diagpos_y = 0;
  if (vLo == BC_DIR && vUp == BC_DIR) {
    H.yin = slice(H.y, 1, Ny); H.hyd = hy; H.gyi = slice(gy, 1, Ny); diagpos_y = 1;
  } else if (vLo == BC_DIR && vUp == BC_PRES) {
    H.yin = slice(H.y, 1, Ny + 1); H.hyd = cat({hy, {hy[Ny - 1]}}); H.gyi = slice(gy, 1, Ny + 1); diagpos_y = 1;
  } else if (vLo == BC_PRES && vUp == BC_DIR) {
    H.yin = slice(H.y, 0, Ny); H.hyd = cat({{hy[0]}, hy}); H.gyi = slice(gy, 0, Ny); diagpos_y = 0;
  } else if (vLo == BC_PRES && vUp == BC_PRES) {
    H.yin = H.y; H.hyd = cat({{hy[0]}, hy, {hy[Ny - 1]}}); H.gyi = gy; diagpos_y = 0;
  } else if (vLo == BC_PER && vUp == BC_PER) {
    H.yin = slice(H.y, 0, Ny);
    H.hyd = cat({{hy[Ny - 1]}, hy});
    H.gyi = cat({{gy[0] + gy[Ny]}, slice(gy, 1, Ny)});
    H.gyd[0] = (hy[0] + hy[Ny - 1]) / 2;
    H.gyd[Ny] = (hy[0] + hy[Ny - 1]) / 2;
    diagpos_y = 0;
  } else {
    fail("unsupported v-low/v-up combination");
  }
  const Sp Bvux = spdiags({ones(Nvx_t - 1)}, {diagpos_x}, Nux_in, Nvx_t - 1);
  const Sp Buvy = spdiags({ones(Nuy_t - 1)}, {diagpos_y}, Nvy_in, Nuy_t - 1);

  auto half2 = [](int n) { return std::vector<std::vector<double>>{std::vector<double>((size_t)n, 0.5),
                                                                    std::vector<double>((size_t)n, 0.5)}; };
  auto recip = [](const std::vector<double> &v) {
    std::vector<double> r(v.size());
    for (size_t i = 0; i < v.size(); ++i) r[i] = 1.0 / v[i];
    return r;
  };
  auto neg = [](std::vector<double> v) {
    for (auto &e : v) e = -e;
    return v;
  };
  const double hx0 = hx[0], hxN = hx[Nx - 1], hy0 = hy[0], hyN = hy[Ny - 1];

  // --- u-component --------------------------------------------------------
  const BC1 Bux = bc_general(Nux_t, Nux_in, 2, uL, uR, hx0, hxN);
  const BC1 Buy = bc_general_stag(Nuy_t, Nuy_in, 2, uLo, uUp, hy0, hyN);
  // Au_ux (operator_averaging.m:32-42)
  H.AUX = make_table(spdiags(half2(Nux_t), {0, 1}, Nux_t - 1, Nux_t), Bux, "Au_ux");
  // Su_ux (operator_convection_diffusion.m:132-142)
  {
    auto d = recip(H.hxd);
    H.SUX = make_table(spdiags({neg(d), d}, {0, 1}, Nux_t - 1, Nux_t), Bux, "Su_ux");
  }
  // Mx (operator_divergence.m:54-89)
  {
    Sp M1D = spdiags({neg(ones(Nux_t)), ones(Nux_t)}, {0, 1}, Nux_t - 1, Nux_t);
    int dp = 0;
    if (uR == BC_PRES && uL == BC_PRES) dp = 1;
    if (uR != BC_PRES && uL == BC_PRES) dp = 1;
    if (uR == BC_PRES && uL != BC_PRES) dp = 0;
    if (uR == BC_PER && uL == BC_PER) dp = 1;
    Sp BMx = spdiags({ones(Nx)}, {dp}, Nx, Nux_t - 1);
    H.MX = make_table(mul(BMx, M1D), Bux, "Mx");
    H.MXT = make_table(transpose(H.MX.T), "Gx");
  }
  // Au_uy (operator_averaging.m:45-55)
  H.AUY = make_table(spdiags(half2(Nuy_t), {0, 1}, Nuy_t - 1, Nuy_t), Buy, "Au_uy");
  // Su_uy with BC_diff_stag (operator_convection_diffusion.m:146-159)
  {
    auto d = recip(H.gyd);
    H.SUY = make_table(spdiags({neg(d), d}, {0, 1}, Nuy_t - 1, Nuy_t), Buy, "Su_uy");
  }
  // Iv_uy = kron(B1D_lu, Bvux*I1D*mat_hx2*B1D_lr) (operator_interpolation.m:237-271)
  {
    Sp I1D = spdiags(half2(Nvx_t), {0, 1}, Nvx_t - 1, Nvx_t);
    if (uR == BC_PRES) I1D = scale_rows(I1D, I1D.m - 1, 0.5);
    if (uL == BC_PRES) I1D = scale_rows(I1D, 0, 0.5);
    std::vector<double> h2 = (uL == BC_PER && uR == BC_PER) ? cat({{hxN}, hx, {hx0}}) : cat({{hx0}, hx, {hxN}});
    Sp Ir = mul(mul(Bvux, I1D), Sp::diag(h2));
    BC1 lr = bc_general_stag(Nvx_t, Nvx_in, 2, vL, vR, hx0, hxN);
    H.IVX = make_table(Ir, lr, "Iv_uy(x)");
    int Nb = Nuy_in + 1 - Nvy_in;
    BC1 lu = bc_general(Nuy_in + 1, Nvy_in, Nb, vLo, vUp, hy0, hyN);
    H.IVY = make_table(Sp::eye(Nuy_in + 1), lu, "Iv_uy(y)");
  }

  // --- v-component --------------------------------------------------------
  const BC1 Bvx = bc_general_stag(Nvx_t, Nvx_in, 2, vL, vR, hx0, hxN);
  const BC1 Bvy = bc_general(Nvy_t, Nvy_in, 2, vLo, vUp, hy0, hyN);
  H.AVX = make_table(spdiags(half2(Nvx_t), {0, 1}, Nvx_t - 1, Nvx_t), Bvx, "Av_vx");
  {
    auto d = recip(H.gxd);
    H.SVX = make_table(spdiags({neg(d), d}, {0, 1}, Nvx_t - 1, Nvx_t), Bvx, "Sv_vx");
  }
  H.AVY = make_table(spdiags(half2(Nvy_t), {0, 1}, Nvy_t - 1, Nvy_t), Bvy, "Av_vy");
  {
    auto d = recip(H.hyd);
    H.SVY = make_table(spdiags({neg(d), d}, {0, 1}, Nvy_t - 1, Nvy_t), Bvy, "Sv_vy");
  }
  {
    Sp M1D = spdiags({neg(ones(Nvy_t)), ones(Nvy_t)}, {0, 1}, Nvy_t - 1, Nvy_t);
    int dp = 0;
    if (vUp == BC_PRES && vLo == BC_PRES) dp = 1;
    if (vUp != BC_PRES && vLo == BC_PRES) dp = 1;
    if (vUp == BC_PRES && vLo != BC_PRES) dp = 0;
    if (vUp == BC_PER && vLo == BC_PER) dp = 1;
    Sp BMy = spdiags({ones(Ny)}, {dp}, Ny, Nvy_t - 1);
    H.MY = make_table(mul(BMy, M1D), Bvy, "My");
    H.MYT = make_table(transpose(H.MY.T), "Gy");
  }
  // Iu_vx = kron(Buvy*I1D*mat_hy2*B1D_lu, B1D_lr) (operator_interpolation.m:277-308)
  {
    Sp I1D = spdiags(half2(Nuy_t), {0, 1}, Nuy_t - 1, Nuy_t);
    if (vUp == BC_PRES) I1D = scale_rows(I1D, I1D.m - 1, 0.5);
    if (vLo == BC_PRES) I1D = scale_rows(I1D, 0, 0.5);
    std::vector<double> h2 = (vLo == BC_PER && vUp == BC_PER) ? cat({{hyN}, hy, {hy0}}) : cat({{hy0}, hy, {hyN}});
    Sp Ir = mul(mul(Buvy, I1D), Sp::diag(h2));
    BC1 lu = bc_general_stag(Nuy_t, Nuy_in, 2, uLo, uUp, hy0, hyN);
    H.IUY = make_table(Ir, lu, "Iu_vx(y)");
    int Nb = Nvx_in + 1 - Nux_in;
    BC1 lr = bc_general(Nvx_in + 1, Nux_in, Nb, uL, uR, hx0, hxN);
    H.IUX = make_table(Sp::eye(Nvx_in + 1), lr, "Iu_vx(x)");
  }

  // shared column sets for the averaging/difference pairs of one field
  align_pair(H.AUX, H.SUX, "Au_ux/Su_ux");
  align_pair(H.AUY, H.SUY, "Au_uy/Su_uy");
  align_pair(H.AVX, H.SVX, "Av_vx/Sv_vx");
  align_pair(H.AVY, H.SVY, "Av_vy/Sv_vy");
  H.rAUX = intersect(find_regular(H.AUX), find_regular(H.SUX));
  H.rAUY = intersect(find_regular(H.AUY), find_regular(H.SUY));
  H.rAVX = intersect(find_regular(H.AVX), find_regular(H.SVX));
  H.rAVY = intersect(find_regular(H.AVY), find_regular(H.SVY));
  H.rIVX = find_regular(H.IVX);
  H.rIVY = find_regular(H.IVY);
  H.rIUX = find_regular(H.IUX);
  H.rIUY = find_regular(H.IUY);
  H.rMXT = find_regular(H.MXT);
  H.rMYT = find_regular(H.MYT);
  H.rMX = find_regular(H.MX);
  H.rMY = find_regular(H.MY);

  // --- Laplacian A = M*Om_inv*G (operator_divergence.m:208) -----------------
  H.TX = make_table(mul(mul(H.MX.T, Sp::diag(recip(H.gxi))), transpose(H.MX.T)), "A(x)");
  H.TY = make_table(mul(mul(H.MY.T, Sp::diag(recip(H.gyi))), transpose(H.MY.T)), "A(y)");
  H.TXd.assign(Nx, 0.0);
  H.TYd.assign(Ny, 0.0);
  for (int i = 0; i < Nx; ++i) {
    auto it = H.TX.T.rows[i].find(i);
    H.TXd[i] = it == H.TX.T.rows[i].end() ? 0.0 : it->second;
  }
  for (int j = 0; j < Ny; ++j) {
    auto it = H.TY.T.rows[j].find(j);
    H.TYd[j] = it == H.TY.T.rows[j].end() ? 0.0 : it->second;
  }

  // --- pressure BC patterns (set_bc_vectors.m:157-176) ---------------------
  H.pxl.assign(Nux_in, 0.0);
  H.pxr.assign(Nux_in, 0.0);
  if (uL == BC_PRES) H.pxl[0] = -1;
  if (uR == BC_PRES) H.pxr[Nux_in - 1] = 1;
  H.pyl.assign(Nvy_in, 0.0);
  H.pyu.assign(Nvy_in, 0.0);
  if (vLo == BC_PRES) H.pyl[0] = -1;
  if (vUp == BC_PRES) H.pyu[Nvy_in - 1] = 1;

  // --- FFT symbol (operator_divergence.m:268-291) ----------------------------
  H.fft_ok = false;
  if (uL == BC_PER && uR == BC_PER && vLo == BC_PER && vUp == BC_PER) {
    double mdx = 0, mdy = 0;
    for (int i = 1; i < Nx; ++i) mdx = std::max(mdx, std::fabs(hx[i] - hx[i - 1]));
    for (int j = 1; j < Ny; ++j) mdy = std::max(mdy, std::fabs(hy[j] - hy[j - 1]));
    if (mdx <= 1e-14 && mdy <= 1e-14) {
      H.fft_ok = true;
      const double dx = hx[0], dy = hy[0];
      H.fft_dxdy = dx * dy;
      H.fft_ax.resize(Nx);
      H.fft_ay.resize(Ny);
      for (int I = 0; I < Nx; ++I) {
        double s = std::sin((double)I * M_PI / Nx);
        H.fft_ax[I] = (1.0 / (dx * dx)) * (s * s);
      }
      for (int J = 0; J < Ny; ++J) {
        double s = std::sin((double)J * M_PI / Ny);
        H.fft_ay[J] = (1.0 / (dy * dy)) * (s * s);
      }
    }
  }
}

}  // namespace ins2d
