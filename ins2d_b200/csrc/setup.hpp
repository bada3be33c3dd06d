// Host-side derivation of the INS2D operators as 1D row tables.
//
// Every 2D operator of the reference is a Kronecker product of 1D operators
// (identity or diagonal metric factors on one axis), with the boundary
// conditions folded in by the elimination u = B1D*u_in + Btemp*ybc
// (BC_general.m:124-125).  This file restates that 1D algebra exactly and
// emits, per 1D operator, a table of at most kTab entries per row plus the
// two boundary-coefficient vectors Pre*Btemp*ybc1 and Pre*Btemp*ybc2, so the
// device kernels apply the operators matrix-free.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace ins2d {

constexpr int kTab = 3;  // max entries per row of a 1D operator table

enum BcType { BC_DIR = 0, BC_PRES = 1, BC_PER = 2, BC_SYM = 3 };

// Row-sparse matrix (host, setup only).
struct Sp {
  int m = 0, n = 0;
  std::vector<std::map<int, double>> rows;
  Sp() = default;
  Sp(int m_, int n_) : m(m_), n(n_), rows(m_) {}
  void set(int i, int j, double v);  // MATLAB A(i,j) = v (0-based)
  static Sp eye(int n);
  static Sp diag(const std::vector<double> &d);
};
Sp mul(const Sp &A, const Sp &B);
Sp sub(const Sp &A, const Sp &B);
Sp transpose(const Sp &A);
Sp scale_rows(const Sp &A, int row, double s);
// MATLAB spdiags(B,d,m,n) create form (column-indexed values when m>=n,
// row-indexed when m<n).
Sp spdiags(const std::vector<std::vector<double>> &Bcols, const std::vector<int> &d, int m, int n);
std::vector<double> matvec(const Sp &A, const std::vector<double> &x);

struct BC1 {
  Sp B1D, Btemp;
  std::vector<double> ybc1, ybc2;
};
BC1 bc_general(int Nt, int Nin, int Nb, int t1, int t2, double h1, double h2);
BC1 bc_general_stag(int Nt, int Nin, int Nb, int t1, int t2, double h1, double h2);

// A device-ready 1D operator: T = Pre*B1D with <= kTab entries per row,
// b1 = Pre*Btemp*ybc1, b2 = Pre*Btemp*ybc2.
struct Table {
  int nrows = 0, ncols = 0;
  std::vector<int32_t> col;  // nrows*kTab
  std::vector<double> w;     // nrows*kTab
  std::vector<double> b1, b2;
  Sp T;  // kept for host-side products (Laplacian, BC pre-products)
  // weights of columns r+s and r+s+1 for the rows of the regular range
  // (find_regular), zero elsewhere
  std::vector<double> rw0, rw1;
};
Table make_table(const Sp &Pre, const BC1 &bc, const std::string &name);
Table make_table(const Sp &T, const std::string &name);
// Interior structure of a table: rows r in [lo,hi) have all entries at
// columns r+s and r+s+1 (weight w1 may be zero), and no boundary
// coefficients.  two = some row in the range uses column r+s+1.
struct Regular {
  int s = 0, lo = 0, hi = 0, two = 0;
};
Regular find_regular(Table &T);  // also fills T.rw0 / T.rw1
Regular intersect(const Regular &a, const Regular &b);

// Re-encodes two tables with the same number of rows on the union of their
// column sets per row, so one set of loads serves both (e.g. Au_ux and Su_ux,
// which share the boundary elimination of u in x).
void align_pair(Table &A, Table &B, const std::string &name);

// All operators of one grid + BC combination (operator_mesh/averaging/
// interpolation/divergence/convection_diffusion.m, order4=0, laminar).
struct HostOps {
  int Nx = 0, Ny = 0;
  int Nux = 0, Nuy = 0, Nvx = 0, Nvy = 0, Npx = 0, Npy = 0;
  int bc[8] = {0};  // u.left,u.right,u.low,u.up,v.left,v.right,v.low,v.up
  double Re = 1.0;
  std::vector<double> x, y, xp, yp, hx, hy, gx, gy;
  std::vector<double> xin, yin, hxd, hyd, gxi, gyi, gxd, gyd;
  // u-momentum tables
  Table AUX, SUX, AUY, SUY, IVX, IVY, MX, MXT;
  // v-momentum tables
  Table AVX, SVX, AVY, SVY, IUX, IUY, MY, MYT;
  // Laplacian A = M Om^-1 G = -(diag(hy) (x) TX + TY (x) diag(hx))
  Table TX, TY;
  std::vector<double> TXd, TYd;  // diagonals of TX, TY
  // y_px / y_py patterns (set_bc_vectors.m:154-176)
  std::vector<double> pxl, pxr, pyl, pyu;
  // regular interior ranges (pairs intersected): used by the fast walker
  Regular rAUX, rAUY, rIVX, rIVY, rMXT, rAVX, rAVY, rIUX, rIUY, rMYT, rMX, rMY;
  // FFT Poisson symbol factors (operator_divergence.m:268-291)
  bool fft_ok = false;
  std::vector<double> fft_ax, fft_ay;  // (1/dx^2) sin^2(I pi/Npx), (1/dy^2) sin^2(J pi/Npy)
  double fft_dxdy = 0.0;
  int64_t Nu() const { return (int64_t)Nux * Nuy; }
  int64_t Nv() const { return (int64_t)Nvx * Nvy; }
  int64_t Np() const { return (int64_t)Npx * Npy; }
};

// Throws std::runtime_error with a message on invalid input.
void build_host_ops(HostOps &H, int Nx, int Ny, const double *x, const double *y,
                    const int bc[8], double Re);

}  // namespace ins2d
