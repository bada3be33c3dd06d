// Host side of the multigrid preconditioner: the level hierarchy of the
// separable pressure matrix by 1D Galerkin aggregation and the dense
// pseudo-inverse of the coarsest level (plain C++; the device set-up is in
// mg.cu).
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "mg_host.hpp"

namespace ins2d {

namespace {

// 1D operator rows (entries at i-1, i, i+1, periodic wrap when per) from a
// host table of the pressure Laplacian factor.
void from_table(const Table &T, int n, bool per, std::vector<double> &m, std::vector<double> &z0,
                std::vector<double> &p) {
  m.assign(n, 0.0);
  z0.assign(n, 0.0);
  p.assign(n, 0.0);
  if (T.nrows != n) throw std::runtime_error("multigrid: table size mismatch");
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < kTab; ++k) {
      const double w = T.w[(size_t)i * kTab + k];
      if (w == 0.0) continue;
      const int c = T.col[(size_t)i * kTab + k];
      if (c == i)
        z0[i] += w;
      else if ((i > 0 && c == i - 1) || (per && i == 0 && c == n - 1))
        m[i] += w;
      else if ((i < n - 1 && c == i + 1) || (per && i == n - 1 && c == 0))
        p[i] += w;
      else
        throw std::runtime_error("multigrid: pressure operator is not tridiagonal in one direction");
    }
  }
}

// Galerkin product Pc' T Pc for pairwise aggregation (I = {2I, 2I+1}).
void coarsen_1d(int n, bool per, const std::vector<double> &m, const std::vector<double> &z0,
                const std::vector<double> &p, const std::vector<double> &h, std::vector<double> &mc,
                std::vector<double> &z0c, std::vector<double> &pc, std::vector<double> &hc) {
  const int nc = (n + 1) / 2;
  mc.assign(nc, 0.0);
  z0c.assign(nc, 0.0);
  pc.assign(nc, 0.0);
  hc.assign(nc, 0.0);
  auto add = [&](int I, int J, double w) {
    if (w == 0.0) return;
    if (J == I)
      z0c[I] += w;
    else if ((I > 0 && J == I - 1) || (per && I == 0 && J == nc - 1))
      mc[I] += w;
    else if ((I < nc - 1 && J == I + 1) || (per && I == nc - 1 && J == 0))
      pc[I] += w;
    else
      throw std::runtime_error("multigrid: coarse operator is not tridiagonal");
  };
  for (int i = 0; i < n; ++i) {
    const int I = i / 2;
    z0c[I] += z0[i];
    hc[I] += h[i];
    if (i > 0 || per) add(I, ((i - 1 + n) % n) / 2, m[i]);
    if (i < n - 1 || per) add(I, ((i + 1) % n) / 2, p[i]);
  }
}

bool can_coarsen(int n, bool per) { return per ? n >= 6 : n >= 4; }

// symmetric eigen-decomposition by cyclic Jacobi rotations (n small)
void jacobi_eig(int n, std::vector<double> &a, std::vector<double> &v) {
  v.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        tot += a[(size_t)i * n + j] * a[(size_t)i * n + j];
        if (i != j) off += a[(size_t)i * n + j] * a[(size_t)i * n + j];
      }
    if (off <= 1e-30 * tot) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a[(size_t)p * n + q];
        if (apq == 0.0) continue;
        const double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {  // A = J' A J
          const double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
          a[(size_t)k * n + p] = c * akp - s * akq;
          a[(size_t)k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
          a[(size_t)p * n + k] = c * apk - s * aqk;
          a[(size_t)q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
          v[(size_t)k * n + p] = c * vkp - s * vkq;
          v[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
  }
}

}  // namespace

std::vector<MgHostLevel> mg_build_levels(const HostOps &H) {
  const bool perx = H.bc[0] == BC_PER, pery = H.bc[6] == BC_PER;
  if (H.Npx < 3 || H.Npy < 3) throw std::runtime_error("multigrid needs at least 3 pressure cells per direction");
  std::vector<MgHostLevel> lv(1);
  MgHostLevel &L0 = lv[0];
  L0.nx = H.Npx;
  L0.ny = H.Npy;
  L0.perx = perx;
  L0.pery = pery;
  from_table(H.TX, H.Npx, perx, L0.xm, L0.x0, L0.xp);
  from_table(H.TY, H.Npy, pery, L0.ym, L0.y0, L0.yp);
  L0.hx = H.hx;
  L0.hy = H.hy;
  for (;;) {
    MgHostLevel &F = lv.back();
    const bool cx = can_coarsen(F.nx, F.perx), cy = can_coarsen(F.ny, F.pery);
    if ((long long)F.nx * F.ny <= kMgCoarseMaxHost || (!cx && !cy)) break;
    if ((int)lv.size() == kMgMaxLevelsHost) throw std::runtime_error("multigrid: too many levels");
    MgHostLevel C;
    C.perx = F.perx;
    C.pery = F.pery;
    F.cx = cx ? 2 : 1;
    F.cy = cy ? 2 : 1;
    if (cx) {
      coarsen_1d(F.nx, F.perx, F.xm, F.x0, F.xp, F.hx, C.xm, C.x0, C.xp, C.hx);
    } else {
      C.xm = F.xm;
      C.x0 = F.x0;
      C.xp = F.xp;
      C.hx = F.hx;
    }
    if (cy) {
      coarsen_1d(F.ny, F.pery, F.ym, F.y0, F.yp, F.hy, C.ym, C.y0, C.yp, C.hy);
    } else {
      C.ym = F.ym;
      C.y0 = F.y0;
      C.yp = F.yp;
      C.hy = F.hy;
    }
    C.nx = (int)C.x0.size();
    C.ny = (int)C.y0.size();
    lv.push_back(std::move(C));
  }
  if ((long long)lv.back().nx * lv.back().ny > kMgCoarseMaxHost)
    throw std::runtime_error("multigrid: coarsest level too large");
  return lv;
}

std::vector<double> mg_dense(const MgHostLevel &L) {
  const int nx = L.nx, ny = L.ny, n = nx * ny;
  std::vector<double> A((size_t)n * n, 0.0);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const int r = j * nx + i;
      auto add = [&](int ii, int jj, double w) { A[(size_t)r * n + jj * nx + ii] += w; };
      const double hx = L.hx[i], hy = L.hy[j];
      add(i, j, -(hy * L.x0[i] + hx * L.y0[j]));
      if (i > 0 || L.perx) add((i - 1 + nx) % nx, j, -hy * L.xm[i]);
      if (i < nx - 1 || L.perx) add((i + 1) % nx, j, -hy * L.xp[i]);
      if (j > 0 || L.pery) add(i, (j - 1 + ny) % ny, -hx * L.ym[j]);
      if (j < ny - 1 || L.pery) add(i, (j + 1) % ny, -hx * L.yp[j]);
    }
  return A;
}

std::vector<double> mg_pinv(std::vector<double> A, int n) {
  std::vector<double> V;
  jacobi_eig(n, A, V);
  double lmax = 0.0;
  for (int i = 0; i < n; ++i) lmax = std::max(lmax, std::fabs(A[(size_t)i * n + i]));
  std::vector<double> P((size_t)n * n, 0.0);
  for (int k = 0; k < n; ++k) {
    const double lam = A[(size_t)k * n + k];
    if (std::fabs(lam) <= 1e-10 * lmax) continue;  // null space (all-Neumann / periodic)
    const double il = 1.0 / lam;
    for (int r = 0; r < n; ++r) {
      const double vr = V[(size_t)r * n + k] * il;
      for (int c = 0; c < n; ++c) P[(size_t)r * n + c] += vr * V[(size_t)c * n + k];
    }
  }
  return P;
}

}  // namespace ins2d
