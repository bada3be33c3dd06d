// Host side of the multigrid preconditioner (mg.cu): level hierarchy of the
// separable pressure matrix and its device set-up.
#pragma once

#include <functional>
#include <vector>

#include "setup.hpp"

namespace ins2d {

// One level: 1D operator rows (entries at i-1, i, i+1) and cell widths per
// direction; cx, cy = aggregation factors to the next level (0 on the coarsest).
struct MgHostLevel {
  int nx = 0, ny = 0;
  bool perx = false, pery = false;
  int cx = 0, cy = 0;
  std::vector<double> xm, x0, xp, hx, ym, y0, yp, hy;
};

// Throws std::runtime_error when the grid is too small for the hierarchy.
std::vector<MgHostLevel> mg_build_levels(const HostOps &H);
// dense matrix of a (small) level, row-major
std::vector<double> mg_dense(const MgHostLevel &L);
// Moore-Penrose pseudo-inverse of a symmetric n x n matrix
std::vector<double> mg_pinv(std::vector<double> A, int n);
// level limits of the device hierarchy (mg.cuh)
constexpr int kMgMaxLevelsHost = 20;
constexpr int kMgCoarseMaxHost = 64;

}  // namespace ins2d
