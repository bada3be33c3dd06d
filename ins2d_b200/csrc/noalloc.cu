// FFT pressure-Poisson solve that allocates no device memory.
//
// Some callers cannot allocate device memory: applications that hand all of
// the GPU's memory to their own pool or arena up front, plugins loaded into a
// host that owns the device allocator, and real-time loops in which a
// cudaMalloc (which may synchronise the device) is not allowed.  For them this
// entry point keeps its scratch -- the half spectrum, the twiddle and symbol
// tables and the max|fhat| word -- in one file-scope device array of fixed
// size, which every GPU that loads the library holds until the process exits.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "ins2d.h"
#include "kernels.cuh"

using namespace ins2d;

namespace {

// limits of the static scratch (see INS2D_NOALLOC_* in ins2d.h)
constexpr int kMaxN = INS2D_NOALLOC_MAX_N;
constexpr long long kMaxCells = INS2D_NOALLOC_MAX_CELLS;
// layout in double2 units: spectrum ((Nx/2+1)*Ny <= kMaxCells/2 + kMaxN),
// twiddle tables x and y (2N <= 2 kMaxN each), symbol factors x and y
// (<= kMaxN doubles each = kMaxN/2 double2), max|fhat| (one double, padded to
// a double2)
constexpr size_t kSpec = (size_t)(kMaxCells / 2 + kMaxN);
constexpr size_t kTotal = kSpec + 4 * (size_t)kMaxN + (size_t)kMaxN + 1;

static __device__ __align__(256) double2 g_scratch[kTotal];

constexpr int kMaxDevices = 64;
double2 *g_scratch_addr[kMaxDevices] = {nullptr};
// the (Nx, Ny, dx, dy) whose twiddle and symbol tables the device's scratch
// holds, so repeated calls of one size upload nothing
struct TableKey {
  int Nx = 0, Ny = 0;
  double dx = 0.0, dy = 0.0;
};
TableKey g_tables[kMaxDevices];
std::mutex g_setup_mu;

int log2_exact(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return ((1 << l) == n) ? l : -1;
}

}  // namespace

extern "C" int ins2d_fft_poisson_noalloc(const double *f, double *dp, int32_t Nx, int32_t Ny, double dx, double dy,
                                         void *stream) {
  if (!f || !dp) return INS2D_EINVAL;
  if (Nx < 2 || Ny < 2 || Nx > kMaxN || Ny > kMaxN || (long long)Nx * Ny > kMaxCells) return INS2D_EINVAL;
  if (!fft_supported(Nx, Ny)) return INS2D_EINVAL;
  if (!(dx > 0) || !(dy > 0)) return INS2D_EINVAL;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return INS2D_ECUDA;
  // once per device, with that device current: the device address of the
  // static array (its host-side name is only a stand-in) and the kernels'
  // shared-memory limits
  double2 *base = nullptr;
  bool upload = true;
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
      void *ptr = nullptr;
      if (cudaGetSymbolAddress(&ptr, g_scratch) != cudaSuccess || !ptr) return INS2D_ECUDA;
      if (fft_prepare() != cudaSuccess) return INS2D_ECUDA;
      g_scratch_addr[dev] = (double2 *)ptr;
    }
    base = g_scratch_addr[dev];
    const TableKey &k = g_tables[dev];
    upload = !(k.Nx == Nx && k.Ny == Ny && k.dx == dx && k.dy == dy);
    // forget the key until the new tables are uploaded: a failed upload must
    // not leave a key that claims them
    if (upload) g_tables[dev] = TableKey{};
  }
  cudaStream_t s = (cudaStream_t)stream;
  double2 *spec = base;
  double2 *twx = base + kSpec;
  double2 *twy = twx + 2 * (size_t)kMaxN;
  double *axd = (double *)(twy + 2 * (size_t)kMaxN);  // kMaxN doubles
  double *ayd = axd + kMaxN;                           // kMaxN doubles
  double *maxabs = (double *)(base + kSpec + 5 * (size_t)kMaxN);
  if (upload) {
    // twiddle tables and the symbol factors (1/dx^2) sin^2(I pi/Nx),
    // (1/dy^2) sin^2(J pi/Ny) of operator_divergence.m:283, as in the context path
    const std::vector<double> tx = fft_twiddle_table(Nx), ty = fft_twiddle_table(Ny);
    std::vector<double> ax((size_t)Nx), ay((size_t)Ny);
    for (int k = 0; k < Nx; ++k) {
      const double sn = std::sin((double)k * M_PI / Nx);
      ax[k] = (1.0 / (dx * dx)) * (sn * sn);
    }
    for (int k = 0; k < Ny; ++k) {
      const double sn = std::sin((double)k * M_PI / Ny);
      ay[k] = (1.0 / (dy * dy)) * (sn * sn);
    }
    if (cudaMemcpyAsync(twx, tx.data(), tx.size() * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(twy, ty.data(), ty.size() * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(axd, ax.data(), ax.size() * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(ayd, ay.data(), ay.size() * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
      return INS2D_ECUDA;
    // the host vectors are released at the end of this block: wait for the
    // copies (pageable sources may still be read by the copy engine)
    if (cudaStreamSynchronize(s) != cudaSuccess) return INS2D_ECUDA;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    g_tables[dev] = TableKey{Nx, Ny, dx, dy};
  }
  DevOps P{};
  P.fft_ax = axd;
  P.fft_ay = ayd;
  P.fft_dxdy = dx * dy;
  FftPlan plan;
  plan.Nx = Nx;
  plan.Ny = Ny;
  plan.logx = log2_exact(Nx);
  plan.logy = log2_exact(Ny);
  plan.twx = twx;
  plan.twy = twy;
  plan.spec = spec;
  plan.maxabs = maxabs;  // zeroed by the first transform pass of each solve
  // An error already pending on this thread belongs to the caller: it is
  // neither cleared nor taken for a failure of this call.  Without one, an
  // error after the launches is this call's own (and is consumed).
  const cudaError_t pending = cudaPeekAtLastError();
  if (launch_fft_poisson(P, plan, f, dp, false, s) != cudaSuccess) return INS2D_ECUDA;
  if (pending == cudaSuccess && cudaPeekAtLastError() != cudaSuccess) {
    cudaGetLastError();
    return INS2D_ECUDA;
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return INS2D_ECUDA;
  return INS2D_OK;
}
