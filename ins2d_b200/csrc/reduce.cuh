// Deterministic grid-wide reduction used by the stencil and PCG kernels:
// warp shuffles, then per-block partials in global memory; the last block to
// finish (atomic ticket) combines the partials with a fixed assignment and a
// fixed tree, so results do not depend on block scheduling.
#pragma once

#include <cfloat>

#include "kernels.cuh"

namespace ins2d {


enum RedOp { R_SUM = 0, R_MAX = 1, R_MIN = 2 };

static __device__ __forceinline__ double red_combine(double a, double b, int op) {
  return op == R_SUM ? a + b : (op == R_MAX ? fmax(a, b) : fmin(a, b));
}
static __host__ __device__ __forceinline__ double red_identity(int op) {
  return op == R_SUM ? 0.0 : (op == R_MAX ? -DBL_MAX : DBL_MAX);
}

// Block-level reduction of NQ values followed by the grid-level finish: the
// last block to arrive combines all partials in block order.  Every thread
// of every block must call it.
template <int NQ>
__device__ bool grid_reduce(double (&v)[NQ], const int (&ops)[NQ], const RedScratch &red, double (&out)[NQ]) {
  __shared__ double sh[32][NQ];
  __shared__ bool last;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int lane = tid & 31, warp = tid >> 5, nw = (blockDim.x * blockDim.y) >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q)
    for (int off = 16; off > 0; off >>= 1) v[q] = red_combine(v[q], __shfl_down_sync(0xffffffffu, v[q], off), ops[q]);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NQ; ++q) sh[warp][q] = v[q];
  __syncthreads();
  const int bid = blockIdx.x + gridDim.x * blockIdx.y;
  const int nb = gridDim.x * gridDim.y;
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double a = sh[0][q];
      for (int w = 1; w < nw; ++w) a = red_combine(a, sh[w][q], ops[q]);
      red.partials[(size_t)bid * NQ + q] = a;
    }
    __threadfence();
    unsigned int ticket = atomicAdd(red.counter, 1u);
    last = (ticket == (unsigned)nb - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  // the last block: each thread combines a fixed strided subset of the
  // partials in order, then a fixed-shape tree -> deterministic result
  const int nthr = blockDim.x * blockDim.y;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double a = red_identity(ops[q]);
    // partials read through L2 (ld.global.cg: written by other blocks before
    // their fence), four loads in flight, combined in block order
    int b = tid;
    for (; b + 3 * nthr < nb; b += 4 * nthr) {
      const double v0 = __ldcg(red.partials + (size_t)b * NQ + q);
      const double v1 = __ldcg(red.partials + (size_t)(b + nthr) * NQ + q);
      const double v2 = __ldcg(red.partials + (size_t)(b + 2 * nthr) * NQ + q);
      const double v3 = __ldcg(red.partials + (size_t)(b + 3 * nthr) * NQ + q);
      a = red_combine(a, v0, ops[q]);
      a = red_combine(a, v1, ops[q]);
      a = red_combine(a, v2, ops[q]);
      a = red_combine(a, v3, ops[q]);
    }
    for (; b < nb; b += nthr) a = red_combine(a, __ldcg(red.partials + (size_t)b * NQ + q), ops[q]);
    for (int off = 16; off > 0; off >>= 1) a = red_combine(a, __shfl_down_sync(0xffffffffu, a, off), ops[q]);
    if (lane == 0) sh[warp][q] = a;
  }
  __syncthreads();
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double a = sh[0][q];
      for (int w = 1; w < nw; ++w) a = red_combine(a, sh[w][q], ops[q]);
      red.result[q] = a;
      out[q] = a;
    }
    *red.counter = 0u;
  }
  return tid == 0;
}

// Variant for callers that only need red.result.
template <int NQ>
__device__ __forceinline__ void grid_reduce(double (&v)[NQ], const int (&ops)[NQ], const RedScratch &red) {
  double out[NQ];
  grid_reduce<NQ>(v, ops, red, out);
}


}  // namespace ins2d
