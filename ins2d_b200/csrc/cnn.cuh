// The learned part of the pressure solve: a small convolutional network
// (six 3x3 convolutions, 1 -> 32 -> 32 -> 32 -> 32 -> 32 -> 1 channels, ReLU
// between them, no biases, zero padding) that maps the Jacobi-scaled Poisson
// right-hand side to an approximation of the solution.  The four 32 -> 32
// layers (forward, backward-data and weight gradient) are BF16 tensor-core
// implicit GEMMs accumulating in FP32 (cnn.cu); the 1 -> 32 and 32 -> 1 layers
// are FP32 CUDA-core kernels.  The PCG uses the network's output as its
// initial guess (ctx.cu: solve_learned) and still iterates to the same
// relative residual, so results are unchanged within the CG tolerance.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "device.cuh"
#include "ins2d.h"

namespace ins2d {
namespace cnn {

constexpr int kC = 32;                 // hidden channels
constexpr int kTaps = 9;               // 3x3 taps, t = (dy+1)*3 + (dx+1)
constexpr int kK = kTaps * kC;         // 288: GEMM depth of a 32 -> 32 layer
constexpr int kMid = 4;                // 32 -> 32 layers
constexpr int kOffW1 = 0;              // [32 co][9 t]
constexpr int kOffWm = kC * kTaps;     // kMid x [32 co][9 t][32 ci]
constexpr int kSzWm = kC * kK;         // 9216
constexpr int kOffW6 = kOffWm + kMid * kSzWm;  // [9 t][32 ci]
constexpr int kNParam = kOffW6 + kK;   // 37440

}  // namespace cnn
}  // namespace ins2d

struct ins2d_cnn {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // master weights, gradient, Adam moments
  __nv_bfloat16 *wf = nullptr, *wb = nullptr;  // packed 32->32 weights: forward, backward-data
  bool packed = false;
  long long adam_t = 0;
  float out_scale = 1.0f;
  long long cap = 0;                     // pixels the activation buffers hold
  __nv_bfloat16 *act[5] = {};            // post-ReLU activations of layers 1..5, NHWC
  __nv_bfloat16 *dz[2] = {};             // pre-activation gradients (ping-pong)
  float *y = nullptr, *dy = nullptr;     // output and its gradient
  float *dres = nullptr;                 // residual A y - diag(A) in of the residual loss
  float *in1 = nullptr;                  // single-field input of the solver's guess
  long long in1_cap = 0;
  float *partials = nullptr;             // weight-gradient partials
  int part_rows = 0;
  double *red = nullptr;                 // reduction scratch (partials + results)
  unsigned *flag = nullptr;              // set by a tensor-core kernel whose wait gave up
  int sms = 148;
  int path = INS2D_CNN_PATH_TCGEN05;     // tensor-core instructions of the 32 -> 32 layers
};

namespace ins2d {
namespace cnn {

// CUDA runtime failures inside the network code
struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
// doubles of reduction scratch the helpers below need
size_t red_doubles();

// network inputs (and targets) from a Poisson right-hand side f (and its
// solution p) on the pressure grid of P: in = (f / diag A) / s with
// s = rms(f / diag A); tgt = (p - center * mean(p)) / s.  p, tgt may be null.
void prepare(const DevOps &P, const double *f, const double *p, int center, float *in, float *tgt, double *red,
             cudaStream_t s);
// forward pass over B fields of H x W (in: fp32 [B][H][W]); output in net->y
void forward(ins2d_cnn *net, const float *in, int B, int H, int W, cudaStream_t s);
// loss (after a stream synchronisation) and gradient in net->g.  P = null:
// mean((y - tgt)^2); P = a context's operators: the residual loss
// mean((A y - diag(A) in)^2) on that grid (tgt unused), gradient 2 A (.) / n.
double loss_grad(ins2d_cnn *net, const float *in, const float *tgt, int B, int H, int W, cudaStream_t s,
                 const DevOps *P);
// one Adam step from net->g
void adam(ins2d_cnn *net, float lr, cudaStream_t s);
// the solver's initial guess: x0 = (N(v) - N(-v)) / 2 with v = prepare(f),
// the odd part of the network N (A^-1 is linear, so the odd part of an
// approximation of it is never a worse approximation), as fp64
void guess(ins2d_cnn *net, const DevOps &P, const double *f, double *x0, cudaStream_t s);
// ensures the buffers hold `pixels` pixels (throws std::bad_alloc)
void reserve(ins2d_cnn *net, long long pixels);
// throws when a tensor-core kernel reported a wait that gave up (synchronises)
void check(ins2d_cnn *net, cudaStream_t s);
// reductions for the Rayleigh-Ritz scaling of the guess (results copied to
// the host; synchronises the stream):
//   d[0] = x.f, d[1] = x.q, d[2] = f.f, d[3] = max|f|
void dots(long long n, const double *x, const double *f, const double *q, double *red, double d[4], cudaStream_t s);
// z = M(r): the odd part of the network applied to r (prepared like f),
// rescaled by the rms of r / diag A so that M(c r) = c M(r) for every real c
void precond(ins2d_cnn *net, const DevOps &P, const double *r, double *z, cudaStream_t s);
// a[n + k] = -a[k] for k < n
void negate_tail(float *a, long long n, cudaStream_t s);
// n standard normal values (counter-based generator with this seed)
void gaussian(float *a, long long n, uint64_t seed, cudaStream_t s);
// sum of squares of n floats (synchronises)
double sumsq(const float *a, long long n, double *red, cudaStream_t s);
// flexible CG steps (each synchronises and returns its reductions):
//   d = {p.q, p.r};  x += a p, r -= a q, d = {r.r, max|r|};  z.q;  p = z + b p
void fcg_pq(long long n, const double *p, const double *q, const double *r, double *red, double d[2],
            cudaStream_t s);
void fcg_update(long long n, double a, double *x, double *r, const double *p, const double *q, double *red,
                double d[2], cudaStream_t s);
double fcg_zq(long long n, const double *z, const double *q, double *red, cudaStream_t s);
void fcg_p(long long n, double b, const double *z, double *p, cudaStream_t s);
//   r = f - a q, x *= a; d[0] = r.r, d[1] = max|r|
void residual(long long n, const double *f, const double *q, double a, double *x, double *r, double *red,
              double d[2], cudaStream_t s);

}  // namespace cnn
}  // namespace ins2d
