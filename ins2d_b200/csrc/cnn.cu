// The learned initial guess of the pressure solve: a six-layer 3x3
// convolutional network trained on the solver's own (right-hand side,
// pressure) pairs.  There is no counterpart in the reference (its solves start
// from zero, pressure_poisson.m:61-70); the network only changes where CG
// starts, never the stopping rule.
//
// Layout: activations NHWC on the pressure grid (pixel (i,j) at j*Npx + i,
// x fastest, then the 32 channels of the pixel: 64 bytes of BF16), a batch of
// B fields one after another.  Master weights are FP32 in one flat vector:
//   W1 [32 co][9 t]            (1 -> 32)
//   W2..W5 [32 co][9 t][32 ci] (32 -> 32, ReLU after each)
//   W6 [9 t][32 ci]            (32 -> 1, scaled by out_scale)
// with t = (dy+1)*3 + (dx+1) and out(p) = sum_t W[t] in(p + (dx,dy)) (zero
// padding).  Rounding points (the oracle emulates them): layer outputs 1..5
// and the gradients dZ1..dZ5 are stored as BF16 (round to nearest even);
// everything else is FP32.
//
// Tensor cores: the 32 -> 32 layers are implicit GEMMs on BF16 tensor cores
// with FP32 accumulators:
//   forward        Z[p][co]   = sum_{t,ci} W[co][t][ci] A[p+t][ci]    M = pixels, N = 32, K = 288
//   backward-data  dA[p][ci]  = sum_{t,co} W[co][8-t][ci] dZ[p+t][co] (the same kernel, transposed weights)
//   weight grad    dW[co][t,ci] = sum_p dZ[p][co] A[p+t][ci]          M = 32, N = 288, K = pixels
// The first two run on tcgen05.mma with TMEM accumulators (k_conv_mid_tc,
// the default) or on mma.sync m16n8k16 (k_conv_mid); the weight gradient on
// mma.sync (k_wgrad_mid).  The 1 -> 32 and 32 -> 1 layers (2 x 288 MACs per
// pixel), the losses (squared error; the residual loss with the context's
// operator tables), the solver's odd-part application and Adam are FP32 /
// FP64 CUDA-core kernels.  Per pixel and 32 -> 32 layer the traffic is one
// read of the input activations and one write of the output (64 bytes each
// in BF16).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <stdexcept>
#include <vector>

#include "cnn.cuh"
#include "ins2d.h"
#include "kernels.cuh"

namespace ins2d {
namespace cnn {

namespace {

using bf16 = __nv_bfloat16;

constexpr int TW = 16, TH = 8;             // output tile of the 32 -> 32 kernels
constexpr int HWD = TW + 2, HHT = TH + 2;  // halo tile
constexpr int PSTR = 40;                   // bf16 per halo pixel in shared memory (32 + 8: no bank conflicts)
constexpr int WSTR = kK + 8;               // bf16 per output channel of the shared weights
constexpr int kRedBlocks = 1184;           // capacity of the reduction partials (148 x 8)
constexpr int kWgBlocks = 592;             // weight-gradient blocks (148 x 4)

#define CK(x)                                                                                 \
  do {                                                                                        \
    cudaError_t e_ = (x);                                                                     \
    if (e_ != cudaSuccess) throw CudaError(std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&h);
}
__device__ __forceinline__ uint32_t pack2h(bf16 lo, bf16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}
__device__ __forceinline__ void unpack8(const uint4 &v, float (&o)[8]) {
  const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    o[2 * k] = __uint_as_float(w[k] << 16);
    o[2 * k + 1] = __uint_as_float(w[k] & 0xffff0000u);
  }
}

// --- layer 1: 1 -> 32, ReLU --------------------------------------------------
__global__ void __launch_bounds__(256) k_conv_in(const float *__restrict__ in, const float *__restrict__ w1,
                                                 bf16 *__restrict__ out, int B, int H, int W) {
  __shared__ float ws[kC * kTaps];
  for (int i = threadIdx.x; i < kC * kTaps; i += blockDim.x) ws[i] = w1[i];
  __syncthreads();
  const long long n = (long long)B * H * W;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(p % W);
    const int y = (int)((p / W) % H);
    float v[kTaps];
#pragma unroll
    for (int t = 0; t < kTaps; ++t) {
      const int xx = x + t % 3 - 1, yy = y + t / 3 - 1;
      v[t] = (xx >= 0 && xx < W && yy >= 0 && yy < H) ? in[p + (long long)(t / 3 - 1) * W + (t % 3 - 1)] : 0.0f;
    }
    uint32_t o[16];
#pragma unroll
    for (int c = 0; c < kC; c += 2) {
      float z0 = 0.0f, z1 = 0.0f;
#pragma unroll
      for (int t = 0; t < kTaps; ++t) {
        z0 = fmaf(ws[c * kTaps + t], v[t], z0);
        z1 = fmaf(ws[(c + 1) * kTaps + t], v[t], z1);
      }
      o[c / 2] = pack2(fmaxf(z0, 0.0f), fmaxf(z1, 0.0f));
    }
    uint4 *dst = reinterpret_cast<uint4 *>(out + p * kC);
#pragma unroll
    for (int k = 0; k < 4; ++k) dst[k] = make_uint4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
  }
}

// --- 32 -> 32 on tensor cores ---------------------------------------------------
// One block: a 16 x 8 pixel tile of one field; warp w computes tile row w
// (M = 16 pixels) for all 32 output channels (4 n-tiles of 8), K = 9 taps x
// 32 input channels in 18 steps of 16.  The halo tile and the weights sit in
// shared memory with padded strides so that the 32-bit fragment loads of a
// warp hit 32 different banks.
// MODE 0: out = bf16(ReLU(Z)).  MODE 1 (backward-data): out = bf16(Z * [mask > 0]).
template <int MODE>
__global__ void __launch_bounds__(256) k_conv_mid(const bf16 *__restrict__ in, const bf16 *__restrict__ wt,
                                                  const bf16 *__restrict__ mask, bf16 *__restrict__ out, int H,
                                                  int W) {
  __shared__ __align__(16) bf16 sin_[HHT * HWD * PSTR];
  __shared__ __align__(16) bf16 sw[kC * WSTR];
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  const long long fbase = (long long)blockIdx.z * H * W;
  for (int i = tid; i < kC * (kK / 8); i += 256) {
    const int co = i / (kK / 8), ch = i % (kK / 8);
    *reinterpret_cast<uint4 *>(&sw[co * WSTR + ch * 8]) = *reinterpret_cast<const uint4 *>(&wt[co * kK + ch * 8]);
  }
  for (int i = tid; i < HHT * HWD * 4; i += 256) {
    const int hp = i >> 2, part = i & 3;
    const int gy = y0 - 1 + hp / HWD, gx = x0 - 1 + hp % HWD;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (gy >= 0 && gy < H && gx >= 0 && gx < W)
      v = *reinterpret_cast<const uint4 *>(&in[(fbase + (long long)gy * W + gx) * kC + part * 8]);
    *reinterpret_cast<uint4 *>(&sin_[hp * PSTR + part * 8]) = v;
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
  float acc[4][4];
#pragma unroll
  for (int nt = 0; nt < 4; ++nt)
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[nt][k] = 0.0f;
#pragma unroll
  for (int tap = 0; tap < kTaps; ++tap) {
    const bf16 *rowp = &sin_[((warp + tap / 3) * HWD + tap % 3) * PSTR];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int kc = h * 16 + 2 * t4;
      const uint32_t a0 = *reinterpret_cast<const uint32_t *>(&rowp[g * PSTR + kc]);
      const uint32_t a1 = *reinterpret_cast<const uint32_t *>(&rowp[(g + 8) * PSTR + kc]);
      const uint32_t a2 = *reinterpret_cast<const uint32_t *>(&rowp[g * PSTR + kc + 8]);
      const uint32_t a3 = *reinterpret_cast<const uint32_t *>(&rowp[(g + 8) * PSTR + kc + 8]);
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const bf16 *wp = &sw[(nt * 8 + g) * WSTR + tap * kC + kc];
        const uint32_t b0 = *reinterpret_cast<const uint32_t *>(wp);
        const uint32_t b1 = *reinterpret_cast<const uint32_t *>(wp + 8);
        mma_bf16(acc[nt], a0, a1, a2, a3, b0, b1);
      }
    }
  }
  const int y = y0 + warp;
  if (y >= H) return;
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    const int x = x0 + g + 8 * half;
    if (x >= W) continue;
    const long long pix = fbase + (long long)y * W + x;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int ch = nt * 8 + 2 * t4;
      float v0 = acc[nt][2 * half], v1 = acc[nt][2 * half + 1];
      if (MODE == 0) {
        v0 = fmaxf(v0, 0.0f);
        v1 = fmaxf(v1, 0.0f);
      } else {
        const uint32_t m = *reinterpret_cast<const uint32_t *>(&mask[pix * kC + ch]);
        if (!(__uint_as_float(m << 16) > 0.0f)) v0 = 0.0f;
        if (!(__uint_as_float(m & 0xffff0000u) > 0.0f)) v1 = 0.0f;
      }
      *reinterpret_cast<uint32_t *>(&out[pix * kC + ch]) = pack2(v0, v1);
    }
  }
}

// --- 32 -> 32 on the 5th-generation tensor cores (tcgen05, TMEM accumulators) --------
// Persistent blocks of 256 threads, several per SM.  Per tile of 8 x 16
// pixels (M = 128 rows, m = py * 8 + px): all threads stage the 10 x 18 halo
// tile in shared memory as four channel planes (plane c8 holds channels
// 8 c8 .. 8 c8 + 7 of every halo pixel, 16 bytes per pixel, rows of 10
// pixels).  That is the canonical K-major layout without swizzle for every
// tap at once: a core matrix is 8 consecutive pixels of one tile row (16
// bytes apart), the next tile row is kTcSbo = 160 bytes further, the next 8
// channels kTcLbo = 2880 bytes further, and tap (dy, dx) only moves the start
// address by (dy * 10 + dx) * 16 bytes.  So the A operands of the 18 MMAs of
// K = 16 (9 taps x 2 channel halves) are descriptors over one halo tile, with
// no im2col copy.  One thread issues them (N = 32, FP32 accumulators in 32
// TMEM columns) and commits to an mbarrier; after the (bounded) wait, warp w
// reads TMEM lanes 32 (w % 4) .. +31 (its pixels), columns 16 (w / 4) .. +15
// (its channels), applies ReLU (MODE 0) or the mask (MODE 1) and stores BF16.
// The weights (B: 32 x 288; core matrices of 8 output channels, next 8 input
// channels kBLbo bytes further) are loaded once per block.
constexpr int kTcM = 128;
constexpr int kTcTW = 8, kTcTH = 16;           // tile: 8 pixels wide, 16 rows
constexpr int kTcHW = kTcTW + 2, kTcHH = kTcTH + 2;
constexpr int kTcSbo = kTcHW * 16;             // 160: next tile row
constexpr int kTcLbo = kTcHH * kTcSbo;         // 2880: next 8 channels (plane)
constexpr int kABytes = (kC / 8) * kTcLbo;     // 11520 per halo buffer (two: double-buffered)
constexpr int kBLbo = (kC / 8) * 128;          // 512: next 8 K-elements of B
constexpr int kBBytes = (kK / 8) * kBLbo;      // 18432
// Dynamic shared memory: A (halo planes), B, the mbarrier and the TMEM slot
constexpr int kTcSmem = 2 * kABytes + kBBytes + 16;
constexpr int kTcBlocksPerSm = 5;
// kind::f16 instruction descriptor: FP32 accumulate (bits 4-5 = 1), A and B
// BF16 (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at
// bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kC >> 3) << 17) |
                            ((uint32_t)(kTcM >> 4) << 24);
constexpr long long kTcWaitLimit = 1LL << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// shared-memory matrix descriptor: start, leading (K) and stride (M/N) byte
// offsets in 16-byte units, descriptor version 1 (bit 46), no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
// 16-byte asynchronous copy global -> shared; src_bytes = 0 writes zeros
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(addr), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

template <int MODE>
__global__ void __launch_bounds__(256, kTcBlocksPerSm) k_conv_mid_tc(const bf16 *__restrict__ in, const bf16 *__restrict__ wt,
                                                        const bf16 *__restrict__ mask, bf16 *__restrict__ out, int B,
                                                        int H, int W, int tiles_x, int tiles_y,
                                                        unsigned *__restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *sA = smem;  // two halo buffers of kABytes
  uint8_t *sB = smem + 2 * kABytes;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + 2 * kABytes + kBBytes);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + 2 * kABytes + kBBytes + 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // B: element (n = co, k) at (k / 8) * kBLbo + co * 16 + (k % 8) * 2
  for (int i = tid; i < kC * (kK / 8); i += 256) {
    const int co = i % kC, kc = i / kC;
    *reinterpret_cast<uint4 *>(sB + kc * kBLbo + co * 16) = *reinterpret_cast<const uint4 *>(&wt[co * kK + kc * 8]);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                 "r"(kC)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  const uint32_t mb = smem_u32(mbar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mb), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t taddr = *tslot;
  const uint32_t aBase = smem_u32(sA), bBase = smem_u32(sB);
  uint32_t phase = 0;
  const long long per_field = (long long)tiles_x * tiles_y;
  const long long ntiles = per_field * B;
  // halo planes of a tile into buffer buf: channels 8 c8 .. 8 c8 + 7 of halo
  // pixel hp at c8 * kTcLbo + hp * 16 (zeros outside the field)
  auto load_halo = [&](long long tl, int buf) {
    const int bb = (int)(tl / per_field);
    const int rm = (int)(tl % per_field);
    const int hx0 = (rm % tiles_x) * kTcTW - 1, hy0 = (rm / tiles_x) * kTcTH - 1;
    const long long fb = (long long)bb * H * W;
    for (int i = tid; i < kTcHW * kTcHH * 4; i += 256) {
      const int hp = i >> 2, c8 = i & 3;
      const int gx = hx0 + hp % kTcHW, gy = hy0 + hp / kTcHW;
      const bool inside = gx >= 0 && gx < W && gy >= 0 && gy < H;
      const bf16 *src = inside ? &in[(fb + (long long)gy * W + gx) * kC + c8 * 8] : in;
      cp_async16(aBase + buf * kABytes + c8 * kTcLbo + hp * 16, src, inside ? 16u : 0u);
    }
  };
  if ((long long)blockIdx.x < ntiles) load_halo(blockIdx.x, 0);
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  int it = 0;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
    const int buf = it & 1;
    // the next tile's halo loads overlap this tile's MMAs and epilogue
    if (tile + gridDim.x < ntiles) load_halo(tile + gridDim.x, buf ^ 1);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    const int b = (int)(tile / per_field);
    const int rem = (int)(tile % per_field);
    const int x0 = (rem % tiles_x) * kTcTW, y0 = (rem / tiles_x) * kTcTH;
    const long long fbase = (long long)b * H * W;
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
      for (int ks = 0; ks < kK / 16; ++ks) {
        const int t = ks >> 1, h = ks & 1;
        const uint32_t a0 = aBase + buf * kABytes + 2 * h * kTcLbo + ((t / 3) * kTcHW + t % 3) * 16;
        tc_mma(taddr, smem_desc(a0, kTcLbo, kTcSbo), smem_desc(bBase + 2 * ks * kBLbo, kBLbo, 128), kIdesc,
               ks > 0 ? 1u : 0u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mb)
                   : "memory");
    }
    bool ok = false;
    for (long long it = 0; it < kTcWaitLimit && !ok; ++it) ok = mbar_try(mb, phase);
    if (!__syncthreads_and(ok)) {
      // give the MMAs a second bounded wait before the TMEM is freed
      if (tid == 0) atomicExch(err, 1u);
      for (long long it = 0; it < kTcWaitLimit && !ok; ++it) ok = mbar_try(mb, phase);
      break;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    uint32_t r[16];
    const int ch0 = 16 * (warp >> 2);
    tmem_ld16(taddr + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)ch0, r);
    const int m = 32 * (warp & 3) + lane;
    const int gx = x0 + (m & (kTcTW - 1)), gy = y0 + (m >> 3);
    if (gx < W && gy < H) {
      const long long pix = fbase + (long long)gy * W + gx;
      float v[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
      if (MODE == 0) {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j], 0.0f);
      } else {
        const uint4 *mp = reinterpret_cast<const uint4 *>(&mask[pix * kC + ch0]);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          float mv[8];
          unpack8(mp[q], mv);
#pragma unroll
          for (int e = 0; e < 8; ++e)
            if (!(mv[e] > 0.0f)) v[q * 8 + e] = 0.0f;
        }
      }
      uint4 *dst = reinterpret_cast<uint4 *>(&out[pix * kC + ch0]);
      dst[0] = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
      dst[1] = make_uint4(pack2(v[8], v[9]), pack2(v[10], v[11]), pack2(v[12], v[13]), pack2(v[14], v[15]));
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(kC) : "memory");
}

// --- layer 6: 32 -> 1 ------------------------------------------------------------
__global__ void __launch_bounds__(256) k_conv_out(const bf16 *__restrict__ a5, const float *__restrict__ w6,
                                                  float scale, float *__restrict__ y, int B, int H, int W) {
  __shared__ float ws[kK];
  for (int i = threadIdx.x; i < kK; i += blockDim.x) ws[i] = w6[i];
  __syncthreads();
  const long long n = (long long)B * H * W;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(p % W);
    const int yy0 = (int)((p / W) % H);
    float acc = 0.0f;
#pragma unroll
    for (int t = 0; t < kTaps; ++t) {
      const int xx = x + t % 3 - 1, yy = yy0 + t / 3 - 1;
      if (xx < 0 || xx >= W || yy < 0 || yy >= H) continue;
      const uint4 *src = reinterpret_cast<const uint4 *>(a5 + (p + (long long)(t / 3 - 1) * W + (t % 3 - 1)) * kC);
#pragma unroll
      for (int part = 0; part < 4; ++part) {
        float a[8];
        unpack8(src[part], a);
#pragma unroll
        for (int e = 0; e < 8; ++e) acc = fmaf(ws[t * kC + part * 8 + e], a[e], acc);
      }
    }
    y[p] = scale * acc;
  }
}

// --- block reductions (fixed order: deterministic) ----------------------------
template <int NQ>
__device__ void block_sum(double (&v)[NQ], const bool (&is_max)[NQ], double *out) {
  __shared__ double sh[32][NQ];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q)
    for (int off = 16; off > 0; off >>= 1) {
      const double o = __shfl_down_sync(0xffffffffu, v[q], off);
      v[q] = is_max[q] ? fmax(v[q], o) : v[q] + o;
    }
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NQ; ++q) sh[warp][q] = v[q];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double a = sh[0][q];
      for (int w = 1; w < nw; ++w) a = is_max[q] ? fmax(a, sh[w][q]) : a + sh[w][q];
      out[q] = a;
    }
}

// out[q] = combination over rows of part[row * NQ + q] (one block, fixed order)
template <int NQ>
__global__ void k_finish(const double *__restrict__ part, int rows, const int max_mask, double *__restrict__ out) {
  bool is_max[NQ];
  double v[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    is_max[q] = (max_mask >> q) & 1;
    v[q] = is_max[q] ? -INFINITY : 0.0;
  }
  for (int r = threadIdx.x; r < rows; r += blockDim.x)
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = is_max[q] ? fmax(v[q], part[r * NQ + q]) : v[q] + part[r * NQ + q];
  block_sum<NQ>(v, is_max, out);
}

// loss = sum (y - tgt)^2 / n; dy = dL/d(layer-6 output) = 2 (y - tgt) / n * scale
__global__ void __launch_bounds__(256) k_loss(const float *__restrict__ y, const float *__restrict__ tgt,
                                              float *__restrict__ dy, float gscale, long long n,
                                              double *__restrict__ part) {
  double v[1] = {0.0};
  const bool mx[1] = {false};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const float d = y[p] - tgt[p];
    dy[p] = gscale * d;
    v[0] += (double)d * d;
  }
  block_sum<1>(v, mx, part + blockIdx.x);
}

// The pressure Laplacian A = M Om^-1 G of a context (its 1D row tables, the
// form of lap() in device.cuh) applied to one FP32 field
__device__ __forceinline__ float lap_f(const DevOps &P, const float *__restrict__ f, int i, int j) {
  const int32_t *cx = P.TX.c + kT * i;
  const double *wx = P.TX.w + kT * i;
  const int32_t *cy = P.TY.c + kT * j;
  const double *wy = P.TY.w + kT * j;
  const long long row = (long long)j * P.Npx;
  const float sx = (float)__ldg(wx) * f[row + __ldg(cx)] + (float)__ldg(wx + 1) * f[row + __ldg(cx + 1)] +
                   (float)__ldg(wx + 2) * f[row + __ldg(cx + 2)];
  const float sy = (float)__ldg(wy) * f[(long long)__ldg(cy) * P.Npx + i] +
                   (float)__ldg(wy + 1) * f[(long long)__ldg(cy + 1) * P.Npx + i] +
                   (float)__ldg(wy + 2) * f[(long long)__ldg(cy + 2) * P.Npx + i];
  return -((float)__ldg(P.hy + j) * sx + (float)__ldg(P.hx + i) * sy);
}

// residual loss, pass 1: d = A y - diag(A) in per field (in = f / (diag(A) s),
// so diag(A) in = f / s); partial sums of d^2
__global__ void __launch_bounds__(256) k_res_loss(const __grid_constant__ DevOps P, const float *__restrict__ y,
                                                  const float *__restrict__ in, float *__restrict__ d, int B,
                                                  double *__restrict__ part) {
  double v[1] = {0.0};
  const bool mx[1] = {false};
  const long long n = (long long)B * P.Np;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const long long b = k / P.Np, kk = k % P.Np;
    const int i = (int)(kk % P.Npx), j = (int)(kk / P.Npx);
    const float dv = lap_f(P, y + b * P.Np, i, j) - (float)lap_diag(P, i, j) * in[k];
    d[k] = dv;
    v[0] += (double)dv * dv;
  }
  block_sum<1>(v, mx, part + blockIdx.x);
}
// pass 2: dy = g A d (A is symmetric)
__global__ void __launch_bounds__(256) k_res_grad(const __grid_constant__ DevOps P, const float *__restrict__ d,
                                                  float *__restrict__ dy, float g, int B) {
  const long long n = (long long)B * P.Np;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const long long b = k / P.Np, kk = k % P.Np;
    dy[k] = g * lap_f(P, d + b * P.Np, (int)(kk % P.Npx), (int)(kk / P.Npx));
  }
}

// dZ5[p][ci] = (sum_t W6[t][ci] dy[p - t]) [A5[p][ci] > 0]
__global__ void __launch_bounds__(256) k_bwd_out(const float *__restrict__ dy, const float *__restrict__ w6,
                                                 const bf16 *__restrict__ a5, bf16 *__restrict__ dz, int B, int H,
                                                 int W) {
  __shared__ float ws[kK];
  for (int i = threadIdx.x; i < kK; i += blockDim.x) ws[i] = w6[i];
  __syncthreads();
  const long long n = (long long)B * H * W;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(p % W);
    const int y = (int)((p / W) % H);
    float s[kC];
#pragma unroll
    for (int c = 0; c < kC; ++c) s[c] = 0.0f;
#pragma unroll
    for (int t = 0; t < kTaps; ++t) {
      const int ddx = t % 3 - 1, ddy = t / 3 - 1;
      const int xx = x - ddx, yy = y - ddy;
      if (xx < 0 || xx >= W || yy < 0 || yy >= H) continue;
      const float d = dy[p - (long long)ddy * W - ddx];
#pragma unroll
      for (int c = 0; c < kC; ++c) s[c] = fmaf(ws[t * kC + c], d, s[c]);
    }
    const uint4 *m = reinterpret_cast<const uint4 *>(a5 + p * kC);
    uint4 *dst = reinterpret_cast<uint4 *>(dz + p * kC);
#pragma unroll
    for (int part = 0; part < 4; ++part) {
      float a[8];
      unpack8(m[part], a);
      uint32_t o[4];
#pragma unroll
      for (int e = 0; e < 8; e += 2)
        o[e / 2] = pack2(a[e] > 0.0f ? s[part * 8 + e] : 0.0f, a[e + 1] > 0.0f ? s[part * 8 + e + 1] : 0.0f);
      dst[part] = make_uint4(o[0], o[1], o[2], o[3]);
    }
  }
}

// Weight gradients of the edge layers, thread (t, c) of a 288-thread block
// summing over a contiguous pixel range:
//   LAYER 1: dW1[c][t] = sum_p dZ1[p][c] in[p + t]     (stored as part[t*32 + c])
//   LAYER 6: dW6[t][c] = sum_p dy[p] A5[p + t][c]
template <int LAYER>
__global__ void __launch_bounds__(kK) k_wgrad_edge(const bf16 *__restrict__ dz1, const float *__restrict__ in0,
                                                   const float *__restrict__ dy, const bf16 *__restrict__ a5,
                                                   float *__restrict__ part, int B, int H, int W, long long chunk) {
  const int tid = threadIdx.x, t = tid >> 5, c = tid & 31;
  const int ddy = t / 3 - 1, ddx = t % 3 - 1;
  const long long n = (long long)B * H * W;
  const long long p0 = blockIdx.x * chunk;
  const long long p1 = p0 + chunk < n ? p0 + chunk : n;
  float acc = 0.0f;
  for (long long p = p0; p < p1; ++p) {
    const int x = (int)(p % W);
    const int y = (int)((p / W) % H);
    const int xx = x + ddx, yy = y + ddy;
    if (xx < 0 || xx >= W || yy < 0 || yy >= H) continue;
    const long long q = p + (long long)ddy * W + ddx;
    if (LAYER == 1)
      acc = fmaf(__bfloat162float(dz1[p * kC + c]), in0[q], acc);
    else
      acc = fmaf(dy[p], __bfloat162float(a5[q * kC + c]), acc);
  }
  part[(long long)blockIdx.x * kK + tid] = acc;
}

// Weight gradient of a 32 -> 32 layer on tensor cores: D[co][t, ci] =
// sum_p dZ[p][co] A[p + t][ci].  Block = 9 warps, warp = tap t (M = 32 output
// channels in 2 m-tiles, N = 32 input channels in 4 n-tiles); K = the 128
// pixels of a 16 x 8 tile in 8 steps of one tile row.  Both operands are
// staged channel-major (transposed) in shared memory so that the fragments'
// pixel pairs are adjacent; blocks loop over tiles and write one partial sum.
__global__ void __launch_bounds__(kK) k_wgrad_mid(const bf16 *__restrict__ dz, const bf16 *__restrict__ a,
                                                  float *__restrict__ part, int B, int H, int W, int tiles_x,
                                                  int tiles_y) {
  constexpr int DZS = TW * TH + 8;    // 136
  constexpr int AS = HHT * HWD + 4;   // 184
  __shared__ __align__(16) bf16 sdz[kC * DZS];
  __shared__ __align__(16) bf16 sa[kC * AS];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
  const int dyo = warp / 3, dxo = warp % 3;
  float acc[2][4][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[mt][nt][k] = 0.0f;
  const long long per_field = (long long)tiles_x * tiles_y;
  const long long ntiles = per_field * B;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int b = (int)(tile / per_field);
    const int rem = (int)(tile % per_field);
    const int x0 = (rem % tiles_x) * TW, y0 = (rem / tiles_x) * TH;
    const long long fbase = (long long)b * H * W;
    __syncthreads();
    for (int i = tid; i < TW * TH * 4; i += kK) {
      const int pix = i >> 2, prt = i & 3;
      const int gx = x0 + pix % TW, gy = y0 + pix / TW;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (gx < W && gy < H) v = *reinterpret_cast<const uint4 *>(&dz[(fbase + (long long)gy * W + gx) * kC + prt * 8]);
      const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        sdz[(prt * 8 + 2 * e) * DZS + pix] = __ushort_as_bfloat16((unsigned short)(w4[e] & 0xffffu));
        sdz[(prt * 8 + 2 * e + 1) * DZS + pix] = __ushort_as_bfloat16((unsigned short)(w4[e] >> 16));
      }
    }
    for (int i = tid; i < HHT * HWD * 4; i += kK) {
      const int hp = i >> 2, prt = i & 3;
      const int gy = y0 - 1 + hp / HWD, gx = x0 - 1 + hp % HWD;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (gy >= 0 && gy < H && gx >= 0 && gx < W)
        v = *reinterpret_cast<const uint4 *>(&a[(fbase + (long long)gy * W + gx) * kC + prt * 8]);
      const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        sa[(prt * 8 + 2 * e) * AS + hp] = __ushort_as_bfloat16((unsigned short)(w4[e] & 0xffffu));
        sa[(prt * 8 + 2 * e + 1) * AS + hp] = __ushort_as_bfloat16((unsigned short)(w4[e] >> 16));
      }
    }
    __syncthreads();
#pragma unroll 2
    for (int ks = 0; ks < TH; ++ks) {
      uint32_t af[2][4];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const bf16 *r0 = &sdz[(mt * 16 + g) * DZS + ks * TW + 2 * t4];
        const bf16 *r1 = r0 + 8 * DZS;
        af[mt][0] = *reinterpret_cast<const uint32_t *>(r0);
        af[mt][1] = *reinterpret_cast<const uint32_t *>(r1);
        af[mt][2] = *reinterpret_cast<const uint32_t *>(r0 + 8);
        af[mt][3] = *reinterpret_cast<const uint32_t *>(r1 + 8);
      }
      const int hb = (ks + dyo) * HWD + dxo + 2 * t4;
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const bf16 *s = &sa[(nt * 8 + g) * AS + hb];
        const uint32_t b0 = pack2h(s[0], s[1]);
        const uint32_t b1 = pack2h(s[8], s[9]);
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) mma_bf16(acc[mt][nt], af[mt][0], af[mt][1], af[mt][2], af[mt][3], b0, b1);
      }
    }
  }
  float *dst = part + (long long)blockIdx.x * kSzWm;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int co = mt * 16 + g, ci = nt * 8 + 2 * t4;
      dst[co * kK + warp * kC + ci] = acc[mt][nt][0];
      dst[co * kK + warp * kC + ci + 1] = acc[mt][nt][1];
      dst[(co + 8) * kK + warp * kC + ci] = acc[mt][nt][2];
      dst[(co + 8) * kK + warp * kC + ci + 1] = acc[mt][nt][3];
    }
}

// out[j] = sum over rows of part[row * cols + j] in row order; remap9 maps
// the edge kernel's (t*32 + c) index to W1's [c][t] layout
__global__ void k_reduce_rows(const float *__restrict__ part, int rows, int cols, float *__restrict__ out,
                              int remap9) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cols) return;
  float s = 0.0f;
  for (int r = 0; r < rows; ++r) s += part[(long long)r * cols + j];
  out[remap9 ? (j & 31) * kTaps + (j >> 5) : j] = s;
}

// BF16 copies of the 32 -> 32 weights: forward [co][t][ci] and the
// backward-data form [ci][8 - t][co]
__global__ void k_pack(const float *__restrict__ w, bf16 *__restrict__ wf, bf16 *__restrict__ wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMid * kSzWm) return;
  const int l = i / kSzWm, r = i % kSzWm;
  const int co = r / kK, t = (r / kC) % kTaps, ci = r % kC;
  const bf16 v = __float2bfloat16_rn(w[kOffWm + i]);
  wf[i] = v;
  wb[l * kSzWm + ci * kK + (kTaps - 1 - t) * kC + co] = v;
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, int n, float lr, float b1, float b2, float c1, float c2, float eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// --- inputs from (f, p) --------------------------------------------------------
__global__ void __launch_bounds__(256) k_prep_stats(const __grid_constant__ DevOps P, const double *__restrict__ f,
                                                    const double *__restrict__ p, double *__restrict__ part) {
  double v[2] = {0.0, 0.0};
  const bool mx[2] = {false, false};
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < P.Np; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % P.Npx), j = (int)(k / P.Npx);
    const double s = f[k] / lap_diag(P, i, j);
    v[0] += s * s;
    if (p) v[1] += p[k];
  }
  block_sum<2>(v, mx, part + 2 * blockIdx.x);
}

__global__ void __launch_bounds__(256) k_prep_write(const __grid_constant__ DevOps P, const double *__restrict__ f,
                                                    const double *__restrict__ p, int center,
                                                    const double *__restrict__ stats, float *__restrict__ in,
                                                    float *__restrict__ tgt) {
  const double n = (double)P.Np;
  const double rms = sqrt(stats[0] / n);
  const double inv = rms > 0.0 ? 1.0 / rms : 1.0;
  const double mean = center ? stats[1] / n : 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < P.Np; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % P.Npx), j = (int)(k / P.Npx);
    in[k] = (float)(f[k] / lap_diag(P, i, j) * inv);
    if (tgt) tgt[k] = (float)((p[k] - mean) * inv);
  }
}

// second field of a pair = -first (the odd part of the network needs both)
__global__ void k_negate(float *__restrict__ a, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    a[n + k] = -a[k];
}

// standard normal values from a counter-based generator (splitmix64 of the
// index and the seed, Box-Muller), for the noise fields of training batches
__device__ __forceinline__ double u01(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return ((z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
__global__ void k_gaussian(float *__restrict__ a, long long n, unsigned long long seed) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double u1 = u01(seed ^ (2ull * (unsigned long long)k)), u2 = u01(seed ^ (2ull * (unsigned long long)k + 1));
    a[k] = (float)(sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
  }
}
__global__ void __launch_bounds__(256) k_sumsq_f(const float *__restrict__ a, long long n, double *__restrict__ part) {
  double v[1] = {0.0};
  const bool mx[1] = {false};
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    v[0] += (double)a[k] * a[k];
  block_sum<1>(v, mx, part + blockIdx.x);
}

__global__ void __launch_bounds__(256) k_dots(long long n, const double *__restrict__ x, const double *__restrict__ f,
                                              const double *__restrict__ q, double *__restrict__ part) {
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  const bool mx[4] = {false, false, false, true};
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double xv = x[k], fv = f[k];
    v[0] += xv * fv;
    v[1] += xv * q[k];
    v[2] += fv * fv;
    v[3] = fmax(v[3], fabs(fv));
  }
  block_sum<4>(v, mx, part + 4 * blockIdx.x);
}

__global__ void __launch_bounds__(256) k_resid(long long n, const double *__restrict__ f, const double *__restrict__ q,
                                               double a, double *__restrict__ x, double *__restrict__ r,
                                               double *__restrict__ part) {
  double v[2] = {0.0, 0.0};
  const bool mx[2] = {false, true};
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double rv = f[k] - a * q[k];
    r[k] = rv;
    x[k] *= a;
    v[0] += rv * rv;
    v[1] = fmax(v[1], fabs(rv));
  }
  block_sum<2>(v, mx, part + 2 * blockIdx.x);
}

template <int MODE>
void launch_mid(ins2d_cnn *net, const bf16 *in, const bf16 *wt, const bf16 *mask, bf16 *out, int B, int H, int W,
                cudaStream_t s) {
  if (net->path == INS2D_CNN_PATH_TCGEN05) {
    const int tx = (W + kTcTW - 1) / kTcTW, ty = (H + kTcTH - 1) / kTcTH;
    const long long nt = (long long)tx * ty * B;
    const int grid = (int)std::min<long long>(nt, (long long)kTcBlocksPerSm * net->sms);
    k_conv_mid_tc<MODE><<<grid, 256, kTcSmem, s>>>(in, wt, mask, out, B, H, W, tx, ty, net->flag);
  } else {
    const int tiles_x = (W + TW - 1) / TW, tiles_y = (H + TH - 1) / TH;
    k_conv_mid<MODE><<<dim3(tiles_x, tiles_y, B), 256, 0, s>>>(in, wt, mask, out, H, W);
  }
}

// z = rms * y: the network output rescaled by the rms of its unscaled input
// (stats[0] = sum of squares over n_stat cells), so z = M(r) is homogeneous
// of degree one in r
// x = s (y[k] - y[n + k]) / 2: the odd part of the network over the pair
// (r, -r), rescaled by s = rms of the unscaled input (stats[0] = its sum of
// squares over n_stat cells) when stats is given, so that the result is odd
// and homogeneous of degree one in r
__global__ void k_widen_odd(const float *__restrict__ y, double *__restrict__ x, long long n,
                            const double *__restrict__ stats, double n_stat) {
  const double s = stats ? sqrt(stats[0] / n_stat) : 1.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    x[k] = 0.5 * s * ((double)y[k] - (double)y[n + k]);
}

// flexible CG vector steps (each with its block partials)
__global__ void __launch_bounds__(256) k_fcg_pq(long long n, const double *__restrict__ p,
                                                const double *__restrict__ q, const double *__restrict__ r,
                                                double *__restrict__ part) {
  double v[2] = {0.0, 0.0};
  const bool mx[2] = {false, false};
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double pv = p[k];
    v[0] += pv * q[k];
    v[1] += pv * r[k];
  }
  block_sum<2>(v, mx, part + 2 * blockIdx.x);
}
__global__ void __launch_bounds__(256) k_fcg_update(long long n, double a, double *__restrict__ x,
                                                    double *__restrict__ r, const double *__restrict__ p,
                                                    const double *__restrict__ q, double *__restrict__ part) {
  double v[2] = {0.0, 0.0};
  const bool mx[2] = {false, true};
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    x[k] += a * p[k];
    const double rv = r[k] - a * q[k];
    r[k] = rv;
    v[0] += rv * rv;
    v[1] = fmax(v[1], fabs(rv));
  }
  block_sum<2>(v, mx, part + 2 * blockIdx.x);
}
__global__ void __launch_bounds__(256) k_fcg_zq(long long n, const double *__restrict__ z,
                                                const double *__restrict__ q, double *__restrict__ part) {
  double v[1] = {0.0};
  const bool mx[1] = {false};
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    v[0] += z[k] * q[k];
  block_sum<1>(v, mx, part + blockIdx.x);
}
__global__ void k_fcg_p(long long n, double b, const double *__restrict__ z, double *__restrict__ p) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    p[k] = z[k] + b * p[k];
}

unsigned stride_blocks(long long n, int per_sm = 8) {
  long long b = (n + 255) / 256;
  const long long cap = std::min<long long>(148LL * per_sm, kRedBlocks);
  if (b > cap) b = cap;
  return (unsigned)(b < 1 ? 1 : b);
}

void pack(ins2d_cnn *net, cudaStream_t s) {
  if (net->packed) return;
  k_pack<<<(kMid * kSzWm + 255) / 256, 256, 0, s>>>(net->w, net->wf, net->wb);
  CK(cudaGetLastError());
  net->packed = true;
}

}  // namespace

void check(ins2d_cnn *net, cudaStream_t s);

void reserve(ins2d_cnn *net, long long pixels) {
  if (pixels <= net->cap) return;
  for (auto *&a : net->act) cudaFree(a), a = nullptr;
  for (auto *&a : net->dz) cudaFree(a), a = nullptr;
  cudaFree(net->y);
  cudaFree(net->dy);
  cudaFree(net->dres);
  net->y = net->dy = net->dres = nullptr;
  net->cap = 0;
  const size_t nb = (size_t)pixels * kC * sizeof(bf16);
  for (auto *&a : net->act)
    if (cudaMalloc(&a, nb) != cudaSuccess) throw std::bad_alloc();
  for (auto *&a : net->dz)
    if (cudaMalloc(&a, nb) != cudaSuccess) throw std::bad_alloc();
  if (cudaMalloc(&net->y, pixels * sizeof(float)) != cudaSuccess) throw std::bad_alloc();
  if (cudaMalloc(&net->dy, pixels * sizeof(float)) != cudaSuccess) throw std::bad_alloc();
  if (cudaMalloc(&net->dres, pixels * sizeof(float)) != cudaSuccess) throw std::bad_alloc();
  net->cap = pixels;
}

void forward(ins2d_cnn *net, const float *in, int B, int H, int W, cudaStream_t s) {
  const long long n = (long long)B * H * W;
  reserve(net, n);
  pack(net, s);
  const unsigned gb = stride_blocks(n, 16);
  k_conv_in<<<gb, 256, 0, s>>>(in, net->w + kOffW1, net->act[0], B, H, W);
  for (int l = 0; l < kMid; ++l)
    launch_mid<0>(net, net->act[l], net->wf + l * kSzWm, nullptr, net->act[l + 1], B, H, W, s);
  k_conv_out<<<gb, 256, 0, s>>>(net->act[4], net->w + kOffW6, net->out_scale, net->y, B, H, W);
  CK(cudaGetLastError());
}

// loss (returned, after a stream synchronisation) and the gradient in net->g
double loss_grad(ins2d_cnn *net, const float *in, const float *tgt, int B, int H, int W, cudaStream_t s,
                 const DevOps *P) {
  const long long n = (long long)B * H * W;
  forward(net, in, B, H, W, s);
  const unsigned gb = stride_blocks(n, 16);
  double *part = net->red, *res = net->red + 4 * kRedBlocks;
  const float g = (float)(2.0 / (double)n) * net->out_scale;
  if (P) {
    k_res_loss<<<gb, 256, 0, s>>>(*P, net->y, in, net->dres, B, part);
    k_res_grad<<<gb, 256, 0, s>>>(*P, net->dres, net->dy, g, B);
  } else {
    k_loss<<<gb, 256, 0, s>>>(net->y, tgt, net->dy, g, n, part);
  }
  k_finish<1><<<1, 256, 0, s>>>(part, (int)gb, 0, res);
  // layer 6
  k_bwd_out<<<gb, 256, 0, s>>>(net->dy, net->w + kOffW6, net->act[4], net->dz[0], B, H, W);
  const int eb = (int)std::min<long long>(kWgBlocks, (n + 255) / 256);
  const long long chunk = (n + eb - 1) / eb;
  k_wgrad_edge<6><<<eb, kK, 0, s>>>(nullptr, nullptr, net->dy, net->act[4], net->partials, B, H, W, chunk);
  k_reduce_rows<<<(kK + 255) / 256, 256, 0, s>>>(net->partials, eb, kK, net->g + kOffW6, 0);
  // layers 5..2: dZ_l in dz[cur]; weight gradient from (dZ_l, A_{l-1}); dZ_{l-1}
  const int tiles_x = (W + TW - 1) / TW, tiles_y = (H + TH - 1) / TH;
  const long long ntiles = (long long)tiles_x * tiles_y * B;
  const int wb = (int)std::min<long long>(kWgBlocks, ntiles);
  int cur = 0;
  for (int l = kMid - 1; l >= 0; --l) {
    // layer index l: input act[l], output act[l + 1], gradient dZ in dz[cur]
    k_wgrad_mid<<<wb, kK, 0, s>>>(net->dz[cur], net->act[l], net->partials, B, H, W, tiles_x, tiles_y);
    k_reduce_rows<<<(kSzWm + 255) / 256, 256, 0, s>>>(net->partials, wb, kSzWm, net->g + kOffWm + l * kSzWm, 0);
    launch_mid<1>(net, net->dz[cur], net->wb + l * kSzWm, net->act[l], net->dz[cur ^ 1], B, H, W, s);
    cur ^= 1;
  }
  // layer 1
  k_wgrad_edge<1><<<eb, kK, 0, s>>>(net->dz[cur], in, nullptr, nullptr, net->partials, B, H, W, chunk);
  k_reduce_rows<<<(kK + 255) / 256, 256, 0, s>>>(net->partials, eb, kK, net->g + kOffW1, 1);
  CK(cudaGetLastError());
  double h = 0.0;
  CK(cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  check(net, s);
  return h / (double)n;
}

void check(ins2d_cnn *net, cudaStream_t s) {
  unsigned f = 0;
  CK(cudaMemcpyAsync(&f, net->flag, sizeof f, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (f) {
    CK(cudaMemsetAsync(net->flag, 0, sizeof(unsigned), s));
    throw CudaError("cnn: a tensor-core wait gave up (tcgen05 MMA did not complete)");
  }
}

void adam(ins2d_cnn *net, float lr, cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f;
  net->adam_t += 1;
  const float c1 = 1.0f - std::pow(b1, (float)net->adam_t), c2 = 1.0f - std::pow(b2, (float)net->adam_t);
  k_adam<<<(kNParam + 255) / 256, 256, 0, s>>>(net->w, net->g, net->m, net->v, kNParam, lr, b1, b2, c1, c2, 1e-8f);
  CK(cudaGetLastError());
  net->packed = false;
}

void prepare(const DevOps &P, const double *f, const double *p, int center, float *in, float *tgt, double *red,
             cudaStream_t s) {
  const unsigned gb = stride_blocks(P.Np);
  double *part = red, *res = red + 4 * kRedBlocks;
  k_prep_stats<<<gb, 256, 0, s>>>(P, f, p, part);
  k_finish<2><<<1, 256, 0, s>>>(part, (int)gb, 0, res);
  k_prep_write<<<gb, 256, 0, s>>>(P, f, p, center, res, in, tgt);
  CK(cudaGetLastError());
}

namespace {
// the network's odd part applied to the prepared field v (f or r):
// out = scaled (N(v) - N(-v)) / 2, one forward pass over the pair
void apply_odd(ins2d_cnn *net, const DevOps &P, const double *v, double *out, bool rescale, cudaStream_t s) {
  reserve(net, 2 * P.Np);
  if (net->in1_cap < 2 * P.Np) {
    cudaFree(net->in1);
    net->in1 = nullptr;
    net->in1_cap = 0;
    if (cudaMalloc(&net->in1, 2 * P.Np * sizeof(float)) != cudaSuccess) throw std::bad_alloc();
    net->in1_cap = 2 * P.Np;
  }
  prepare(P, v, nullptr, 0, net->in1, nullptr, net->red, s);
  k_negate<<<stride_blocks(P.Np), 256, 0, s>>>(net->in1, P.Np);
  forward(net, net->in1, 2, P.Npy, P.Npx, s);
  k_widen_odd<<<stride_blocks(P.Np), 256, 0, s>>>(net->y, out, P.Np, rescale ? net->red + 4 * kRedBlocks : nullptr,
                                                   (double)P.Np);
  CK(cudaGetLastError());
}
}  // namespace

void guess(ins2d_cnn *net, const DevOps &P, const double *f, double *x0, cudaStream_t s) {
  apply_odd(net, P, f, x0, false, s);
}

void precond(ins2d_cnn *net, const DevOps &P, const double *r, double *z, cudaStream_t s) {
  apply_odd(net, P, r, z, true, s);
}

namespace {
void finish_read(int nq, unsigned gb, int max_mask, double *red, double *d, cudaStream_t s) {
  double *part = red, *res = red + 4 * kRedBlocks;
  if (nq == 1)
    k_finish<1><<<1, 256, 0, s>>>(part, (int)gb, max_mask, res);
  else
    k_finish<2><<<1, 256, 0, s>>>(part, (int)gb, max_mask, res);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(d, res, nq * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
}
}  // namespace

void fcg_pq(long long n, const double *p, const double *q, const double *r, double *red, double d[2],
            cudaStream_t s) {
  const unsigned gb = stride_blocks(n);
  k_fcg_pq<<<gb, 256, 0, s>>>(n, p, q, r, red);
  finish_read(2, gb, 0, red, d, s);
}
void fcg_update(long long n, double a, double *x, double *r, const double *p, const double *q, double *red,
                double d[2], cudaStream_t s) {
  const unsigned gb = stride_blocks(n);
  k_fcg_update<<<gb, 256, 0, s>>>(n, a, x, r, p, q, red);
  finish_read(2, gb, 2, red, d, s);
}
double fcg_zq(long long n, const double *z, const double *q, double *red, cudaStream_t s) {
  const unsigned gb = stride_blocks(n);
  k_fcg_zq<<<gb, 256, 0, s>>>(n, z, q, red);
  double d = 0.0;
  finish_read(1, gb, 0, red, &d, s);
  return d;
}
void fcg_p(long long n, double b, const double *z, double *p, cudaStream_t s) {
  k_fcg_p<<<stride_blocks(n), 256, 0, s>>>(n, b, z, p);
  CK(cudaGetLastError());
}

void negate_tail(float *a, long long n, cudaStream_t s) {
  k_negate<<<stride_blocks(n), 256, 0, s>>>(a, n);
  CK(cudaGetLastError());
}

void gaussian(float *a, long long n, uint64_t seed, cudaStream_t s) {
  k_gaussian<<<stride_blocks(n), 256, 0, s>>>(a, n, (unsigned long long)seed);
  CK(cudaGetLastError());
}

double sumsq(const float *a, long long n, double *red, cudaStream_t s) {
  const unsigned gb = stride_blocks(n);
  double *part = red, *res = red + 4 * kRedBlocks;
  k_sumsq_f<<<gb, 256, 0, s>>>(a, n, part);
  k_finish<1><<<1, 256, 0, s>>>(part, (int)gb, 0, res);
  CK(cudaGetLastError());
  double h = 0.0;
  CK(cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return h;
}

void dots(long long n, const double *x, const double *f, const double *q, double *red, double d[4], cudaStream_t s) {
  const unsigned gb = stride_blocks(n);
  double *part = red, *res = red + 4 * kRedBlocks;
  k_dots<<<gb, 256, 0, s>>>(n, x, f, q, part);
  k_finish<4><<<1, 256, 0, s>>>(part, (int)gb, 8, res);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(d, res, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
}

void residual(long long n, const double *f, const double *q, double a, double *x, double *r, double *red,
              double d[2], cudaStream_t s) {
  const unsigned gb = stride_blocks(n);
  double *part = red, *res = red + 4 * kRedBlocks;
  k_resid<<<gb, 256, 0, s>>>(n, f, q, a, x, r, part);
  k_finish<2><<<1, 256, 0, s>>>(part, (int)gb, 2, res);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(d, res, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
}

size_t red_doubles() { return 4 * (size_t)kRedBlocks + 8; }

}  // namespace cnn
}  // namespace ins2d

// ---------------------------------------------------------------------------
// C-ABI: the network object
using namespace ins2d;
using cnn::CudaError;

namespace {

int cnn_fail(ins2d_cnn *n, int code, const std::string &msg) {
  if (n) n->err = msg;
  return code;
}

// He-normal initial weights from a seeded generator (splitmix64 + Box-Muller)
void init_weights(std::vector<float> &w, uint64_t seed) {
  uint64_t st = seed;
  auto next = [&]() {
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return ((z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  };
  auto normal = [&]() {
    const double u1 = next(), u2 = next();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  };
  w.assign(cnn::kNParam, 0.0f);
  for (int i = 0; i < cnn::kOffWm; ++i) w[i] = (float)(normal() * std::sqrt(2.0 / cnn::kTaps));
  for (int i = cnn::kOffWm; i < cnn::kOffW6; ++i) w[i] = (float)(normal() * std::sqrt(2.0 / cnn::kK));
  for (int i = cnn::kOffW6; i < cnn::kNParam; ++i) w[i] = (float)(normal() * std::sqrt(1.0 / cnn::kK));
}

bool dev_ptr(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int check_shape(ins2d_cnn *n, const void *a, const void *b, int32_t B, int32_t H, int32_t W) {
  if (B < 1 || H < 1 || W < 1) return cnn_fail(n, INS2D_EINVAL, "cnn: batch and field sizes must be positive");
  if ((long long)B * H * W > (1LL << 31) / cnn::kC)
    return cnn_fail(n, INS2D_EINVAL, "cnn: B*H*W too large (at most 2^26 pixels per call)");
  if (H > 8 * 65535 || B > 65535) return cnn_fail(n, INS2D_EINVAL, "cnn: H or B beyond the launch limits");
  if (!a || !dev_ptr(a) || (b && !dev_ptr(b)))
    return cnn_fail(n, INS2D_EINVAL, "cnn: inputs, targets and outputs must be device arrays");
  return INS2D_OK;
}

}  // namespace

extern "C" {

int ins2d_cnn_create(int32_t device, uint64_t seed, ins2d_cnn **out) {
  if (!out) return INS2D_EINVAL;
  *out = nullptr;
  ins2d_cnn *n = new (std::nothrow) ins2d_cnn();
  if (!n) return INS2D_ENOMEM;
  try {
    n->device = device;
    DeviceGuard dg(device);
    CK(dg.err);
    const size_t pb = cnn::kNParam * sizeof(float);
    for (float **p : {&n->w, &n->g, &n->m, &n->v})
      if (cudaMalloc(p, pb) != cudaSuccess) throw std::bad_alloc();
    if (cudaMalloc(&n->wf, cnn::kMid * cnn::kSzWm * sizeof(__nv_bfloat16)) != cudaSuccess) throw std::bad_alloc();
    if (cudaMalloc(&n->wb, cnn::kMid * cnn::kSzWm * sizeof(__nv_bfloat16)) != cudaSuccess) throw std::bad_alloc();
    if (cudaMalloc(&n->partials, (size_t)cnn::kWgBlocks * cnn::kSzWm * sizeof(float)) != cudaSuccess)
      throw std::bad_alloc();
    if (cudaMalloc(&n->red, cnn::red_doubles() * sizeof(double)) != cudaSuccess) throw std::bad_alloc();
    if (cudaMalloc(&n->flag, sizeof(unsigned)) != cudaSuccess) throw std::bad_alloc();
    CK(cudaMemset(n->flag, 0, sizeof(unsigned)));
    CK(cudaDeviceGetAttribute(&n->sms, cudaDevAttrMultiProcessorCount, device));
    std::vector<float> w;
    init_weights(w, seed);
    CK(cudaMemcpy(n->w, w.data(), pb, cudaMemcpyHostToDevice));
    CK(cudaMemset(n->m, 0, pb));
    CK(cudaMemset(n->v, 0, pb));
    CK(cudaMemset(n->g, 0, pb));
  } catch (const std::bad_alloc &) {
    ins2d_cnn_destroy(n);
    return INS2D_ENOMEM;
  } catch (const std::exception &) {
    ins2d_cnn_destroy(n);
    return INS2D_ECUDA;
  }
  *out = n;
  return INS2D_OK;
}

int ins2d_cnn_destroy(ins2d_cnn *n) {
  if (!n) return INS2D_OK;
  DeviceGuard dg(n->device);
  for (float *p : {n->w, n->g, n->m, n->v, n->y, n->dy, n->dres, n->in1, n->partials}) cudaFree(p);
  cudaFree(n->wf);
  cudaFree(n->wb);
  cudaFree(n->red);
  cudaFree(n->flag);
  for (auto *a : n->act) cudaFree(a);
  for (auto *a : n->dz) cudaFree(a);
  delete n;
  return INS2D_OK;
}

const char *ins2d_cnn_last_error(const ins2d_cnn *n) { return n ? n->err.c_str() : "null network"; }

int ins2d_cnn_set_stream(ins2d_cnn *n, void *stream) {
  if (!n) return INS2D_EINVAL;
  n->stream = (cudaStream_t)stream;
  return INS2D_OK;
}

int ins2d_cnn_set_path(ins2d_cnn *n, int32_t path) {
  if (!n) return INS2D_EINVAL;
  if (path != INS2D_CNN_PATH_TCGEN05 && path != INS2D_CNN_PATH_MMA_SYNC)
    return cnn_fail(n, INS2D_EINVAL, "cnn_set_path: unknown tensor-core path");
  n->path = path;
  return INS2D_OK;
}

int ins2d_cnn_get_params(ins2d_cnn *n, float *w, float *out_scale) {
  if (!n) return INS2D_EINVAL;
  try {
    DeviceGuard dg(n->device);
    CK(dg.err);
    if (w) {
      CK(cudaMemcpyAsync(w, n->w, cnn::kNParam * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
      CK(cudaStreamSynchronize(n->stream));
    }
    if (out_scale) *out_scale = n->out_scale;
  } catch (const std::exception &e) {
    return cnn_fail(n, INS2D_ECUDA, e.what());
  }
  return INS2D_OK;
}

int ins2d_cnn_set_params(ins2d_cnn *n, const float *w, float out_scale) {
  if (!n) return INS2D_EINVAL;
  if (!(out_scale > 0.0f) || !std::isfinite(out_scale)) return cnn_fail(n, INS2D_EINVAL, "cnn: out_scale must be > 0");
  try {
    DeviceGuard dg(n->device);
    CK(dg.err);
    if (w) {
      CK(cudaMemcpyAsync(n->w, w, cnn::kNParam * sizeof(float), cudaMemcpyHostToDevice, n->stream));
      CK(cudaStreamSynchronize(n->stream));
      n->packed = false;
    }
    n->out_scale = out_scale;
  } catch (const std::exception &e) {
    return cnn_fail(n, INS2D_ECUDA, e.what());
  }
  return INS2D_OK;
}

int ins2d_cnn_forward(ins2d_cnn *n, const float *in, float *y, int32_t B, int32_t H, int32_t W) {
  if (!n) return INS2D_EINVAL;
  int rc = check_shape(n, in, y, B, H, W);
  if (rc) return rc;
  if (!y) return cnn_fail(n, INS2D_EINVAL, "cnn_forward: null output");
  try {
    DeviceGuard dg(n->device);
    CK(dg.err);
    cnn::forward(n, in, B, H, W, n->stream);
    CK(cudaMemcpyAsync(y, n->y, (size_t)B * H * W * sizeof(float), cudaMemcpyDeviceToDevice, n->stream));
    CK(cudaStreamSynchronize(n->stream));
    cnn::check(n, n->stream);
  } catch (const std::bad_alloc &) {
    return cnn_fail(n, INS2D_ENOMEM, "cnn_forward: out of device memory");
  } catch (const std::exception &e) {
    return cnn_fail(n, INS2D_ECUDA, e.what());
  }
  return INS2D_OK;
}

int ins2d_cnn_get_activations(ins2d_cnn *n, int32_t layer, int64_t pixels, uint16_t *out) {
  if (!n) return INS2D_EINVAL;
  if (layer < 1 || layer > 5 || !out || pixels < 1 || pixels > n->cap)
    return cnn_fail(n, INS2D_EINVAL, "cnn_get_activations: layer 1..5, pixels of the last forward pass");
  try {
    DeviceGuard dg(n->device);
    CK(dg.err);
    CK(cudaMemcpyAsync(out, n->act[layer - 1], (size_t)pixels * cnn::kC * sizeof(uint16_t), cudaMemcpyDeviceToHost,
                       n->stream));
    CK(cudaStreamSynchronize(n->stream));
  } catch (const std::exception &e) {
    return cnn_fail(n, INS2D_ECUDA, e.what());
  }
  return INS2D_OK;
}

int ins2d_cnn_loss_grad(ins2d_cnn *n, const float *in, const float *tgt, int32_t B, int32_t H, int32_t W,
                        double *loss, float *grad) {
  if (!n) return INS2D_EINVAL;
  int rc = check_shape(n, in, tgt, B, H, W);
  if (rc) return rc;
  if (!tgt) return cnn_fail(n, INS2D_EINVAL, "cnn_loss_grad: null targets");
  try {
    DeviceGuard dg(n->device);
    CK(dg.err);
    const double l = cnn::loss_grad(n, in, tgt, B, H, W, n->stream, nullptr);
    if (loss) *loss = l;
    if (grad) {
      CK(cudaMemcpyAsync(grad, n->g, cnn::kNParam * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
      CK(cudaStreamSynchronize(n->stream));
    }
  } catch (const std::bad_alloc &) {
    return cnn_fail(n, INS2D_ENOMEM, "cnn_loss_grad: out of device memory");
  } catch (const std::exception &e) {
    return cnn_fail(n, INS2D_ECUDA, e.what());
  }
  return INS2D_OK;
}

int ins2d_cnn_train_step(ins2d_cnn *n, const float *in, const float *tgt, int32_t B, int32_t H, int32_t W, float lr,
                         double *loss) {
  if (!n) return INS2D_EINVAL;
  int rc = check_shape(n, in, tgt, B, H, W);
  if (rc) return rc;
  if (!tgt) return cnn_fail(n, INS2D_EINVAL, "cnn_train_step: null targets");
  if (!(lr > 0.0f) || !std::isfinite(lr)) return cnn_fail(n, INS2D_EINVAL, "cnn_train_step: lr must be > 0");
  try {
    DeviceGuard dg(n->device);
    CK(dg.err);
    const double l = cnn::loss_grad(n, in, tgt, B, H, W, n->stream, nullptr);
    if (!std::isfinite(l)) return cnn_fail(n, INS2D_ENONFINITE, "cnn_train_step: non-finite loss");
    cnn::adam(n, lr, n->stream);
    if (loss) *loss = l;
  } catch (const std::bad_alloc &) {
    return cnn_fail(n, INS2D_ENOMEM, "cnn_train_step: out of device memory");
  } catch (const std::exception &e) {
    return cnn_fail(n, INS2D_ECUDA, e.what());
  }
  return INS2D_OK;
}

}  // extern "C"
