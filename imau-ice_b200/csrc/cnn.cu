// cnn.cu -- the learned warm start of the DIVA solve (include/diva_cnn.h): a small
// encoder-decoder network on the a-grid, trained on solutions of this solver, whose
// prediction sets u_vav_cx / v_vav_cy before the viscosity iteration starts.
//
// Every 3x3 convolution is an implicit GEMM on the 5th-generation tensor cores:
//   forward  D[pixel][cout] = sum_(tap,cin)  X[pixel+tap][cin]     W[tap][cout][cin]
//   dgrad    D[pixel][cin]  = sum_(tap,cout) dZ[pixel-tap][cout]   W[tap][cout][cin]
//   wgrad    D[cout][cin]   = sum_pixel      dZ[pixel][cout]       X[pixel+tap][cin]
// (dZ = dY masked by the ReLU of the layer's output).  A CTA of 128 threads owns one
// 128-row tile of D in tensor memory (FP32 accumulators, tcgen05.alloc), its threads
// gather the BF16 operand tiles for one tap (or one 64-pixel slice) from HBM into
// shared memory in the no-swizzle K-major core-matrix layout -- 8 rows x 16 bytes
// per core matrix, rows 16 bytes apart, K halves LBO apart, 8-row groups SBO apart --
// while the tensor core works on the other of two stages; one elected thread issues
// the tcgen05.mma instructions (M = 128, K = 16 each) and commits them to the stage's
// mbarrier.  The epilogue reads the accumulators with tcgen05.ld (warp w owns lanes
// 32w..32w+31 = rows), adds the bias and applies the ReLU, and stores BF16 (forward,
// dgrad) or FP32 partial sums (wgrad, one slice of pixels per CTA, reduced in a fixed
// order afterwards so that training is deterministic).
//
// Pooling, upsampling + concatenation, the 1x1 head with the masked squared-error
// loss, and Adam are elementwise or reduction kernels on CUDA cores.  Every mbarrier
// wait is bounded; on time-out the kernel raises the network's error flag and frees
// its tensor memory, and the host returns DIVA_TIMEOUT.
#include <cuda_bf16.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>
#include "ctx.hpp"
#include "../../include/diva_cnn.h"

namespace diva {
namespace cnn {

using bf16 = __nv_bfloat16;

constexpr int kInC = 16;            // input channels (8 used)
constexpr double kVelScale = 10.0;  // m/yr; outputs are asinh(u / kVelScale)
constexpr long kSpin = 1L << 22;    // mbarrier polls before a wait gives up
constexpr int kPixChunk = 64;       // wgrad K slice (pixels) per stage

// ---------------------------------------------------------------------------
// PTX wrappers (sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
  for (long it = 0; it < kSpin; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// D[tmem] (+)= A[smem] * B[smem]^T, both K-major; acc = 0 overwrites D
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
// 16 consecutive FP32 columns of this thread's lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// Shared-memory matrix descriptor, no swizzle: start, leading (K) and stride (8-row)
// byte offsets in 16-byte units, descriptor version 1 (bit 46).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor, kind::f16: D FP32 (bits 4-5 = 1), A and B BF16 (bits 7-9,
// 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

template <int N>
__host__ __device__ constexpr int tmem_cols() {
  return N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
}

// zero the lanes of v whose BF16 gate value is not > 0 (ReLU derivative)
__device__ __forceinline__ uint4 relu_gate(uint4 v, uint4 g) {
  uint32_t* pv = &v.x;
  const uint32_t* pg = &g.x;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint32_t m = 0;
    if ((int16_t)(pg[q] & 0xFFFFu) > 0) m |= 0x0000FFFFu;
    if ((int16_t)(pg[q] >> 16) > 0) m |= 0xFFFF0000u;
    pv[q] &= m;
  }
  return v;
}

__device__ __forceinline__ unsigned char* align1024(unsigned char* p) {
  return reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

// Occupancy guard: dynamic shared memory large enough that the CTAs resident on one
// SM never ask for more than its 512 tensor-memory columns together.
__host__ constexpr int smem_floor(int ncols) { return ncols >= 128 ? 47 * 1024 : ncols >= 64 ? 27 * 1024 : 0; }

// ---------------------------------------------------------------------------
// forward / dgrad 3x3 convolution
// ---------------------------------------------------------------------------
struct ConvArgs {
  const bf16* x;     // [n][H][W][KC]: forward input, or dY of the layer (dgrad)
  const bf16* gate;  // dgrad: the layer's forward output [n][H][W][KC]
  const bf16* w;     // forward: W [9][COUT][CIN]; dgrad: W^T [9][CIN][COUT]
  const float* bias; // forward: [COUT]
  bf16* y;           // [n][H][W][NO]
  int n, H, W, relu;
  int* err;
};

template <int KC, int NO>
__host__ __device__ constexpr int conv_smem() {
  return 2 * (128 * KC * 2 + NO * KC * 2) + 64 + 1024;
}

template <int KC, int NO, bool DGRAD>
__global__ void __launch_bounds__(128) k_conv3x3(ConvArgs a) {
  static_assert(KC % 16 == 0 && NO % 16 == 0 && NO <= 128, "tile shape");
  constexpr int A_BYTES = 128 * KC * 2, B_BYTES = NO * KC * 2, STAGE = A_BYTES + B_BYTES;
  constexpr int NCOL = tmem_cols<NO>();
  constexpr uint32_t IDESC = idesc_bf16(128, NO);
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = align1024(smem_raw);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + 2 * STAGE);
  uint32_t* taddr_s = reinterpret_cast<uint32_t*>(bar + 2);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int H = a.H, W = a.W;
  const long npix = (long)a.n * H * W;
  const long p = (long)blockIdx.x * 128 + tid;  // this thread's row of D
  const bool pin = p < npix;
  int pb = 0, py = 0, px = 0;
  if (pin) {
    px = (int)(p % W);
    const long q = p / W;
    py = (int)(q % H);
    pb = (int)(q / H);
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  if (warp == 0) tc_alloc(taddr_s, NCOL);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *taddr_s;

  bool ok = true;
  for (int t = 0; t < 9; ++t) {
    const int s = t & 1;
    unsigned char* As = sm + s * STAGE;
    unsigned char* Bs = As + A_BYTES;
    if (t >= 2 && !mbar_wait(&bar[s], ((t - 2) >> 1) & 1)) ok = false;  // stage free again
    int dy = t / 3 - 1, dx = t % 3 - 1;
    if (DGRAD) { dy = -dy; dx = -dx; }
    const int yy = py + dy, xx = px + dx;
    const bool in = pin && yy >= 0 && yy < H && xx >= 0 && xx < W;
    const long src = (((long)pb * H + yy) * W + xx) * KC;
#pragma unroll 4
    for (int kc = 0; kc < KC / 8; ++kc) {
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (in) {
        v = *reinterpret_cast<const uint4*>(a.x + src + kc * 8);
        if (DGRAD) v = relu_gate(v, *reinterpret_cast<const uint4*>(a.gate + src + kc * 8));
      }
      *reinterpret_cast<uint4*>(As + kc * 2048 + tid * 16) = v;
    }
    // B(n, k) = w[t][n][k]: forward, W[t][cout][cin]; dgrad, the transposed copy
    // W^T[t][cin][cout] (k_transpose_w), so both stage contiguous 16-byte rows
    for (int c = tid; c < NO * (KC / 8); c += 128) {
      const int n = c % NO, kc = c / NO;
      const uint4 v = *reinterpret_cast<const uint4*>(a.w + ((long)t * NO + n) * KC + kc * 8);
      *reinterpret_cast<uint4*>(Bs + kc * (NO * 16) + n * 16) = v;
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int k = 0; k < KC / 16; ++k) {
        const uint64_t da = sdesc(smem_u32(As) + 2 * k * 2048, 2048, 128);
        const uint64_t db = sdesc(smem_u32(Bs) + 2 * k * (NO * 16), NO * 16, 128);
        tc_mma(tmem, da, db, IDESC, (t > 0 || k > 0) ? 1u : 0u);
      }
      tc_commit(&bar[s]);
    }
  }
  if (!mbar_wait(&bar[0], 0)) ok = false;  // tap 8: fifth phase of barrier 0
  tc_fence_after();
  ok = __syncthreads_and(ok);
  if (ok) {
#pragma unroll 1
    for (int n0 = 0; n0 < NO; n0 += 16) {
      float v[16];
      tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)n0, v);
      if (pin) {
        __align__(16) bf16 o[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          float f = v[q];
          if (!DGRAD) {
            f += a.bias[n0 + q];
            if (a.relu) f = fmaxf(f, 0.0f);
          }
          o[q] = __float2bfloat16_rn(f);
        }
        uint4* dst = reinterpret_cast<uint4*>(a.y + p * NO + n0);
        dst[0] = reinterpret_cast<const uint4*>(o)[0];
        dst[1] = reinterpret_cast<const uint4*>(o)[1];
      }
    }
  } else if (tid == 0) {
    atomicExch(a.err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tc_dealloc(tmem, NCOL);
  }
}

// ---------------------------------------------------------------------------
// wgrad: D[cout (rows, padded to 128)][cin] over a slice of pixels, per tap
// ---------------------------------------------------------------------------
struct WgradArgs {
  const bf16* x;     // the layer's input [n][H][W][CI]
  const bf16* dy;    // gradient of the layer's output [n][H][W][CO]
  const bf16* gate;  // the layer's output (ReLU mask)
  float* part;       // [nsplit][9][CO][CI]
  int n, H, W, nsplit;
  int* err;
};

template <int CI>
__host__ __device__ constexpr int wgrad_smem() {
  return 2 * (128 * kPixChunk * 2 + CI * kPixChunk * 2) + 64 + 1024;
}

template <int CI, int CO>
__global__ void __launch_bounds__(128) k_conv3x3_wgrad(WgradArgs a) {
  static_assert(CI % 16 == 0 && CO % 8 == 0 && CO <= 128 && CI <= 128, "tile shape");
  constexpr int A_BYTES = 128 * kPixChunk * 2, B_BYTES = CI * kPixChunk * 2, STAGE = A_BYTES + B_BYTES;
  constexpr int NCOL = tmem_cols<CI>();
  constexpr uint32_t IDESC = idesc_bf16(128, CI);
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = align1024(smem_raw);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + 2 * STAGE);
  uint32_t* taddr_s = reinterpret_cast<uint32_t*>(bar + 2);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int t = blockIdx.y, split = blockIdx.x;
  const int dy = t / 3 - 1, dx = t % 3 - 1;
  const int H = a.H, W = a.W;
  const long npix = (long)a.n * H * W;
  const long nchunk = (npix + kPixChunk - 1) / kPixChunk;
  const long per = (nchunk + a.nsplit - 1) / a.nsplit;
  const long c0 = split * per, c1 = c0 + per < nchunk ? c0 + per : nchunk;
  const int nloc = c1 > c0 ? (int)(c1 - c0) : 0;

  // rows CO..127 of A stay zero in both stages
  if constexpr (CO < 128) {
    constexpr int PAD = 128 - CO;
    for (int i = tid; i < 2 * PAD * (kPixChunk / 8); i += 128) {
      const int st = i / (PAD * (kPixChunk / 8));
      const int r = i % (PAD * (kPixChunk / 8));
      const int m = CO + r % PAD, kc = r / PAD;
      *reinterpret_cast<uint4*>(sm + st * STAGE + kc * 2048 + m * 16) = make_uint4(0u, 0u, 0u, 0u);
    }
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  if (warp == 0) tc_alloc(taddr_s, NCOL);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *taddr_s;

  bool ok = true;
  for (int c = 0; c < nloc; ++c) {
    const int s = c & 1;
    unsigned char* As = sm + s * STAGE;
    unsigned char* Bs = As + A_BYTES;
    if (c >= 2 && !mbar_wait(&bar[s], ((c - 2) >> 1) & 1)) ok = false;
    const long pbase = (c0 + c) * kPixChunk;
    // A(m = cout, k = pixel) = dY * (gate > 0)
    for (int i = tid; i < kPixChunk * (CO / 8); i += 128) {
      const int kk = i % kPixChunk, mc = i / kPixChunk;
      const long p = pbase + kk;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (p < npix)
        v = relu_gate(*reinterpret_cast<const uint4*>(a.dy + p * CO + mc * 8),
                      *reinterpret_cast<const uint4*>(a.gate + p * CO + mc * 8));
      const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
      for (int q = 0; q < 8; ++q)
        *reinterpret_cast<bf16*>(As + (kk >> 3) * 2048 + (mc * 8 + q) * 16 + (kk & 7) * 2) = e[q];
    }
    // B(n = cin, k = pixel) = X[pixel + tap]
    for (int i = tid; i < kPixChunk * (CI / 8); i += 128) {
      const int kk = i % kPixChunk, nc = i / kPixChunk;
      const long p = pbase + kk;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (p < npix) {
        const int px = (int)(p % W);
        const long q = p / W;
        const int py = (int)(q % H), pb = (int)(q / H);
        const int yy = py + dy, xx = px + dx;
        if (yy >= 0 && yy < H && xx >= 0 && xx < W)
          v = *reinterpret_cast<const uint4*>(a.x + (((long)pb * H + yy) * W + xx) * CI + nc * 8);
      }
      const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
      for (int q = 0; q < 8; ++q)
        *reinterpret_cast<bf16*>(Bs + (kk >> 3) * (CI * 16) + (nc * 8 + q) * 16 + (kk & 7) * 2) = e[q];
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int k = 0; k < kPixChunk / 16; ++k) {
        const uint64_t da = sdesc(smem_u32(As) + 2 * k * 2048, 2048, 128);
        const uint64_t db = sdesc(smem_u32(Bs) + 2 * k * (CI * 16), CI * 16, 128);
        tc_mma(tmem, da, db, IDESC, (c > 0 || k > 0) ? 1u : 0u);
      }
      tc_commit(&bar[s]);
    }
  }
  if (nloc > 0 && !mbar_wait(&bar[(nloc - 1) & 1], ((nloc - 1) >> 1) & 1)) ok = false;
  tc_fence_after();
  ok = __syncthreads_and(ok);
  const int m = warp * 32 + (tid & 31);
  float* dst = a.part + (((long)split * 9 + t) * CO + m) * CI;
  if (ok) {
#pragma unroll 1
    for (int n0 = 0; n0 < CI; n0 += 16) {
      float v[16];
      if (nloc > 0) {
        tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)n0, v);
      } else {
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = 0.0f;
      }
      if (m < CO) {
#pragma unroll
        for (int q = 0; q < 16; ++q) dst[n0 + q] = v[q];
      }
    }
  } else if (tid == 0) {
    atomicExch(a.err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tc_dealloc(tmem, NCOL);
  }
}

// ---------------------------------------------------------------------------
// reductions, elementwise layers, head + loss, Adam
// ---------------------------------------------------------------------------
// out[c] = sum over r of part[r][c], r in order (deterministic)
__global__ void k_sum_rows(const float* part, int nrows, int ncols, float* out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncols) return;
  float s = 0.0f;
  for (int r = 0; r < nrows; ++r) s += part[(long)r * ncols + c];
  out[c] = s;
}

// per-block partial sums of dZ = dY * (Y > 0) over a slice of pixels, one thread per channel
__global__ void k_bias_part(const bf16* dy, const bf16* gate, long npix, int C, int nblk, float* part) {
  const int c = threadIdx.x;
  if (c >= C) return;
  const long per = (npix + nblk - 1) / nblk;
  const long p0 = blockIdx.x * per, p1 = p0 + per < npix ? p0 + per : npix;
  float s = 0.0f;
  for (long p = p0; p < p1; ++p) {
    const float g = __bfloat162float(gate[p * C + c]);
    if (g > 0.0f) s += __bfloat162float(dy[p * C + c]);
  }
  part[(long)blockIdx.x * C + c] = s;
}

// 2x2 average pool, 8 channels per thread
__global__ void k_pool(const bf16* x, bf16* y, int n, int H, int W, int C) {
  const int H2 = H / 2, W2 = W / 2, C8 = C / 8;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)n * H2 * W2 * C8) return;
  const int c8 = (int)(i % C8);
  long q = i / C8;
  const int X = (int)(q % W2);
  q /= W2;
  const int Y = (int)(q % H2), b = (int)(q / H2);
  float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int d = 0; d < 4; ++d) {
    const long src = (((long)b * H + 2 * Y + (d >> 1)) * W + 2 * X + (d & 1)) * C + c8 * 8;
    const uint4 v = *reinterpret_cast<const uint4*>(x + src);
    const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
    for (int k = 0; k < 8; ++k) s[k] += __bfloat162float(e[k]);
  }
  __align__(16) bf16 o[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) o[k] = __float2bfloat16_rn(0.25f * s[k]);
  *reinterpret_cast<uint4*>(y + (((long)b * H2 + Y) * W2 + X) * C + c8 * 8) = *reinterpret_cast<uint4*>(o);
}

// g_hi += 0.25 * g_lo (nearest), the adjoint of the 2x2 average pool
__global__ void k_pool_bwd_add(const bf16* glo, bf16* ghi, int n, int H, int W, int C) {
  const int C8 = C / 8;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)n * H * W * C8) return;
  const int c8 = (int)(i % C8);
  long q = i / C8;
  const int x = (int)(q % W);
  q /= W;
  const int y = (int)(q % H), b = (int)(q / H);
  const long dst = (((long)b * H + y) * W + x) * C + c8 * 8;
  const long src = (((long)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c8 * 8;
  uint4 vh = *reinterpret_cast<const uint4*>(ghi + dst);
  const uint4 vl = *reinterpret_cast<const uint4*>(glo + src);
  bf16* eh = reinterpret_cast<bf16*>(&vh);
  const bf16* el = reinterpret_cast<const bf16*>(&vl);
#pragma unroll
  for (int k = 0; k < 8; ++k) eh[k] = __float2bfloat16_rn(__bfloat162float(eh[k]) + 0.25f * __bfloat162float(el[k]));
  *reinterpret_cast<uint4*>(ghi + dst) = vh;
}

// out[..][0:C1] = lo (nearest x2), out[..][C1:C1+C2] = skip
__global__ void k_upcat(const bf16* lo, const bf16* skip, bf16* out, int n, int H, int W, int C1, int C2) {
  const int C = C1 + C2, C8 = C / 8;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)n * H * W * C8) return;
  const int c8 = (int)(i % C8);
  long q = i / C8;
  const int x = (int)(q % W);
  q /= W;
  const int y = (int)(q % H), b = (int)(q / H);
  const int c = c8 * 8;
  uint4 v;
  if (c < C1)
    v = *reinterpret_cast<const uint4*>(lo + (((long)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C1 + c);
  else
    v = *reinterpret_cast<const uint4*>(skip + (((long)b * H + y) * W + x) * C2 + (c - C1));
  *reinterpret_cast<uint4*>(out + (((long)b * H + y) * W + x) * C + c) = v;
}

// adjoint of k_upcat: g_lo = sum of the 4 children, g_skip = its slice (written)
__global__ void k_upcat_bwd(const bf16* gout, bf16* glo, bf16* gskip, int n, int H, int W, int C1, int C2) {
  const int C = C1 + C2;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nlo = (long)n * (H / 2) * (W / 2) * (C1 / 8);
  const long nsk = (long)n * H * W * (C2 / 8);
  if (i < nlo) {
    const int c8 = (int)(i % (C1 / 8));
    long q = i / (C1 / 8);
    const int X = (int)(q % (W / 2));
    q /= (W / 2);
    const int Y = (int)(q % (H / 2)), b = (int)(q / (H / 2));
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int d = 0; d < 4; ++d) {
      const uint4 v = *reinterpret_cast<const uint4*>(
          gout + (((long)b * H + 2 * Y + (d >> 1)) * W + 2 * X + (d & 1)) * C + c8 * 8);
      const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
      for (int k = 0; k < 8; ++k) s[k] += __bfloat162float(e[k]);
    }
    __align__(16) bf16 o[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) o[k] = __float2bfloat16_rn(s[k]);
    *reinterpret_cast<uint4*>(glo + (((long)b * (H / 2) + Y) * (W / 2) + X) * C1 + c8 * 8) =
        *reinterpret_cast<uint4*>(o);
  } else if (i < nlo + nsk) {
    const long r = i - nlo;
    const int c8 = (int)(r % (C2 / 8));
    const long pix = r / (C2 / 8);
    *reinterpret_cast<uint4*>(gskip + pix * C2 + c8 * 8) =
        *reinterpret_cast<const uint4*>(gout + pix * C + C1 + c8 * 8);
  }
}

// The 1x1 head (FP32 weights, BF16 input): out[o] = sum_c W[o][c] d1[c] + b[o] for the
// kOut state channels.  With targets: the masked squared error (per-block partial sums
// into part[block]), dL/d(out) into dout (FP32, for the weight gradient) and dL/d(d1)
// (BF16).  Channel validity: 0 and 2 on cx points (x < nx-1, y < ny), 1 and 3 on cy
// points (y < ny-1, x < nx), 4 .. 4+nz-1 on a points, the rest never.
constexpr int kHeadC = 32;
constexpr int kOut = 20;
constexpr int kMaxNzOut = kOut - 4;
__device__ __forceinline__ bool out_valid(int o, int x, int y, int nx, int ny, int nz) {
  if (o == 0 || o == 2) return x < nx - 1 && y < ny;
  if (o == 1 || o == 3) return y < ny - 1 && x < nx;
  return o < 4 + nz && x < nx && y < ny;
}
struct LossWeights {
  float w[kOut];
};

__global__ void __launch_bounds__(128) k_head(const bf16* d1, const float* wh, const float* bh, float* out,
                                              const float* tgt, float* dout, bf16* gd1, float* part, int n, int H,
                                              int W, int ny, int nx, int nz, float inv_count, LossWeights lw) {
  __shared__ float red[4];
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long npix = (long)n * H * W;
  float se = 0.0f;
  if (p < npix) {
    float f[kHeadC];
#pragma unroll
    for (int c8 = 0; c8 < kHeadC / 8; ++c8) {
      const uint4 v = *reinterpret_cast<const uint4*>(d1 + p * kHeadC + c8 * 8);
      const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
      for (int k = 0; k < 8; ++k) f[c8 * 8 + k] = __bfloat162float(e[k]);
    }
    float o[kOut];
#pragma unroll
    for (int j = 0; j < kOut; ++j) {
      float s = bh[j];
#pragma unroll
      for (int c = 0; c < kHeadC; ++c) s = fmaf(wh[j * kHeadC + c], f[c], s);
      o[j] = s;
    }
    if (out) {
#pragma unroll
      for (int j = 0; j < kOut; ++j) out[p * kOut + j] = o[j];
    }
    if (tgt) {
      const int x = (int)(p % W), y = (int)((p / W) % H);
      float gd[kHeadC];
#pragma unroll
      for (int c = 0; c < kHeadC; ++c) gd[c] = 0.0f;
#pragma unroll
      for (int j = 0; j < kOut; ++j) {
        const float e = out_valid(j, x, y, nx, ny, nz) ? o[j] - tgt[p * kOut + j] : 0.0f;
        const float g = 2.0f * lw.w[j] * e * inv_count;
        se += lw.w[j] * e * e;
        dout[p * kOut + j] = g;
#pragma unroll
        for (int c = 0; c < kHeadC; ++c) gd[c] = fmaf(g, wh[j * kHeadC + c], gd[c]);
      }
      __align__(16) bf16 gb[kHeadC];
#pragma unroll
      for (int c = 0; c < kHeadC; ++c) gb[c] = __float2bfloat16_rn(gd[c]);
#pragma unroll
      for (int c8 = 0; c8 < kHeadC / 8; ++c8)
        *reinterpret_cast<uint4*>(gd1 + p * kHeadC + c8 * 8) = reinterpret_cast<const uint4*>(gb)[c8];
    }
  }
  if (!tgt) return;
  for (int o = 16; o > 0; o >>= 1) se += __shfl_down_sync(0xffffffffu, se, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = se;
  __syncthreads();
  if (threadIdx.x == 0) part[blockIdx.x] = ((red[0] + red[1]) + red[2]) + red[3];
}

// per-block partial sums of the head's gradient: thread t < kOut*kHeadC sums
// dout[p][t / kHeadC] * d1[p][t % kHeadC], thread kOut*kHeadC + o sums dout[p][o]
constexpr int kHeadGrad = kOut * kHeadC + kOut;
__global__ void __launch_bounds__(kHeadGrad) k_head_wgrad(const float* dout, const bf16* d1, long npix, int nblk,
                                                          float* part) {
  const int t = threadIdx.x;
  const long per = (npix + nblk - 1) / nblk;
  const long p0 = blockIdx.x * per, p1 = p0 + per < npix ? p0 + per : npix;
  float s = 0.0f;
  if (t < kOut * kHeadC) {
    const int o = t / kHeadC, c = t % kHeadC;
    for (long p = p0; p < p1; ++p) s = fmaf(dout[p * kOut + o], __bfloat162float(d1[p * kHeadC + c]), s);
  } else {
    const int o = t - kOut * kHeadC;
    for (long p = p0; p < p1; ++p) s += dout[p * kOut + o];
  }
  part[(long)blockIdx.x * kHeadGrad + t] = s;
}

__global__ void k_adam(float* w, const float* g, float* m, float* v, bf16* wb, long n, float lr, float c1,
                       float c2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = 0.9f * m[i] + 0.1f * gi;
  const float vi = 0.999f * v[i] + 0.001f * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
  w[i] = wi;
  wb[i] = __float2bfloat16_rn(wi);
}

__global__ void k_to_bf16(const float* w, bf16* wb, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) wb[i] = __float2bfloat16_rn(w[i]);
}

// W^T[t][ci][co] = bf16(W[t][co][ci]) of one 3x3 layer: the dgrad operand
__global__ void k_transpose_w(const float* w, bf16* wt, int cin, int cout) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 9L * cin * cout) return;
  const int co = (int)(i % cout);
  const long r = i / cout;
  const int ci = (int)(r % cin), t = (int)(r / cin);
  wt[i] = __float2bfloat16_rn(w[((long)t * cout + co) * cin + ci]);
}

// ---------------------------------------------------------------------------
// the context's fields <-> network tensors
// ---------------------------------------------------------------------------
struct FieldPtrs {
  const double *Hi, *Hb, *dx, *dy, *A, *beta;
  const int *sheet, *shelf;
};

__global__ void k_features(Dims d, FieldPtrs f, bf16* feat, int Hp, int Wp) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x;  // j
  const int x = blockIdx.y * blockDim.y + threadIdx.y;  // i
  if (y >= Hp || x >= Wp) return;
  __align__(16) bf16 o[kInC];
#pragma unroll
  for (int c = 0; c < kInC; ++c) o[c] = __float2bfloat16_rn(0.0f);
  if (y < d.ny && x < d.nx) {
    const long long q = d.at(y, x);
    o[0] = __float2bfloat16_rn((float)(f.Hi[q] / 1000.0));
    o[1] = __float2bfloat16_rn((float)(f.Hb[q] / 1000.0));
    o[2] = __float2bfloat16_rn((float)(f.dx[q] * 100.0));
    o[3] = __float2bfloat16_rn((float)(f.dy[q] * 100.0));
    o[4] = __float2bfloat16_rn((float)(log10(fmax(f.A[q], 1e-30)) + 17.0));
    o[5] = __float2bfloat16_rn((float)(log10(fmax(f.beta[q], 1e-30)) - 4.0));
    o[6] = __float2bfloat16_rn((float)f.sheet[q]);
    o[7] = __float2bfloat16_rn((float)f.shelf[q]);
  }
  uint4* dst = reinterpret_cast<uint4*>(feat + ((long)y * Wp + x) * kInC);
  dst[0] = reinterpret_cast<const uint4*>(o)[0];
  dst[1] = reinterpret_cast<const uint4*>(o)[1];
}

struct StatePtrs {
  double *ucx, *vcy, *tbx, *tby, *visc;
};
constexpr double kTauScale = 1000.0;  // Pa; outputs 2, 3 are asinh(taub / kTauScale)
constexpr double kViscShift = 8.0;    // outputs 4.. are log10(visc_eff) - kViscShift

__global__ void k_targets(Dims d, StatePtrs s, float* tgt, int Hp, int Wp) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x;
  const int x = blockIdx.y * blockDim.y + threadIdx.y;
  if (y >= Hp || x >= Wp) return;
  float t[kOut];
#pragma unroll
  for (int o = 0; o < kOut; ++o) t[o] = 0.0f;
  if (y < d.ny && x < d.nx - 1) {
    t[0] = (float)asinh(s.ucx[d.at(y, x)] / kVelScale);
    t[2] = (float)asinh(s.tbx[d.at(y, x)] / kTauScale);
  }
  if (y < d.ny - 1 && x < d.nx) {
    t[1] = (float)asinh(s.vcy[d.at(y, x)] / kVelScale);
    t[3] = (float)asinh(s.tby[d.at(y, x)] / kTauScale);
  }
  if (y < d.ny && x < d.nx)
    for (int k = 0; k < d.nz && k < kMaxNzOut; ++k)
      t[4 + k] = (float)(log10(fmax(s.visc[k * d.plane + d.at(y, x)], 1e-30)) - kViscShift);
#pragma unroll
  for (int o = 0; o < kOut; ++o) tgt[((long)y * Wp + x) * kOut + o] = t[o];
}

// an output clamped to [-lim, lim]; a non-finite one becomes 0
__device__ __forceinline__ double clamp_out(float v, double lim) {
  const double x = (double)v;
  return x == x ? fmax(-lim, fmin(lim, x)) : 0.0;
}

// the predicted state into the context's fields, within physical bounds (velocities
// within the solver's DIVA_vel_max, |taub| <= 1e7 Pa, viscosity in [1e3, 1e18]) so that
// a poorly trained network cannot hand the solve an overflow; velocities_only: u, v
__global__ void k_apply(Dims d, const float* pred, StatePtrs s, int Wp, int velocities_only, double vmax) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x;
  const int x = blockIdx.y * blockDim.y + threadIdx.y;
  if (y >= d.ny || x >= d.nx) return;
  const float* q = pred + ((long)y * Wp + x) * kOut;
  const double ulim = asinh(vmax / kVelScale), tlim = asinh(1e7 / kTauScale);
  if (x < d.nx - 1) s.ucx[d.at(y, x)] = kVelScale * sinh(clamp_out(q[0], ulim));
  if (y < d.ny - 1) s.vcy[d.at(y, x)] = kVelScale * sinh(clamp_out(q[1], ulim));
  if (velocities_only) return;
  if (x < d.nx - 1) s.tbx[d.at(y, x)] = kTauScale * sinh(clamp_out(q[2], tlim));
  if (y < d.ny - 1) s.tby[d.at(y, x)] = kTauScale * sinh(clamp_out(q[3], tlim));
  for (int k = 0; k < d.nz; ++k) {
    const double l = fmax(3.0 - kViscShift, fmin(18.0 - kViscShift, clamp_out(q[4 + k], 1e30)));
    s.visc[k * d.plane + d.at(y, x)] = pow(10.0, l + kViscShift);
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <int KC, int NO, bool DG>
int launch_conv(const ConvArgs& a, cudaStream_t st) {
  constexpr int need = conv_smem<KC, NO>();
  constexpr int floor_ = smem_floor(tmem_cols<NO>());
  constexpr int smem = need > floor_ ? need : floor_;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_conv3x3<KC, NO, DG>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
        cudaSuccess)
      return DIVA_CUDA_ERROR;
    attr = true;
  }
  const long npix = (long)a.n * a.H * a.W;
  k_conv3x3<KC, NO, DG><<<(unsigned)((npix + 127) / 128), 128, smem, st>>>(a);
  return DIVA_OK;
}

template <int CI, int CO>
int launch_wgrad(const WgradArgs& a, cudaStream_t st) {
  constexpr int need = wgrad_smem<CI>();
  constexpr int floor_ = smem_floor(tmem_cols<CI>());
  constexpr int smem = need > floor_ ? need : floor_;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_conv3x3_wgrad<CI, CO>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
        cudaSuccess)
      return DIVA_CUDA_ERROR;
    attr = true;
  }
  k_conv3x3_wgrad<CI, CO><<<dim3(a.nsplit, 9), 128, smem, st>>>(a);
  return DIVA_OK;
}

int conv_fwd(int cin, int cout, const ConvArgs& a, cudaStream_t st) {
#define FWD(KC, NO) \
  if (cin == KC && cout == NO) return launch_conv<KC, NO, false>(a, st);
  FWD(16, 32) FWD(32, 32) FWD(32, 64) FWD(64, 64) FWD(64, 128) FWD(128, 64) FWD(64, 32)
#undef FWD
  return DIVA_UNSUPPORTED;
}
int conv_dgrad(int cin, int cout, const ConvArgs& a, cudaStream_t st) {
#define DGR(KC, NO) \
  if (cout == KC && cin == NO) return launch_conv<KC, NO, true>(a, st);
  DGR(32, 32) DGR(32, 64) DGR(64, 128) DGR(128, 64) DGR(64, 64) DGR(64, 32)
#undef DGR
  return DIVA_UNSUPPORTED;
}
int conv_wgrad(int cin, int cout, const WgradArgs& a, cudaStream_t st) {
#define WGR(CI, CO) \
  if (cin == CI && cout == CO) return launch_wgrad<CI, CO>(a, st);
  WGR(16, 32) WGR(32, 32) WGR(32, 64) WGR(64, 64) WGR(64, 128) WGR(128, 64) WGR(64, 32)
#undef WGR
  return DIVA_UNSUPPORTED;
}

// tensors of the network (index, level, channels)
enum T { T_IN, T_A1, T_E1, T_P1, T_A2, T_E2, T_P2, T_B1, T_B2, T_U2, T_C2, T_D2, T_U1, T_C1, T_D1, T_N };
constexpr int kTLevel[T_N] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 1, 1, 1, 0, 0, 0};
constexpr int kTChan[T_N] = {16, 32, 32, 32, 64, 64, 64, 128, 64, 128, 64, 32, 64, 32, 32};

struct Layer {
  int cin, cout, in, out;
  long woff, boff;
};
constexpr int kNL = 10;
constexpr int kLayerDef[kNL][4] = {{16, 32, T_IN, T_A1}, {32, 32, T_A1, T_E1}, {32, 64, T_P1, T_A2},
                                   {64, 64, T_A2, T_E2}, {64, 128, T_P2, T_B1}, {128, 64, T_B1, T_B2},
                                   {128, 64, T_U2, T_C2}, {64, 32, T_C2, T_D2}, {64, 32, T_U1, T_C1},
                                   {32, 32, T_C1, T_D1}};

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double unit(uint64_t& s) { return ((splitmix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

}  // namespace cnn
}  // namespace diva

using namespace diva;
using namespace diva::cnn;

struct diva_cnn {
  int ny = 0, nx = 0, nz = 0, Hp = 0, Wp = 0, batch = 0, capacity = 0, nsamples = 0;
  Layer L[kNL];
  long head_w = 0, head_b = 0, nw = 0;
  cudaStream_t stream = nullptr;
  void* arena = nullptr;
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  bf16* wb = nullptr;
  bf16* wbt = nullptr;   // per-layer transposed BF16 weights (dgrad)
  bf16* act[T_N] = {};
  bf16* grad[T_N] = {};
  float *out = nullptr, *tgt = nullptr, *dout = nullptr, *part = nullptr, *loss = nullptr, *loss_hist = nullptr;
  long part_floats = 0;
  bf16* ds_feat = nullptr;
  float* ds_tgt = nullptr;
  int* err = nullptr;
  long adam_t = 0;
  LossWeights lw{};

  // valid output entries of n samples (the loss is their mean squared error)
  long valid(int n) const {
    return (long)n * (2L * ny * (nx - 1) + 2L * (ny - 1) * nx + (long)nz * ny * nx);
  }
  int lvH(int l) const { return Hp >> l; }
  int lvW(int l) const { return Wp >> l; }
  long tsize(int t) const { return (long)lvH(kTLevel[t]) * lvW(kTLevel[t]) * kTChan[t]; }
  int wgrad_split(long npix) const {
    const long nchunk = (npix + kPixChunk - 1) / kPixChunk;
    long s = nchunk < 64 ? nchunk : 64;
    return (int)(s < 1 ? 1 : s);
  }
};

namespace {

#define CK(x)                                              \
  do {                                                     \
    if ((x) != cudaSuccess) return DIVA_CUDA_ERROR;        \
  } while (0)
#define RET(x)                                             \
  do {                                                     \
    const int _st = (x);                                   \
    if (_st != DIVA_OK) return _st;                        \
  } while (0)

inline unsigned nblk(long n, int b) { return (unsigned)((n + b - 1) / b); }
constexpr int kHeadBlocks = 148;

int forward(diva_cnn_t* N, const bf16* in, float* out, int n, cudaStream_t st) {
  auto tens = [&](int t) -> const bf16* { return t == T_IN ? in : N->act[t]; };
  auto conv = [&](int l) {
    const Layer& ly = N->L[l];
    const int lv = kTLevel[ly.out];
    ConvArgs a{tens(ly.in), nullptr, N->wb + ly.woff, N->w + ly.boff, N->act[ly.out], n, N->lvH(lv), N->lvW(lv),
               1, N->err};
    return conv_fwd(ly.cin, ly.cout, a, st);
  };
  auto pool = [&](int src, int dst) {
    const int lv = kTLevel[src];
    const long cnt = (long)n * (N->lvH(lv) / 2) * (N->lvW(lv) / 2) * (kTChan[src] / 8);
    k_pool<<<nblk(cnt, 256), 256, 0, st>>>(N->act[src], N->act[dst], n, N->lvH(lv), N->lvW(lv), kTChan[src]);
  };
  auto upcat = [&](int lo, int skip, int dst) {
    const int lv = kTLevel[dst];
    const long cnt = (long)n * N->lvH(lv) * N->lvW(lv) * (kTChan[dst] / 8);
    k_upcat<<<nblk(cnt, 256), 256, 0, st>>>(N->act[lo], N->act[skip], N->act[dst], n, N->lvH(lv), N->lvW(lv),
                                            kTChan[lo], kTChan[skip]);
  };
  RET(conv(0));
  RET(conv(1));
  pool(T_E1, T_P1);
  RET(conv(2));
  RET(conv(3));
  pool(T_E2, T_P2);
  RET(conv(4));
  RET(conv(5));
  upcat(T_B2, T_E2, T_U2);
  RET(conv(6));
  RET(conv(7));
  upcat(T_D2, T_E1, T_U1);
  RET(conv(8));
  RET(conv(9));
  if (out) {
    const long npix = (long)n * N->Hp * N->Wp;
    k_head<<<nblk(npix, 128), 128, 0, st>>>(N->act[T_D1], N->w + N->head_w, N->w + N->head_b, out, nullptr,
                                            nullptr, nullptr, nullptr, n, N->Hp, N->Wp, N->ny, N->nx, N->nz, 0.0f,
                                            N->lw);
  }
  CK(cudaGetLastError());
  return DIVA_OK;
}

// gradient of the batch loss into N->g, the batch's squared-error sum into *loss_dst
int backward(diva_cnn_t* N, const bf16* in, const float* tgt, int n, cudaStream_t st, float* loss_dst) {
  const long npix0 = (long)n * N->Hp * N->Wp;
  const unsigned hb = nblk(npix0, 128);
  if ((long)hb > N->part_floats - 128 || (long)kHeadBlocks * kHeadGrad > N->part_floats - 128) return DIVA_BAD_INPUT;
  k_head<<<hb, 128, 0, st>>>(N->act[T_D1], N->w + N->head_w, N->w + N->head_b, nullptr, tgt, N->dout,
                             N->grad[T_D1], N->part, n, N->Hp, N->Wp, N->ny, N->nx, N->nz,
                             1.0f / (float)N->valid(n), N->lw);
  k_sum_rows<<<1, 32, 0, st>>>(N->part, (int)hb, 1, loss_dst);
  k_head_wgrad<<<kHeadBlocks, kHeadGrad, 0, st>>>(N->dout, N->act[T_D1], npix0, kHeadBlocks, N->part);
  k_sum_rows<<<nblk(kHeadGrad, 256), 256, 0, st>>>(N->part, kHeadBlocks, kHeadGrad, N->g + N->head_w);

  auto tens = [&](int t) -> const bf16* { return t == T_IN ? in : N->act[t]; };
  auto layer_bwd = [&](int l, bool dgrad) -> int {
    const Layer& ly = N->L[l];
    const int lv = kTLevel[ly.out];
    const int H = N->lvH(lv), W = N->lvW(lv);
    const long npix = (long)n * H * W;
    const int ns = N->wgrad_split(npix);
    const long wn = 9L * ly.cout * ly.cin;
    if ((long)ns * wn > N->part_floats - 128) return DIVA_BAD_INPUT;
    WgradArgs wa{tens(ly.in), N->grad[ly.out], N->act[ly.out], N->part, n, H, W, ns, N->err};
    RET(conv_wgrad(ly.cin, ly.cout, wa, st));
    k_sum_rows<<<nblk(wn, 256), 256, 0, st>>>(N->part, ns, (int)wn, N->g + ly.woff);
    const int nb = 128;
    k_bias_part<<<nb, 128, 0, st>>>(N->grad[ly.out], N->act[ly.out], npix, ly.cout, nb, N->part);
    k_sum_rows<<<1, 128, 0, st>>>(N->part, nb, ly.cout, N->g + ly.boff);
    if (dgrad) {
      ConvArgs a{N->grad[ly.out], N->act[ly.out], N->wbt + ly.woff, nullptr, N->grad[ly.in], n, H, W, 0, N->err};
      RET(conv_dgrad(ly.cin, ly.cout, a, st));
    }
    return DIVA_OK;
  };
  auto upcat_bwd = [&](int dst, int lo, int skip) {
    const int lv = kTLevel[dst];
    const int H = N->lvH(lv), W = N->lvW(lv);
    const long cnt = (long)n * (H / 2) * (W / 2) * (kTChan[lo] / 8) + (long)n * H * W * (kTChan[skip] / 8);
    k_upcat_bwd<<<nblk(cnt, 256), 256, 0, st>>>(N->grad[dst], N->grad[lo], N->grad[skip], n, H, W, kTChan[lo],
                                                kTChan[skip]);
  };
  auto pool_bwd = [&](int lo, int hi) {
    const int lv = kTLevel[hi];
    const long cnt = (long)n * N->lvH(lv) * N->lvW(lv) * (kTChan[hi] / 8);
    k_pool_bwd_add<<<nblk(cnt, 256), 256, 0, st>>>(N->grad[lo], N->grad[hi], n, N->lvH(lv), N->lvW(lv),
                                                   kTChan[hi]);
  };
  RET(layer_bwd(9, true));   // d1b -> g_c1
  RET(layer_bwd(8, true));   // d1a -> g_u1
  upcat_bwd(T_U1, T_D2, T_E1);
  RET(layer_bwd(7, true));   // d2b -> g_c2
  RET(layer_bwd(6, true));   // d2a -> g_u2
  upcat_bwd(T_U2, T_B2, T_E2);
  RET(layer_bwd(5, true));   // bb -> g_b1
  RET(layer_bwd(4, true));   // ba -> g_p2
  pool_bwd(T_P2, T_E2);
  RET(layer_bwd(3, true));   // e2b -> g_a2
  RET(layer_bwd(2, true));   // e2a -> g_p1
  pool_bwd(T_P1, T_E1);
  RET(layer_bwd(1, true));   // e1b -> g_a1
  RET(layer_bwd(0, false));  // e1a
  CK(cudaGetLastError());
  return DIVA_OK;
}

void transpose_weights(diva_cnn_t* N, cudaStream_t st) {
  for (int l = 0; l < kNL; ++l) {
    const Layer& ly = N->L[l];
    k_transpose_w<<<nblk(9L * ly.cin * ly.cout, 256), 256, 0, st>>>(N->w + ly.woff, N->wbt + ly.woff, ly.cin,
                                                                    ly.cout);
  }
}

int adam(diva_cnn_t* N, float lr, cudaStream_t st) {
  N->adam_t += 1;
  const float c1 = 1.0f - powf(0.9f, (float)N->adam_t), c2 = 1.0f - powf(0.999f, (float)N->adam_t);
  k_adam<<<nblk(N->nw, 256), 256, 0, st>>>(N->w, N->g, N->m, N->v, N->wb, N->nw, lr, c1, c2);
  transpose_weights(N, st);
  CK(cudaGetLastError());
  return DIVA_OK;
}

int check_err(diva_cnn_t* N) {
  int e = 0;
  CK(cudaMemcpy(&e, N->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    CK(cudaMemset(N->err, 0, sizeof(int)));
    return DIVA_TIMEOUT;
  }
  return DIVA_OK;
}

FieldPtrs field_ptrs(const Ctx* c) {
  return FieldPtrs{c->D(DIVA_F_HI_A),     c->D(DIVA_F_HB_A),       c->D(DIVA_F_DHS_DX_A),
                   c->D(DIVA_F_DHS_DY_A), c->D(DIVA_F_A_FLOW_VAV_A), c->D(DIVA_F_BETA_SQ_A),
                   static_cast<const int*>(c->f[DIVA_F_MASK_SHEET_A]),
                   static_cast<const int*>(c->f[DIVA_F_MASK_SHELF_A])};
}

StatePtrs state_ptrs(Ctx* c) {
  return StatePtrs{c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY), c->D(DIVA_F_TAUB_CX), c->D(DIVA_F_TAUB_CY),
                   c->D(DIVA_F_VISC_EFF_3D_A)};
}

dim3 img_grid(int Hp, int Wp) { return dim3((Hp + kBX - 1) / kBX, (Wp + kBY - 1) / kBY); }

}  // namespace

extern "C" {

int32_t diva_cnn_create(diva_cnn_t** out, int32_t ny, int32_t nx, int32_t nz, int32_t batch, int32_t capacity,
                        uint64_t seed) {
  if (!out || ny < 2 || nx < 2 || nz < 2 || batch < 1 || capacity < 0) return DIVA_BAD_INPUT;
  *out = nullptr;
  if (nz > kMaxNzOut) return DIVA_UNSUPPORTED;
  diva_cnn_t* N = new (std::nothrow) diva_cnn_t();
  if (!N) return DIVA_CUDA_ERROR;
  N->ny = ny;
  N->nx = nx;
  N->nz = nz;
  N->Hp = (ny + 3) / 4 * 4;
  N->Wp = (nx + 3) / 4 * 4;
  N->batch = batch;
  N->capacity = capacity;
  for (int o = 0; o < kOut; ++o) N->lw.w[o] = 1.0f;
  long off = 0;
  for (int l = 0; l < kNL; ++l) {
    Layer& ly = N->L[l];
    ly.cin = kLayerDef[l][0];
    ly.cout = kLayerDef[l][1];
    ly.in = kLayerDef[l][2];
    ly.out = kLayerDef[l][3];
    ly.woff = off;
    off += 9L * ly.cin * ly.cout;
    ly.boff = off;
    off += ly.cout;
  }
  N->head_w = off;
  off += (long)kOut * kHeadC;
  N->head_b = off;
  off += kOut;
  N->nw = off;

  // wgrad partials: up to 64 slices of the largest layer; head partials
  long part = 64L * 9 * 128 * 64;
  const long hb = (long)nblk((long)batch * N->Hp * N->Wp, 128);
  if (hb > part) part = hb;
  if ((long)kHeadBlocks * kHeadGrad > part) part = (long)kHeadBlocks * kHeadGrad;
  if (128L * 128 > part) part = 128L * 128;
  N->part_floats = part + 128;

  const long img = (long)N->Hp * N->Wp;
  size_t bytes = 0;
  auto carve = [&](size_t b) {
    const size_t o = bytes;
    bytes += (b + 255) / 256 * 256;
    return o;
  };
  const size_t o_w = carve(N->nw * 4), o_g = carve(N->nw * 4), o_m = carve(N->nw * 4), o_v = carve(N->nw * 4);
  const size_t o_wb = carve(N->nw * 2), o_wbt = carve(N->nw * 2);
  size_t o_act[T_N], o_grad[T_N];
  for (int t = 0; t < T_N; ++t) {
    o_act[t] = carve((size_t)batch * N->tsize(t) * 2);
    o_grad[t] = t == T_IN ? 0 : carve((size_t)batch * N->tsize(t) * 2);
  }
  const size_t o_out = carve((size_t)batch * img * kOut * 4), o_tgt = carve((size_t)batch * img * kOut * 4);
  const size_t o_dout = carve((size_t)batch * img * kOut * 4);
  const size_t o_part = carve(N->part_floats * 4), o_loss = carve(256), o_err = carve(256);
  const size_t o_lh = carve((size_t)(capacity + 1) * 4);
  const size_t o_dsf = carve((size_t)capacity * img * kInC * 2), o_dst = carve((size_t)capacity * img * kOut * 4);
  if (cudaMalloc(&N->arena, bytes) != cudaSuccess) {
    delete N;
    return DIVA_CUDA_ERROR;
  }
  char* base = static_cast<char*>(N->arena);
  N->w = reinterpret_cast<float*>(base + o_w);
  N->g = reinterpret_cast<float*>(base + o_g);
  N->m = reinterpret_cast<float*>(base + o_m);
  N->v = reinterpret_cast<float*>(base + o_v);
  N->wb = reinterpret_cast<bf16*>(base + o_wb);
  N->wbt = reinterpret_cast<bf16*>(base + o_wbt);
  for (int t = 0; t < T_N; ++t) {
    N->act[t] = reinterpret_cast<bf16*>(base + o_act[t]);
    N->grad[t] = t == T_IN ? nullptr : reinterpret_cast<bf16*>(base + o_grad[t]);
  }
  N->out = reinterpret_cast<float*>(base + o_out);
  N->tgt = reinterpret_cast<float*>(base + o_tgt);
  N->dout = reinterpret_cast<float*>(base + o_dout);
  N->part = reinterpret_cast<float*>(base + o_part);
  N->loss = reinterpret_cast<float*>(base + o_loss);
  N->err = reinterpret_cast<int*>(base + o_err);
  N->loss_hist = reinterpret_cast<float*>(base + o_lh);
  N->ds_feat = reinterpret_cast<bf16*>(base + o_dsf);
  N->ds_tgt = reinterpret_cast<float*>(base + o_dst);
  if (cudaStreamCreateWithFlags(&N->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMemset(N->arena, 0, bytes) != cudaSuccess) {
    diva_cnn_destroy(N);
    return DIVA_CUDA_ERROR;
  }
  // He-normal weights from the seed, zero biases
  std::vector<float> h(N->nw, 0.0f);
  uint64_t s = seed;
  auto normal = [&]() {
    const double u1 = unit(s), u2 = unit(s);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
  };
  for (int l = 0; l < kNL; ++l) {
    const double sd = std::sqrt(2.0 / (9.0 * N->L[l].cin));
    for (long i = 0; i < 9L * N->L[l].cin * N->L[l].cout; ++i) h[N->L[l].woff + i] = (float)(sd * normal());
  }
  for (int i = 0; i < kOut * kHeadC; ++i) h[N->head_w + i] = (float)(std::sqrt(1.0 / kHeadC) * normal());
  const int st = diva_cnn_weights(N, h.data(), N->nw, 1);
  if (st != DIVA_OK) {
    diva_cnn_destroy(N);
    return st;
  }
  *out = N;
  return DIVA_OK;
}

int32_t diva_cnn_destroy(diva_cnn_t* N) {
  if (!N) return DIVA_BAD_INPUT;
  if (N->stream) cudaStreamSynchronize(N->stream);
  if (N->arena) cudaFree(N->arena);
  if (N->stream) cudaStreamDestroy(N->stream);
  delete N;
  return DIVA_OK;
}

int32_t diva_cnn_num_weights(const diva_cnn_t* N, int64_t* n) {
  if (!N || !n) return DIVA_BAD_INPUT;
  *n = N->nw;
  return DIVA_OK;
}

int32_t diva_cnn_padded_shape(const diva_cnn_t* N, int32_t* Hp, int32_t* Wp) {
  if (!N || !Hp || !Wp) return DIVA_BAD_INPUT;
  *Hp = N->Hp;
  *Wp = N->Wp;
  return DIVA_OK;
}

int32_t diva_cnn_num_samples(const diva_cnn_t* N, int32_t* n) {
  if (!N || !n) return DIVA_BAD_INPUT;
  *n = N->nsamples;
  return DIVA_OK;
}

int32_t diva_cnn_weights(diva_cnn_t* N, float* host, int64_t n, int32_t direction) {
  if (!N || !host || n != N->nw || (direction != 0 && direction != 1)) return DIVA_BAD_INPUT;
  CK(cudaStreamSynchronize(N->stream));
  if (direction == 0) {
    CK(cudaMemcpy(host, N->w, n * 4, cudaMemcpyDeviceToHost));
    return DIVA_OK;
  }
  CK(cudaMemcpy(N->w, host, n * 4, cudaMemcpyHostToDevice));
  CK(cudaMemset(N->m, 0, n * 4));
  CK(cudaMemset(N->v, 0, n * 4));
  N->adam_t = 0;
  k_to_bf16<<<nblk(n, 256), 256, 0, N->stream>>>(N->w, N->wb, n);
  transpose_weights(N, N->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(N->stream));
  return DIVA_OK;
}

int32_t diva_cnn_grads(diva_cnn_t* N, float* host, int64_t n) {
  if (!N || !host || n != N->nw) return DIVA_BAD_INPUT;
  CK(cudaStreamSynchronize(N->stream));
  CK(cudaMemcpy(host, N->g, n * 4, cudaMemcpyDeviceToHost));
  return DIVA_OK;
}

int32_t diva_cnn_set_loss_weights(diva_cnn_t* N, const float* w, int32_t n) {
  if (!N || !w || n != kOut) return DIVA_BAD_INPUT;
  for (int o = 0; o < kOut; ++o)
    if (!(w[o] >= 0.0f) || std::isinf(w[o])) return DIVA_BAD_INPUT;
  CK(cudaStreamSynchronize(N->stream));
  for (int o = 0; o < kOut; ++o) N->lw.w[o] = w[o];
  return DIVA_OK;
}

int32_t diva_cnn_add_sample(diva_cnn_t* N, diva_ctx_t* ctx) {
  if (!N || !ctx) return DIVA_BAD_INPUT;
  Ctx* c = &ctx->c;
  if (c->d.ny != N->ny || c->d.nx != N->nx || c->d.nz != N->nz || N->nsamples >= N->capacity)
    return DIVA_BAD_INPUT;
  const long img = (long)N->Hp * N->Wp;
  const int k = N->nsamples;
  k_features<<<img_grid(N->Hp, N->Wp), block2d(), 0, c->stream>>>(c->d, field_ptrs(c), N->ds_feat + k * img * kInC,
                                                                   N->Hp, N->Wp);
  k_targets<<<img_grid(N->Hp, N->Wp), block2d(), 0, c->stream>>>(c->d, state_ptrs(c), N->ds_tgt + k * img * kOut,
                                                                  N->Hp, N->Wp);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  N->nsamples += 1;
  return DIVA_OK;
}

int32_t diva_cnn_predict(diva_cnn_t* N, diva_ctx_t* ctx, int32_t complete_sweeps) {
  if (!N || !ctx || complete_sweeps < 0 || complete_sweeps > 10000) return DIVA_BAD_INPUT;
  Ctx* c = &ctx->c;
  if (c->d.ny != N->ny || c->d.nx != N->nx || c->d.nz != N->nz) return DIVA_BAD_INPUT;
  CK(cudaStreamSynchronize(N->stream));
  k_features<<<img_grid(N->Hp, N->Wp), block2d(), 0, c->stream>>>(c->d, field_ptrs(c), N->act[T_IN], N->Hp,
                                                                   N->Wp);
  RET(forward(N, N->act[T_IN], N->out, 1, c->stream));
  k_apply<<<img_grid(N->ny, N->nx), block2d(), 0, c->stream>>>(c->d, N->out, state_ptrs(c), N->Wp,
                                                                complete_sweeps > 0, c->c.DIVA_vel_max);
  // the context's launch count includes the network's kernels run on its stream: features,
  // 10 convolutions, 2 pools, 2 up-concatenations, the head and the state write
  c->launches += 17;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  RET(check_err(N));
  return complete_sweeps > 0 ? diva_complete_state(ctx, complete_sweeps) : DIVA_OK;
}

int32_t diva_cnn_forward(diva_cnn_t* N, const void* feat, float* out, int32_t n) {
  if (!N || !feat || !out || n < 1 || n > N->batch) return DIVA_BAD_INPUT;
  RET(forward(N, static_cast<const bf16*>(feat), out, n, N->stream));
  CK(cudaStreamSynchronize(N->stream));
  return check_err(N);
}

int32_t diva_cnn_train_step(diva_cnn_t* N, const void* feat, const float* tgt, int32_t n, float lr, float* loss) {
  if (!N || !feat || !tgt || n < 1 || n > N->batch || !(lr >= 0.0f)) return DIVA_BAD_INPUT;
  const bf16* in = static_cast<const bf16*>(feat);
  RET(forward(N, in, nullptr, n, N->stream));
  RET(backward(N, in, tgt, n, N->stream, N->loss));
  float l = 0.0f;
  CK(cudaMemcpyAsync(&l, N->loss, 4, cudaMemcpyDeviceToHost, N->stream));
  RET(adam(N, lr, N->stream));
  CK(cudaStreamSynchronize(N->stream));
  if (loss) *loss = l / (float)N->valid(n);
  return check_err(N);
}

int32_t diva_cnn_train(diva_cnn_t* N, int32_t epochs, float lr, uint64_t seed, float* loss) {
  if (!N || epochs < 0 || !(lr >= 0.0f) || N->nsamples < 1) return DIVA_BAD_INPUT;
  const long img = (long)N->Hp * N->Wp;
  std::vector<int> order(N->nsamples);
  for (int i = 0; i < N->nsamples; ++i) order[i] = i;
  uint64_t s = seed;
  std::vector<float> batch_loss;
  double last = 0.0;
  for (int e = 0; e < epochs; ++e) {
    for (int i = N->nsamples - 1; i > 0; --i) {
      const int j = (int)(splitmix(s) % (uint64_t)(i + 1));
      const int t = order[i];
      order[i] = order[j];
      order[j] = t;
    }
    const int nb = (N->nsamples + N->batch - 1) / N->batch;
    batch_loss.assign(nb, 0.0f);
    for (int b = 0; b < nb; ++b) {
      const int n = std::min(N->batch, N->nsamples - b * N->batch);
      for (int k = 0; k < n; ++k) {
        const int smp = order[b * N->batch + k];
        CK(cudaMemcpyAsync(N->act[T_IN] + k * img * kInC, N->ds_feat + smp * img * kInC, img * kInC * 2,
                           cudaMemcpyDeviceToDevice, N->stream));
        CK(cudaMemcpyAsync(N->tgt + k * img * kOut, N->ds_tgt + smp * img * kOut, img * kOut * 4,
                           cudaMemcpyDeviceToDevice, N->stream));
      }
      RET(forward(N, N->act[T_IN], nullptr, n, N->stream));
      RET(backward(N, N->act[T_IN], N->tgt, n, N->stream, N->loss_hist + b));
      RET(adam(N, lr, N->stream));
    }
    CK(cudaMemcpyAsync(batch_loss.data(), N->loss_hist, nb * 4, cudaMemcpyDeviceToHost, N->stream));
    CK(cudaStreamSynchronize(N->stream));
    RET(check_err(N));
    double sum = 0.0;
    for (int b = 0; b < nb; ++b) sum += batch_loss[b];
    last = sum / (double)N->valid(N->nsamples);
    if (!(last == last) || std::isinf(last)) {   // diverged: the weights are no longer usable
      if (loss) *loss = (float)last;
      return DIVA_NAN_DETECTED;
    }
  }
  if (loss) *loss = (float)last;
  return DIVA_OK;
}

}  // extern "C"
