// noalloc.cu -- the viscosity-iteration step norm without any allocation.
//
// diva_visc_iter_uv_resid_noalloc() computes the step norm of one viscosity
// iteration (calc_visc_iter_UV_resid, ice_velocity_module.f90:1530-1601) from
// device arrays the caller owns, for callers that cannot let a library call
// cudaMalloc: a host model that budgets all device memory through its own pool
// allocator, or code that must not trigger allocation while it runs alongside
// other work on the device.  The reduction needs per-block partial sums; they
// live in the file-scope array below instead of a context arena.
//
// Scratch: kResidMaxBlocks * 3 doubles = 384 KiB, held by every GPU that loads
// the library until the process exits.  All calls share it, so calls that
// overlap on the GPU (different streams, or host threads) race on it; serialise
// them.  Each call writes every partial it later reads, so nothing has to be
// cleared between calls.
#include <cuda.h>   // CUcontext and CUresult, for the context id of the set-up
#include <mutex>
#include "common.cuh"

namespace {

constexpr int kResidMaxBlocks = 16384;   // blocks of 32 x 8 columns

static __device__ __align__(256) double g_resid_scratch[kResidMaxBlocks * 3];

// per-block partial sums of (u - u_prev)^2, (u + u_prev)^2 and the count of
// points with |u| above the tolerance, over the cx and cy points of the block
__global__ void k_resid_partials(int nx, int ny, const double* __restrict__ u, const double* __restrict__ up,
                                 int ldu, const double* __restrict__ v, const double* __restrict__ vp, int ldv,
                                 double* partials) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  double s[3] = {0.0, 0.0, 0.0};
  if (j < ny && i < nx) {
    if (i < nx - 1) {
      const long long q = (long long)i * ldu + j;
      const double a = u[q], b = up[q];
      if (fabs(a) > diva::kVelTol) {
        s[2] += 1.0;
        s[0] += (a - b) * (a - b);
        s[1] += (a + b) * (a + b);
      }
    }
    if (j < ny - 1) {
      const long long q = (long long)i * ldv + j;
      const double a = v[q], b = vp[q];
      if (fabs(a) > diva::kVelTol) {
        s[2] += 1.0;
        s[0] += (a - b) * (a - b);
        s[1] += (a + b) * (a + b);
      }
    }
  }
  diva::block_sum<3>(s);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const int b = blockIdx.y * gridDim.x + blockIdx.x;
    partials[3 * b + 0] = s[0];
    partials[3 * b + 1] = s[1];
    partials[3 * b + 2] = s[2];
  }
}

// fixed-order sum of the partials and the norm itself
__global__ void k_resid_final(const double* partials, int nblocks, double* out) {
  __shared__ double sh[3][256];
  double s[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int q = 0; q < 3; ++q) s[q] += partials[3 * b + q];
  for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] = s[q];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double r1 = sh[0][0], r2 = sh[1][0], n = sh[2][0];
    out[0] = (n > 0.0) ? 2.0 * sqrt(r1) / diva::max_ref(sqrt(r2), 1E-8) : 0.0;
  }
}

// Device address of the scratch array, set up by the first call in each CUDA context:
// cudaGetSymbolAddress with the device current, checked, and cached with the context's
// unique id (cuCtxGetId, never reused within a process).  A cudaDeviceReset, or a caller
// that makes another context current on the same device, gives a new id, and the next
// call sets up again (the module, and with it the array, may sit at a new address).
// The driver calls are resolved through the runtime, so the library needs no link
// against the driver library.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;

// id of the context current on this thread; 0 if none is current yet
int current_context_id(unsigned long long* id) {
  if (!g_ctx_current || !g_ctx_id) {
    void* f0 = nullptr;
    void* f1 = nullptr;
    cudaDriverEntryPointQueryResult q0, q1;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0) != cudaSuccess ||
        q0 != cudaDriverEntryPointSuccess || !f0)
      return DIVA_CUDA_ERROR;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || !f1)
      return DIVA_CUDA_ERROR;
    g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f0);
    g_ctx_id = reinterpret_cast<CtxGetIdFn>(f1);
  }
  CUcontext ctx = nullptr;
  if (g_ctx_current(&ctx) != CUDA_SUCCESS) return DIVA_CUDA_ERROR;
  *id = 0;
  if (ctx && g_ctx_id(ctx, id) != CUDA_SUCCESS) return DIVA_CUDA_ERROR;
  return DIVA_OK;
}

int scratch_for_current_device(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DIVA_CUDA_ERROR;
  std::lock_guard<std::mutex> lock(g_mu);
  unsigned long long id = 0;
  int st = current_context_id(&id);
  if (st) return st;
  if (id == 0 || id != g_scratch_ctx[dev] || !g_scratch_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_resid_scratch) != cudaSuccess || !p) return DIVA_CUDA_ERROR;
    if ((st = current_context_id(&id))) return st;   // the look-up made the primary context current
    g_scratch_ptr[dev] = static_cast<double*>(p);
    g_scratch_ctx[dev] = id;
  }
  *out = g_scratch_ptr[dev];
  return DIVA_OK;
}

}  // namespace

extern "C" int diva_visc_iter_uv_resid_noalloc(int32_t nx, int32_t ny, const double* u_cx, const double* u_cx_prev,
                                               int32_t ld_cx, const double* v_cy, const double* v_cy_prev,
                                               int32_t ld_cy, double* resid_uv, void* stream) {
  if (nx < 2 || ny < 2 || ld_cx < ny || ld_cy < ny - 1 || !u_cx || !u_cx_prev || !v_cy || !v_cy_prev || !resid_uv)
    return DIVA_BAD_INPUT;
  const dim3 block(diva::kBX, diva::kBY);
  const dim3 grid((ny + diva::kBX - 1) / diva::kBX, (nx + diva::kBY - 1) / diva::kBY);
  const long long nblocks = (long long)grid.x * grid.y;
  if (nblocks > kResidMaxBlocks) return DIVA_BAD_INPUT;   // grid larger than the static scratch covers
  double* scratch = nullptr;
  const int st = scratch_for_current_device(&scratch);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_resid_partials<<<grid, block, 0, s>>>(nx, ny, u_cx, u_cx_prev, ld_cx, v_cy, v_cy_prev, ld_cy, scratch);
  k_resid_final<<<1, 256, 0, s>>>(scratch, (int)nblocks, resid_uv);
  return cudaGetLastError() == cudaSuccess ? DIVA_OK : DIVA_CUDA_ERROR;
}
