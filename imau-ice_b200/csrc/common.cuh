// common.cuh -- layout, constants and helpers shared by the B200 kernels.
//
// Device layout.  Every 2D field (a, cx, cy and b grid alike) lives on one
// padded plane of nx columns x ld rows, element (j,i) at [i*ld + j] with j
// fastest -- the order of the reference's Fortran arrays (ny,nx), so a warp
// over j reads 32 consecutive doubles.  A cx field uses columns 0..nx-2, a
// cy field rows 0..ny-2, a b field both.  3D fields are layer-major:
// (k,j,i) at [k*plane + i*ld + j], so each zeta layer is one coalesced plane.
// ld is ny rounded up to 16 elements (128-byte rows for doubles).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/diva.h"

namespace diva {

// parameters_module.f90:10-23
constexpr double kPi = 3.141592653589793;
constexpr double kT0 = 273.16;
constexpr double kCC = 8.7E-04;
constexpr double kGrav = 9.81;
constexpr double kRhoI = 910.0;
constexpr double kRhoSW = 1028.0;
constexpr double kRGas = 8.314;
// DIVA_vel_tolerance = 1e-6 is a default-REAL literal in ice_velocity_module.f90:1547
constexpr double kVelTol = (double)1e-6f;

constexpr int kMaxNz = 64;

struct Dims {
  int nx, ny, nz, ld;
  long long plane;  // nx * ld
  double dx;
  __host__ __device__ long long at(int j, int i) const { return (long long)i * ld + j; }
};

// zeta tables passed by value to kernels
struct Zeta {
  int nz;
  double z[kMaxNz];    // C%zeta
  double z2[kMaxNz];   // zeta**2 (computed on the host with pow, as the reference's zeta**n)
  double zn[kMaxNz];   // zeta**n_flow
};

// MAX and MIN as gfortran expands them for the reference (mvar = a; if (b > mvar
// .OR. isnan(mvar)) mvar = b): a NaN argument never wins.  Written out with an
// explicit NaN test so that the result does not depend on how min/max
// instructions are selected for NaN operands.
__host__ __device__ __forceinline__ double max_ref(double a, double b) { return (b > a || a != a) ? b : a; }
__host__ __device__ __forceinline__ double min_ref(double a, double b) { return (b < a || a != a) ? b : a; }

__device__ __forceinline__ double stag_margin(double v0, double v1, double H0, double H1) {
  // calc_staggered_margin, ice_velocity_module.f90:1300-1319
  if (H0 > 0.0 && H1 == 0.0) return v0;
  if (H0 == 0.0 && H1 > 0.0) return v1;
  return 0.5 * (v0 + v1);
}

// 2D launch helpers: threadIdx.x -> j (coalesced), threadIdx.y / blockIdx.y -> i
constexpr int kBX = 32, kBY = 8;
inline dim3 grid2d(int nj, int ni) { return dim3((nj + kBX - 1) / kBX, (ni + kBY - 1) / kBY); }
inline dim3 block2d() { return dim3(kBX, kBY); }

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of up to 4 values; result valid in thread 0.  blockDim <= 1024.
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N]) {
  __shared__ double sh[N][32];
  const int lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31;
  const int warp = (threadIdx.x + threadIdx.y * blockDim.x) >> 5;
  const int nwarp = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
  for (int q = 0; q < N; ++q) v[q] = warp_sum(v[q]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < N; ++q) sh[q][warp] = v[q];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < N; ++q) {
      double t = lane < nwarp ? sh[q][lane] : 0.0;
      v[q] = warp_sum(t);
    }
  }
}

}  // namespace diva
