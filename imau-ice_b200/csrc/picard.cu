// picard.cu -- the per-iteration physics of solve_DIVA / solve_SSA and the
// velocity fields computed after the viscosity iteration.
//
//   K1 k_column_prep, k_layer_viscosity, k_column_integrals (+ k_shear_rates once per solve)
//                             calc_vertical_shear_strain_rates   ice_velocity_module.f90:664-721
//                             calc_effective_viscosity (a-grid)   :722-818
//                             calc_sliding_term_beta + laws       :900-959, basal_conditions_and_sliding_module.f90:908-1236
//                             calc_F_integral(n=2)                :960-1013
//                             calc_beta_eff (a-grid)              :1014-1061
//      k_face_coefficients    N_b (:820-874), N_cx/N_cy (:876-880), beta_eff on cx/cy (:1063-1076)
//   K4 k_picard_update        apply_velocity_limits :1432-1498, relax :1499-1529,
//                             calc_visc_iter_UV_resid :1530-1601 (block partials),
//                             estimate_visc_iter_UV_errors :1602-1652,
//                             calc_basal_stress :1087-1120, calc_basal_velocities :1121-1199
//   K5 k_f1 / k_u3d           calc_3D_horizontal_velocities_DIVA  :1200-1298
//   K6 k_faces_prelude / k_secondary
//                             calc_secondary_velocities :377-533, calc_3D_vertical_velocities :534-661,
//                             map_velocity_from_c*_to_a_* :2592-2811
//   K7 k_sia                  solve_SIA :36-105
//
// One thread owns one a-grid column (j,i) and, with it, the cx face (j,i) east
// of it and the cy face (j,i) north of it.  Column loops run over the zeta
// layers, each a coalesced plane.
#include <algorithm>
#include <cmath>
#include <math_constants.h>
#include "ctx.hpp"

namespace diva {
namespace {

struct CoefArgs {
  Dims d;
  Zeta zt;
  // config
  int diva, bc_margin, sliding, gl_subgrid, basal_freezing, prescribed_tauc, n_is_3, crossterms;
  double n_flow, eps0, visc_min, beta_max, delta_v, wm, q_plastic, u_thr, zi_ut, zi_p, dT_freeze, Fmin;
  // inputs
  const double *u, *v, *visc_prev, *taub_cx, *taub_cy, *Hi, *afac;
  const int *mask_ice, *mask_ocean;
  const double *beta_sq, *phi_fric, *alpha_sq, *Neff, *Ti, *Tpmp;
  // outputs
  double *dudz, *dvdz, *visc, *visc_int, *Na, *beta, *F2, *beta_eff, *tauc;
  // per-column scratch between the three launches
  double* col_eps;
  int* col_flags;
  // the basal stress each column's shear read, kept (keep_seen) so that the shear strain
  // rates of the viscosity loop's last iteration can be written after the loop
  int keep_seen;
  double *taub_seen_cx, *taub_seen_cy;
};

// strain rates of the depth-averaged velocity on the a-grid,
// ddx_cx_to_a / ddy_cx_to_a / ddx_cy_to_a / ddy_cy_to_a (derivatives_and_grids_module.f90:755-939)
__device__ __forceinline__ double ddx_cx_to_a(const Dims& d, const double* u, int j, int i) {
  const int ii = i == 0 ? 1 : (i == d.nx - 1 ? d.nx - 2 : i);
  return (u[d.at(j, ii)] - u[d.at(j, ii - 1)]) / d.dx;
}
__device__ __forceinline__ double ddy_cy_to_a(const Dims& d, const double* v, int j, int i) {
  const int jj = j == 0 ? 1 : (j == d.ny - 1 ? d.ny - 2 : j);
  return (v[d.at(jj, i)] - v[d.at(jj - 1, i)]) / d.dx;
}
__device__ __forceinline__ double ddy_cx_to_a(const Dims& d, const double* u, int j, int i) {
  const int nx = d.nx, ny = d.ny;
  const double dx = d.dx;
  auto U = [&](int jj, int ii) { return u[d.at(jj, ii)]; };
  if (i > 0 && i < nx - 1) {
    if (j > 0 && j < ny - 1) return (U(j + 1, i - 1) + U(j + 1, i) - U(j - 1, i - 1) - U(j - 1, i)) / (4.0 * dx);
    if (j == 0) return (U(1, i - 1) + U(1, i) - U(0, i - 1) - U(0, i)) / (4.0 * dx);
    return (U(ny - 1, i - 1) + U(ny - 1, i) - U(ny - 2, i - 1) - U(ny - 2, i)) / (4.0 * dx);
  }
  const int ic = (i == 0) ? 0 : nx - 2;
  if (j > 0 && j < ny - 1) return (U(j + 1, ic) - U(j - 1, ic)) / (2.0 * dx);
  if (j == 0) return (U(1, ic) - U(0, ic)) / dx;
  return (U(ny - 1, ic) - U(ny - 2, ic)) / dx;
}
__device__ __forceinline__ double ddx_cy_to_a(const Dims& d, const double* v, int j, int i) {
  const int nx = d.nx, ny = d.ny;
  const double dx = d.dx;
  auto V = [&](int jj, int ii) { return v[d.at(jj, ii)]; };
  if (j > 0 && j < ny - 1) {
    if (i > 0 && i < nx - 1) return (V(j - 1, i + 1) + V(j, i + 1) - V(j - 1, i - 1) - V(j, i - 1)) / (4.0 * dx);
    if (i == 0) return (V(j - 1, 1) + V(j, 1) - V(j - 1, 0) - V(j, 0)) / (4.0 * dx);
    return (V(j - 1, nx - 1) + V(j, nx - 1) - V(j - 1, nx - 2) - V(j, nx - 2)) / (4.0 * dx);
  }
  const int jc = (j == 0) ? 0 : ny - 2;
  if (i > 0 && i < nx - 1) return (V(jc, i + 1) - V(jc, i - 1)) / (2.0 * dx);
  if (i == 0) return (V(jc, 1) - V(jc, 0)) / dx;
  return (V(jc, nx - 1) - V(jc, nx - 2)) / dx;
}

__device__ __forceinline__ double sliding_beta(const CoefArgs& a, long long q, double ua, double va) {
  const double uabs = sqrt(a.delta_v * a.delta_v + ua * ua + va * va);
  switch (a.sliding) {
    case DIVA_SLIDING_NONE: return 0.0;
    case DIVA_SLIDING_WEERTMAN: return a.beta_sq[q] * pow(uabs, 1.0 / a.wm - 1.0);
    case DIVA_SLIDING_COULOMB: {
      double tc = a.prescribed_tauc ? a.tauc[q] : tan((kPi / 180.0) * a.phi_fric[q]) * a.Neff[q];
      if (!a.prescribed_tauc) a.tauc[q] = tc;
      return tc / uabs;
    }
    case DIVA_SLIDING_COULOMB_REGULARISED: {
      const double tc = tan((kPi / 180.0) * a.phi_fric[q]) * a.Neff[q];
      a.tauc[q] = tc;
      return tc * pow(uabs, a.q_plastic - 1.0) / pow(a.u_thr, a.q_plastic);
    }
    case DIVA_SLIDING_TSAI2015:
      return min_ref(a.alpha_sq[q] * a.Neff[q], a.beta_sq[q] * pow(uabs, 1.0 / a.wm)) * pow(uabs, -1.0);
    case DIVA_SLIDING_SCHOOF2005: {
      const double a2 = a.alpha_sq[q], b2 = a.beta_sq[q], m = a.wm;
      return ((b2 * pow(uabs, 1.0 / m) * a2 * a.Neff[q]) / (pow(pow(b2, m) * uabs + pow(a2 * a.Neff[q], m), 1.0 / m))) *
             pow(uabs, -1.0);
    }
    case DIVA_SLIDING_ZOET_IVERSON:
      return a.Neff[q] * tan((kPi / 180.0) * a.phi_fric[q]) * (pow(uabs, 1.0 / a.zi_p - 1.0)) *
             (pow(uabs + a.zi_ut, -1.0 / a.zi_p));
  }
  return CUDART_NAN;
}

// Block shape of the layer-parallel kernels: a warp over 32 rows, 8 grid columns.
constexpr int kColLanes = 32, kColRows = 8;

// Per-column decisions of the layer step, packed by k_column_prep (and kept for k_shear_rates):
//   bits 0-3   the E, W, N, S shear face carries ice (FACE_*)
//   bits 4-11  per face, which side the staggered viscosity takes (calc_staggered_margin
//              :1300-1319): 0 the mean of both, 1 the first (west/south) side, 2 the second
//   bits 12-15 the same choice for the column's own x and y staggering of du/dz, dv/dz,
//              including the first/last grid column and row, which take one face only
//   bit 16     no viscosity in this column (BC margins outside the ice)
enum { FACE_E = 1, FACE_W = 2, FACE_N = 4, FACE_S = 8, COL_SKIP = 1 << 16 };
constexpr int kModeShift = 4, kStagXShift = 12, kStagYShift = 14;

__device__ __forceinline__ int margin_mode(double H0, double H1) {
  if (H0 > 0.0 && H1 == 0.0) return 1;
  if (H0 == 0.0 && H1 > 0.0) return 2;
  return 0;
}
// calc_staggered_margin with the side choice made beforehand (same values as stag_margin)
__device__ __forceinline__ double stag_mode(int mode, double v0, double v1) {
  return mode == 1 ? v0 : (mode == 2 ? v1 : 0.5 * (v0 + v1));
}

// K1 in three launches.  (a) k_column_prep, one thread per column: the strain rates
// of the depth-averaged flow and which of the column's four shear faces have ice.
// (b) k_layer_viscosity, one thread per (column, layer), a warp over 32 neighbouring
// rows j of one grid column i and one layer: the shear of the column's own east and
// north faces, the west face, and the south face as the north face of the lane below
// (shuffle), then the viscosity of the layer.  (c) k_column_integrals, one thread per
// column: the vertical integrals in layer order (as the sequential quadrature does), N_a,
// the sliding law, F2 and beta_eff.  The middle step is layer-parallel (15 x the threads
// of a column kernel): a single column kernel walking the layers, measured, took 104 us
// per iteration on the 321 x 561 ice cap against 75 us for the three launches, whose extra
// read of the viscosity is cheaper than the lost parallelism.  The shear strain rates
// du/dz, dv/dz (:664-721) are written by the layer step only with WRITE_SHEAR; inside the
// viscosity loop (K1_LOOP) k_column_prep keeps the basal stress it saw instead, and
// k_shear_rates writes the last iteration's shear once after the loop.
__global__ void __launch_bounds__(256) k_column_prep(CoefArgs a) {
  const Dims d = a.d;
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const int nx = d.nx, ny = d.ny;
  const long long q = d.at(j, i);
  const int* __restrict__ mask = a.mask_ice;
  const double* __restrict__ Hi = a.Hi;
  const bool ice = mask[q] == 1;
  const bool skip_visc = a.bc_margin && !ice;  // BC margins: no viscosity outside the ice (:759-764)
  // strain rates of the depth-averaged flow (calc_effective_viscosity :751-754)
  double eps_h = 0.0;
  if (!skip_visc) {
    const double du_dx = ddx_cx_to_a(d, a.u, j, i), dv_dy = ddy_cy_to_a(d, a.v, j, i);
    const double du_dy = ddy_cx_to_a(d, a.u, j, i), dv_dx = ddx_cy_to_a(d, a.v, j, i);
    eps_h = du_dx * du_dx + dv_dy * dv_dy + du_dx * dv_dy + 0.25 * ((du_dy + dv_dx) * (du_dy + dv_dx));
  }
  const double H = Hi[q];
  int flags = skip_visc ? COL_SKIP : 0;
  auto face = [&](int bit, int f, long long p0, long long p1) {
    // a face carries shear if either side has ice (calc_vertical_shear_strain_rates :685-695)
    if (a.diva && !(mask[p0] == 0 && mask[p1] == 0)) flags |= bit;
    flags |= margin_mode(Hi[p0], Hi[p1]) << (kModeShift + 2 * f);
  };
  if (i < nx - 1) face(FACE_E, 0, q, d.at(j, i + 1));
  if (i > 0) face(FACE_W, 1, d.at(j, i - 1), q);
  if (j < ny - 1) face(FACE_N, 2, q, d.at(j + 1, i));
  if (j > 0) face(FACE_S, 3, d.at(j - 1, i), q);
  // a-grid staggering of the face values: first column/row the east/north face alone (2),
  // last column/row the west/south face alone (1), else the margin rule
  const int mx = i == 0 ? 2 : (i == nx - 1 ? 1 : margin_mode(Hi[d.at(j, i - 1)], H));
  const int my = j == 0 ? 2 : (j == ny - 1 ? 1 : margin_mode(Hi[d.at(j - 1, i)], H));
  flags |= (mx << kStagXShift) | (my << kStagYShift);
  a.col_eps[q] = eps_h;
  a.col_flags[q] = flags;
  if (a.keep_seen && a.diva) {   // the basal stress this iteration's shear reads (k_shear_rates)
    if (i < nx - 1) a.taub_seen_cx[q] = a.taub_cx[q];
    if (j < ny - 1) a.taub_seen_cy[q] = a.taub_cy[q];
  }
}

// The layer step's arithmetic type R: double, or float for precision 'mixed' (the
// viscosity of the linearisation in FP32: face shears, strain rate, the rate factor's
// power and the viscosity bound; inputs and the stored viscosity stay FP64 fields).
template <class R> __device__ __forceinline__ R stag_mode_t(int mode, R v0, R v1) {
  return mode == 1 ? v0 : (mode == 2 ? v1 : R(0.5) * (v0 + v1));
}
template <class R> __device__ __forceinline__ R max_ref_t(R a, R b) { return (b > a || a != a) ? b : a; }
__device__ __forceinline__ double rcbrt_t(double x) { return rcbrt(x); }
__device__ __forceinline__ float rcbrt_t(float x) { return rcbrtf(x); }
__device__ __forceinline__ double pow_t(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float pow_t(float x, float y) { return powf(x, y); }

template <bool WRITE_SHEAR, class R>
__global__ void __launch_bounds__(kColLanes * kColRows) k_layer_viscosity(CoefArgs a) {
  const Dims d = a.d;
  const int lane = threadIdx.x;
  // the layer is the fastest grid index: blocks running together share their columns'
  // 2D inputs in L1/L2 instead of streaming them once per layer
  const int k = blockIdx.x, j = blockIdx.y * kColLanes + lane, i = blockIdx.z * kColRows + threadIdx.y;
  const bool row = i < d.nx;   // whole warps: i is uniform across a warp; idle warps stay for the barrier
  const bool col = row && j < d.ny;   // lanes past the last row stay for the shuffle
  const int nx = d.nx, ny = d.ny, ld = d.ld;
  const int q = (row ? i : nx - 1) * ld + (j < ny ? j : ny - 1);   // plane index (planes hold < 2^31 points)
  const long long off = (long long)k * d.plane;
  const double* __restrict__ vp = a.visc_prev + off;
  const R zk = (R)a.zt.z[k];
  const int flags = a.col_flags[q];
  const bool has_e = col && i < nx - 1, has_w = col && i > 0, has_n = col && j < ny - 1, has_s = col && j > 0;
  auto mode = [&](int f) { return (flags >> (kModeShift + 2 * f)) & 3; };
  auto shear = [&](double tb, double v0, double v1, int m) { return ((R)tb / stag_mode_t<R>(m, (R)v0, (R)v1)) * zk; };
  // the west face of column i is the east face of column i-1: the warp below in the block
  // computed it (the same operands, so the same value), the block's first warp computes it
  __shared__ R east[kColRows][kColLanes];
  R dudz_e = R(0), dvdz_n = R(0), dvdz_s = R(0), dudz_w = R(0);
  if (a.diva) {
    const double vq = vp[q];
    if (has_e) {
      if (flags & FACE_E) dudz_e = shear(a.taub_cx[q], vq, vp[q + ld], mode(0));
      if (WRITE_SHEAR) a.dudz[off + q] = (double)dudz_e;
    }
    east[threadIdx.y][lane] = dudz_e;
    if (has_n) {
      if (flags & FACE_N) dvdz_n = shear(a.taub_cy[q], vq, vp[q + 1], mode(2));
      if (WRITE_SHEAR) a.dvdz[off + q] = (double)dvdz_n;
    }
    dvdz_s = __shfl_up_sync(0xffffffffu, dvdz_n, 1);   // north face of row j-1
    if (lane == 0 && has_s) dvdz_s = (flags & FACE_S) ? shear(a.taub_cy[q - 1], vp[q - 1], vq, mode(3)) : R(0);
    __syncthreads();
    if (has_w && (flags & FACE_W))
      dudz_w = threadIdx.y > 0 ? east[threadIdx.y - 1][lane] : shear(a.taub_cx[q - ld], vp[q - ld], vq, mode(1));
  }
  if (!col) return;
  R eta = R(0);
  if (!(flags & COL_SKIP)) {
    const int mx = (flags >> kStagXShift) & 3, my = (flags >> kStagYShift) & 3;
    R du_dz_a, dv_dz_a;
    if (a.diva) {
      du_dz_a = stag_mode_t<R>(mx, dudz_w, dudz_e);
      dv_dz_a = stag_mode_t<R>(my, dvdz_s, dvdz_n);
    } else {
      // solve_SSA calls calc_effective_viscosity without refreshing du/dz: use the stored fields
      const double* dudz = a.dudz + off;
      const double* dvdz = a.dvdz + off;
      du_dz_a = stag_mode_t<R>(mx, (R)(i > 0 ? dudz[q - ld] : 0.0), (R)(i < nx - 1 ? dudz[q] : 0.0));
      dv_dz_a = stag_mode_t<R>(my, (R)(j > 0 ? dvdz[q - 1] : 0.0), (R)(j < ny - 1 ? dvdz[q] : 0.0));
    }
    const R eps_sq = (R)a.col_eps[q] + R(0.25) * (du_dz_a * du_dz_a + dv_dz_a * dv_dz_a) + (R)a.eps0;
    const R pe = a.n_is_3 ? rcbrt_t(eps_sq) : pow_t(eps_sq, (R)((1.0 - a.n_flow) / (2.0 * a.n_flow)));
    eta = max_ref_t<R>((R)a.afac[off + q] * pe, (R)a.visc_min);   // NaN (first cold iteration) -> visc_min
  }
  a.visc[off + q] = (double)eta;
}

// NZ > 0: the layer count known at compile time (the default 15 layers), so the loop is
// unrolled and every layer's load is in flight at once; NZ = 0: any layer count.
template <int NZ, class R>
__global__ void __launch_bounds__(256) k_column_integrals(CoefArgs a) {
  const Dims d = a.d;
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const int nx = d.nx, ny = d.ny, nz = NZ > 0 ? NZ : d.nz;
  const long long q = d.at(j, i);
  const double H = a.Hi[q];
  const bool ice = a.mask_ice[q] == 1;
  const bool skip_visc = a.bc_margin && !ice;
  const double* __restrict__ visc = a.visc;
  double vint = 0.0, fint = 0.0, vprev = 0.0, fprev = 0.0;
#pragma unroll
  for (int k = 0; k < nz; ++k) {
    const double eta = visc[(long long)k * d.plane + q];
    const double zk = a.zt.z[k];
    if (k > 0) vint = vint + 0.5 * (eta + vprev) * (zk - a.zt.z[k - 1]);
    vprev = eta;
    if (a.diva) {
      const double fk = (double)(((R)H / (R)eta) * (R)a.zt.z2[k]);
      if (k > 0) fint = fint + 0.5 * (fk + fprev) * (zk - a.zt.z[k - 1]);
      fprev = fk;
    }
  }
  if (!skip_visc) {
    a.visc_int[q] = vint;
    a.Na[q] = a.bc_margin ? vint * H : vint * max_ref(0.1, H);
  }
  // sliding (calc_sliding_term_beta :924-951)
  double ua, va;
  if (i == 0) ua = a.u[d.at(j, 0)];
  else if (i == nx - 1) ua = a.u[d.at(j, nx - 2)];
  else ua = (a.u[d.at(j, i - 1)] + a.u[q]) / 2.0;
  if (j == 0) va = a.v[d.at(0, i)];
  else if (j == ny - 1) va = a.v[d.at(ny - 2, i)];
  else va = (a.v[d.at(j - 1, i)] + a.v[q]) / 2.0;
  double beta = min_ref(sliding_beta(a, q, ua, va), a.beta_max);
  if (!a.gl_subgrid && a.mask_ocean[q] == 1) beta = 0.0;
  a.beta[q] = beta;
  if (a.diva) {
    double F2;
    if (ice) F2 = max_ref(a.Fmin, fint);
    else F2 = a.bc_margin ? 0.0 : a.Fmin;
    a.F2[q] = F2;
    double be;
    if (a.sliding == DIVA_SLIDING_NONE) {
      be = 1.0 / F2;
    } else {
      be = beta / (1.0 + beta * F2);
      if (a.basal_freezing) {
        const long long ob = (long long)(nz - 1) * d.plane + q;
        if (a.Tpmp[ob] - a.Ti[ob] > a.dT_freeze) be = 1.0 / F2;
      }
    }
    a.beta_eff[q] = be;
  } else {
    a.beta_eff[q] = beta;   // solve_SSA :193
  }
}


// The shear strain rates du/dz, dv/dz (calc_vertical_shear_strain_rates :664-721) of the last
// viscosity iteration, from the flags and basal stress its fused K1 kept and the viscosity
// it read: the values a K1 that writes them would have left.  Layer-parallel.
template <class R>
__global__ void __launch_bounds__(kColLanes * kColRows) k_shear_rates(CoefArgs a) {
  const Dims d = a.d;
  const int lane = threadIdx.x;
  const int k = blockIdx.x, j = blockIdx.y * kColLanes + lane, i = blockIdx.z * kColRows + threadIdx.y;
  if (i >= d.nx) return;
  const bool col = j < d.ny;
  const int nx = d.nx, ny = d.ny, ld = d.ld;
  const long long q = d.at(col ? j : ny - 1, i);
  const long long off = (long long)k * d.plane;
  const double* __restrict__ vp = a.visc_prev + off;
  const R zk = (R)a.zt.z[k];
  const int flags = a.col_flags[q];
  auto mode = [&](int f) { return (flags >> (kModeShift + 2 * f)) & 3; };
  auto shear = [&](double tb, double v0, double v1, int m) { return ((R)tb / stag_mode_t<R>(m, (R)v0, (R)v1)) * zk; };
  if (!col) return;
  if (i < nx - 1) a.dudz[off + q] = (double)((flags & FACE_E) ? shear(a.taub_seen_cx[q], vp[q], vp[q + ld], mode(0)) : R(0));
  if (j < ny - 1) a.dvdz[off + q] = (double)((flags & FACE_N) ? shear(a.taub_seen_cy[q], vp[q], vp[q + 1], mode(2)) : R(0));
}

struct FaceArgs {
  Dims d;
  int bc_margin, apply_fgrnd, crossterms;
  const double *vint, *Hb_i, *beta_eff, *fcx, *fcy, *Na;
  const int* mask_ice;
  double *visc_int_b, *Nb, *bex, *bey, *Ncx, *Ncy;
  double *lvBx, *lvBy, *lvNa, *lvNb;   // level-0 operator coefficients (Bx = beta_eff_cx * dx^2)
};

__global__ void __launch_bounds__(256) k_face_coefficients(FaceArgs a) {
  const Dims d = a.d;
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  const double dx2 = d.dx * d.dx;
  if (i < d.nx - 1 && j < d.ny - 1) {
    // the 3D viscosity staggered to the b-grid and integrated over the column (:820-874).
    // The staggering is a fixed weighting of the four corner columns and the trapezoid rule
    // is linear, so the integral is the same weighting of the corners' integrals (equal up
    // to rounding): the 3D viscosity is not read again.
    const long long q1 = d.at(j, i + 1), q2 = d.at(j + 1, i), q3 = d.at(j + 1, i + 1);
    double s;
    if (a.bc_margin) {
      const int m0 = a.mask_ice[q] == 1, m1 = a.mask_ice[q1] == 1, m2 = a.mask_ice[q2] == 1, m3 = a.mask_ice[q3] == 1;
      const double w = (double)m0 + (double)m1 + (double)m2 + (double)m3;
      double vb = 0.0;
      if (m0) vb = vb + a.vint[q];
      if (m1) vb = vb + a.vint[q1];
      if (m2) vb = vb + a.vint[q2];
      if (m3) vb = vb + a.vint[q3];
      s = w > 0.0 ? vb / w : 0.0;
    } else {
      s = (a.vint[q] + a.vint[q1] + a.vint[q2] + a.vint[q3]) / 4.0;
    }
    a.visc_int_b[q] = s;
    const double nb = a.bc_margin ? s * a.Hb_i[q] : s * max_ref(0.1, a.Hb_i[q]);
    a.Nb[q] = nb;
    a.lvNb[q] = a.crossterms ? nb : 1.0;
  }
  if (i < d.nx - 1) {
    double b = (a.beta_eff[q] + a.beta_eff[d.at(j, i + 1)]) / 2.0;
    if (a.apply_fgrnd) b = b * (a.fcx[q] * a.fcx[q]);
    a.bex[q] = b;
    if (a.crossterms) {
      a.lvBx[q] = b * dx2;
    } else {
      const double ncx = (a.Na[q] + a.Na[d.at(j, i + 1)]) / 2.0;
      a.Ncx[q] = ncx;
      a.lvBx[q] = dx2 * b / ncx;
    }
  }
  if (j < d.ny - 1) {
    double b = (a.beta_eff[q] + a.beta_eff[d.at(j + 1, i)]) / 2.0;
    if (a.apply_fgrnd) b = b * (a.fcy[q] * a.fcy[q]);
    a.bey[q] = b;
    if (a.crossterms) {
      a.lvBy[q] = b * dx2;
    } else {
      const double ncy = (a.Na[q] + a.Na[d.at(j + 1, i)]) / 2.0;
      a.Ncy[q] = ncy;
      a.lvBy[q] = dx2 * b / ncy;
    }
  }
  a.lvNa[q] = a.crossterms ? a.Na[q] : 1.0;
}

// 0.5 * A^(-1/n): constant over one solve, so the pow of A is taken once per solve
__global__ void k_afac(Dims d, double n_flow, const double* A, double* afac) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const double e = -1.0 / n_flow;
  for (int k = 0; k < d.nz; ++k) {
    const long long o = (long long)k * d.plane + d.at(j, i);
    afac[o] = 0.5 * pow(A[o], e);
  }
}

// apply_velocity_limits (:1432-1498) of the linear solution at a cx point: |u| with v mapped
// to the cx grid (map_cy_to_cx_2D :1757-1797), scaled down to vmax
__device__ __forceinline__ double limited_u(const Dims& d, const double* xu, const double* xv, double vmax, int j,
                                            int i) {
  const int ny = d.ny;
  auto XV = [&](int jj, int ii) { return xv[d.at(jj, ii)]; };
  double vcx;
  if (j > 0 && j < ny - 1) vcx = (XV(j - 1, i) + XV(j - 1, i + 1) + XV(j, i) + XV(j, i + 1)) / 4.0;
  else if (j == 0) vcx = (XV(0, i) + XV(0, i + 1)) / 2.0;
  else vcx = (XV(ny - 2, i) + XV(ny - 2, i + 1)) / 2.0;
  double un = xu[d.at(j, i)];
  const double uabs = sqrt(un * un + vcx * vcx);
  if (uabs > vmax) un = un * vmax / uabs;
  return un;
}
// the same at a cy point, u mapped to the cy grid (map_cx_to_cy_2D :1718-1756)
__device__ __forceinline__ double limited_v(const Dims& d, const double* xu, const double* xv, double vmax, int j,
                                            int i) {
  const int nx = d.nx;
  auto XU = [&](int jj, int ii) { return xu[d.at(jj, ii)]; };
  double ucy;
  if (i > 0 && i < nx - 1) ucy = (XU(j, i - 1) + XU(j, i) + XU(j + 1, i - 1) + XU(j + 1, i)) / 4.0;
  else if (i == 0) ucy = (XU(j, 0) + XU(j + 1, 0)) / 2.0;
  else ucy = (XU(j, nx - 2) + XU(j + 1, nx - 2)) / 2.0;
  double vn = xv[d.at(j, i)];
  const double vabs = sqrt(ucy * ucy + vn * vn);
  if (vabs > vmax) vn = vn * vmax / vabs;
  return vn;
}

// ---- Anderson mixing of the viscosity iteration (picard_anderson_m > 0) --------------
// No counterpart in the reference, whose update is the relaxation :1499-1529.  The map is
// one unrelaxed Picard step, g(u) = velocity-limited solution of A(u) x = b(u); with the
// residual f = g(u) - u and the differences dF_i = f_i+1 - f_i, dG_i = g_i+1 - g_i of the
// last m iterations, the next iterate is g - sum_i gamma_i dG_i, gamma the least-squares
// minimiser of |f - sum_i gamma_i dF_i| (u on the cx points and v on the cy points make
// one vector).  k_aa_prepare writes g, f and the newest difference columns and reduces
// the inner products of the newest dF and of f with every history column; k_aa_solve
// updates the Gram matrix and solves for gamma on one thread; k_picard_update mixes.
struct AAArgs {
  Dims d;
  int m, nblk_x;
  double vmax;
  const double *u, *v, *xu, *xv;
  double *dFu[kAAMax], *dFv[kAAMax], *dGu[kAAMax], *dGv[kAAMax];
  double *fu, *fv, *gu, *gv;   // previous f, g on entry; this iteration's on exit
  const double* sc;
  double* partials;            // kAAPartials per block: dF_i . dF_new, then dF_i . f
};

__global__ void __launch_bounds__(256) k_aa_prepare(AAArgs a) {
  const Dims d = a.d;
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  const bool have = a.sc[SC_AA_HAVE] != 0.0;
  const int s = (int)a.sc[SC_AA_HEAD];
  double acc[kAAPartials];
#pragma unroll
  for (int k = 0; k < kAAPartials; ++k) acc[k] = 0.0;
  if (j < d.ny && i < d.nx) {
    const long long q = d.at(j, i);
    auto point = [&](double g, double x, double* fp, double* gp, double* const* dF, double* const* dG) {
      const double f = g - x;
      if (have) {
        const double df = f - fp[q];
#pragma unroll
        for (int k = 0; k < kAAMax; ++k)
          if (k == s) {
            dF[k][q] = df;
            dG[k][q] = g - gp[q];
          }
#pragma unroll
        for (int k = 0; k < kAAMax; ++k) {
          if (k < a.m) {
            const double c = (k == s) ? df : dF[k][q];
            acc[k] += c * df;
            acc[kAAMax + k] += c * f;
          }
        }
      }
      fp[q] = f;
      gp[q] = g;
    };
    if (i < d.nx - 1) point(limited_u(d, a.xu, a.xv, a.vmax, j, i), a.u[q], a.fu, a.gu, a.dFu, a.dGu);
    if (j < d.ny - 1) point(limited_v(d, a.xu, a.xv, a.vmax, j, i), a.v[q], a.fv, a.gv, a.dFv, a.dGv);
  }
  // block sums in groups of at most four values (block_sum keeps one shared array per width)
  double* out = a.partials + (long long)kAAPartials * (blockIdx.y * a.nblk_x + blockIdx.x);
  for (int base = 0; base < kAAPartials; base += 4) {
    double v4[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) v4[k] = base + k < kAAPartials ? acc[base + k] : 0.0;
    block_sum<4>(v4);
    if (threadIdx.x == 0 && threadIdx.y == 0)
      for (int k = 0; k < 4 && base + k < kAAPartials; ++k) out[base + k] = v4[k];
    __syncthreads();
  }
}

// One thread: fixed-order sums of the partials, the Gram matrix update and the mixing
// coefficients.  Shared with the oracle's restatement (aa_coefficients).
__global__ void k_aa_solve(const double* partials, int nblocks, int m, double* sc) {
  __shared__ double sh[kAAPartials][256];
  double t[kAAPartials];
#pragma unroll
  for (int k = 0; k < kAAPartials; ++k) t[k] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int k = 0; k < kAAPartials; ++k) t[k] += partials[(long long)kAAPartials * b + k];
  for (int k = 0; k < kAAPartials; ++k) sh[k][threadIdx.x] = t[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < kAAPartials; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  double dots[kAAPartials];
  for (int k = 0; k < kAAPartials; ++k) dots[k] = sh[k][0];
  aa_coefficients(sc, m, dots);
}

struct UpdArgs {
  Dims d;
  int diva, sliding_none, basal_freezing, nblk_x;
  double vmax, rel, dT_freeze;
  const double *xu, *xv;           // linear solution
  double *u, *v, *up, *vp;         // velocities (relaxed in place) and the previous iterate
  // Anderson mixing (aa_m > 0): the iterate is g - sum gamma_i dG_i instead of the relaxation
  int aa_m;
  const double* sc;
  const double *gu, *gv;
  const double *dGu[kAAMax], *dGv[kAAMax];
  const double *uchk, *vchk;       // fields tested by estimate_visc_iter_UV_errors
  double *errx, *erry;             // DIVA_err candidates
  const double *bex, *bey, *F2, *Hi, *Ti, *Tpmp;
  double *taubx, *tauby, *ubx, *vby;
  double* partials;                // 3 per block
};

__global__ void __launch_bounds__(256) k_picard_update(UpdArgs a) {
  const Dims d = a.d;
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  double sums[3] = {0.0, 0.0, 0.0};
  if (j < d.ny && i < d.nx) {
    const int nx = d.nx, ny = d.ny;
    const long long q = d.at(j, i);
    bool frozen = false;
    if (a.diva && a.basal_freezing) {
      const long long ob = (long long)(d.nz - 1) * d.plane + q;
      frozen = a.Tpmp[ob] - a.Ti[ob] > a.dT_freeze;
    }
    if (i < nx - 1) {
      const double uo = a.u[q];
      double un;
      if (a.aa_m > 0 && a.sc[SC_AA_OFF] != 0.0) {
        un = a.rel * a.gu[q] + (1.0 - a.rel) * uo;   // mixing given up: the relaxation of g
      } else if (a.aa_m > 0) {
        un = a.gu[q];
        for (int k = 0; k < a.aa_m; ++k) un -= a.sc[SC_AA_GAMMA + k] * a.dGu[k][q];
      } else {
        un = limited_u(d, a.xu, a.xv, a.vmax, j, i);
        un = a.rel * un + (1.0 - a.rel) * uo;
      }
      a.up[q] = uo;
      a.u[q] = un;
      if (fabs(un) > kVelTol) {
        sums[2] += 1.0;
        sums[0] += (un - uo) * (un - uo);
        sums[1] += (un + uo) * (un + uo);
      }
      const double chk = a.diva ? un : a.uchk[q];
      a.errx[q] = (fabs(chk) > kVelTol) ? 2.0 * fabs(un - uo) / fabs(un + uo + 1E-5) : 0.0;
      if (a.diva) {
        const double tb = a.bex[q] * un;
        a.taubx[q] = tb;
        if (a.sliding_none) {
          a.ubx[q] = 0.0;
        } else {
          const double F2s = stag_margin(a.F2[q], a.F2[d.at(j, i + 1)], a.Hi[q], a.Hi[d.at(j, i + 1)]);
          a.ubx[q] = frozen ? 0.0 : un - tb * F2s;
        }
      }
    }
    if (j < ny - 1) {
      const double vo = a.v[q];
      double vn;
      if (a.aa_m > 0 && a.sc[SC_AA_OFF] != 0.0) {
        vn = a.rel * a.gv[q] + (1.0 - a.rel) * vo;
      } else if (a.aa_m > 0) {
        vn = a.gv[q];
        for (int k = 0; k < a.aa_m; ++k) vn -= a.sc[SC_AA_GAMMA + k] * a.dGv[k][q];
      } else {
        vn = limited_v(d, a.xu, a.xv, a.vmax, j, i);
        vn = a.rel * vn + (1.0 - a.rel) * vo;
      }
      a.vp[q] = vo;
      a.v[q] = vn;
      if (fabs(vn) > kVelTol) {
        sums[2] += 1.0;
        sums[0] += (vn - vo) * (vn - vo);
        sums[1] += (vn + vo) * (vn + vo);
      }
      const double chk = a.diva ? vn : a.vchk[q];
      a.erry[q] = (fabs(chk) > kVelTol) ? 2.0 * fabs(vn - vo) / fabs(vn + vo + 1E-5) : 0.0;
      if (a.diva) {
        const double tb = a.bey[q] * vn;
        a.tauby[q] = tb;
        if (a.sliding_none) {
          a.vby[q] = 0.0;
        } else {
          const double F2s = stag_margin(a.F2[q], a.F2[d.at(j + 1, i)], a.Hi[q], a.Hi[d.at(j + 1, i)]);
          a.vby[q] = frozen ? 0.0 : vn - tb * F2s;
        }
      }
    }
  }
  block_sum<3>(sums);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const int b = blockIdx.y * a.nblk_x + blockIdx.x;
    a.partials[3 * b + 0] = sums[0];
    a.partials[3 * b + 1] = sums[1];
    a.partials[3 * b + 2] = sums[2];
  }
}

// fixed-order sum of block partials (deterministic)
__global__ void k_sum_partials(const double* partials, int nblocks, int width, double* out) {
  __shared__ double sh[256];
  for (int w = 0; w < width; ++w) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partials[(long long)width * b + w];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[w] = sh[0];
    __syncthreads();
  }
}

// calc_basal_stress + calc_basal_velocities at the current velocities (used when
// the viscosity iteration stops on the nonlinear residual before a linear solve)
__global__ void k_basal_stress_velocities(Dims d, int sliding_none, int basal_freezing, double dT, const double* u,
                                          const double* v, const double* bex, const double* bey, const double* F2,
                                          const double* Hi, const double* Ti, const double* Tpmp, double* tbx,
                                          double* tby, double* ubx, double* vby, const double* pred) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  if (pred && *pred == 0.0) return;   // graph launch: only when the iteration stopped on the nonlinear residual
  const long long q = d.at(j, i);
  bool frozen = false;
  if (basal_freezing) {
    const long long ob = (long long)(d.nz - 1) * d.plane + q;
    frozen = Tpmp[ob] - Ti[ob] > dT;
  }
  if (i < d.nx - 1) {
    const double tb = bex[q] * u[q];
    tbx[q] = tb;
    const double F2s = stag_margin(F2[q], F2[d.at(j, i + 1)], Hi[q], Hi[d.at(j, i + 1)]);
    ubx[q] = sliding_none ? 0.0 : (frozen ? 0.0 : u[q] - tb * F2s);
  }
  if (j < d.ny - 1) {
    const double tb = bey[q] * v[q];
    tby[q] = tb;
    const double F2s = stag_margin(F2[q], F2[d.at(j + 1, i)], Hi[q], Hi[d.at(j + 1, i)]);
    vby[q] = sliding_none ? 0.0 : (frozen ? 0.0 : v[q] - tb * F2s);
  }
}

// visc_eff_3D_b of the last viscosity iteration (:820-858), written once per solve
__global__ void k_visc_b(Dims d, int bc_margin, const double* visc, const int* mask_ice, double* vb) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny - 1 || i >= d.nx - 1) return;
  const long long q = d.at(j, i), q1 = d.at(j, i + 1), q2 = d.at(j + 1, i), q3 = d.at(j + 1, i + 1);
  int m0 = 1, m1 = 1, m2 = 1, m3 = 1;
  double w = 0.0;
  if (bc_margin) {
    m0 = mask_ice[q] == 1; m1 = mask_ice[q1] == 1; m2 = mask_ice[q2] == 1; m3 = mask_ice[q3] == 1;
    w = (double)m0 + (double)m1 + (double)m2 + (double)m3;
  }
  for (int k = 0; k < d.nz; ++k) {
    const long long o = (long long)k * d.plane;
    double s;
    if (bc_margin) {
      s = 0.0;
      if (m0) s = s + visc[o + q];
      if (m1) s = s + visc[o + q1];
      if (m2) s = s + visc[o + q2];
      if (m3) s = s + visc[o + q3];
      if (w > 0.0) s = s / w;
    } else {
      s = (visc[o + q] + visc[o + q1] + visc[o + q2] + visc[o + q3]) / 4.0;
    }
    vb[o + q] = s;
  }
}

// F1(zeta) = int_base^zeta (-H/eta) zeta dzeta on the a-grid (:1222-1227)
__global__ void k_f1(Dims d, Zeta zt, const double* Hi, const double* visc, double* F1) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  const double H = Hi[q];
  const int nz = d.nz;
  double acc = 0.0;
  double fk1 = (-H / visc[(long long)(nz - 1) * d.plane + q]) * zt.z[nz - 1];
  F1[(long long)(nz - 1) * d.plane + q] = 0.0;
  for (int k = nz - 2; k >= 0; --k) {
    const double fk = (-H / visc[(long long)k * d.plane + q]) * zt.z[k];
    acc = acc - 0.5 * (fk1 + fk) * (zt.z[k + 1] - zt.z[k]);
    F1[(long long)k * d.plane + q] = acc;
    fk1 = fk;
  }
}

// u_3D = u_base + taub * F1_stag (:1229-1289)
__global__ void k_u3d(Dims d, int bc_margin, const double* Hi, const double* F1, const double* ubx, const double* vby,
                      const double* tbx, const double* tby, double* u3, double* v3) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  if (i < d.nx - 1) {
    const long long q1 = d.at(j, i + 1);
    const double H0 = Hi[q], H1 = Hi[q1];
    for (int k = 0; k < d.nz; ++k) {
      const long long o = (long long)k * d.plane;
      const double f0 = F1[o + q], f1 = F1[o + q1];
      double s;
      if (bc_margin) {
        if (H0 > 0.0 && H1 == 0.0) s = f0;
        else if (H0 == 0.0 && H1 > 0.0) s = f1;
        else if (H0 > 0.0 && H1 > 0.0) s = 0.5 * (f0 + f1);
        else s = 0.0;
      } else {
        s = 0.5 * (f0 + f1);
      }
      u3[o + q] = ubx[q] + tbx[q] * s;
    }
  }
  if (j < d.ny - 1) {
    const long long q1 = d.at(j + 1, i);
    const double H0 = Hi[q], H1 = Hi[q1];
    for (int k = 0; k < d.nz; ++k) {
      const long long o = (long long)k * d.plane;
      const double f0 = F1[o + q], f1 = F1[o + q1];
      double s;
      if (bc_margin) {
        if (H0 > 0.0 && H1 == 0.0) s = f0;
        else if (H0 == 0.0 && H1 > 0.0) s = f1;
        else if (H0 > 0.0 && H1 > 0.0) s = 0.5 * (f0 + f1);
        else s = 0.0;
      } else {
        s = 0.5 * (f0 + f1);
      }
      v3[o + q] = vby[q] + tby[q] * s;
    }
  }
}

// Per-face part of calc_secondary_velocities (:393-485): the 3D cx/cy fields per
// mode, base velocities, surface velocities and (SIA, SIA/SSA) vertical averages.
__global__ void k_faces_prelude(Dims d, Zeta zt, int dyn, double* u3, double* v3, const double* u3s,
                                const double* v3s, const double* uS, const double* vS, double* ub, double* vb,
                                double* us, double* vs, double* uv, double* vv) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  for (int face = 0; face < 2; ++face) {
    if (face == 0 && i >= d.nx - 1) continue;
    if (face == 1 && j >= d.ny - 1) continue;
    double* f3 = face == 0 ? u3 : v3;
    const double* s3 = face == 0 ? u3s : v3s;
    const double sS = face == 0 ? uS[q] : vS[q];
    double* base = face == 0 ? ub : vb;
    double* surf = face == 0 ? us : vs;
    double* vav = face == 0 ? uv : vv;
    if (dyn == DIVA_DYN_SIA) {
      for (int k = 0; k < d.nz; ++k) f3[(long long)k * d.plane + q] = s3[(long long)k * d.plane + q];
      base[q] = 0.0;
    } else if (dyn == DIVA_DYN_SSA) {
      base[q] = sS;
      vav[q] = sS;
      for (int k = 0; k < d.nz; ++k) f3[(long long)k * d.plane + q] = sS;
    } else if (dyn == DIVA_DYN_SIA_SSA) {
      for (int k = 0; k < d.nz; ++k) f3[(long long)k * d.plane + q] = s3[(long long)k * d.plane + q] + sS;
      base[q] = sS;
    }
    surf[q] = f3[q];
    if (dyn == DIVA_DYN_SIA || dyn == DIVA_DYN_SIA_SSA) {
      double avg = 0.0;
      for (int k = 0; k < d.nz - 1; ++k)
        avg = avg + 0.5 * (f3[(long long)(k + 1) * d.plane + q] + f3[(long long)k * d.plane + q]) *
                        (zt.z[k + 1] - zt.z[k]);
      vav[q] = avg;
    }
  }
}

struct SecArgs {
  Dims d;
  Zeta zt;
  int dyn, do_w;
  const double *u3, *v3, *Hs, *Hi, *dHs_dx, *dHs_dy, *dHi_dx, *dHi_dy, *dHb_dt;
  const double *uv, *vv, *us, *vs, *ub, *vb;
  const int *sheet, *ice;
  double *w, *ws, *wb, *u3a, *v3a, *uva, *vva, *usa, *vsa, *uba, *vba, *abv, *abs_, *abb, *Rs;
};

// map_velocity_from_cx_to_a (:2592-2701) for one value, mask_ice along x
__device__ __forceinline__ double map_cx_a(const Dims& d, const int* ice, const double* f, long long off, int j, int i) {
  if (i == 0) return ice[d.at(j, 0)] == 1 ? f[off + d.at(j, 0)] : 0.0;
  if (i == d.nx - 1) return ice[d.at(j, i)] == 1 ? f[off + d.at(j, i - 1)] : 0.0;
  const int m0 = ice[d.at(j, i - 1)], m1 = ice[d.at(j, i)], m2 = ice[d.at(j, i + 1)];
  if (m0 == 1 && m1 == 1 && m2 == 1) return 0.5 * (f[off + d.at(j, i - 1)] + f[off + d.at(j, i)]);
  if (m0 == 0 && m1 == 1 && m2 == 1) return f[off + d.at(j, i)];
  if (m0 == 1 && m1 == 1 && m2 == 0) return f[off + d.at(j, i - 1)];
  return 0.0;
}
// map_velocity_from_cy_to_a (:2702-2811), mask_ice along y
__device__ __forceinline__ double map_cy_a(const Dims& d, const int* ice, const double* f, long long off, int j, int i) {
  if (j == 0) return ice[d.at(0, i)] == 1 ? f[off + d.at(0, i)] : 0.0;
  if (j == d.ny - 1) return ice[d.at(j, i)] == 1 ? f[off + d.at(j - 1, i)] : 0.0;
  const int m0 = ice[d.at(j - 1, i)], m1 = ice[d.at(j, i)], m2 = ice[d.at(j + 1, i)];
  if (m0 == 1 && m1 == 1 && m2 == 1) return 0.5 * (f[off + d.at(j - 1, i)] + f[off + d.at(j, i)]);
  if (m0 == 0 && m1 == 1 && m2 == 1) return f[off + d.at(j, i)];
  if (m0 == 1 && m1 == 1 && m2 == 0) return f[off + d.at(j - 1, i)];
  return 0.0;
}

__global__ void __launch_bounds__(256) k_secondary(SecArgs a) {
  const Dims d = a.d;
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const long long q = d.at(j, i), P = d.plane;
  const double dx = d.dx;
  if (a.do_w) {
    // calc_3D_vertical_velocities :562-650; surface/thickness slopes recomputed from Hs, Hi (:563-566)
    auto A = [&](const double* f, int jj, int ii) { return f[d.at(jj, ii)]; };
    double sx, sy, hx, hy;
    if (i > 0 && i < nx - 1) { sx = (A(a.Hs, j, i + 1) - A(a.Hs, j, i - 1)) / (2 * dx); hx = (A(a.Hi, j, i + 1) - A(a.Hi, j, i - 1)) / (2 * dx); }
    else if (i == 0) { sx = (A(a.Hs, j, 1) - A(a.Hs, j, 0)) / dx; hx = (A(a.Hi, j, 1) - A(a.Hi, j, 0)) / dx; }
    else { sx = (A(a.Hs, j, nx - 1) - A(a.Hs, j, nx - 2)) / dx; hx = (A(a.Hi, j, nx - 1) - A(a.Hi, j, nx - 2)) / dx; }
    if (j > 0 && j < ny - 1) { sy = (A(a.Hs, j + 1, i) - A(a.Hs, j - 1, i)) / (2 * dx); hy = (A(a.Hi, j + 1, i) - A(a.Hi, j - 1, i)) / (2 * dx); }
    else if (j == 0) { sy = (A(a.Hs, 1, i) - A(a.Hs, 0, i)) / dx; hy = (A(a.Hi, 1, i) - A(a.Hi, 0, i)) / dx; }
    else { sy = (A(a.Hs, ny - 1, i) - A(a.Hs, ny - 2, i)) / dx; hy = (A(a.Hi, ny - 1, i) - A(a.Hi, ny - 2, i)) / dx; }
    const double dHbase_dx = sx - hx, dHbase_dy = sy - hy;
    const long long ob = (long long)(nz - 1) * P;
    double ubase, vbase;
    if (i == 0) ubase = a.u3[ob + d.at(j, 0)];
    else if (i == nx - 1) ubase = a.u3[ob + d.at(j, nx - 2)];
    else ubase = 0.5 * (a.u3[ob + d.at(j, i - 1)] + a.u3[ob + d.at(j, i)]);
    if (j == 0) vbase = a.v3[ob + d.at(0, i)];
    else if (j == ny - 1) vbase = a.v3[ob + d.at(ny - 2, i)];
    else vbase = 0.5 * (a.v3[ob + d.at(j - 1, i)] + a.v3[ob + d.at(j, i)]);
    double wk1 = (ubase * dHbase_dx) + (vbase * dHbase_dy);
    if (a.sheet[q] == 1) wk1 = wk1 + a.dHb_dt[q];
    a.w[ob + q] = wk1;
    // x and y index pairs of the divergence stencil (:603-622)
    const int ia = (i == 0) ? 1 : (i == nx - 1 ? nx - 2 : i), ib = ia - 1;
    const int ja = (j == 0) ? 1 : (j == ny - 1 ? ny - 2 : j), jb = ja - 1;
    const double H = a.Hi[q], Hm = max_ref(0.1, H);
    const double gsx = a.dHs_dx[q], gsy = a.dHs_dy[q], gix = a.dHi_dx[q], giy = a.dHi_dy[q];
    double du_kp1 = (a.u3[ob + d.at(j, ia)] - a.u3[ob + d.at(j, ib)]) / dx;
    double dv_kp1 = (a.v3[ob + d.at(ja, i)] - a.v3[ob + d.at(jb, i)]) / dx;
    double ua_kp1 = a.u3a[ob + q], va_kp1 = a.v3a[ob + q];   // stale a-grid velocities (read before refresh)
    for (int k = nz - 2; k >= 0; --k) {
      const long long o = (long long)k * P;
      const double du_k = (a.u3[o + d.at(j, ia)] - a.u3[o + d.at(j, ib)]) / dx;
      const double dv_k = (a.v3[o + d.at(ja, i)] - a.v3[o + d.at(jb, i)]) / dx;
      const double ua_k = a.u3a[o + q], va_k = a.v3a[o + q];
      const double w1 = (du_k + du_kp1) / 2.0, w2 = (dv_k + dv_kp1) / 2.0;
      const double dz = a.zt.z[k + 1] - a.zt.z[k], zm = 0.5 * (a.zt.z[k + 1] + a.zt.z[k]);
      const double w3 = ((gsx - zm * gix) / Hm) * ((ua_kp1 - ua_k) / dz);
      const double w4 = ((gsy - zm * giy) / Hm) * ((va_kp1 - va_k) / dz);
      const double wk = wk1 - H * (w1 + w2 + w3 + w4) * dz;
      a.w[o + q] = wk;
      wk1 = wk;
      du_kp1 = du_k; dv_kp1 = dv_k; ua_kp1 = ua_k; va_kp1 = va_k;
    }
    a.ws[q] = a.w[q];
    a.wb[q] = a.w[ob + q];
  }
  // a-grid maps of the 3D field (own column only: safe after the stale reads above)
  for (int k = 0; k < nz; ++k) {
    const long long o = (long long)k * P;
    a.u3a[o + q] = map_cx_a(d, a.ice, a.u3, o, j, i);
    a.v3a[o + q] = map_cy_a(d, a.ice, a.v3, o, j, i);
  }
  const double uva = map_cx_a(d, a.ice, a.uv, 0, j, i), vva = map_cy_a(d, a.ice, a.vv, 0, j, i);
  const double usa = map_cx_a(d, a.ice, a.us, 0, j, i), vsa = map_cy_a(d, a.ice, a.vs, 0, j, i);
  const double uba = map_cx_a(d, a.ice, a.ub, 0, j, i), vba = map_cy_a(d, a.ice, a.vb, 0, j, i);
  a.uva[q] = uva; a.vva[q] = vva; a.usa[q] = usa; a.vsa[q] = vsa; a.uba[q] = uba; a.vba[q] = vba;
  const double av = sqrt(uva * uva + vva * vva), as = sqrt(usa * usa + vsa * vsa), ab = sqrt(uba * uba + vba * vba);
  a.abv[q] = av; a.abs_[q] = as; a.abb[q] = ab;
  double R;
  if (a.dyn == DIVA_DYN_SIA) R = 1.0;
  else if (a.dyn == DIVA_DYN_SSA) R = 0.0;
  else R = (a.ice[q] == 1) ? max_ref(0.0, min_ref(1.0, (1.0 - ab / as))) : 0.0;
  a.Rs[q] = R;
}

// solve_SIA 3D velocities (:60-105)
__global__ void k_sia(Dims d, Zeta zt, double n, const int* sheet, const double* Hcx, const double* Hcy,
                      const double* sxcx, const double* sycx, const double* sxcy, const double* sycy,
                      const double* Acx, const double* Acy, double* u3, double* v3) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i), P = d.plane;
  const int nz = d.nz;
  for (int face = 0; face < 2; ++face) {
    if (face == 0 && i >= d.nx - 1) continue;
    if (face == 1 && j >= d.ny - 1) continue;
    const long long qn = face == 0 ? d.at(j, i + 1) : d.at(j + 1, i);
    double* out = face == 0 ? u3 : v3;
    if (sheet[q] == 0 && sheet[qn] == 0) {
      for (int k = 0; k < nz; ++k) out[(long long)k * P + q] = 0.0;
      continue;
    }
    const double H = face == 0 ? Hcx[q] : Hcy[q];
    const double sx = face == 0 ? sxcx[q] : sxcy[q], sy = face == 0 ? sycx[q] : sycy[q];
    const double* A = face == 0 ? Acx : Acy;
    const double slope = face == 0 ? sx : sy;
    const double D0 = pow(kRhoI * kGrav * H, n) * pow((sx * sx + sy * sy), (n - 1.0) / 2.0);
    // D(zeta) = 2 H int_base^zeta A zeta^n (vertical_integration_from_bottom_to_zeta)
    double acc = 0.0, fk1 = A[(long long)(nz - 1) * P + q] * zt.zn[nz - 1];
    out[(long long)(nz - 1) * P + q] = max_ref(D0 * (2.0 * H * 0.0), -1E5) * slope;
    for (int k = nz - 2; k >= 0; --k) {
      const double fk = A[(long long)k * P + q] * zt.zn[k];
      acc = acc - 0.5 * (fk1 + fk) * (zt.z[k + 1] - zt.z[k]);
      out[(long long)k * P + q] = max_ref(D0 * (2.0 * H * acc), -1E5) * slope;
      fk1 = fk;
    }
  }
}

__global__ void k_count_sheet(Dims d, const int* sheet, int* out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  if (sheet[d.at(j, i)] != 0) atomicOr(out, 1);
}

__global__ void k_zero_uv(Dims d, double* u, double* v) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  if (i < d.nx - 1) u[d.at(j, i)] = 0.0;
  if (j < d.ny - 1) v[d.at(j, i)] = 0.0;
}

}  // namespace

#define G2 grid2d(c->d.ny, c->d.nx), block2d(), 0, c->stream

// Whether K1 computes the viscosity of the linearisation in FP32 (precision 'mixed').
#ifndef DIVA_K1_FP32
#define DIVA_K1_FP32 1
#endif
static bool k1_fp32(const diva_config_t& C) { return DIVA_K1_FP32 && C.precision == DIVA_PREC_MIXED; }

int launch_prepare_afac(Ctx* c) {
  k_afac<<<G2>>>(c->d, c->c.n_flow, c->D(DIVA_F_A_FLOW_3D_A), c->afac); c->launches++;
  DIVA_LAUNCHED(c, "k_afac");
  return DIVA_OK;
}

static void fill_coef_args(Ctx* c, CoefArgs& a, const double* u, const double* v, bool diva) {
  const diva_config_t& C = c->c;
  a.d = c->d;
  a.zt = c->zt;
  a.diva = diva;
  a.bc_margin = C.choice_ice_margin == DIVA_MARGIN_BC;
  a.sliding = C.choice_sliding_law;
  a.gl_subgrid = C.do_GL_subgrid_friction;
  a.basal_freezing = C.include_basal_freezing;
  a.prescribed_tauc = C.prescribed_tauc;
  a.n_is_3 = C.n_flow == 3.0;
  a.crossterms = C.include_SSADIVA_crossterms;
  a.n_flow = C.n_flow;
  a.eps0 = C.DIVA_epsilon_sq_0;
  a.visc_min = C.DIVA_visc_eff_min;
  a.beta_max = C.DIVA_beta_max;
  a.delta_v = C.slid_delta_v;
  a.wm = C.slid_Weertman_m;
  a.q_plastic = C.slid_Coulomb_reg_q_plastic;
  a.u_thr = C.slid_Coulomb_reg_u_threshold;
  a.zi_ut = C.slid_ZI_ut;
  a.zi_p = C.slid_ZI_p;
  a.dT_freeze = C.deltaT_basal_freezing;
  {
    // F_int_min = vertical_integrate( (1/visc_eff_min) * zeta**2) (:980)
    double s = 0.0;
    for (int k = 1; k < c->d.nz; ++k) {
      const double f0 = (1.0 / C.DIVA_visc_eff_min) * c->zt.z2[k - 1], f1 = (1.0 / C.DIVA_visc_eff_min) * c->zt.z2[k];
      s = s + 0.5 * (f1 + f0) * (c->zt.z[k] - c->zt.z[k - 1]);
    }
    a.Fmin = s;
  }
  a.u = u; a.v = v;
  a.visc_prev = c->visc_prev;
  a.taub_cx = c->D(DIVA_F_TAUB_CX); a.taub_cy = c->D(DIVA_F_TAUB_CY);
  a.Hi = c->D(DIVA_F_HI_A); a.afac = c->afac;
  a.mask_ice = c->I(DIVA_F_MASK_ICE_A); a.mask_ocean = c->I(DIVA_F_MASK_OCEAN_A);
  a.beta_sq = c->D(DIVA_F_BETA_SQ_A); a.phi_fric = c->D(DIVA_F_PHI_FRIC_A); a.alpha_sq = c->D(DIVA_F_ALPHA_SQ_A);
  a.Neff = c->D(DIVA_F_NEFF_A); a.Ti = c->D(DIVA_F_TI_A); a.Tpmp = c->D(DIVA_F_TI_PMP_A);
  a.dudz = c->D(DIVA_F_DU_DZ_3D_CX); a.dvdz = c->D(DIVA_F_DV_DZ_3D_CY);
  a.visc = c->D(DIVA_F_VISC_EFF_3D_A); a.visc_int = c->D(DIVA_F_VISC_EFF_INT_A); a.Na = c->D(DIVA_F_N_A);
  a.beta = c->D(DIVA_F_BETA_A); a.F2 = c->D(DIVA_F_F2_A); a.beta_eff = c->D(DIVA_F_BETA_EFF_A);
  a.tauc = c->D(DIVA_F_TAUC_A);
  a.col_eps = c->col_eps;
  a.col_flags = c->col_flags;
  a.taub_seen_cx = c->taub_seen[0];
  a.taub_seen_cy = c->taub_seen[1];
}

int launch_diva_coefficients(Ctx* c, const double* u, const double* v, bool diva, int what) {
  const diva_config_t& C = c->c;
  // Picard double buffering of visc_eff_3D_a: read the previous, write the new
  std::swap(c->f[DIVA_F_VISC_EFF_3D_A], *reinterpret_cast<void**>(&c->visc_prev));
  CoefArgs a{};
  fill_coef_args(c, a, u, v, diva);
  if (C.choice_ice_margin == DIVA_MARGIN_BC) {
    // BC margins keep visc_eff_int_a / N_a of ice-free points from before: the
    // previous buffer's content is not carried over by the swap, so copy it.
    DIVA_CUDA(c, cudaMemcpyAsync(c->D(DIVA_F_VISC_EFF_3D_A), c->visc_prev, sizeof(double) * c->d.plane * c->d.nz,
                                 cudaMemcpyDeviceToDevice, c->stream));
  }
  a.keep_seen = what != K1_WRITE_SHEAR;
  k_column_prep<<<G2>>>(a); c->launches++;
  {
    const dim3 block(kColLanes, kColRows);
    const dim3 grid(c->d.nz, (c->d.ny + kColLanes - 1) / kColLanes, (c->d.nx + kColRows - 1) / kColRows);
    const bool f32 = k1_fp32(C);
    if (what == K1_WRITE_SHEAR) {
      if (f32) k_layer_viscosity<true, float><<<grid, block, 0, c->stream>>>(a);
      else k_layer_viscosity<true, double><<<grid, block, 0, c->stream>>>(a);
    } else {
      if (f32) k_layer_viscosity<false, float><<<grid, block, 0, c->stream>>>(a);
      else k_layer_viscosity<false, double><<<grid, block, 0, c->stream>>>(a);
    }
    c->launches++;
  }
  if (k1_fp32(C)) {
    if (c->d.nz == 15) k_column_integrals<15, float><<<G2>>>(a);
    else k_column_integrals<0, float><<<G2>>>(a);
  } else {
    if (c->d.nz == 15) k_column_integrals<15, double><<<G2>>>(a);
    else k_column_integrals<0, double><<<G2>>>(a);
  }
  c->launches++;
  if (what == K1_COLUMNS_ONLY) {   // timing of the column launches alone (diva_profile_kernel)
    DIVA_LAUNCHED(c, "column coefficients");
    return DIVA_OK;
  }
  DIVA_LAUNCHED(c, "column coefficients");
  FaceArgs fa{};
  fa.d = c->d;
  fa.bc_margin = a.bc_margin;
  fa.apply_fgrnd = diva ? C.do_GL_subgrid_friction : 1;   // solve_SSA always applies f_grnd^2 (:200-205)
  fa.crossterms = C.include_SSADIVA_crossterms;
  fa.vint = c->D(DIVA_F_VISC_EFF_INT_A); fa.Hb_i = c->D(DIVA_F_HI_B); fa.beta_eff = c->D(DIVA_F_BETA_EFF_A);
  fa.fcx = c->D(DIVA_F_F_GRND_CX); fa.fcy = c->D(DIVA_F_F_GRND_CY); fa.Na = c->D(DIVA_F_N_A);
  fa.mask_ice = c->I(DIVA_F_MASK_ICE_A);
  fa.visc_int_b = c->D(DIVA_F_VISC_EFF_INT_B); fa.Nb = c->D(DIVA_F_N_B);
  fa.bex = c->D(DIVA_F_BETA_EFF_CX); fa.bey = c->D(DIVA_F_BETA_EFF_CY);
  fa.Ncx = c->D(DIVA_F_N_CX); fa.Ncy = c->D(DIVA_F_N_CY);
  fa.lvBx = c->lv[0].Bx; fa.lvBy = c->lv[0].By; fa.lvNa = c->lv[0].Na; fa.lvNb = c->lv[0].Nb;
  k_face_coefficients<<<G2>>>(fa); c->launches++;
  DIVA_LAUNCHED(c, "k_face_coefficients");
  return DIVA_OK;
}

int launch_picard_update(Ctx* c, double* u, double* v, const double* xu, const double* xv, bool diva) {
  const diva_config_t& C = c->c;
  UpdArgs a{};
  a.d = c->d;
  a.diva = diva;
  a.sliding_none = C.choice_sliding_law == DIVA_SLIDING_NONE;
  a.basal_freezing = C.include_basal_freezing;
  dim3 g = grid2d(c->d.ny, c->d.nx);
  a.nblk_x = g.x;
  a.vmax = C.DIVA_vel_max;
  a.rel = C.DIVA_visc_it_relax;
  a.dT_freeze = C.deltaT_basal_freezing;
  a.xu = xu; a.xv = xv; a.u = u; a.v = v;
  a.up = c->D(DIVA_F_U_CX_PREV); a.vp = c->D(DIVA_F_V_CY_PREV);
  a.uchk = c->D(DIVA_F_U_VAV_CX); a.vchk = c->D(DIVA_F_V_VAV_CY);
  a.errx = c->err_cand[0]; a.erry = c->err_cand[1];
  a.bex = c->D(DIVA_F_BETA_EFF_CX); a.bey = c->D(DIVA_F_BETA_EFF_CY); a.F2 = c->D(DIVA_F_F2_A);
  a.Hi = c->D(DIVA_F_HI_A); a.Ti = c->D(DIVA_F_TI_A); a.Tpmp = c->D(DIVA_F_TI_PMP_A);
  a.taubx = c->D(DIVA_F_TAUB_CX); a.tauby = c->D(DIVA_F_TAUB_CY);
  a.ubx = c->D(DIVA_F_U_BASE_CX); a.vby = c->D(DIVA_F_V_BASE_CY);
  a.partials = c->partials;
  a.aa_m = C.picard_anderson_m;
  a.sc = c->scal;
  a.gu = c->aa_g[0]; a.gv = c->aa_g[1];
  for (int k = 0; k < kAAMax; ++k) { a.dGu[k] = c->aa_dG[k][0]; a.dGv[k] = c->aa_dG[k][1]; }
  k_picard_update<<<g, block2d(), 0, c->stream>>>(a); c->launches++;
  DIVA_LAUNCHED(c, "k_picard_update");
  k_sum_partials<<<1, 256, 0, c->stream>>>(c->partials, (int)(g.x * g.y), 3, c->scal + SC_RES1); c->launches++;
  DIVA_LAUNCHED(c, "k_sum_partials");
  return DIVA_OK;
}

int launch_anderson_prepare(Ctx* c, const double* u, const double* v, const double* xu, const double* xv) {
  const diva_config_t& C = c->c;
  AAArgs a{};
  a.d = c->d;
  a.m = C.picard_anderson_m;
  const dim3 g = grid2d(c->d.ny, c->d.nx);
  a.nblk_x = g.x;
  a.vmax = C.DIVA_vel_max;
  a.u = u; a.v = v; a.xu = xu; a.xv = xv;
  for (int k = 0; k < kAAMax; ++k) {
    a.dFu[k] = c->aa_dF[k][0]; a.dFv[k] = c->aa_dF[k][1];
    a.dGu[k] = c->aa_dG[k][0]; a.dGv[k] = c->aa_dG[k][1];
  }
  a.fu = c->aa_f[0]; a.fv = c->aa_f[1]; a.gu = c->aa_g[0]; a.gv = c->aa_g[1];
  a.sc = c->scal;
  a.partials = c->partials;
  k_aa_prepare<<<g, block2d(), 0, c->stream>>>(a); c->launches++;
  DIVA_LAUNCHED(c, "k_aa_prepare");
  k_aa_solve<<<1, 256, 0, c->stream>>>(c->partials, (int)(g.x * g.y), a.m, c->scal); c->launches++;
  DIVA_LAUNCHED(c, "k_aa_solve");
  return DIVA_OK;
}

// start of a solve: empty history, zeroed columns (unused slots then mix in nothing)
int anderson_reset(Ctx* c) {
  if (c->c.picard_anderson_m <= 0) return DIVA_OK;
  for (int q = 0; q < 2; ++q)
    for (int k = 0; k < kAAMax; ++k) {
      DIVA_CUDA(c, cudaMemsetAsync(c->aa_dF[k][q], 0, sizeof(double) * c->d.plane, c->stream));
      DIVA_CUDA(c, cudaMemsetAsync(c->aa_dG[k][q], 0, sizeof(double) * c->d.plane, c->stream));
    }
  return DIVA_OK;
}

int launch_commit_err(Ctx* c) {
  std::swap(c->f[DIVA_F_DIVA_ERR_CX], *reinterpret_cast<void**>(&c->err_cand[0]));
  std::swap(c->f[DIVA_F_DIVA_ERR_CY], *reinterpret_cast<void**>(&c->err_cand[1]));
  return DIVA_OK;
}

int launch_basal_stress_velocities(Ctx* c) {
  const diva_config_t& C = c->c;
  k_basal_stress_velocities<<<G2>>>(c->d, C.choice_sliding_law == DIVA_SLIDING_NONE, C.include_basal_freezing,
                                    C.deltaT_basal_freezing, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY),
                                    c->D(DIVA_F_BETA_EFF_CX), c->D(DIVA_F_BETA_EFF_CY), c->D(DIVA_F_F2_A),
                                    c->D(DIVA_F_HI_A), c->D(DIVA_F_TI_A), c->D(DIVA_F_TI_PMP_A),
                                    c->D(DIVA_F_TAUB_CX), c->D(DIVA_F_TAUB_CY), c->D(DIVA_F_U_BASE_CX),
                                    c->D(DIVA_F_V_BASE_CY), nullptr); c->launches++;
  DIVA_LAUNCHED(c, "k_basal_stress_velocities");
  return DIVA_OK;
}

int launch_basal_pred(Ctx* c) {
  const diva_config_t& C = c->c;
  k_basal_stress_velocities<<<G2>>>(c->d, C.choice_sliding_law == DIVA_SLIDING_NONE, C.include_basal_freezing,
                                    C.deltaT_basal_freezing, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY),
                                    c->D(DIVA_F_BETA_EFF_CX), c->D(DIVA_F_BETA_EFF_CY), c->D(DIVA_F_F2_A),
                                    c->D(DIVA_F_HI_A), c->D(DIVA_F_TI_A), c->D(DIVA_F_TI_PMP_A),
                                    c->D(DIVA_F_TAUB_CX), c->D(DIVA_F_TAUB_CY), c->D(DIVA_F_U_BASE_CX),
                                    c->D(DIVA_F_V_BASE_CY), c->scal + SC_EXIT_RELRES); c->launches++;
  DIVA_LAUNCHED(c, "k_basal_stress_velocities");
  return DIVA_OK;
}

// end of a graph-launched viscosity iteration: the step norm from the summed
// partials (calc_visc_iter_UV_resid :1588-1596) and the stop test (:346-351)
__global__ void k_ctl_end(double* sc, int relmode, double tol, int nit) {
  const double r1 = sc[SC_RES1], r2 = sc[SC_RES2], cnt = sc[SC_RES1 + 2];
  if (!isfinite(r1) || !isfinite(r2)) sc[SC_NAN] = 1.0;
  const double resid = (cnt > 0.0) ? 2.0 * sqrt(r1) / max_ref(sqrt(r2), 1E-8) : 0.0;
  sc[SC_RESID] = resid;
  bool conv = false;
  if (!relmode && resid < tol) conv = true;
  else if (sc[SC_PIC_IT] >= (double)nit) conv = true;
  sc[SC_CONVERGED] = conv ? 1.0 : 0.0;
}

// DIVA_err of this iteration becomes the field unless the iteration converged (:353-355)
__global__ void k_err_commit(Dims d, const double* sc, const double* cx, const double* cy, double* fx, double* fy) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  if (sc[SC_CONVERGED] != 0.0) return;
  const long long q = d.at(j, i);
  fx[q] = cx[q];
  fy[q] = cy[q];
}

int launch_ctl_end(Ctx* c, bool relmode) {
  k_ctl_end<<<1, 1, 0, c->stream>>>(c->scal, relmode, c->c.DIVA_visc_it_norm_dUV_tol, c->c.DIVA_visc_it_nit); c->launches++;
  DIVA_LAUNCHED(c, "k_ctl_end");
  return DIVA_OK;
}

int launch_err_commit_pred(Ctx* c) {
  k_err_commit<<<G2>>>(c->d, c->scal, c->err_cand[0], c->err_cand[1], c->D(DIVA_F_DIVA_ERR_CX),
                       c->D(DIVA_F_DIVA_ERR_CY)); c->launches++;
  DIVA_LAUNCHED(c, "k_err_commit");
  return DIVA_OK;
}

int launch_shear_rates(Ctx* c) {
  CoefArgs a{};
  fill_coef_args(c, a, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY), true);
  const dim3 block(kColLanes, kColRows);
  const dim3 grid(c->d.nz, (c->d.ny + kColLanes - 1) / kColLanes, (c->d.nx + kColRows - 1) / kColRows);
  if (k1_fp32(c->c)) k_shear_rates<float><<<grid, block, 0, c->stream>>>(a);
  else k_shear_rates<double><<<grid, block, 0, c->stream>>>(a);
  c->launches++;
  DIVA_LAUNCHED(c, "k_shear_rates");
  return DIVA_OK;
}

int launch_visc_b_output(Ctx* c) {
  // the shear strain rates the last viscosity iteration's K1 saw (the loop does not write them)
  int st;
  if ((st = launch_shear_rates(c))) return st;
  k_visc_b<<<G2>>>(c->d, c->c.choice_ice_margin == DIVA_MARGIN_BC, c->D(DIVA_F_VISC_EFF_3D_A),
                   c->I(DIVA_F_MASK_ICE_A), c->D(DIVA_F_VISC_EFF_3D_B)); c->launches++;
  DIVA_LAUNCHED(c, "k_visc_b");
  return DIVA_OK;
}

int launch_3d_horizontal_velocities(Ctx* c) {
  k_f1<<<G2>>>(c->d, c->zt, c->D(DIVA_F_HI_A), c->D(DIVA_F_VISC_EFF_3D_A), c->D(DIVA_F_F1_3D_A)); c->launches++;
  DIVA_LAUNCHED(c, "k_f1");
  k_u3d<<<G2>>>(c->d, c->c.choice_ice_margin == DIVA_MARGIN_BC, c->D(DIVA_F_HI_A), c->D(DIVA_F_F1_3D_A),
                c->D(DIVA_F_U_BASE_CX), c->D(DIVA_F_V_BASE_CY), c->D(DIVA_F_TAUB_CX), c->D(DIVA_F_TAUB_CY),
                c->D(DIVA_F_U_3D_CX), c->D(DIVA_F_V_3D_CY)); c->launches++;
  DIVA_LAUNCHED(c, "k_u3d");
  return DIVA_OK;
}

int launch_secondary_velocities(Ctx* c) {
  const int dyn = c->c.choice_ice_dynamics;
  k_faces_prelude<<<G2>>>(c->d, c->zt, dyn, c->D(DIVA_F_U_3D_CX), c->D(DIVA_F_V_3D_CY), c->D(DIVA_F_U_3D_SIA_CX),
                          c->D(DIVA_F_V_3D_SIA_CY), c->D(DIVA_F_U_SSA_CX), c->D(DIVA_F_V_SSA_CY),
                          c->D(DIVA_F_U_BASE_CX), c->D(DIVA_F_V_BASE_CY), c->D(DIVA_F_U_SURF_CX),
                          c->D(DIVA_F_V_SURF_CY), c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY)); c->launches++;
  DIVA_LAUNCHED(c, "k_faces_prelude");
  SecArgs a{};
  a.d = c->d; a.zt = c->zt; a.dyn = dyn; a.do_w = dyn != DIVA_DYN_SSA;
  a.u3 = c->D(DIVA_F_U_3D_CX); a.v3 = c->D(DIVA_F_V_3D_CY); a.Hs = c->D(DIVA_F_HS_A); a.Hi = c->D(DIVA_F_HI_A);
  a.dHs_dx = c->D(DIVA_F_DHS_DX_A); a.dHs_dy = c->D(DIVA_F_DHS_DY_A);
  a.dHi_dx = c->D(DIVA_F_DHI_DX_A); a.dHi_dy = c->D(DIVA_F_DHI_DY_A); a.dHb_dt = c->D(DIVA_F_DHB_DT_A);
  a.uv = c->D(DIVA_F_U_VAV_CX); a.vv = c->D(DIVA_F_V_VAV_CY); a.us = c->D(DIVA_F_U_SURF_CX);
  a.vs = c->D(DIVA_F_V_SURF_CY); a.ub = c->D(DIVA_F_U_BASE_CX); a.vb = c->D(DIVA_F_V_BASE_CY);
  a.sheet = c->I(DIVA_F_MASK_SHEET_A); a.ice = c->I(DIVA_F_MASK_ICE_A);
  a.w = c->D(DIVA_F_W_3D_A); a.ws = c->D(DIVA_F_W_SURF_A); a.wb = c->D(DIVA_F_W_BASE_A);
  a.u3a = c->D(DIVA_F_U_3D_A); a.v3a = c->D(DIVA_F_V_3D_A);
  a.uva = c->D(DIVA_F_U_VAV_A); a.vva = c->D(DIVA_F_V_VAV_A); a.usa = c->D(DIVA_F_U_SURF_A);
  a.vsa = c->D(DIVA_F_V_SURF_A); a.uba = c->D(DIVA_F_U_BASE_A); a.vba = c->D(DIVA_F_V_BASE_A);
  a.abv = c->D(DIVA_F_UABS_VAV_A); a.abs_ = c->D(DIVA_F_UABS_SURF_A); a.abb = c->D(DIVA_F_UABS_BASE_A);
  a.Rs = c->D(DIVA_F_R_SHEAR);
  k_secondary<<<G2>>>(a); c->launches++;
  DIVA_LAUNCHED(c, "k_secondary");
  return DIVA_OK;
}

int launch_sia(Ctx* c) {
  k_sia<<<G2>>>(c->d, c->zt, c->c.n_flow, c->I(DIVA_F_MASK_SHEET_A), c->D(DIVA_F_HI_CX), c->D(DIVA_F_HI_CY),
                c->D(DIVA_F_DHS_DX_CX), c->D(DIVA_F_DHS_DY_CX), c->D(DIVA_F_DHS_DX_CY), c->D(DIVA_F_DHS_DY_CY),
                c->D(DIVA_F_A_FLOW_3D_CX), c->D(DIVA_F_A_FLOW_3D_CY), c->D(DIVA_F_U_3D_SIA_CX),
                c->D(DIVA_F_V_3D_SIA_CY)); c->launches++;
  DIVA_LAUNCHED(c, "k_sia");
  return DIVA_OK;
}

int launch_zero_velocities(Ctx* c, double* u, double* v) {
  k_zero_uv<<<G2>>>(c->d, u, v); c->launches++;
  DIVA_LAUNCHED(c, "k_zero_uv");
  return DIVA_OK;
}

int launch_any_sheet(Ctx* c, int* result) {
  int* flag = c->ff_flag;
  DIVA_CUDA(c, cudaMemsetAsync(flag, 0, sizeof(int), c->stream));
  k_count_sheet<<<G2>>>(c->d, c->I(DIVA_F_MASK_SHEET_A), flag); c->launches++;
  DIVA_LAUNCHED(c, "k_count_sheet");
  int h = 0;
  DIVA_CUDA(c, cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  *result = h;
  return DIVA_OK;
}

}  // namespace diva
