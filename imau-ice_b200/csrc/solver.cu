// solver.cu -- the linear solve of solve_DIVA_stag_linearised
// (ice_velocity_module.f90:1656-1761), which the reference assembles as a CSR
// matrix (rows :1762-2589) and hands to PETSc KSP or SOR
// (utilities_module.f90:600-718, petsc_module.F90:23-90).
//
// Here the matrix is never formed.  The operator is applied matrix-free from
// N_a, N_b and beta_eff (the coefficients of the reference's free rows,
// :2342-2467), and the domain-boundary rows (:1932-2191: u - u_in = 0,
// u = 0, u - u_opp = 0) are eliminated exactly: a boundary unknown is read
// through its source (the inner or opposite unknown, or zero), so only
// interior unknowns are solved for and the boundary values are filled from
// them afterwards.  The solver is BiCGStab, right-preconditioned with one
// geometric-multigrid V-cycle:
//   * levels coarsen the a-grid by 2 in each direction with at least 9 points
//     (semi-coarsening once one direction is small), so cells may become
//     anisotropic; the coarse operator is the same staggered discretisation
//     rediscretised on the coarse grid with cell aspect hy/hx and averaged
//     N_a, N_b, beta_eff;
//   * transfers are bilinear on the staggered u (cx) and v (cy) points,
//     restriction = transpose of prolongation;
//   * smoothing is 4-colour Gauss-Seidel (u red/black, v red/black), with the
//     exact diagonal of the reduced system;
//   * the larger levels are smoothed by tile kernels (two launches per level and
//     V-cycle, halo recomputed instead of exchanged), the coarse levels whose
//     data fit in 200 KB run out of one thread block's shared memory (one launch
//     per V-cycle), and the coarsest level is solved directly with its inverse,
//     formed once per viscosity iteration.
// All reductions are two-stage (block partials, then one fixed-order sum) so
// results are bit-reproducible from run to run.
#include <cmath>
#include <cstdio>
#include <utility>
#include <vector>
#include "ctx.hpp"

namespace diva {
namespace {

#ifndef DIVA_SUB_THREADS
#define DIVA_SUB_THREADS 1024
#endif
constexpr int kSubThreads = DIVA_SUB_THREADS;   // threads of the one-block coarse-level kernel

// A level's operator.  R is the type of its coefficients and of the x values it is
// applied to: double everywhere, float for the finest level's smoother copies of the
// mixed-precision preconditioner (precision = DIVA_PREC_MIXED).
template <class R>
struct OpT {
  Dims d;
  BCs bc;
  double ax, ay;   // hy/hx and hx/hy of the level's cells (1 on the fine grid)
  const R *Na, *Nb, *Bx, *By;
  // 'BC' ice margins (finest level only, else null): the type of each u and v row
  const int8_t *rtu, *rtv;
  double inv_dx;
};
using Op = OpT<double>;

// Row types of the finest level with choice_ice_margin 'BC' (solve_DIVA_stag_linearised
// :1683-1727): a free row, u = 0 (shelf next to land, or a front cell with ocean on both
// sides), or the calving-front stress row of list_DIVA_matrix_coefficients_eq_1_margin
// (:2192-2266) / eq_2_margin (:2267-2341) with the ice on the lower (west/south) or upper
// side of the face.
enum : int8_t { RT_FREE = 0, RT_IDENT = 1, RT_MARGIN_LO = 2, RT_MARGIN_HI = 3 };

__host__ __device__ __forceinline__ bool u_int(const Dims& d, int j, int i) {
  return i >= 1 && i <= d.nx - 3 && j >= 1 && j <= d.ny - 2;
}
__host__ __device__ __forceinline__ bool v_int(const Dims& d, int j, int i) {
  return i >= 1 && i <= d.nx - 2 && j >= 1 && j <= d.ny - 3;
}
__host__ __device__ __forceinline__ int bc_pick(int a, int b) {
  if (a == DIVA_BC_ZERO || b == DIVA_BC_ZERO) return DIVA_BC_ZERO;
  if (a == DIVA_BC_INFINITE || b == DIVA_BC_INFINITE) return DIVA_BC_INFINITE;
  return DIVA_BC_PERIODIC;
}
// Source of u(j,i) (list_DIVA_matrix_coefficients_eq_1_boundary :1932-2061); false = zero.
__host__ __device__ __forceinline__ bool u_src(const Dims& d, const BCs& b, int j, int i, int& js, int& is) {
  if (u_int(d, j, i)) { js = j; is = i; return true; }
  const bool W = i == 0, E = i == d.nx - 2, S = j == 0, N = j == d.ny - 1;
  int t;
  if (W && S) t = bc_pick(b.uS, b.uW);
  else if (E && S) t = bc_pick(b.uS, b.uE);
  else if (W && N) t = bc_pick(b.uN, b.uW);
  else if (E && N) t = bc_pick(b.uN, b.uE);
  else if (W) t = b.uW;
  else if (E) t = b.uE;
  else if (S) t = b.uS;
  else t = b.uN;
  if (t == DIVA_BC_ZERO) return false;
  if (t == DIVA_BC_INFINITE) { is = W ? 1 : (E ? d.nx - 3 : i); js = S ? 1 : (N ? d.ny - 2 : j); }
  else { is = W ? d.nx - 3 : (E ? 1 : i); js = S ? d.ny - 2 : (N ? 1 : j); }
  return true;
}
// Source of v(j,i) (list_DIVA_matrix_coefficients_eq_2_boundary :2062-2191).
__host__ __device__ __forceinline__ bool v_src(const Dims& d, const BCs& b, int j, int i, int& js, int& is) {
  if (v_int(d, j, i)) { js = j; is = i; return true; }
  const bool W = i == 0, E = i == d.nx - 1, S = j == 0, N = j == d.ny - 2;
  int t;
  if (W && S) t = bc_pick(b.vS, b.vW);
  else if (E && S) t = bc_pick(b.vS, b.vE);
  else if (W && N) t = bc_pick(b.vN, b.vW);
  else if (E && N) t = bc_pick(b.vN, b.vE);
  else if (W) t = b.vW;
  else if (E) t = b.vE;
  else if (S) t = b.vS;
  else t = b.vN;
  if (t == DIVA_BC_ZERO) return false;
  if (t == DIVA_BC_INFINITE) { is = W ? 1 : (E ? d.nx - 2 : i); js = S ? 1 : (N ? d.ny - 3 : j); }
  else { is = W ? d.nx - 2 : (E ? 1 : i); js = S ? d.ny - 3 : (N ? 1 : j); }
  return true;
}
// Where the x values of the (j,i) point live: a full plane of the level (GIx), or
// a shared-memory tile whose origin is (j0,i0) and whose rows hold rj points (TIx).
struct GIx {
  Dims d;
  __device__ __forceinline__ long long operator()(int j, int i) const { return d.at(j, i); }
};
struct TIx {
  int j0, i0, rj;
  __device__ __forceinline__ int operator()(int j, int i) const { return (i - i0) * rj + (j - j0); }
};

// Read a u (v) value through the boundary elimination (RAW = false), or as
// stored (RAW = true: the reference's assembled rows reference stored values).
template <bool RAW, class R, class IX>
__device__ __forceinline__ R LUx(const OpT<R>& o, const R* x, const IX& ix, int j, int i) {
  if (RAW) return x[ix(j, i)];
  int js, is;
  return u_src(o.d, o.bc, j, i, js, is) ? x[ix(js, is)] : R(0);
}
template <bool RAW, class R, class IX>
__device__ __forceinline__ R LVx(const OpT<R>& o, const R* x, const IX& ix, int j, int i) {
  if (RAW) return x[ix(j, i)];
  int js, is;
  return v_src(o.d, o.bc, j, i, js, is) ? x[ix(js, is)] : R(0);
}
template <bool RAW = false>
__device__ __forceinline__ double LU(const Op& o, const double* x, int j, int i) {
  return LUx<RAW>(o, x, GIx{o.d}, j, i);
}
template <bool RAW = false>
__device__ __forceinline__ double LV(const Op& o, const double* x, int j, int i) {
  return LVx<RAW>(o, x, GIx{o.d}, j, i);
}

// Sum of the nine stencil terms, accumulated with explicit fused multiply-adds in a
// fixed order, so every code path (boundary-mapped reads, plain reads, the row
// tables of the sub-cycle) rounds identically whatever the compiler would contract.
__device__ __forceinline__ double fma_r(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fma_r(float a, float b, float c) { return fmaf(a, b, c); }

template <class R>
__device__ __forceinline__ R stencil9(R c0, R x0, R c1, R x1, R c2, R x2, R c3, R x3, R c4, R x4, R c5, R x5, R c6,
                                      R x6, R c7, R x7, R c8, R x8) {
  R s = c0 * x0;
  s = fma_r(c1, x1, s);
  s = fma_r(c2, x2, s);
  s = fma_r(c3, x3, s);
  s = fma_r(c4, x4, s);
  s = fma_r(c5, x5, s);
  s = fma_r(c6, x6, s);
  s = fma_r(c7, x7, s);
  return fma_r(c8, x8, s);
}

template <class R>
__device__ __forceinline__ R stencil4(R c0, R x0, R c1, R x1, R c2, R x2, R c3, R x3) {
  R s = c0 * x0;
  s = fma_r(c1, x1, s);
  s = fma_r(c2, x2, s);
  return fma_r(c3, x3, s);
}

// (A x) of the u row at interior (j,i) (list_DIVA_matrix_coefficients_eq_1_free :2342-2404)
// IX places x values, CX the coefficients N_a, N_b, B (a level plane or a shared-memory tile)
// (the constants are written R(k) so that R = double performs exactly the double
// operations of the reference's rows and R = float stays in single precision)
template <bool RAW, bool FRONT = true, class R, class IX, class CX>
__device__ __forceinline__ R AuXC(const OpT<R>& o, const R* xu, const R* xv, const IX& ix, const CX& cx, int j,
                                  int i) {
  if (FRONT && o.rtu) {
    const int t = o.rtu[o.d.at(j, i)];
    if (t == RT_IDENT) return xu[ix(j, i)];
    if (t != RT_FREE) {   // front row: -4N u(i1-1) + 4N u(i1) - 2N v(j-1,i1) + 2N v(j,i1), N = N_a(i1)/dx
      const int i1 = t == RT_MARGIN_LO ? i : i + 1;
      const R N = o.Na[cx(j, i1)], idx = R(o.inv_dx);
      return stencil4(R(-4) * idx * N, LUx<RAW>(o, xu, ix, j, i1 - 1), R(4) * idx * N, LUx<RAW>(o, xu, ix, j, i1),
                      R(-2) * idx * N, LVx<RAW>(o, xv, ix, j - 1, i1), R(2) * idx * N, LVx<RAW>(o, xv, ix, j, i1));
    }
  }
  const R Ae = o.Na[cx(j, i + 1)], Aw = o.Na[cx(j, i)], Bn = o.Nb[cx(j, i)], Bs = o.Nb[cx(j - 1, i)];
  const R ax = R(o.ax), ay = R(o.ay);
  const R cE = R(4) * ax * Ae, cW = R(4) * ax * Aw, cN = ay * Bn, cS = ay * Bs;
  const R diag = -(cE + cW + cN + cS) - o.Bx[cx(j, i)];
  return stencil9(cE, LUx<RAW>(o, xu, ix, j, i + 1), cW, LUx<RAW>(o, xu, ix, j, i - 1), cN,
                  LUx<RAW>(o, xu, ix, j + 1, i), cS, LUx<RAW>(o, xu, ix, j - 1, i), diag, xu[ix(j, i)],
                  R(-2) * Aw - Bn, LVx<RAW>(o, xv, ix, j, i), R(2) * Ae + Bn, LVx<RAW>(o, xv, ix, j, i + 1),
                  R(2) * Aw + Bs, LVx<RAW>(o, xv, ix, j - 1, i), R(-2) * Ae - Bs, LVx<RAW>(o, xv, ix, j - 1, i + 1));
}
// (A x) of the v row at interior (j,i) (list_DIVA_matrix_coefficients_eq_2_free :2405-2467)
template <bool RAW, bool FRONT = true, class R, class IX, class CX>
__device__ __forceinline__ R AvXC(const OpT<R>& o, const R* xu, const R* xv, const IX& ix, const CX& cx, int j,
                                  int i) {
  if (FRONT && o.rtv) {
    const int t = o.rtv[o.d.at(j, i)];
    if (t == RT_IDENT) return xv[ix(j, i)];
    if (t != RT_FREE) {   // front row: -4N v(j1-1) + 4N v(j1) - 2N u(j1,i-1) + 2N u(j1,i), N = N_a(j1)/dx
      const int j1 = t == RT_MARGIN_LO ? j : j + 1;
      const R N = o.Na[cx(j1, i)], idx = R(o.inv_dx);
      return stencil4(R(-4) * idx * N, LVx<RAW>(o, xv, ix, j1 - 1, i), R(4) * idx * N, LVx<RAW>(o, xv, ix, j1, i),
                      R(-2) * idx * N, LUx<RAW>(o, xu, ix, j1, i - 1), R(2) * idx * N, LUx<RAW>(o, xu, ix, j1, i));
    }
  }
  const R An = o.Na[cx(j + 1, i)], As = o.Na[cx(j, i)], Be = o.Nb[cx(j, i)], Bw = o.Nb[cx(j, i - 1)];
  const R ax = R(o.ax), ay = R(o.ay);
  const R cN = R(4) * ay * An, cS = R(4) * ay * As, cE = ax * Be, cW = ax * Bw;
  const R diag = -(cN + cS + cE + cW) - o.By[cx(j, i)];
  return stencil9(cN, LVx<RAW>(o, xv, ix, j + 1, i), cS, LVx<RAW>(o, xv, ix, j - 1, i), cE,
                  LVx<RAW>(o, xv, ix, j, i + 1), cW, LVx<RAW>(o, xv, ix, j, i - 1), diag, xv[ix(j, i)],
                  R(-2) * An - Bw, LUx<RAW>(o, xu, ix, j + 1, i - 1), R(2) * An + Be, LUx<RAW>(o, xu, ix, j + 1, i),
                  R(2) * As + Bw, LUx<RAW>(o, xu, ix, j, i - 1), R(-2) * As - Be, LUx<RAW>(o, xu, ix, j, i));
}
template <bool RAW, class IX>
__device__ __forceinline__ double AuX(const Op& o, const double* xu, const double* xv, const IX& ix, int j, int i) {
  return AuXC<RAW>(o, xu, xv, ix, GIx{o.d}, j, i);
}
template <bool RAW, class IX>
__device__ __forceinline__ double AvX(const Op& o, const double* xu, const double* xv, const IX& ix, int j, int i) {
  return AvXC<RAW>(o, xu, xv, ix, GIx{o.d}, j, i);
}
template <bool RAW = false>
__device__ __forceinline__ double Au(const Op& o, const double* xu, const double* xv, int j, int i) {
  return AuX<RAW>(o, xu, xv, GIx{o.d}, j, i);
}
template <bool RAW = false>
__device__ __forceinline__ double Av(const Op& o, const double* xu, const double* xv, int j, int i) {
  return AvX<RAW>(o, xu, xv, GIx{o.d}, j, i);
}
// effective diagonal of the reduced system: couplings to boundary unknowns whose source is the row itself fold in
__device__ __forceinline__ double diag_u(const Op& o, int j, int i) {
  const Dims& d = o.d;
  if (o.rtu) {
    const int t = o.rtu[d.at(j, i)];
    if (t == RT_IDENT) return 1.0;
    if (t != RT_FREE) {   // the u terms of the front row whose source is this row
      const int i1 = t == RT_MARGIN_LO ? i : i + 1;
      const double N = o.Na[d.at(j, i1)];
      double dg = 0.0;
      int js, is;
      if (u_src(d, o.bc, j, i1 - 1, js, is) && js == j && is == i) dg += -4.0 * o.inv_dx * N;
      if (u_src(d, o.bc, j, i1, js, is) && js == j && is == i) dg += 4.0 * o.inv_dx * N;
      return dg;
    }
  }
  const double Ae = o.Na[d.at(j, i + 1)], Aw = o.Na[d.at(j, i)], Bn = o.Nb[d.at(j, i)], Bs = o.Nb[d.at(j - 1, i)];
  const double cE = 4.0 * o.ax * Ae, cW = 4.0 * o.ax * Aw, cN = o.ay * Bn, cS = o.ay * Bs;
  double dg = -(cE + cW + cN + cS) - o.Bx[d.at(j, i)];
  int js, is;
  if (!u_int(d, j, i + 1) && u_src(d, o.bc, j, i + 1, js, is) && js == j && is == i) dg += cE;
  if (!u_int(d, j, i - 1) && u_src(d, o.bc, j, i - 1, js, is) && js == j && is == i) dg += cW;
  if (!u_int(d, j + 1, i) && u_src(d, o.bc, j + 1, i, js, is) && js == j && is == i) dg += cN;
  if (!u_int(d, j - 1, i) && u_src(d, o.bc, j - 1, i, js, is) && js == j && is == i) dg += cS;
  return dg;
}
__device__ __forceinline__ double diag_v(const Op& o, int j, int i) {
  const Dims& d = o.d;
  if (o.rtv) {
    const int t = o.rtv[d.at(j, i)];
    if (t == RT_IDENT) return 1.0;
    if (t != RT_FREE) {
      const int j1 = t == RT_MARGIN_LO ? j : j + 1;
      const double N = o.Na[d.at(j1, i)];
      double dg = 0.0;
      int js, is;
      if (v_src(d, o.bc, j1 - 1, i, js, is) && js == j && is == i) dg += -4.0 * o.inv_dx * N;
      if (v_src(d, o.bc, j1, i, js, is) && js == j && is == i) dg += 4.0 * o.inv_dx * N;
      return dg;
    }
  }
  const double An = o.Na[d.at(j + 1, i)], As = o.Na[d.at(j, i)], Be = o.Nb[d.at(j, i)], Bw = o.Nb[d.at(j, i - 1)];
  const double cN = 4.0 * o.ay * An, cS = 4.0 * o.ay * As, cE = o.ax * Be, cW = o.ax * Bw;
  double dg = -(cN + cS + cE + cW) - o.By[d.at(j, i)];
  int js, is;
  if (!v_int(d, j + 1, i) && v_src(d, o.bc, j + 1, i, js, is) && js == j && is == i) dg += cN;
  if (!v_int(d, j - 1, i) && v_src(d, o.bc, j - 1, i, js, is) && js == j && is == i) dg += cS;
  if (!v_int(d, j, i + 1) && v_src(d, o.bc, j, i + 1, js, is) && js == j && is == i) dg += cE;
  if (!v_int(d, j, i - 1) && v_src(d, o.bc, j, i - 1, js, is) && js == j && is == i) dg += cW;
  return dg;
}

#define IDX2D                                                            \
  const int j = blockIdx.x * blockDim.x + threadIdx.x;                   \
  const int i = blockIdx.y * blockDim.y + threadIdx.y;

// Gauss-Seidel update of one point of one component (comp 0 = u, 1 = v).  Every smoother
// (these per-colour kernels, the tiles, the sub-cycle) forms x + (b - A x) / diag as one
// explicit fused multiply-add, so all of them round alike.
__device__ __forceinline__ void gs_point(const Op& o, double* xu, double* xv, const double* bu, const double* bv,
                                         const double* idu, const double* idv, int comp, int j, int i) {
  const long long q = o.d.at(j, i);
  if (comp == 0) {
    if (u_int(o.d, j, i)) xu[q] = fma(bu[q] - Au(o, xu, xv, j, i), idu[q], xu[q]);
  } else {
    if (v_int(o.d, j, i)) xv[q] = fma(bv[q] - Av(o, xu, xv, j, i), idv[q], xv[q]);
  }
}

// one colour of Gauss-Seidel: comp 0 = u, 1 = v; colour = (i+j) parity
__global__ void k_gs(Op o, double* xu, double* xv, const double* bu, const double* bv, const double* idu,
                     const double* idv, int comp, int color) {
  const int jj = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  const int j = 2 * jj + ((i + color) & 1);
  if (j >= o.d.ny || i >= o.d.nx) return;
  gs_point(o, xu, xv, bu, bv, idu, idv, comp, j, i);
}

// block-wide pass over all points of one colour (the caller synchronises)
__device__ __forceinline__ void block_gs_pass(const Op& o, double* xu, double* xv, const double* bu, const double* bv,
                                              const double* idu, const double* idv, int comp, int color) {
  const Dims& d = o.d;
  const int hj = (d.ny + 1) / 2, n = hj * d.nx;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const int i = t / hj, j = 2 * (t % hj) + ((i + color) & 1);
    if (j < d.ny) gs_point(o, xu, xv, bu, bv, idu, idv, comp, j, i);
  }
}

// relaxation of the coarsest level by one block: `sweeps` symmetric sweeps u0 u1 v0 v1 | v1 v0 u1 u0
__device__ __forceinline__ void block_coarse_relax(const Op& o, double* xu, double* xv, const double* bu,
                                                   const double* bv, const double* idu, const double* idv,
                                                   int sweeps) {
  for (int s = 0; s < sweeps; ++s) {
    for (int pass = 0; pass < 8; ++pass) {
      const int p = pass < 4 ? pass : 7 - pass;
      block_gs_pass(o, xu, xv, bu, bv, idu, idv, p >> 1, p & 1);
      __syncthreads();
    }
  }
}

__global__ void k_coarse_solve(Op o, double* xu, double* xv, const double* bu, const double* bv, const double* idu,
                               const double* idv, int sweeps) {
  block_coarse_relax(o, xu, xv, bu, bv, idu, idv, sweeps);
}

// r = b - A x on the interior (zero elsewhere)
__device__ __forceinline__ void residual_point(const Op& o, const double* xu, const double* xv, const double* bu,
                                               const double* bv, double* ru, double* rv, int j, int i) {
  const long long q = o.d.at(j, i);
  ru[q] = u_int(o.d, j, i) ? bu[q] - Au(o, xu, xv, j, i) : 0.0;
  rv[q] = v_int(o.d, j, i) ? bv[q] - Av(o, xu, xv, j, i) : 0.0;
}
__global__ void k_residual(Op o, const double* xu, const double* xv, const double* bu, const double* bv, double* ru,
                           double* rv) {
  IDX2D
  if (j >= o.d.ny || i >= o.d.nx) return;
  residual_point(o, xu, xv, bu, bv, ru, rv, j, i);
}

// 1D transfer weights.  "cell" direction: u along x, v along y; "node": u along y, v along x.
// Gather form of the restriction: coarse C collects fine f with weight w; tap k of at most
// 4 (cell) or 3 (node), or the single tap f = C, w = 1 where the level is not coarsened
// along that direction (f2 = 1).  The taps are formed in registers, one at a time, and
// summed with explicit fused multiply-adds (the weights' products are exact), so every
// kernel that restricts or prolongs rounds alike.
__device__ __forceinline__ int gather_cell_n(int f2) { return f2 == 1 ? 1 : 4; }
__device__ __forceinline__ int gather_node_n(int f2) { return f2 == 1 ? 1 : 3; }
__device__ __forceinline__ void gather_cell(int C, int f2, int k, int& f, double& w) {
  if (f2 == 1) { f = C; w = 1.0; return; }
  f = 2 * C - 1 + k; w = (k == 0 || k == 3) ? 0.25 : 0.75;
}
__device__ __forceinline__ void gather_node(int C, int f2, int k, int& f, double& w) {
  if (f2 == 1) { f = C; w = 1.0; return; }
  f = 2 * C - 1 + k; w = k == 1 ? 1.0 : 0.5;
}
// Scatter form (prolongation): fine f takes coarse C with weight w; tap k of at most 2.
__host__ __device__ __forceinline__ int scatter_cell_n(int f, int f2) { return f2 == 1 ? 1 : 2; }
__host__ __device__ __forceinline__ int scatter_node_n(int f, int f2) { return f2 == 1 ? 1 : ((f & 1) == 0 ? 1 : 2); }
__host__ __device__ __forceinline__ void scatter_cell(int f, int f2, int k, int& C, double& w) {
  if (f2 == 1) { C = f; w = 1.0; return; }
  const int c = f >> 1;
  C = k == 0 ? c : ((f & 1) == 0 ? c - 1 : c + 1);
  w = k == 0 ? 0.75 : 0.25;
}
__host__ __device__ __forceinline__ void scatter_node(int f, int f2, int k, int& C, double& w) {
  if (f2 == 1) { C = f; w = 1.0; return; }
  const int c = f >> 1;
  if ((f & 1) == 0) { C = c; w = 1.0; return; }
  C = c + k; w = 0.5;
}

// b_c = P^T r_f on coarse interior points; x_c = 0
// (P^T r_f) at the coarse point (j,i): the restricted u and v residuals (zero off the coarse interior)
template <class RR>
__device__ __forceinline__ void restrict_values(const Dims& df, const Dims& dc, int fx, int fy, const RR* ru,
                                                const RR* rv, int j, int i, double& bu, double& bv) {
  double s = 0.0;
  if (u_int(dc, j, i)) {
    const int ni = gather_cell_n(fx), nj = gather_node_n(fy);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (a >= nj) break;
      int fj; double wj;
      gather_node(j, fy, a, fj, wj);
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        if (b >= ni) break;
        int fi; double wi;
        gather_cell(i, fx, b, fi, wi);
        if (u_int(df, fj, fi)) s = fma(wj * wi, (double)ru[df.at(fj, fi)], s);
      }
    }
  }
  bu = s;
  s = 0.0;
  if (v_int(dc, j, i)) {
    const int ni = gather_node_n(fx), nj = gather_cell_n(fy);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      if (a >= nj) break;
      int fj; double wj;
      gather_cell(j, fy, a, fj, wj);
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        if (b >= ni) break;
        int fi; double wi;
        gather_node(i, fx, b, fi, wi);
        if (v_int(df, fj, fi)) s = fma(wj * wi, (double)rv[df.at(fj, fi)], s);
      }
    }
  }
  bv = s;
}
// b_c = P^T r_f on coarse interior points; x_c = 0
__device__ __forceinline__ void restrict_point(const Dims& df, const Dims& dc, int fx, int fy, const double* ru,
                                               const double* rv, double* bu, double* bv, double* xu, double* xv,
                                               int j, int i) {
  const long long q = dc.at(j, i);
  restrict_values(df, dc, fx, fy, ru, rv, j, i, bu[q], bv[q]);
  xu[q] = 0.0;
  xv[q] = 0.0;
}
__global__ void k_restrict(Dims df, Dims dc, int fx, int fy, const double* ru, const double* rv, double* bu,
                           double* bv, double* xu, double* xv) {
  IDX2D
  if (j >= dc.ny || i >= dc.nx) return;
  restrict_point(df, dc, fx, fy, ru, rv, bu, bv, xu, xv, j, i);
}

// P x_c at the fine point (j,i): increments of u and v (coarse values read through the
// coarse boundary mapping); zero off the fine interior
__device__ __forceinline__ void prolong_delta(const Op& oc, const Dims& df, int fx, int fy, const double* xcu,
                                              const double* xcv, int j, int i, double& du, double& dv) {
  const Dims& dc = oc.d;
  du = 0.0;
  dv = 0.0;
  if (u_int(df, j, i)) {
    const int ni = scatter_cell_n(i, fx), nj = scatter_node_n(j, fy);
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      if (a >= nj) break;
      int Cj; double wj;
      scatter_node(j, fy, a, Cj, wj);
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        if (b >= ni) break;
        int Ci; double wi;
        scatter_cell(i, fx, b, Ci, wi);
        const int J = min(max(Cj, 0), dc.ny - 1), I = min(max(Ci, 0), dc.nx - 2);
        s = fma(wj * wi, LU(oc, xcu, J, I), s);
      }
    }
    du = s;
  }
  if (v_int(df, j, i)) {
    const int ni = scatter_node_n(i, fx), nj = scatter_cell_n(j, fy);
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      if (a >= nj) break;
      int Cj; double wj;
      scatter_cell(j, fy, a, Cj, wj);
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        if (b >= ni) break;
        int Ci; double wi;
        scatter_node(i, fx, b, Ci, wi);
        const int J = min(max(Cj, 0), dc.ny - 2), I = min(max(Ci, 0), dc.nx - 1);
        s = fma(wj * wi, LV(oc, xcv, J, I), s);
      }
    }
    dv = s;
  }
}
// P x_c at the fine point (j,i) of a level coarsened by 2 in both directions, from the
// coarse correction staged in shared memory: cu/cv hold, for the coarse region whose
// origin is (CJ0,CI0) (CRJ rows per column), the values prolong_delta reads (the clamped
// position read through the coarse boundary mapping).  The same taps, weights and order.
__device__ __forceinline__ void prolong_delta_staged(const Dims& df, const double* cu, const double* cv, int CJ0,
                                                     int CI0, int CRJ, int j, int i, double& du, double& dv) {
  du = 0.0;
  dv = 0.0;
  if (u_int(df, j, i)) {
    const int ni = scatter_cell_n(i, 2), nj = scatter_node_n(j, 2);
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      if (a >= nj) break;
      int Cj; double wj;
      scatter_node(j, 2, a, Cj, wj);
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        if (b >= ni) break;
        int Ci; double wi;
        scatter_cell(i, 2, b, Ci, wi);
        s = fma(wj * wi, cu[(Ci - CI0) * CRJ + (Cj - CJ0)], s);
      }
    }
    du = s;
  }
  if (v_int(df, j, i)) {
    const int ni = scatter_node_n(i, 2), nj = scatter_cell_n(j, 2);
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      if (a >= nj) break;
      int Cj; double wj;
      scatter_cell(j, 2, a, Cj, wj);
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        if (b >= ni) break;
        int Ci; double wi;
        scatter_node(i, 2, b, Ci, wi);
        s = fma(wj * wi, cv[(Ci - CI0) * CRJ + (Cj - CJ0)], s);
      }
    }
    dv = s;
  }
}
// x_f += P x_c on fine interior points
__device__ __forceinline__ void prolong_point(const Op& oc, const Dims& df, int fx, int fy, const double* xcu,
                                              const double* xcv, double* xu, double* xv, int j, int i) {
  const long long q = df.at(j, i);
  double du, dv;
  prolong_delta(oc, df, fx, fy, xcu, xcv, j, i, du, dv);
  if (u_int(df, j, i)) xu[q] += du;
  if (v_int(df, j, i)) xv[q] += dv;
}
__global__ void k_prolong(Op oc, Dims df, int fx, int fy, const double* xcu, const double* xcv, double* xu,
                          double* xv) {
  IDX2D
  if (j >= df.ny || i >= df.nx) return;
  prolong_point(oc, df, fx, fy, xcu, xcv, xu, xv, j, i);
}

// ---- tiled smoothing of the large levels ---------------------------------------------
// One block owns a TJ x TI tile of a level and keeps x and b of the tile plus a
// halo of H points on every side in shared memory (H = 4 nu + 1 for nu sweeps per
// phase: kHalo for two, kHaloOne for one).  Colour pass q of a smoothing phase
// updates the points within H-1-q of the tile.  Every value
// a row reads -- its stencil neighbours and, on an 'infinite' or 'zero' side, the
// inner point a boundary unknown is mapped to -- lies within one point of the row,
// so after the 8 passes of V(2,2)'s pre- or post-smoothing the tile and one ring
// around it hold exactly what the level-wide colour sweeps produce, and the
// residual of the tile follows from them.  The halo is recomputed by the
// neighbouring blocks instead of exchanged.  A periodic side maps a boundary
// unknown across the domain, so such grids use the per-colour kernels.
constexpr int kHalo = 9;        // the widest halo: 2 sweeps (8 colour passes) + 1
constexpr int kHaloOne = 5;     // the halo of 1 sweep (4 colour passes) + 1
constexpr int kTileThreads = 512;
// the halo a tile kernel needs for `sweeps` smoothing sweeps per phase
inline int halo_for(int sweeps) { return sweeps <= 1 ? kHaloOne : kHalo; }

// STAGE: the region's coefficients (N_a, N_b, B_x, B_y and the inverse diagonals)
// are staged in shared memory too, so the colour passes touch no global memory.
// R: the type of the tile's values and coefficients (float on the finest level of the
// mixed-precision preconditioner, else double).
template <int TJ, int TI, bool STAGE, class R = double, int H = kHalo>
struct TileGeom {
  static constexpr int RJ = TJ + 2 * H, RI = TI + 2 * H, N = RJ * RI;
  static constexpr size_t smem = (STAGE ? 10 : 4) * N * sizeof(R);   // x, b (+ 6 coefficient planes)
  // the post-smoothing kernel also stages the coarse correction under its region (a
  // level coarsened by 2 in both directions): CRJ x CRI coarse points, u and v, in double
  static constexpr int CRJ = RJ / 2 + 3, CRI = RI / 2 + 3;
  static constexpr size_t coarse_off = (smem + 7) / 8;   // in doubles
  static constexpr size_t smem_up = (coarse_off + 2 * CRJ * CRI) * sizeof(double);
};

// A block whose whole region lies in the interior of both components (u: 1 <= i <=
// nx-3, 1 <= j <= ny-2; v: 1 <= i <= nx-2, 1 <= j <= ny-3) reads every stencil value
// as stored: the boundary mapping is the identity there, so DEEP blocks skip it and
// the interior tests (the same values, decided once per block).
constexpr bool kTileDeepPath = true;
template <int TJ, int TI, int H>
__device__ __forceinline__ bool tile_deep(const TIx& ix, const Dims& d) {
  constexpr int RJ = TJ + 2 * H, RI = TI + 2 * H;
  return kTileDeepPath && ix.i0 >= 1 && ix.i0 + RI - 1 <= d.nx - 3 && ix.j0 >= 1 && ix.j0 + RJ - 1 <= d.ny - 3;
}

// The shared-memory planes of a tile kernel and the operator reading from them.
// FRONT: the operator may carry 'BC' front rows (only the finest level's kernels with
// choice_ice_margin 'BC'); without it the row-type test is compiled out.
template <int TJ, int TI, bool STAGE, bool FRONT, class R, int H>
struct TileMem {
  R *xu, *xv, *bu, *bv;
  const R *iu, *iv;   // inverse diagonals: staged plane or the level's
  OpT<R> os;          // the level's operator, coefficients staged when STAGE
  __device__ TileMem(R* sm, const OpT<R>& o, const R* idu, const R* idv) {
    using G = TileGeom<TJ, TI, STAGE, R, H>;
    xu = sm; xv = sm + G::N; bu = sm + 2 * G::N; bv = sm + 3 * G::N;
    os = o;
    iu = idu; iv = idv;
    if (STAGE) {
      os.Na = sm + 4 * G::N; os.Nb = sm + 5 * G::N; os.Bx = sm + 6 * G::N; os.By = sm + 7 * G::N;
      iu = sm + 8 * G::N; iv = sm + 9 * G::N;
    }
  }
  // stage the region's coefficients (out-of-domain points are never read)
  __device__ void stage(const OpT<R>& o, const R* idu, const R* idv, const TIx& ix, int t, bool in, long long q) {
    if (!STAGE) return;
    using G = TileGeom<TJ, TI, STAGE, R, H>;
    R* sm = xu;
    sm[4 * G::N + t] = in ? o.Na[q] : R(0);
    sm[5 * G::N + t] = in ? o.Nb[q] : R(0);
    sm[6 * G::N + t] = in ? o.Bx[q] : R(0);
    sm[7 * G::N + t] = in ? o.By[q] : R(0);
    sm[8 * G::N + t] = in ? idu[q] : R(0);
    sm[9 * G::N + t] = in ? idv[q] : R(0);
  }
  template <bool RAW>
  __device__ __forceinline__ R Au(const TIx& ix, int j, int i) const {
    if (STAGE) return AuXC<RAW, FRONT>(os, xu, xv, ix, ix, j, i);
    return AuXC<RAW, FRONT>(os, xu, xv, ix, GIx{os.d}, j, i);
  }
  template <bool RAW>
  __device__ __forceinline__ R Av(const TIx& ix, int j, int i) const {
    if (STAGE) return AvXC<RAW, FRONT>(os, xu, xv, ix, ix, j, i);
    return AvXC<RAW, FRONT>(os, xu, xv, ix, GIx{os.d}, j, i);
  }
  __device__ __forceinline__ R idu(const TIx& ix, int j, int i) const {
    return STAGE ? iu[ix(j, i)] : iu[os.d.at(j, i)];
  }
  __device__ __forceinline__ R idv(const TIx& ix, int j, int i) const {
    return STAGE ? iv[ix(j, i)] : iv[os.d.at(j, i)];
  }
  // Boundary unknowns in the tile ("ghosts").  A u or v value outside its component's
  // interior is read, by the rows next to it, through the boundary elimination (u_src,
  // v_src): as the value of its source point, or as zero.  The tile keeps each such value
  // in its own slot, equal to its source's value, so every row of a block reads its whole
  // stencil as stored, at the domain's edge too.  The elimination maps a row's outside
  // same-component neighbours back to the row itself (read before the row's own update),
  // and cross-component ghosts are read only in the other component's passes, so a
  // component's ghosts are refreshed from their sources (ghost_refresh) after the staging
  // and after each pair of that component's colour passes: every read then sees the value
  // the elimination would read.  (Periodic sides, whose sources lie across the
  // domain, do not use the tiles.)
  __device__ __forceinline__ bool in_region(const TIx& ix, int j, int i) const {
    using G = TileGeom<TJ, TI, STAGE, R, H>;
    return j >= ix.j0 && j < ix.j0 + G::RJ && i >= ix.i0 && i < ix.i0 + G::RI;
  }
  // The new value of the interior u point (j,i) into the ghosts whose source it is: by
  // u_src's rule, the edge point beyond it on an 'infinite' side and the corner beyond it
  // where two such sides meet.
  __device__ __forceinline__ void ghosts_u(const TIx& ix, int j, int i, R val) {
    const Dims& d = os.d;
    const BCs& b = os.bc;
    const bool W = i == 1, E = i == d.nx - 3, S = j == 1, N = j == d.ny - 2;
    if (!(W || E || S || N)) return;
    auto put = [&](int jg, int ig) { if (in_region(ix, jg, ig)) xu[ix(jg, ig)] = val; };
    constexpr int INF = DIVA_BC_INFINITE;
    if (W && b.uW == INF) put(j, 0);
    if (E && b.uE == INF) put(j, d.nx - 2);
    if (S && b.uS == INF) put(0, i);
    if (N && b.uN == INF) put(d.ny - 1, i);
    if (W && S && bc_pick(b.uS, b.uW) == INF) put(0, 0);
    if (E && S && bc_pick(b.uS, b.uE) == INF) put(0, d.nx - 2);
    if (W && N && bc_pick(b.uN, b.uW) == INF) put(d.ny - 1, 0);
    if (E && N && bc_pick(b.uN, b.uE) == INF) put(d.ny - 1, d.nx - 2);
  }
  // Every source point of the region (the interior points on the lines i = 1, the last
  // interior column, j = 1 and the last interior row of each component) writes its current
  // value into its ghosts; one point per thread.
  __device__ __forceinline__ void ghost_refresh(const TIx& ix, int comps = 3) {   // bit 0: u, bit 1: v
    using G = TileGeom<TJ, TI, STAGE, R, H>;
    const Dims& d = os.d;
    // the four lines of each component, clipped to the region: 2 vertical (RJ points each)
    // and 2 horizontal (RI points each)
    const int per = 2 * G::RJ + 2 * G::RI;
    const int t0 = (comps & 1) ? 0 : per, t1 = (comps & 2) ? 2 * per : per;
    for (int t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
      const bool ucomp = t < per;
      const int e = ucomp ? t : t - per;
      int j, i;
      if (e < 2 * G::RJ) {   // a column line: i = 1 or the last interior column
        j = ix.j0 + e % G::RJ;
        i = e < G::RJ ? 1 : (ucomp ? d.nx - 3 : d.nx - 2);
      } else {               // a row line: j = 1 or the last interior row
        const int f = e - 2 * G::RJ;
        i = ix.i0 + f % G::RI;
        j = f < G::RI ? 1 : (ucomp ? d.ny - 2 : d.ny - 3);
      }
      if (!in_region(ix, j, i)) continue;
      if (ucomp) {
        if (u_int(d, j, i)) ghosts_u(ix, j, i, xu[ix(j, i)]);
      } else {
        if (v_int(d, j, i)) ghosts_v(ix, j, i, xv[ix(j, i)]);
      }
    }
  }
  // the same for the interior v point (j,i) (v_src's rule)
  __device__ __forceinline__ void ghosts_v(const TIx& ix, int j, int i, R val) {
    const Dims& d = os.d;
    const BCs& b = os.bc;
    const bool W = i == 1, E = i == d.nx - 2, S = j == 1, N = j == d.ny - 3;
    if (!(W || E || S || N)) return;
    auto put = [&](int jg, int ig) { if (in_region(ix, jg, ig)) xv[ix(jg, ig)] = val; };
    constexpr int INF = DIVA_BC_INFINITE;
    if (W && b.vW == INF) put(j, 0);
    if (E && b.vE == INF) put(j, d.nx - 1);
    if (S && b.vS == INF) put(0, i);
    if (N && b.vN == INF) put(d.ny - 2, i);
    if (W && S && bc_pick(b.vS, b.vW) == INF) put(0, 0);
    if (E && S && bc_pick(b.vS, b.vE) == INF) put(0, d.nx - 1);
    if (W && N && bc_pick(b.vN, b.vW) == INF) put(d.ny - 2, 0);
    if (E && N && bc_pick(b.vN, b.vE) == INF) put(d.ny - 2, d.nx - 1);
  }
};

// one colour pass over the region points within `reach` of the tile
template <bool DEEP, class M>
__device__ __forceinline__ void tile_pass(M& m, const TIx& ix, int TJ, int TI, int tj0, int ti0, int comp, int color,
                                          int reach) {
  const Dims& d = m.os.d;
  // the box of points within `reach` of the tile, one colour of it
  const int bj0 = tj0 - reach, bi0 = ti0 - reach, BJ = TJ + 2 * reach, BI = TI + 2 * reach;
  const int hj = (BJ + 1) / 2;
  for (int t = threadIdx.x; t < hj * BI; t += blockDim.x) {
    const int i = bi0 + t / hj;
    const int j = bj0 + 2 * (t % hj) + ((color + i + bj0) & 1);   // (i + j) & 1 == color
    if (j >= bj0 + BJ) continue;
    if (!DEEP && (j < 0 || j >= d.ny || i < 0 || i >= d.nx)) continue;
    const int k = ix(j, i);
    // every stencil value is read as stored: at the domain's edge the ghosts hold what
    // the boundary elimination would read
    if (comp == 0) {
      if (DEEP || u_int(d, j, i)) m.xu[k] = fma_r(m.bu[k] - m.template Au<true>(ix, j, i), m.idu(ix, j, i), m.xu[k]);
    } else {
      if (DEEP || v_int(d, j, i)) m.xv[k] = fma_r(m.bv[k] - m.template Av<true>(ix, j, i), m.idv(ix, j, i), m.xv[k]);
    }
  }
}
template <int TJ, int TI, class M>
__device__ __forceinline__ void tile_pass_any(bool deep, M& m, const TIx& ix, int tj0, int ti0, int comp, int color,
                                              int reach) {
  if (deep) tile_pass<true>(m, ix, TJ, TI, tj0, ti0, comp, color, reach);
  else tile_pass<false>(m, ix, TJ, TI, tj0, ti0, comp, color, reach);
}

// Source of b for a pre-smoothing kernel: given on the level (the finest), or the
// restriction of the finer level's residual, computed where it is needed.
struct Restriction {
  int on;              // 0: b given in gbu/gbv
  Dims df;             // finer level
  int fx, fy;          // coarsening factors from it
  const void *ru, *rv; // its residual: double, or float (rfloat) from a mixed-precision finest level
  int rfloat;
};
__device__ __forceinline__ void restrict_from(const Restriction& rs, const Dims& dc, int j, int i, double& b0,
                                              double& b1) {
  if (rs.rfloat)
    restrict_values(rs.df, dc, rs.fx, rs.fy, static_cast<const float*>(rs.ru), static_cast<const float*>(rs.rv), j,
                    i, b0, b1);
  else
    restrict_values(rs.df, dc, rs.fx, rs.fy, static_cast<const double*>(rs.ru), static_cast<const double*>(rs.rv),
                    j, i, b0, b1);
}

// pre-smoothing from x = 0 (the descent of a V-cycle enters every level with x = 0):
// `sweeps` forward sweeps (u0 u1 v0 v1), then x, b and r = b - A x of the tile.
// b is read (and, when restricted here, stored) in double; x and r are written in R.
template <int TJ, int TI, bool STAGE, bool FRONT, class R, int H>
__global__ void __launch_bounds__(kTileThreads) k_smooth_down(OpT<R> o, Restriction rs, double* gbu, double* gbv,
                                                              R* gxu, R* gxv, R* gru, R* grv, const R* idu,
                                                              const R* idv, int sweeps) {
  constexpr int RJ = TJ + 2 * H, N = RJ * (TI + 2 * H);
  extern __shared__ double smd[];
  R* sm = reinterpret_cast<R*>(smd);
  TileMem<TJ, TI, STAGE, FRONT, R, H> m(sm, o, idu, idv);
  const Dims& d = o.d;
  const int tj0 = blockIdx.x * TJ, ti0 = blockIdx.y * TI;
  const TIx ix{tj0 - H, ti0 - H, RJ};
  const bool deep = tile_deep<TJ, TI, H>(ix, d);
  for (int t = threadIdx.x; t < N; t += blockDim.x) {
    const int j = ix.j0 + t % RJ, i = ix.i0 + t / RJ;
    const bool in = j >= 0 && j < d.ny && i >= 0 && i < d.nx;
    const long long q = in ? d.at(j, i) : 0;
    double b0 = 0.0, b1 = 0.0;
    if (in) {
      if (rs.on) {
        restrict_from(rs, d, j, i, b0, b1);
      } else {
        b0 = gbu[q];
        b1 = gbv[q];
      }
    }
    m.xu[t] = R(0);
    m.xv[t] = R(0);
    m.bu[t] = R(b0);
    m.bv[t] = R(b1);
    m.stage(o, idu, idv, ix, t, in, q);
  }
  __syncthreads();
  int pass = 0;
  for (int s = 0; s < sweeps; ++s)
    for (int p = 0; p < 4; ++p, ++pass) {
      tile_pass_any<TJ, TI>(deep, m, ix, tj0, ti0, p >> 1, p & 1, H - 1 - pass);
      __syncthreads();
      if (!deep && (p & 1)) {   // a component's pair done: its ghosts from their sources
        m.ghost_refresh(ix, 1 << (p >> 1));
        __syncthreads();
      }
    }
  for (int t = threadIdx.x; t < TJ * TI; t += blockDim.x) {
    const int j = tj0 + t % TJ, i = ti0 + t / TJ;
    if (j >= d.ny || i >= d.nx) continue;
    const long long q = d.at(j, i);
    const int k = ix(j, i);
    gxu[q] = m.xu[k];
    gxv[q] = m.xv[k];
    if (rs.on) {
      gbu[q] = m.bu[k];
      gbv[q] = m.bv[k];
    }
    if (deep) {
      gru[q] = m.bu[k] - m.template Au<true>(ix, j, i);
      grv[q] = m.bv[k] - m.template Av<true>(ix, j, i);
    } else {
      // the ghosts hold the boundary values: stored reads
      gru[q] = u_int(d, j, i) ? m.bu[k] - m.template Au<true>(ix, j, i) : R(0);
      grv[q] = v_int(d, j, i) ? m.bv[k] - m.template Av<true>(ix, j, i) : R(0);
    }
  }
}

// post-smoothing: x += P x_c, then `sweeps` backward sweeps (v1 v0 u1 u0); x of the tile.
// The pre-smoothed x is read over the halo from (gxu, gxv) and the result written to
// (oxu, oxv): separate arrays, since blocks of other tiles may still be reading the
// halo when this block writes (the grid runs in several waves on large levels).  The
// coarse correction and b are double; the smoothing runs in R; the output is double.
template <int TJ, int TI, bool STAGE, bool FRONT, class R, int H>
__global__ void __launch_bounds__(kTileThreads) k_smooth_up(OpT<R> o, Op oc, int fx, int fy, const double* xcu,
                                                            const double* xcv, const double* gbu, const double* gbv,
                                                            const R* gxu, const R* gxv, double* oxu, double* oxv,
                                                            const R* idu, const R* idv, int sweeps) {
  constexpr int RJ = TJ + 2 * H, N = RJ * (TI + 2 * H);
  extern __shared__ double smd[];
  R* sm = reinterpret_cast<R*>(smd);
  TileMem<TJ, TI, STAGE, FRONT, R, H> m(sm, o, idu, idv);
  const Dims& d = o.d;
  const int tj0 = blockIdx.x * TJ, ti0 = blockIdx.y * TI;
  const TIx ix{tj0 - H, ti0 - H, RJ};
  const bool deep = tile_deep<TJ, TI, H>(ix, d);
  // The coarse correction under the region, staged once (a level coarsened by 2 in both
  // directions): each coarse value is read from L2 once per block instead of by every
  // fine point that takes it (up to 8 reads per fine point).
  using G = TileGeom<TJ, TI, STAGE, R, H>;
  const bool staged = fx == 2 && fy == 2;
  const int CJ0 = (ix.j0 >> 1) - 1, CI0 = (ix.i0 >> 1) - 1;
  double* cu = smd + G::coarse_off;
  double* cv = cu + G::CRJ * G::CRI;
  if (staged) {
    const Dims& dc = oc.d;
    for (int t = threadIdx.x; t < G::CRJ * G::CRI; t += blockDim.x) {
      const int J = CJ0 + t % G::CRJ, I = CI0 + t / G::CRJ;
      cu[t] = LU(oc, xcu, min(max(J, 0), dc.ny - 1), min(max(I, 0), dc.nx - 2));
      cv[t] = LV(oc, xcv, min(max(J, 0), dc.ny - 2), min(max(I, 0), dc.nx - 1));
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < N; t += blockDim.x) {
    const int j = ix.j0 + t % RJ, i = ix.i0 + t / RJ;
    const bool in = j >= 0 && j < d.ny && i >= 0 && i < d.nx;
    const long long q = in ? d.at(j, i) : 0;
    double xa = 0.0, xb = 0.0, ba = 0.0, bb = 0.0;
    if (in) {
      double du, dv;
      if (staged) prolong_delta_staged(d, cu, cv, CJ0, CI0, G::CRJ, j, i, du, dv);
      else prolong_delta(oc, d, fx, fy, xcu, xcv, j, i, du, dv);
      xa = gxu[q];
      xb = gxv[q];
      if (u_int(d, j, i)) xa += du;
      if (v_int(d, j, i)) xb += dv;
      ba = gbu[q];
      bb = gbv[q];
    }
    m.xu[t] = R(xa);
    m.xv[t] = R(xb);
    m.bu[t] = R(ba);
    m.bv[t] = R(bb);
    m.stage(o, idu, idv, ix, t, in, q);
  }
  __syncthreads();
  if (!deep) {
    // The ghosts take their sources' staged values: every interior point on the lines next
    // to the domain's edge writes its own ghosts (ghosts_u/ghosts_v), so only those
    // lines are visited.  A 'zero' ghost holds 0 already (the pre-smoothing left it so).
    m.ghost_refresh(ix);
    __syncthreads();
  }
  int pass = 0;
  for (int s = 0; s < sweeps; ++s)
    for (int p = 3; p >= 0; --p, ++pass) {
      tile_pass_any<TJ, TI>(deep, m, ix, tj0, ti0, p >> 1, p & 1, H - 1 - pass);
      __syncthreads();
      if (!deep && !(p & 1)) {   // a component's pair done: its ghosts from their sources
        m.ghost_refresh(ix, 1 << (p >> 1));
        __syncthreads();
      }
    }
  for (int t = threadIdx.x; t < TJ * TI; t += blockDim.x) {
    const int j = tj0 + t % TJ, i = ti0 + t / TJ;
    if (j >= d.ny || i >= d.nx) continue;
    const long long q = d.at(j, i);
    const int k = ix(j, i);
    oxu[q] = (deep || u_int(d, j, i)) ? (double)m.xu[k] : 0.0;   // no ghost values out
    oxv[q] = (deep || v_int(d, j, i)) ? (double)m.xv[k] : 0.0;
  }
}

// ---- direct solve of the coarsest level ------------------------------------------------
// The coarsest level has at most kCoarseDirectMax interior unknowns, numbered u first,
// then v, each in plane order (i outer, j inner).  Once per viscosity iteration its
// reduced matrix is assembled from the sub-cycle's row tables (the operator's nine
// terms per row, boundary reads already mapped to their sources, duplicates summed in
// the operator's own term order) and inverted by Gauss-Jordan elimination with partial
// pivoting, in one launch; the coarse step of every V-cycle is then one matrix-vector
// product.  A pivot below 1e-13 of the largest entry (a singular coarse operator, e.g.
// a free-floating shelf with no fixed boundary) raises the flag and the coarse step
// relaxes instead.
struct CoarseMap {
  int ny, nu, nv;
  __host__ __device__ __forceinline__ int n() const { return nu + nv; }
  __device__ __forceinline__ void point(int r, int& comp, int& j, int& i) const {
    if (r < nu) { comp = 0; i = 1 + r / (ny - 2); j = 1 + r % (ny - 2); }
    else { const int q = r - nu; comp = 1; i = 1 + q / (ny - 3); j = 1 + q % (ny - 3); }
  }
};

// Assembly and inversion of the coarsest level's matrix by one block.  tab is the level's
// row table (kTabCols columns of R = n rows: plane position, 4 same-component and 4
// cross-component mapped reads; the zero element P = nx*ny stands for 'zero' sides).
// Gauss-Jordan step k maps the matrix of step k-1 (buffer k&1) to the next one in one
// pass with one barrier: every warp finds the pivot row p of column k itself, and every
// element takes its value from the old matrix with rows k and p exchanged.
constexpr int kInvThreads = 1024;
constexpr size_t kInvSmem = 2 * kCoarseDirectMax * (kCoarseDirectMax + 1) * sizeof(double);

__device__ __forceinline__ void coarse_setup_block(const Op& o, const CoarseMap& m, const uint16_t* tab,
                                                   double* Ainv, int* singular) {
  constexpr int M = kCoarseDirectMax, LD = M + 1;
  extern __shared__ double inv_buf[];   // two n x n matrices, row stride LD
  __shared__ int perm[M];
  __shared__ double wmax[kInvThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n = m.n(), ny = m.ny, P = o.d.nx * ny;
  const Dims& d = o.d;
  for (int e = tid; e < n * n; e += blockDim.x) inv_buf[(e / n) * LD + e % n] = 0.0;
  __syncthreads();
  // the unknown of a plane position (compact rows of length ny) of a u or v point
  auto unknown = [&](int pos, bool ucomp) {
    const int i = pos / ny, j = pos % ny;
    return ucomp ? (i - 1) * (ny - 2) + (j - 1) : m.nu + (i - 1) * (ny - 3) + (j - 1);
  };
  for (int r = tid; r < n; r += blockDim.x) {
    const int pos = tab[r], i = pos / ny, j = pos % ny;
    int src[8];
    for (int t = 0; t < 8; ++t) src[t] = tab[(1 + t) * n + r];
    double cf[9];
    if (r < m.nu) {
      const double Ae = o.Na[d.at(j, i + 1)], Aw = o.Na[d.at(j, i)], Bn = o.Nb[d.at(j, i)], Bs = o.Nb[d.at(j - 1, i)];
      const double cE = 4.0 * o.ax * Ae, cW = 4.0 * o.ax * Aw, cN = o.ay * Bn, cS = o.ay * Bs;
      cf[0] = cE; cf[1] = cW; cf[2] = cN; cf[3] = cS;
      cf[4] = -(cE + cW + cN + cS) - o.Bx[d.at(j, i)];
      cf[5] = -2.0 * Aw - Bn; cf[6] = 2.0 * Ae + Bn; cf[7] = 2.0 * Aw + Bs; cf[8] = -2.0 * Ae - Bs;
    } else {
      const double An = o.Na[d.at(j + 1, i)], As = o.Na[d.at(j, i)], Be = o.Nb[d.at(j, i)], Bw = o.Nb[d.at(j, i - 1)];
      const double cN = 4.0 * o.ay * An, cS = 4.0 * o.ay * As, cE = o.ax * Be, cW = o.ax * Bw;
      cf[0] = cN; cf[1] = cS; cf[2] = cE; cf[3] = cW;
      cf[4] = -(cN + cS + cE + cW) - o.By[d.at(j, i)];
      cf[5] = -2.0 * An - Bw; cf[6] = 2.0 * An + Be; cf[7] = 2.0 * As + Bw; cf[8] = -2.0 * As - Be;
    }
    const bool u = r < m.nu;
    const int row = unknown(pos, u);
    double* a = inv_buf + row * LD;
    // the terms in the operator's order: 4 same-component reads, the diagonal, 4 cross reads
    for (int t = 0; t < 4; ++t)
      if (src[t] != P) a[unknown(src[t], u)] += cf[t];
    a[row] += cf[4];
    for (int t = 4; t < 8; ++t)
      if (src[t] != P) a[unknown(src[t], !u)] += cf[t + 1];
  }
  __syncthreads();
  double amax = 0.0;
  for (int e = tid; e < n * n; e += blockDim.x) {
    const double v = inv_buf[(e / n) * LD + e % n];
    amax = (fabs(v) > amax || v != v) ? fabs(v) : amax;
  }
  for (int o2 = 16; o2 > 0; o2 >>= 1) {   // largest magnitude; a NaN wins
    const double w = __shfl_xor_sync(0xffffffffu, amax, o2);
    amax = (w > amax || w != w) ? w : amax;
  }
  if (lane == 0) wmax[warp] = amax;
  __syncthreads();
  amax = wmax[0];
  for (int w = 1; w < (int)(blockDim.x >> 5); ++w) amax = (wmax[w] > amax || wmax[w] != wmax[w]) ? wmax[w] : amax;
  const double tiny = 1e-13 * amax;
  bool bad = !(amax > 0.0) || amax != amax;
  int cur = 0;
  for (int k = 0; k < n && !bad; ++k) {
    const double* a = inv_buf + cur * M * LD;
    double* b = inv_buf + (cur ^ 1) * M * LD;
    // pivot: largest |a[r][k]|, r >= k, lowest r on ties (the same in every warp)
    double best = -1.0;
    int br = k;
    for (int r = k + lane; r < n; r += 32)
      if (fabs(a[r * LD + k]) > best) { best = fabs(a[r * LD + k]); br = r; }
    for (int o2 = 16; o2 > 0; o2 >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o2);
      const int orr = __shfl_xor_sync(0xffffffffu, br, o2);
      if (ob > best || (ob == best && orr < br)) { best = ob; br = orr; }
    }
    if (!(best > tiny)) { bad = true; break; }
    const int p = br;
    if (tid == 0) perm[k] = p;
    const double piv = a[p * LD + k];
    for (int e = tid; e < n * n; e += blockDim.x) {
      const int r = e / n, c = e % n;
      const double pk = (c == k ? 1.0 : a[p * LD + c]) / piv;   // normalised pivot row
      if (r == k) {
        b[r * LD + c] = pk;
      } else {
        const int src = r == p ? k : r;   // the row that sits at r after the exchange
        b[r * LD + c] = (c == k ? 0.0 : a[src * LD + c]) - a[src * LD + k] * pk;
      }
    }
    cur ^= 1;
    __syncthreads();
  }
  if (!bad) {
    double* a = inv_buf + cur * M * LD;
    for (int k = n - 1; k >= 0; --k) {
      const int p = perm[k];
      if (p != k)
        for (int r = tid; r < n; r += blockDim.x) {
          const double t = a[r * LD + k];
          a[r * LD + k] = a[r * LD + p];
          a[r * LD + p] = t;
        }
      __syncthreads();
    }
    for (int e = tid; e < n * n; e += blockDim.x) Ainv[e] = a[(e / n) * LD + e % n];
  }
  if (tid == 0) *singular = bad ? 1 : 0;
}


// x = Ainv b on the coarsest level, by one block (the caller synchronises).  The descent
// enters the coarsest level with x = 0, so its residual is b itself.  AinvT is the
// inverse transposed (AinvT[c * n + r] = Ainv[r][c]), in shared memory, so the threads of
// a warp read consecutive elements; the sums run over c in ascending order.
__device__ __forceinline__ void block_coarse_direct(const Op& o, const CoarseMap& m, const double* AinvT, double* xu,
                                                    double* xv, const double* bu, const double* bv) {
  __shared__ double sr[kCoarseDirectMax];
  const int n = m.n();
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    int comp, j, i;
    m.point(r, comp, j, i);
    const long long q = o.d.at(j, i);
    sr[r] = comp == 0 ? bu[q] : bv[q];
  }
  __syncthreads();
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    double s = 0.0;
    for (int c = 0; c < n; ++c) s += AinvT[c * n + r] * sr[c];
    int comp, j, i;
    m.point(r, comp, j, i);
    (comp == 0 ? xu : xv)[o.d.at(j, i)] = s;
  }
}

// The levels from `first` down, run by one thread block out of shared memory with
// barriers between the phases: the same per-point operations in the same order
// as the per-level kernels of vcycle(), without a launch per phase and without a
// global-memory round trip per phase.  Each level keeps kSubArrays compact planes
// (row length ny, one extra element that stays 0) in the block's dynamic shared
// memory; the coefficients of every level and b of the first are staged in at the
// start, x of the first level is written back at the end.
//
// The Gauss-Seidel passes and residuals run from row tables built once on the host
// (they depend on the grid and the boundary conditions only): for each level the
// interior rows grouped by (component, colour), each with its plane position and the
// positions its eight off-diagonal stencil reads map to (boundary unknowns resolved
// to their sources, 'zero' sides to the zero element).  A row update is then table
// reads and the operator's arithmetic, without per-read boundary logic.
enum { SA_NA, SA_NB, SA_BX, SA_BY, SA_IDU, SA_IDV, SA_XU, SA_XV, SA_BU, SA_BV, SA_RU, SA_RV, kSubArrays };
constexpr size_t kSubSmemBudget = 200 * 1024;   // dynamic shared memory of the sub-cycle
constexpr int kTabCols = 9;                      // a row's position and its eight mapped reads
constexpr int kTabProlong = 4;                   // then the row's prolongation taps (coarse positions)

struct SubLevel {
  Op o;                      // global-memory operator of the level
  const double *idu, *idv;   // global inverse diagonals
  int fx, fy;                // coarsening factors to the next level
  int soff;                  // offset of the level's planes in shared memory (doubles)
  int rows;                  // interior rows (u then v)
  int cls[5];                // row ranges of the classes u colour 0, u 1, v 0, v 1
  int toff;                  // offset of the level's row table in the shared table area (uint16)
  const uint16_t* gtab;      // the table in global memory: kTabCols columns of `rows` entries
};
struct SubCycle {
  int first, last, nu1, nu2, coarse_sweeps;
  int direct;                  // coarsest level solved with Ainv unless *singular
  CoarseMap map;
  const double* Ainv;
  const int* singular;
  Restriction rs;              // b of the first level: given, or restricted from the finer residual
  int dbl;                     // doubles of all levels' planes (the table area follows)
  int ainv_off;                // offset (doubles) of the staged, transposed inverse, after the tables
  int tab16;                   // 16-byte vectors of all levels' row tables
  SubLevel L[kMaxLevels];
};

template <class F>
__device__ __forceinline__ void block_for_points(const Dims& d, F f) {
  const int n = d.nx * d.ny;
  for (int t = threadIdx.x; t < n; t += blockDim.x) f(t % d.ny, t / d.ny);
}

// (A x) of table row r: same terms in the same order as AuX / AvX
__device__ __forceinline__ double table_row_apply(const uint16_t* tab, int R, int r, bool urow, int ny, double ax,
                                                  double ay, const double* Na, const double* Nb, const double* Bx,
                                                  const double* By, const double* xu, const double* xv, int& q) {
  q = tab[r];
  const int s0 = tab[R + r], s1 = tab[2 * R + r], s2 = tab[3 * R + r], s3 = tab[4 * R + r];
  const int s4 = tab[5 * R + r], s5 = tab[6 * R + r], s6 = tab[7 * R + r], s7 = tab[8 * R + r];
  if (urow) {
    const double Ae = Na[q + ny], Aw = Na[q], Bn = Nb[q], Bs = Nb[q - 1];
    const double cE = 4.0 * ax * Ae, cW = 4.0 * ax * Aw, cN = ay * Bn, cS = ay * Bs;
    const double diag = -(cE + cW + cN + cS) - Bx[q];
    return stencil9(cE, xu[s0], cW, xu[s1], cN, xu[s2], cS, xu[s3], diag, xu[q], -2.0 * Aw - Bn, xv[s4],
                    2.0 * Ae + Bn, xv[s5], 2.0 * Aw + Bs, xv[s6], -2.0 * Ae - Bs, xv[s7]);
  }
  const double An = Na[q + 1], As = Na[q], Be = Nb[q], Bw = Nb[q - ny];
  const double cN = 4.0 * ay * An, cS = 4.0 * ay * As, cE = ax * Be, cW = ax * Bw;
  const double diag = -(cN + cS + cE + cW) - By[q];
  return stencil9(cN, xv[s0], cS, xv[s1], cE, xv[s2], cW, xv[s3], diag, xv[q], -2.0 * An - Bw, xu[s4],
                  2.0 * An + Be, xu[s5], 2.0 * As + Bw, xu[s6], -2.0 * As - Be, xu[s7]);
}

__global__ void __launch_bounds__(kSubThreads) k_subcycle(SubCycle sc, double* xu0, double* xv0,
                                                          const double* bu0, const double* bv0) {
  extern __shared__ double sm[];
  __shared__ Op so[kMaxLevels];   // operators of the staged levels
  uint16_t* tabs = reinterpret_cast<uint16_t*>(sm + sc.dbl);
  double* AinvT = sm + sc.ainv_off;
  // whether the coarsest level is solved with its inverse (read before the staging, so
  // that the flag's load overlaps it)
  const bool direct = sc.direct && *sc.singular == 0;
  if (threadIdx.x == 0)
    for (int l = sc.first; l <= sc.last; ++l) {
      Op o = sc.L[l].o;
      const int P1 = o.d.nx * o.d.ny + 1;
      o.d.ld = o.d.ny;
      o.d.plane = P1 - 1;
      double* a = sm + sc.L[l].soff;
      o.Na = a + SA_NA * P1;
      o.Nb = a + SA_NB * P1;
      o.Bx = a + SA_BX * P1;
      o.By = a + SA_BY * P1;
      so[l] = o;
    }
  // the staging: one pass over the points of all levels (their loads independent of one
  // another), then the row tables and the coarsest level's inverse
  {
    int total = 0;
    for (int l = sc.first; l <= sc.last; ++l) total += sc.L[l].o.d.nx * sc.L[l].o.d.ny + 1;
    for (int t0 = threadIdx.x; t0 < total; t0 += blockDim.x) {
      int l = sc.first, t = t0;
      while (t >= sc.L[l].o.d.nx * sc.L[l].o.d.ny + 1) { t -= sc.L[l].o.d.nx * sc.L[l].o.d.ny + 1; ++l; }
      const SubLevel& L = sc.L[l];
      const Dims& g = L.o.d;
      const int P = g.nx * g.ny, P1 = P + 1;
      double* a = sm + L.soff;
      if (t == P) {   // the zero element read by 'zero' boundary sides
        a[SA_XU * P1 + t] = 0.0;
        a[SA_XV * P1 + t] = 0.0;
        continue;
      }
      const int jj = t % g.ny, ii = t / g.ny;
      const long long q = g.at(jj, ii);
      a[SA_NA * P1 + t] = L.o.Na[q];
      a[SA_NB * P1 + t] = L.o.Nb[q];
      a[SA_BX * P1 + t] = L.o.Bx[q];
      a[SA_BY * P1 + t] = L.o.By[q];
      a[SA_IDU * P1 + t] = L.idu[q];
      a[SA_IDV * P1 + t] = L.idv[q];
      if (l == sc.first) {   // entered with x = 0
        double b0, b1;
        if (sc.rs.on) {
          restrict_from(sc.rs, g, jj, ii, b0, b1);
        } else {
          b0 = bu0[q];
          b1 = bv0[q];
        }
        a[SA_XU * P1 + t] = 0.0;
        a[SA_XV * P1 + t] = 0.0;
        a[SA_BU * P1 + t] = b0;
        a[SA_BV * P1 + t] = b1;
      }
    }
    {   // the levels' tables are contiguous and padded to 16 bytes in both places
      const uint4* g = reinterpret_cast<const uint4*>(sc.L[sc.first].gtab);
      uint4* t = reinterpret_cast<uint4*>(tabs);
      for (int e = threadIdx.x; e < sc.tab16; e += blockDim.x) t[e] = g[e];
    }
    if (direct) {
      const int n = sc.map.n();
      for (int e = threadIdx.x; e < n * n; e += blockDim.x) AinvT[(e % n) * n + e / n] = sc.Ainv[e];
    }
  }
  __syncthreads();
  auto arr = [&](int l, int k) { return sm + sc.L[l].soff + k * (sc.L[l].o.d.nx * sc.L[l].o.d.ny + 1); };
  // one Gauss-Seidel pass over the rows of class p (0/1: u colours, 2/3: v colours)
  auto gs_pass = [&](int l, int p) {
    const SubLevel& L = sc.L[l];
    const Op& o = so[l];
    const int P1 = L.o.d.nx * L.o.d.ny + 1, ny = L.o.d.ny;
    const double* a = sm + L.soff;
    double* xu = sm + L.soff + SA_XU * P1;
    double* xv = sm + L.soff + SA_XV * P1;
    const uint16_t* tab = tabs + L.toff;
    const bool urow = p < 2;
    for (int r = L.cls[p] + threadIdx.x; r < L.cls[p + 1]; r += blockDim.x) {
      int q;
      const double Ax = table_row_apply(tab, L.rows, r, urow, ny, o.ax, o.ay, a + SA_NA * P1, a + SA_NB * P1,
                                        a + SA_BX * P1, a + SA_BY * P1, xu, xv, q);
      if (urow) xu[q] = fma(a[SA_BU * P1 + q] - Ax, a[SA_IDU * P1 + q], xu[q]);
      else xv[q] = fma(a[SA_BV * P1 + q] - Ax, a[SA_IDV * P1 + q], xv[q]);
    }
  };
  // descend
  for (int l = sc.first; l <= sc.last; ++l) {
    const Op& o = so[l];
    double *xu = arr(l, SA_XU), *xv = arr(l, SA_XV), *bu = arr(l, SA_BU), *bv = arr(l, SA_BV);
    const double *idu = arr(l, SA_IDU), *idv = arr(l, SA_IDV);
    if (l == sc.last) {
      if (direct) {
        block_coarse_direct(o, sc.map, AinvT, xu, xv, bu, bv);
        __syncthreads();
      } else {
        block_coarse_relax(o, xu, xv, bu, bv, idu, idv, sc.coarse_sweeps);
      }
      break;
    }
    for (int s = 0; s < sc.nu1; ++s)
      for (int p = 0; p < 4; ++p) {
        gs_pass(l, p);
        __syncthreads();
      }
    // residual of the interior rows (the restriction reads interior rows only)
    double *ru = arr(l, SA_RU), *rv = arr(l, SA_RV);
    {
      const SubLevel& L = sc.L[l];
      const int P1 = L.o.d.nx * L.o.d.ny + 1;
      const double* a = sm + L.soff;
      const uint16_t* tab = tabs + L.toff;
      for (int r = threadIdx.x; r < L.rows; r += blockDim.x) {
        const bool urow = r < L.cls[2];
        int q;
        const double Ax = table_row_apply(tab, L.rows, r, urow, L.o.d.ny, o.ax, o.ay, a + SA_NA * P1,
                                          a + SA_NB * P1, a + SA_BX * P1, a + SA_BY * P1, xu, xv, q);
        if (urow) ru[q] = bu[q] - Ax;
        else rv[q] = bv[q] - Ax;
      }
    }
    __syncthreads();
    const Op& k = so[l + 1];
    double *kxu = arr(l + 1, SA_XU), *kxv = arr(l + 1, SA_XV), *kbu = arr(l + 1, SA_BU), *kbv = arr(l + 1, SA_BV);
    const int fx = sc.L[l].fx, fy = sc.L[l].fy;
    // the two levels' dimensions in registers for the transfer (not re-read from shared
    // memory for every tap)
    const Dims df = o.d, dc = k.d;
    block_for_points(dc, [&](int j, int i) {
      restrict_point(df, dc, fx, fy, ru, rv, kbu, kbv, kxu, kxv, j, i);
    });
    __syncthreads();
  }
  // ascend
  for (int l = sc.last - 1; l >= sc.first; --l) {
    double *xu = arr(l, SA_XU), *xv = arr(l, SA_XV);
    const double *kxu = arr(l + 1, SA_XU), *kxv = arr(l + 1, SA_XV);
    {   // x += P x_c on the interior rows, from the rows' prolongation taps (coarse positions
        // mapped on the host; the weights formed here, in prolong_delta's order)
      const SubLevel& L = sc.L[l];
      const int fx = L.fx, fy = L.fy, ny = L.o.d.ny, R = L.rows;
      const uint16_t* tab = tabs + L.toff;
      const uint16_t* ptab = tab + kTabCols * R;
      for (int r = threadIdx.x; r < R; r += blockDim.x) {
        const int q = tab[r], j = q % ny, i = q / ny;
        double s = 0.0, wj, wi;
        int k = 0, C;
        if (r < L.cls[2]) {
          const int nj = scatter_node_n(j, fy), ni = scatter_cell_n(i, fx);
          for (int a = 0; a < nj; ++a) {
            scatter_node(j, fy, a, C, wj);
            for (int b = 0; b < ni; ++b, ++k) {
              scatter_cell(i, fx, b, C, wi);
              s = fma(wj * wi, kxu[ptab[k * R + r]], s);
            }
          }
          xu[q] += s;
        } else {
          const int nj = scatter_cell_n(j, fy), ni = scatter_node_n(i, fx);
          for (int a = 0; a < nj; ++a) {
            scatter_cell(j, fy, a, C, wj);
            for (int b = 0; b < ni; ++b, ++k) {
              scatter_node(i, fx, b, C, wi);
              s = fma(wj * wi, kxv[ptab[k * R + r]], s);
            }
          }
          xv[q] += s;
        }
      }
    }
    __syncthreads();
    for (int s = 0; s < sc.nu2; ++s)
      for (int p = 3; p >= 0; --p) {
        gs_pass(l, p);
        __syncthreads();
      }
  }
  {
    const Dims& g = sc.L[sc.first].o.d;
    const int P = g.nx * g.ny;
    const double *xu = arr(sc.first, SA_XU), *xv = arr(sc.first, SA_XV);
    for (int t = threadIdx.x; t < P; t += blockDim.x) {
      const long long q = g.at(t % g.ny, t / g.ny);
      xu0[q] = xu[t];
      xv0[q] = xv[t];
    }
  }
}

// rediscretised coarse coefficients (averages of the fine ones; B scales with the cell area)
__device__ __forceinline__ void coarsen_point(const Dims& df, const Dims& dc, int fx, int fy, const double* Na,
                                              const double* Nb, const double* Bx, const double* By, double* cNa,
                                              double* cNb, double* cBx, double* cBy, int j, int i) {
  const long long q = dc.at(j, i);
  auto cl = [](int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); };
  const double w3[3] = {0.25, 0.5, 0.25};
  {  // N_a: full weighting around fine a (fy*j, fx*i)
    double s = 0.0;
    for (int a = -1; a <= 1; ++a)
      for (int b = -1; b <= 1; ++b) {
        const double wa = fy == 2 ? w3[a + 1] : (a == 0 ? 1.0 : 0.0);
        const double wb = fx == 2 ? w3[b + 1] : (b == 0 ? 1.0 : 0.0);
        if (wa == 0.0 || wb == 0.0) continue;
        s += wa * wb * Na[df.at(cl(fy * j + a, 0, df.ny - 1), cl(fx * i + b, 0, df.nx - 1))];
      }
    cNa[q] = s;
  }
  if (j < dc.ny - 1 && i < dc.nx - 1) {  // N_b: fine b cells inside the coarse b cell
    double s = 0.0;
    const int na = fy, nb = fx;
    for (int a = 0; a < na; ++a)
      for (int b = 0; b < nb; ++b)
        s += Nb[df.at(cl(fy * j + a, 0, df.ny - 2), cl(fx * i + b, 0, df.nx - 2))];
    cNb[q] = s / (double)(na * nb);
  }
  const double area = (double)(fx * fy);
  if (i < dc.nx - 1) {  // Bx: cell along x, node along y
    double s = 0.0;
    for (int a = -1; a <= 1; ++a) {
      const double wa = fy == 2 ? w3[a + 1] : (a == 0 ? 1.0 : 0.0);
      if (wa == 0.0) continue;
      for (int b = 0; b < fx; ++b)
        s += wa * (1.0 / fx) * Bx[df.at(cl(fy * j + a, 0, df.ny - 1), cl(fx * i + b, 0, df.nx - 2))];
    }
    cBx[q] = area * s;
  }
  if (j < dc.ny - 1) {  // By: cell along y, node along x
    double s = 0.0;
    for (int b = -1; b <= 1; ++b) {
      const double wb = fx == 2 ? w3[b + 1] : (b == 0 ? 1.0 : 0.0);
      if (wb == 0.0) continue;
      for (int a = 0; a < fy; ++a)
        s += wb * (1.0 / fy) * By[df.at(cl(fy * j + a, 0, df.ny - 2), cl(fx * i + b, 0, df.nx - 1))];
    }
    cBy[q] = area * s;
  }
}

// the row types of the finest level from the SICO masks (assembly loop :1683-1727)
__global__ void k_row_types(Dims d, const int* combi, const int* inner, const int* outer, int8_t* rtu,
                            int8_t* rtv) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  int8_t t = RT_FREE;
  if (u_int(d, j, i)) {
    const long long q1 = d.at(j, i + 1);
    if ((combi[q] == 3 && combi[q1] == 1) || (combi[q] == 1 && combi[q1] == 3)) {
      t = RT_IDENT;   // shelf next to land
    } else if ((inner[q] == 1 && outer[q1] == 1) || (outer[q] == 1 && inner[q1] == 1)) {
      const int i1 = inner[q] == 1 ? i : i + 1;
      if (outer[d.at(j, i1 - 1)] == 1 && outer[d.at(j, i1 + 1)] == 1) t = RT_IDENT;
      else t = i1 == i ? RT_MARGIN_LO : RT_MARGIN_HI;
    }
  }
  rtu[q] = t;
  t = RT_FREE;
  if (v_int(d, j, i)) {
    const long long q1 = d.at(j + 1, i);
    if ((combi[q] == 3 && combi[q1] == 1) || (combi[q] == 1 && combi[q1] == 3)) {
      t = RT_IDENT;
    } else if ((inner[q] == 1 && outer[q1] == 1) || (outer[q] == 1 && inner[q1] == 1)) {
      const int j1 = inner[q] == 1 ? j : j + 1;
      if (outer[d.at(j1 - 1, i)] == 1 && outer[d.at(j1 + 1, i)] == 1) t = RT_IDENT;
      else t = j1 == j ? RT_MARGIN_LO : RT_MARGIN_HI;
    }
  }
  rtv[q] = t;
}

// rhs of the free rows of the finest level (k_rhs), folded into the first set-up launch;
// with 'BC' margins, 0 for u = 0 rows and the front stress for front rows
struct RhsArgs {
  int on, crossterms;
  const double *tdx, *tdy, *Ncx, *Ncy;
  double *bu, *bv;
  const int8_t *rtu, *rtv;
  const double *Hi, *SL, *Hb;
};

// vertically integrated stress difference across a calving front at the ice cell q
// (0.5 rho_i g H^2 - 0.5 rho_sw g H_ocean^2, :2251-2262)
__device__ __forceinline__ double front_stress(const RhsArgs& r, long long q) {
  const double H = r.Hi[q];
  const double Ho = r.SL[q] > r.Hb[q] ? min_ref(kRhoI / kRhoSW * H, r.SL[q] - r.Hb[q]) : 0.0;
  return 0.5 * kRhoI * kGrav * H * H - 0.5 * kRhoSW * kGrav * Ho * Ho;
}

// Operator set-up of one level in one launch over its points: the inverse diagonals of
// level l, the rediscretised coefficients of level l+1 (coarse points are a subset of
// the fine index range) and, on the finest level, the right-hand side.
// float copies of the finest level's coefficients and inverse diagonals (DIVA_PREC_MIXED)
struct F32Out {
  float *Na, *Nb, *Bx, *By, *idu, *idv;
};

__global__ void k_level_setup(Op o, int coarsen, Dims dc, int fx, int fy, double* cNa, double* cNb, double* cBx,
                              double* cBy, double* idu, double* idv, RhsArgs rhs, F32Out f32) {
  IDX2D
  if (j >= o.d.ny || i >= o.d.nx) return;
  const long long q = o.d.at(j, i);
  idu[q] = u_int(o.d, j, i) ? 1.0 / diag_u(o, j, i) : 0.0;
  idv[q] = v_int(o.d, j, i) ? 1.0 / diag_v(o, j, i) : 0.0;
  if (f32.Na) {
    f32.Na[q] = (float)o.Na[q];
    f32.Nb[q] = (float)o.Nb[q];
    f32.Bx[q] = (float)o.Bx[q];
    f32.By[q] = (float)o.By[q];
    f32.idu[q] = (float)idu[q];
    f32.idv[q] = (float)idv[q];
  }
  if (coarsen && j < dc.ny && i < dc.nx)
    coarsen_point(o.d, dc, fx, fy, o.Na, o.Nb, o.Bx, o.By, cNa, cNb, cBx, cBy, j, i);
  if (rhs.on) {
    const double dx2 = o.d.dx * o.d.dx;
    rhs.bu[q] = u_int(o.d, j, i) ? (rhs.crossterms ? -rhs.tdx[q] * dx2 : -rhs.tdx[q] * dx2 / rhs.Ncx[q]) : 0.0;
    rhs.bv[q] = v_int(o.d, j, i) ? (rhs.crossterms ? -rhs.tdy[q] * dx2 : -rhs.tdy[q] * dx2 / rhs.Ncy[q]) : 0.0;
    if (rhs.rtu) {
      const int tu = rhs.rtu[q], tv = rhs.rtv[q];
      if (tu == RT_IDENT) rhs.bu[q] = 0.0;
      else if (tu != RT_FREE) rhs.bu[q] = front_stress(rhs, o.d.at(j, tu == RT_MARGIN_LO ? i : i + 1));
      if (tv == RT_IDENT) rhs.bv[q] = 0.0;
      else if (tv != RT_FREE) rhs.bv[q] = front_stress(rhs, o.d.at(tv == RT_MARGIN_LO ? j : j + 1, i));
    }
  }
}

// Operator set-up of the sub-cycle levels in one block: per level (one barrier each) the
// inverse diagonals and the coefficients of the next level, then the coarsest level's
// matrix and its inverse.  The same per-point operations as k_level_setup and
// k_coarse_setup.
struct SmallSetup {
  int first, last;           // the levels handled
  int direct;                // assemble and invert the coarsest level's matrix
  // when: 0 every launch; 1 in the viscosity iterations coarse_inverse_due() picks, read from
  // the device iteration counter (graph-launched loop); 2 not in this launch
  int inv_when;
  const double* sc;
  CoarseMap map;
  const uint16_t* tab;       // the coarsest level's row table
  double* Ainv;
  int* singular;
  Op o[kMaxLevels];
  double *idu[kMaxLevels], *idv[kMaxLevels];
  int fx[kMaxLevels], fy[kMaxLevels];
};

__global__ void __launch_bounds__(kInvThreads) k_small_setup(SmallSetup a) {
  for (int l = a.first; l <= a.last; ++l) {
    const Op& o = a.o[l];
    const bool coarsen = l < a.last;
    const Op& k = a.o[coarsen ? l + 1 : l];
    const int n = o.d.nx * o.d.ny;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      const int j = t % o.d.ny, i = t / o.d.ny;
      const long long q = o.d.at(j, i);
      a.idu[l][q] = u_int(o.d, j, i) ? 1.0 / diag_u(o, j, i) : 0.0;
      a.idv[l][q] = v_int(o.d, j, i) ? 1.0 / diag_v(o, j, i) : 0.0;
      if (coarsen && j < k.d.ny && i < k.d.nx)
        coarsen_point(o.d, k.d, a.fx[l], a.fy[l], o.Na, o.Nb, o.Bx, o.By, const_cast<double*>(k.Na),
                      const_cast<double*>(k.Nb), const_cast<double*>(k.Bx), const_cast<double*>(k.By), j, i);
    }
    __syncthreads();
  }
  const bool inv = a.inv_when == 0 || (a.inv_when == 1 && coarse_inverse_due((int)a.sc[SC_PIC_IT]));
  if (a.direct && inv) coarse_setup_block(a.o[a.last], a.map, a.tab, a.Ainv, a.singular);
}

// ---- Krylov kernels (fine level) --------------------------------------------------
constexpr int kPW = 4;   // partial sums per block

__device__ __forceinline__ void store_partials(double (&v)[kPW], double* partials, int nbx) {
  block_sum<kPW>(v);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const int b = blockIdx.y * nbx + blockIdx.x;
#pragma unroll
    for (int q = 0; q < kPW; ++q) partials[kPW * b + q] = v[q];
  }
}

// out = A x ; partial dots: [0] = w1.out, [1] = w2.out, [2] = out.out
__global__ void k_matvec(Op o, const double* xu, const double* xv, double* ou, double* ov, const double* w1u,
                         const double* w1v, const double* w2u, const double* w2v, double* partials, int nbx) {
  IDX2D
  double acc[kPW] = {0.0, 0.0, 0.0, 0.0};
  if (j < o.d.ny && i < o.d.nx) {
    const long long q = o.d.at(j, i);
    if (u_int(o.d, j, i)) {
      const double a = Au(o, xu, xv, j, i);
      ou[q] = a;
      if (w1u) acc[0] += w1u[q] * a;
      if (w2u) acc[1] += w2u[q] * a;
      acc[2] += a * a;
    } else {
      ou[q] = 0.0;
    }
    if (v_int(o.d, j, i)) {
      const double a = Av(o, xu, xv, j, i);
      ov[q] = a;
      if (w1v) acc[0] += w1v[q] * a;
      if (w2v) acc[1] += w2v[q] * a;
      acc[2] += a * a;
    } else {
      ov[q] = 0.0;
    }
  }
  store_partials(acc, partials, nbx);
}

// r = b - A x; rhat = r; partials: [0] r.r, [1] b.b
__global__ void k_init_residual(Op o, const double* xu, const double* xv, const double* bu, const double* bv,
                                double* ru, double* rv, double* hu, double* hv, double* pu, double* pv,
                                double* partials, int nbx) {
  IDX2D
  double acc[kPW] = {0.0, 0.0, 0.0, 0.0};
  if (j < o.d.ny && i < o.d.nx) {
    const long long q = o.d.at(j, i);
    double r = 0.0;
    if (u_int(o.d, j, i)) {
      r = bu[q] - Au(o, xu, xv, j, i);
      acc[0] += r * r;
      acc[1] += bu[q] * bu[q];
    }
    ru[q] = r; hu[q] = r; pu[q] = r;
    r = 0.0;
    if (v_int(o.d, j, i)) {
      r = bv[q] - Av(o, xu, xv, j, i);
      acc[0] += r * r;
      acc[1] += bv[q] * bv[q];
    }
    rv[q] = r; hv[q] = r; pv[q] = r;
  }
  store_partials(acc, partials, nbx);
}

// s = r - alpha v ; partial [0] s.s
__global__ void k_update_s(Dims d, const double* sc, const double* ru, const double* rv, const double* vu,
                           const double* vv, double* su, double* sv, double* partials, int nbx) {
  IDX2D
  double acc[kPW] = {0.0, 0.0, 0.0, 0.0};
  if (j < d.ny && i < d.nx) {
    const long long q = d.at(j, i);
    const double alpha = sc[SC_ALPHA];
    const double a = ru[q] - alpha * vu[q], b = rv[q] - alpha * vv[q];
    su[q] = a; sv[q] = b;
    acc[0] = a * a + b * b;
  }
  store_partials(acc, partials, nbx);
}

// x += alpha phat + omega shat ; r = s - omega t ; partials [0] rhat.r, [1] r.r
__global__ void k_update_xr(Dims d, const double* sc, double* xu, double* xv, const double* phu, const double* phv,
                            const double* shu, const double* shv, const double* su, const double* sv,
                            const double* tu, const double* tv, double* ru, double* rv, const double* hu,
                            const double* hv, double* partials, int nbx) {
  IDX2D
  double acc[kPW] = {0.0, 0.0, 0.0, 0.0};
  if (j < d.ny && i < d.nx) {
    const long long q = d.at(j, i);
    const double alpha = sc[SC_ALPHA], omega = sc[SC_OMEGA];
    if (u_int(d, j, i)) {
      xu[q] += alpha * phu[q] + omega * shu[q];
      const double r = su[q] - omega * tu[q];
      ru[q] = r;
      acc[0] += hu[q] * r;
      acc[1] += r * r;
    }
    if (v_int(d, j, i)) {
      xv[q] += alpha * phv[q] + omega * shv[q];
      const double r = sv[q] - omega * tv[q];
      rv[q] = r;
      acc[0] += hv[q] * r;
      acc[1] += r * r;
    }
  }
  store_partials(acc, partials, nbx);
}

// x += alpha phat (early exit on small s)
__global__ void k_update_x_half(Dims d, const double* sc, double* xu, double* xv, const double* phu,
                                const double* phv) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  const double alpha = sc[SC_ALPHA];
  if (u_int(d, j, i)) xu[q] += alpha * phu[q];
  if (v_int(d, j, i)) xv[q] += alpha * phv[q];
}

// p = r + beta (p - omega v)
__global__ void k_update_p(Dims d, const double* sc, const double* ru, const double* rv, const double* vu,
                           const double* vv, double* pu, double* pv) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  const double beta = sc[SC_BETA], omega = sc[SC_OMEGA];
  pu[q] = ru[q] + beta * (pu[q] - omega * vu[q]);
  pv[q] = rv[q] + beta * (pv[q] - omega * vv[q]);
}

// fixed-order reduction of block partials into sc[dst..dst+3], then the scalar step
enum { ST_INIT = 0, ST_ALPHA, ST_SNORM, ST_OMEGA, ST_RHO };
__global__ void k_reduce(const double* partials, int nblocks, double* sc, int stage) {
  __shared__ double sh[kPW][256];
  double s[kPW] = {0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int q = 0; q < kPW; ++q) s[q] += partials[kPW * b + q];
  for (int q = 0; q < kPW; ++q) sh[q][threadIdx.x] = s[q];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int q = 0; q < kPW; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double r0 = sh[0][0], r1 = sh[1][0];
  switch (stage) {
    case ST_INIT:   // [0] r.r, [1] b.b
      sc[SC_RNORM2] = r0; sc[SC_BNORM2] = r1; sc[SC_RHO] = r0; break;
    case ST_ALPHA:  // [0] rhat.v
      sc[SC_TMP0] = r0;
      sc[SC_ALPHA] = (r0 != 0.0) ? sc[SC_RHO] / r0 : 0.0; break;
    case ST_SNORM:  // [0] s.s
      sc[SC_SNORM2] = r0; break;
    case ST_OMEGA:  // [0] s.t, [2] t.t  (k_matvec with w1 = s)
      sc[SC_OMEGA] = (sh[2][0] != 0.0) ? r0 / sh[2][0] : 0.0; break;
    case ST_RHO: {  // [0] rhat.r, [1] r.r
      const double rho_new = r0;
      const double om = sc[SC_OMEGA], al = sc[SC_ALPHA], rho = sc[SC_RHO];
      sc[SC_BETA] = (rho != 0.0 && om != 0.0) ? (rho_new / rho) * (al / om) : 0.0;
      sc[SC_RHO] = rho_new;
      sc[SC_RNORM2] = r1;
      break;
    }
  }
}

// boundary unknowns = their sources (after a solve)
__global__ void k_fill_boundary(Dims d, BCs bc, double* xu, double* xv) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  Op o;
  o.d = d; o.bc = bc;
  const long long q = d.at(j, i);
  if (i < d.nx - 1 && !u_int(d, j, i)) xu[q] = LU(o, xu, j, i);
  if (j < d.ny - 1 && !v_int(d, j, i)) xv[q] = LV(o, xv, j, i);
}

// nonlinear residual over all rows of the reference matrix: interior rows
// b - A u, boundary rows -(u_b - u_src) (or -u_b for zero); partials [0] r.r, [1] b.b
__global__ void k_relres(Op o, const double* u, const double* v, const double* bu, const double* bv,
                         double* partials, int nbx) {
  IDX2D
  double acc[kPW] = {0.0, 0.0, 0.0, 0.0};
  if (j < o.d.ny && i < o.d.nx) {
    const long long q = o.d.at(j, i);
    if (i < o.d.nx - 1) {
      double r;
      if (u_int(o.d, j, i)) { r = bu[q] - Au<true>(o, u, v, j, i); acc[1] += bu[q] * bu[q]; }
      else r = LU(o, u, j, i) - u[q];
      acc[0] += r * r;
    }
    if (j < o.d.ny - 1) {
      double r;
      if (v_int(o.d, j, i)) { r = bv[q] - Av<true>(o, u, v, j, i); acc[1] += bv[q] * bv[q]; }
      else r = LV(o, v, j, i) - v[q];
      acc[0] += r * r;
    }
  }
  store_partials(acc, partials, nbx);
}

// ---- device-side control of a graph-launched viscosity iteration ------------------
// Single-thread kernels that finish a reduction and set the conditional-node
// handles, so the Krylov loop and the skip of a converged iteration are
// decided on the device without a host round trip.
__device__ __forceinline__ void sum_partials4(const double* partials, int nblocks, double (&out)[kPW]) {
  __shared__ double sh[kPW][256];
  double s[kPW] = {0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int q = 0; q < kPW; ++q) s[q] += partials[kPW * b + q];
  for (int q = 0; q < kPW; ++q) sh[q][threadIdx.x] = s[q];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int q = 0; q < kPW; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + o];
    __syncthreads();
  }
  for (int q = 0; q < kPW; ++q) out[q] = sh[q][0];
}

__global__ void k_ctl_begin(double* sc) {
  sc[SC_PIC_IT] += 1.0;
  sc[SC_EXIT_RELRES] = 0.0;
  sc[SC_LIN_IT] = 0.0;
  sc[SC_LIN_FULL] = 0.0;
  sc[SC_SOLVED] = 0.0;
  sc[SC_CONVERGED] = 0.0;
}

// nonlinear residual of the current iterate; skip the solve when it meets the tolerance
__global__ void k_ctl_relres(const double* partials, int nblocks, double* sc, cudaGraphConditionalHandle h_solve,
                             double tol, int stall_its) {
  double v[kPW];
  sum_partials4(partials, nblocks, v);
  if (threadIdx.x != 0) return;
  const double rr = v[0], bb = v[1];
  const double relres = bb > 0.0 ? sqrt(rr / bb) : sqrt(rr);
  sc[SC_RELRES] = relres;
  sc[SC_ETA] = eta_after(sc[SC_ETA], relres, sc[SC_RELRES_PREV], tol);
  sc[SC_RELRES_PREV] = relres;
  bool stop = false;
  if (!isfinite(relres)) { sc[SC_NAN] = 1.0; stop = true; }
  else if (relres <= tol) { sc[SC_EXIT_RELRES] = 1.0; stop = true; }
  else if (stall_after(relres, sc + SC_STALL_BEST, sc + SC_STALL_SINCE, stall_its)) {
    sc[SC_EXIT_RELRES] = 1.0;   // ends like a converged one (basal stress at this state), flagged
    sc[SC_STALLED] = 1.0;
    stop = true;
  }
  cudaGraphSetConditional(h_solve, stop ? 0u : 1u);
}

// initial Krylov residual and the target of this linear solve
__global__ void k_ctl_lin_init(const double* partials, int nblocks, double* sc, cudaGraphConditionalHandle h_while,
                               int adaptive, double lin_rtol, int maxit) {
  double v[kPW];
  sum_partials4(partials, nblocks, v);
  if (threadIdx.x != 0) return;
  const double rr = v[0], bb = v[1];
  sc[SC_RNORM2] = rr;
  sc[SC_BNORM2] = bb;
  sc[SC_RHO] = rr;
  double rtol = lin_rtol;
  if (adaptive) rtol = max_ref(lin_rtol, sc[SC_ETA] * min_ref(1.0, sc[SC_RELRES]));
  const double t = rtol * (bb > 0.0 ? sqrt(bb) : 1.0);
  sc[SC_TARGET2] = t * t;
  sc[SC_SOLVED] = 1.0;
  if (!isfinite(rr)) sc[SC_NAN] = 1.0;
  cudaGraphSetConditional(h_while, (isfinite(rr) && rr > t * t && maxit > 0) ? 1u : 0u);
}

// after s = r - alpha v: stop at the half step if |s| meets the target
__global__ void k_ctl_half(const double* partials, int nblocks, double* sc, cudaGraphConditionalHandle h_while,
                           cudaGraphConditionalHandle h_half) {
  double v[kPW];
  sum_partials4(partials, nblocks, v);
  if (threadIdx.x != 0) return;
  const double ss = v[0];
  sc[SC_SNORM2] = ss;
  sc[SC_LIN_IT] += 1.0;
  if (!isfinite(ss)) {
    sc[SC_NAN] = 1.0;
    sc[SC_HALFDONE] = 0.0;
    cudaGraphSetConditional(h_half, 0u);
    cudaGraphSetConditional(h_while, 0u);
  } else if (ss <= sc[SC_TARGET2]) {
    sc[SC_HALFDONE] = 1.0;
    sc[SC_RNORM2] = ss;
    cudaGraphSetConditional(h_half, 0u);
    cudaGraphSetConditional(h_while, 0u);
  } else {
    sc[SC_HALFDONE] = 0.0;
    cudaGraphSetConditional(h_half, 1u);
  }
}

__global__ void k_x_half_pred(Dims d, const double* sc, double* xu, double* xv, const double* phu, const double* phv) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  if (sc[SC_HALFDONE] == 0.0) return;
  const long long q = d.at(j, i);
  const double alpha = sc[SC_ALPHA];
  if (u_int(d, j, i)) xu[q] += alpha * phu[q];
  if (v_int(d, j, i)) xv[q] += alpha * phv[q];
}

// after the full step: rho, beta and the continue test
__global__ void k_ctl_full(const double* partials, int nblocks, double* sc, cudaGraphConditionalHandle h_while,
                           int maxit) {
  double v[kPW];
  sum_partials4(partials, nblocks, v);
  if (threadIdx.x != 0) return;
  const double rho_new = v[0], rr = v[1];
  const double om = sc[SC_OMEGA], al = sc[SC_ALPHA], rho = sc[SC_RHO];
  sc[SC_BETA] = (rho != 0.0 && om != 0.0) ? (rho_new / rho) * (al / om) : 0.0;
  sc[SC_RHO] = rho_new;
  sc[SC_RNORM2] = rr;
  sc[SC_LIN_FULL] += 1.0;
  const bool fin = isfinite(rr);
  if (!fin) sc[SC_NAN] = 1.0;
  cudaGraphSetConditional(h_while, (fin && rr > sc[SC_TARGET2] && sc[SC_LIN_IT] < (double)maxit) ? 1u : 0u);
}

__global__ void k_ctl_lin_finish(double* sc) {
  if (sc[SC_RNORM2] > sc[SC_TARGET2]) sc[SC_LIN_FAILED] += 1.0;
}

// ---- host side --------------------------------------------------------------------
Op op_of(const Ctx* c, int l) {
  Op o;
  o.d = c->lv[l].d;
  o.bc = c->bc;
  o.ax = c->lv[l].d.dx;   // placeholders, set below
  o.ay = 1.0;
  o.Na = c->lv[l].Na; o.Nb = c->lv[l].Nb; o.Bx = c->lv[l].Bx; o.By = c->lv[l].By;
  o.inv_dx = 1.0 / c->lv[l].d.dx;
  o.rtu = nullptr;
  o.rtv = nullptr;
  if (l == 0 && c->c.choice_ice_margin == DIVA_MARGIN_BC) {
    o.rtu = c->rtu;
    o.rtv = c->rtv;
  }
  return o;
}

}  // namespace

// per-level cell aspect ratio (hy/hx): kept in Level via d.dx (hx) and a side table
static double level_ax(const Ctx* c, int l) {
  double hx = c->d.dx, hy = c->d.dx;
  for (int q = 1; q <= l; ++q) {
    if (c->lv[q].d.nx != c->lv[q - 1].d.nx) hx *= 2.0;
    if (c->lv[q].d.ny != c->lv[q - 1].d.ny) hy *= 2.0;
  }
  return hy / hx;
}
static Op make_op(const Ctx* c, int l) {
  Op o = op_of(c, l);
  o.ax = level_ax(c, l);
  o.ay = 1.0 / o.ax;
  return o;
}
// The finest level of the mixed-precision preconditioner (DIVA_PREC_MIXED): its smoother runs
// in float on float copies of the coefficients and inverse diagonals (written by the
// finest level's set-up), with the pre-smoothed x and the residual stored as float in
// the level's tu/tv and ru/rv planes.  Everything else stays double.
static int sub_first_level(const Ctx* c);
static bool level_fp32(const Ctx* c, int l) {
  return c->c.precision == DIVA_PREC_MIXED && c->tiled && l < sub_first_level(c);
}
static OpT<float> make_op32(const Ctx* c, int l) {
  const Op o = make_op(c, l);
  OpT<float> f;
  f.d = o.d; f.bc = o.bc; f.ax = o.ax; f.ay = o.ay; f.inv_dx = o.inv_dx; f.rtu = o.rtu; f.rtv = o.rtv;
  f.Na = c->f32[l][F32_NA]; f.Nb = c->f32[l][F32_NB]; f.Bx = c->f32[l][F32_BX]; f.By = c->f32[l][F32_BY];
  return f;
}

static void factors(const Ctx* c, int l, int* fx, int* fy) {
  *fx = (c->lv[l + 1].d.nx != c->lv[l].d.nx) ? 2 : 1;
  *fy = (c->lv[l + 1].d.ny != c->lv[l].d.ny) ? 2 : 1;
}

#define GL(l) grid2d(c->lv[l].d.ny, c->lv[l].d.nx), block2d(), 0, c->stream

static CoarseMap coarse_map(const Ctx* c) {
  const Dims& d = c->lv[c->nlev - 1].d;
  CoarseMap m;
  m.ny = d.ny;
  m.nu = (d.nx > 3 && d.ny > 2) ? (d.nx - 3) * (d.ny - 2) : 0;
  m.nv = (d.nx > 2 && d.ny > 3) ? (d.nx - 2) * (d.ny - 3) : 0;
  return m;
}

static int coarse_direct_n(const Ctx* c) {
  const int n = coarse_map(c).n();
  return n > 0 && n <= kCoarseDirectMax ? n : 0;
}

static int sub_first_level(const Ctx* c);

int solver_setup(Ctx* c, int inv_when) {
  const diva_config_t& C = c->c;
  // the 'BC' front rows live on the finest level only; a grid too small to coarsen
  // would hand that level to the coarse direct solve, whose matrix has no front rows
  if (C.choice_ice_margin == DIVA_MARGIN_BC && c->nlev < 2)
    return set_error(c, DIVA_UNSUPPORTED, "choice_ice_margin 'BC' needs nx or ny of at least 9");
  if (C.precision == DIVA_PREC_MIXED && (c->nlev < 2 || !c->tiled))
    return set_error(c, DIVA_UNSUPPORTED,
                     "precision 'mixed' needs the tiled smoother (no periodic boundary, DIVA_NO_TILES unset) and nx or ny >= 9");
  // level l's diagonal and level l+1's coefficients in one launch; the finest level's
  // launch also forms the right-hand side, so it always runs on its own
  const int first_small = sub_first_level(c) > 1 ? sub_first_level(c) : 1;
  for (int l = 0; l < first_small && l < c->nlev; ++l) {
    const Level& F = c->lv[l];
    const bool coarsen = l + 1 < c->nlev;
    const Level& K = c->lv[coarsen ? l + 1 : l];
    int fx = 1, fy = 1;
    if (coarsen) factors(c, l, &fx, &fy);
    RhsArgs rhs{};
    if (l == 0) {
      rhs.on = 1;
      rhs.crossterms = C.include_SSADIVA_crossterms;
      rhs.tdx = c->D(DIVA_F_TAUDX_CX); rhs.tdy = c->D(DIVA_F_TAUDY_CY);
      rhs.Ncx = c->D(DIVA_F_N_CX); rhs.Ncy = c->D(DIVA_F_N_CY);
      rhs.bu = c->kv[KV_B][0]; rhs.bv = c->kv[KV_B][1];
      if (C.choice_ice_margin == DIVA_MARGIN_BC) {
        rhs.rtu = c->rtu; rhs.rtv = c->rtv;
        rhs.Hi = c->D(DIVA_F_HI_A); rhs.SL = c->D(DIVA_F_SL_A); rhs.Hb = c->D(DIVA_F_HB_A);
      }
    }
    F32Out f32{};
    if (level_fp32(c, l)) {
      float* const* f = c->f32[l];
      f32.Na = f[F32_NA]; f32.Nb = f[F32_NB]; f32.Bx = f[F32_BX]; f32.By = f[F32_BY];
      f32.idu = f[F32_IDU]; f32.idv = f[F32_IDV];
    }
    k_level_setup<<<GL(l)>>>(make_op(c, l), coarsen ? 1 : 0, K.d, fx, fy, K.Na, K.Nb, K.Bx, K.By, F.idu, F.idv,
                             rhs, f32); c->launches++;
    DIVA_LAUNCHED(c, "k_level_setup");
  }
  const CoarseMap m = coarse_map(c);
  c->coarse_n = m.nu + m.nv;
  c->coarse_direct = c->coarse_n > 0 && c->coarse_n <= kCoarseDirectMax;
  SmallSetup a;
  a.first = first_small;
  a.last = c->nlev - 1;
  a.direct = c->coarse_direct ? 1 : 0;
  a.map = m;
  a.tab = c->sub_tab + c->sub_tab_off[c->nlev - 1];
  a.Ainv = c->coarse_inv;
  a.singular = c->coarse_singular;
  a.inv_when = inv_when;
  a.sc = c->scal;
  for (int l = a.first < a.last ? a.first : a.last; l <= a.last; ++l) {   // (first > last on a one-level grid)
    a.o[l] = make_op(c, l);
    a.idu[l] = c->lv[l].idu;
    a.idv[l] = c->lv[l].idv;
    a.fx[l] = a.fy[l] = 1;
    if (l < a.last) factors(c, l, &a.fx[l], &a.fy[l]);
  }
  k_small_setup<<<1, kInvThreads, kInvSmem, c->stream>>>(a); c->launches++;
  DIVA_LAUNCHED(c, "k_small_setup");
  return DIVA_OK;
}

static int gs_sweep(Ctx* c, int l, double* xu, double* xv, const double* bu, const double* bv, bool forward) {
  const Op o = make_op(c, l);
  const Level& L = c->lv[l];
  dim3 g = grid2d((L.d.ny + 1) / 2, L.d.nx);
  for (int p = 0; p < 4; ++p) {
    const int pp = forward ? p : 3 - p;
    k_gs<<<g, block2d(), 0, c->stream>>>(o, xu, xv, bu, bv, L.idu, L.idv, pp >> 1, pp & 1); c->launches++;
  }
  DIVA_LAUNCHED(c, "k_gs");
  c->fine_passes += (double)L.d.plane / (double)c->d.plane;
  return DIVA_OK;
}

// interior rows (u then v) of a level
static int level_rows(const Dims& d) {
  const int nu = (d.nx > 3 && d.ny > 2) ? (d.nx - 3) * (d.ny - 2) : 0;
  const int nv = (d.nx > 2 && d.ny > 3) ? (d.nx - 2) * (d.ny - 3) : 0;
  return nu + nv;
}

// shared memory the sub-cycle needs from level l down: the planes, then the row tables
static size_t sub_dbl(const Ctx* c, int l) {
  size_t n = 0;
  for (int q = l; q < c->nlev; ++q) n += (size_t)kSubArrays * ((size_t)c->lv[q].d.nx * c->lv[q].d.ny + 1);
  return n;
}
// entries of one level's row table, padded to 8 (16 bytes) so that every level's table
// starts 16-byte aligned and the sub-cycle copies the tables as 16-byte vectors
static size_t level_tab_entries(const Dims& d) { return ((size_t)(kTabCols + kTabProlong) * level_rows(d) + 7) / 8 * 8; }
static size_t sub_tab_entries(const Ctx* c, int l) {
  size_t n = 0;
  for (int q = l; q < c->nlev; ++q) n += level_tab_entries(c->lv[q].d);
  return n;
}
// the coarsest level's unknowns when it is solved with its inverse, else 0
static int coarse_direct_n(const Ctx* c);
// doubles of the sub-cycle's table area (16-byte aligned), between the planes and the inverse
static size_t sub_tab_dbl(const Ctx* c, int l) { return ((sub_tab_entries(c, l) * sizeof(uint16_t) + 15) / 16) * 2; }
// dynamic shared memory of the sub-cycle from level l: planes, row tables, the inverse
static size_t sub_bytes(const Ctx* c, int l) {
  const size_t n = (size_t)coarse_direct_n(c);
  return (sub_dbl(c, l) + sub_tab_dbl(c, l) + n * n) * sizeof(double);
}

// the largest level whose levels all fit in the sub-cycle's shared memory (the row
// tables are built from there down, whatever the configuration)
static int sub_first_fit(const Ctx* c) {
  for (int l = 0; l < c->nlev; ++l)
    if (sub_bytes(c, l) <= kSubSmemBudget) return l;
  return c->nlev - 1;
}
// first level of the one-block sub-cycle
static int sub_first_level(const Ctx* c) {
  // the finest level's 'BC' front rows are not in the sub-cycle's row tables, and a
  // mixed-precision finest level is smoothed by the float tile kernels
  const bool own0 = c->c.choice_ice_margin == DIVA_MARGIN_BC || (c->c.precision == DIVA_PREC_MIXED && c->tiled);
  const int l0 = (own0 && c->nlev > 1) ? 1 : 0;
  const int f = sub_first_fit(c);
  return f > l0 ? f : l0;
}

static int vcycle(Ctx* c, int l, double* xu, double* xv, const double* bu, const double* bv,
                  const Restriction& rs);

// tile edge of level l's smoothing kernels: 32 x 32 while that still fills the GPU, else
// 16 x 16, unless the caller chose one (diva_set_tile_edges, e.g. from an autotuner)
static int tile_edge(const Ctx* c, int l) {
  if (c->tile_override[l] == 16 || c->tile_override[l] == 32) return c->tile_override[l];
  const Dims& d = c->lv[l].d;
  const long long b32 = (long long)((d.ny + 31) / 32) * ((d.nx + 31) / 32);
  return b32 >= 148 ? 32 : 16;
}
constexpr int kSMs = 148;   // B200
// Whether level l's tiles are 1.5x wider along i (T x 3T/2): when square tiles give a little
// more than one block per SM (e.g. 198 on the 321 x 561 ice cap's finest level, where 50 SMs
// would run two blocks each and set the kernel's length) and the wider ones fit in one
// block per SM, with less halo per point.  Not when the caller chose the edge.
static bool tile_wide(const Ctx* c, int l) {
  if (c->tile_override[l] == 16 || c->tile_override[l] == 32) return false;
  const Dims& d = c->lv[l].d;
  const int T = tile_edge(c, l), W = 3 * T / 2;
  const long long sq = (long long)((d.ny + T - 1) / T) * ((d.nx + T - 1) / T);
  const long long wide = (long long)((d.ny + T - 1) / T) * ((d.nx + W - 1) / W);
  return sq > kSMs && wide <= kSMs;
}

// Which tile kernels a level uses: the edge (tile_edge), and whether the region's
// coefficients are staged in shared memory (16 x 16 tiles: 92 KB, two blocks per SM;
// 32 x 32 tiles would need 200 KB, one block per SM, so they read the coefficients
// from L2 instead).
constexpr bool kStage16 = true, kStage32 = false;

// H: the tile's halo, 4 nu + 1 for nu sweeps per phase (halo_for); tiles of TJ rows (j)
// by TI columns (i)
template <int TJ, int TI, bool S, class R, int H>
static void tile_down_h(Ctx* c, int l, const OpT<R>& o, const R* idu, const R* idv, const Restriction& rs,
                        const double* bu, const double* bv, int nu) {
  const Level& L = c->lv[l];
  const dim3 grid((L.d.ny + TJ - 1) / TJ, (L.d.nx + TI - 1) / TI);
  // b is written only when it is restricted here (rs.on), which never happens on the finest level
  auto kern = o.rtu ? k_smooth_down<TJ, TI, S, true, R, H> : k_smooth_down<TJ, TI, S, false, R, H>;
  kern<<<grid, kTileThreads, TileGeom<TJ, TI, S, R, H>::smem, c->stream>>>(
      o, rs, const_cast<double*>(bu), const_cast<double*>(bv), reinterpret_cast<R*>(L.tu),
      reinterpret_cast<R*>(L.tv), reinterpret_cast<R*>(L.ru), reinterpret_cast<R*>(L.rv), idu, idv, nu);
  c->launches++;
}
template <int TJ, int TI, bool S, class R, int H>
static void tile_up_h(Ctx* c, int l, const OpT<R>& o, const R* idu, const R* idv, int fx, int fy, const double* bu,
                      const double* bv, double* xu, double* xv, int nu) {
  const Level& L = c->lv[l];
  const Level& K = c->lv[l + 1];
  const dim3 grid((L.d.ny + TJ - 1) / TJ, (L.d.nx + TI - 1) / TI);
  auto kern = o.rtu ? k_smooth_up<TJ, TI, S, true, R, H> : k_smooth_up<TJ, TI, S, false, R, H>;
  kern<<<grid, kTileThreads, TileGeom<TJ, TI, S, R, H>::smem_up, c->stream>>>(
      o, make_op(c, l + 1), fx, fy, K.xu, K.xv, bu, bv, reinterpret_cast<const R*>(L.tu),
      reinterpret_cast<const R*>(L.tv), xu, xv, idu, idv, nu);
  c->launches++;
}
template <int TJ, int TI, bool S, class R>
static void tile_down_r(Ctx* c, int l, const OpT<R>& o, const R* idu, const R* idv, const Restriction& rs,
                        const double* bu, const double* bv, int nu) {
  if (halo_for(nu) == kHaloOne) tile_down_h<TJ, TI, S, R, kHaloOne>(c, l, o, idu, idv, rs, bu, bv, nu);
  else tile_down_h<TJ, TI, S, R, kHalo>(c, l, o, idu, idv, rs, bu, bv, nu);
}
template <int TJ, int TI, bool S, class R>
static void tile_up_r(Ctx* c, int l, const OpT<R>& o, const R* idu, const R* idv, int fx, int fy, const double* bu,
                      const double* bv, double* xu, double* xv, int nu) {
  if (halo_for(nu) == kHaloOne) tile_up_h<TJ, TI, S, R, kHaloOne>(c, l, o, idu, idv, fx, fy, bu, bv, xu, xv, nu);
  else tile_up_h<TJ, TI, S, R, kHalo>(c, l, o, idu, idv, fx, fy, bu, bv, xu, xv, nu);
}
static int tile_down(Ctx* c, int l, const Restriction& rs, const double* bu, const double* bv, double* xu,
                     double* xv, int nu) {
  const Level& L = c->lv[l];
  const int T = tile_edge(c, l);
  const bool W = tile_wide(c, l);
  if (level_fp32(c, l)) {   // float tiles stage their coefficients at every shape (100 KB at 32 x 32)
    const OpT<float> o = make_op32(c, l);
    const float *iu = c->f32[l][F32_IDU], *iv = c->f32[l][F32_IDV];
    if (T == 32) W ? tile_down_r<32, 48, true>(c, l, o, iu, iv, rs, bu, bv, nu) : tile_down_r<32, 32, true>(c, l, o, iu, iv, rs, bu, bv, nu);
    else W ? tile_down_r<16, 24, true>(c, l, o, iu, iv, rs, bu, bv, nu) : tile_down_r<16, 16, true>(c, l, o, iu, iv, rs, bu, bv, nu);
  } else {
    const Op o = make_op(c, l);
    const double *iu = L.idu, *iv = L.idv;
    if (T == 32) W ? tile_down_r<32, 48, kStage32>(c, l, o, iu, iv, rs, bu, bv, nu) : tile_down_r<32, 32, kStage32>(c, l, o, iu, iv, rs, bu, bv, nu);
    else W ? tile_down_r<16, 24, kStage16>(c, l, o, iu, iv, rs, bu, bv, nu) : tile_down_r<16, 16, kStage16>(c, l, o, iu, iv, rs, bu, bv, nu);
  }
  DIVA_LAUNCHED(c, "k_smooth_down");
  return DIVA_OK;
}
static int tile_up(Ctx* c, int l, int fx, int fy, const double* bu, const double* bv, double* xu, double* xv,
                   int nu) {
  const Level& L = c->lv[l];
  const int T = tile_edge(c, l);
  const bool W = tile_wide(c, l);
  if (level_fp32(c, l)) {
    const OpT<float> o = make_op32(c, l);
    const float *iu = c->f32[l][F32_IDU], *iv = c->f32[l][F32_IDV];
    if (T == 32) W ? tile_up_r<32, 48, true>(c, l, o, iu, iv, fx, fy, bu, bv, xu, xv, nu) : tile_up_r<32, 32, true>(c, l, o, iu, iv, fx, fy, bu, bv, xu, xv, nu);
    else W ? tile_up_r<16, 24, true>(c, l, o, iu, iv, fx, fy, bu, bv, xu, xv, nu) : tile_up_r<16, 16, true>(c, l, o, iu, iv, fx, fy, bu, bv, xu, xv, nu);
  } else {
    const Op o = make_op(c, l);
    const double *iu = L.idu, *iv = L.idv;
    if (T == 32) W ? tile_up_r<32, 48, kStage32>(c, l, o, iu, iv, fx, fy, bu, bv, xu, xv, nu) : tile_up_r<32, 32, kStage32>(c, l, o, iu, iv, fx, fy, bu, bv, xu, xv, nu);
    else W ? tile_up_r<16, 24, kStage16>(c, l, o, iu, iv, fx, fy, bu, bv, xu, xv, nu) : tile_up_r<16, 16, kStage16>(c, l, o, iu, iv, fx, fy, bu, bv, xu, xv, nu);
  }
  DIVA_LAUNCHED(c, "k_smooth_up");
  return DIVA_OK;
}

// V-cycle step of a tiled level: 2 launches for the smoothing, the residual and the
// restriction instead of 4 per sweep and 2 more
static int vcycle_tiled(Ctx* c, int l, double* xu, double* xv, const double* bu, const double* bv,
                        const Restriction& rs, int nu1, int nu2) {
  if (4 * nu1 > halo_for(nu1) - 1 || 4 * nu2 > halo_for(nu2) - 1)
    return set_error(c, DIVA_UNSUPPORTED, "tiled smoothing depth");
  const Level& L = c->lv[l];
  const Level& K = c->lv[l + 1];
  int st = tile_down(c, l, rs, bu, bv, xu, xv, nu1);
  if (st) return st;
  Restriction next{};
  next.on = 1;
  next.df = L.d;
  factors(c, l, &next.fx, &next.fy);
  next.ru = L.ru;
  next.rv = L.rv;
  next.rfloat = level_fp32(c, l) ? 1 : 0;   // the float residual of a mixed-precision level
  if ((st = vcycle(c, l + 1, K.xu, K.xv, K.bu, K.bv, next))) return st;
  if ((st = tile_up(c, l, next.fx, next.fy, bu, bv, xu, xv, nu2))) return st;
  c->fine_passes += (nu1 + nu2 + 1) * (double)L.d.plane / (double)c->d.plane;
  return DIVA_OK;
}

// Shared-memory limits of the tiled kernels (the 32 x 32 tiles need 80 KB) and of
// the sub-cycle, and whether the grid's boundary conditions allow tiles at all.
// Row tables of the sub-cycle levels (see k_subcycle), built on the host from the
// level sizes and the boundary conditions and copied to the context's table area.
static int build_sub_tables(Ctx* c) {
  const int first = sub_first_fit(c);
  std::vector<uint16_t> tab(sub_tab_entries(c, first));
  size_t off = 0;
  for (int l = first; l < c->nlev; ++l) {
    Dims d = c->lv[l].d;
    d.ld = d.ny;   // compact planes in shared memory
    const int P = d.nx * d.ny, R = level_rows(d);
    if (P >= 65535) return set_error(c, DIVA_UNSUPPORTED, "sub-cycle level too large for 16-bit row tables");
    c->sub_tab_off[l] = off;
    int r = 0;
    auto put = [&](int j, int i, bool urow) {
      const int js_[4] = {urow ? j : j + 1, urow ? j : j - 1, urow ? j + 1 : j, urow ? j - 1 : j};
      const int is_[4] = {urow ? i + 1 : i, urow ? i - 1 : i, urow ? i : i + 1, urow ? i : i - 1};
      const int jc_[4] = {urow ? j : j + 1, urow ? j : j + 1, urow ? j - 1 : j, urow ? j - 1 : j};
      const int ic_[4] = {urow ? i : i - 1, urow ? i + 1 : i, urow ? i : i - 1, urow ? i + 1 : i};
      tab[off + r] = (uint16_t)d.at(j, i);
      for (int k = 0; k < 4; ++k) {   // same-component neighbours, then the cross-coupled reads
        int js, is;
        const bool on = urow ? u_src(d, c->bc, js_[k], is_[k], js, is) : v_src(d, c->bc, js_[k], is_[k], js, is);
        tab[off + (size_t)(1 + k) * R + r] = on ? (uint16_t)d.at(js, is) : (uint16_t)P;
        const bool on2 = urow ? v_src(d, c->bc, jc_[k], ic_[k], js, is) : u_src(d, c->bc, jc_[k], ic_[k], js, is);
        tab[off + (size_t)(5 + k) * R + r] = on2 ? (uint16_t)d.at(js, is) : (uint16_t)P;
      }
      // the prolongation taps of the row from the next level (prolong_delta's taps in its
      // order, each clamped and read through the coarse level's boundary mapping; the
      // coarse plane's zero element for a 'zero' side or a tap the row does not have)
      if (l + 1 < c->nlev) {
        Dims dc = c->lv[l + 1].d;
        dc.ld = dc.ny;
        const int Pc = dc.nx * dc.ny;
        int fx, fy;
        factors(c, l, &fx, &fy);
        int k = 0, js, is, Cj, Ci;
        double w;
        auto clampi = [](int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); };
        if (urow) {
          for (int a = 0; a < scatter_node_n(j, fy); ++a)
            for (int b = 0; b < scatter_cell_n(i, fx); ++b, ++k) {
              scatter_node(j, fy, a, Cj, w);
              scatter_cell(i, fx, b, Ci, w);
              const bool on = u_src(dc, c->bc, clampi(Cj, 0, dc.ny - 1), clampi(Ci, 0, dc.nx - 2), js, is);
              tab[off + (size_t)(kTabCols + k) * R + r] = on ? (uint16_t)dc.at(js, is) : (uint16_t)Pc;
            }
        } else {
          for (int a = 0; a < scatter_cell_n(j, fy); ++a)
            for (int b = 0; b < scatter_node_n(i, fx); ++b, ++k) {
              scatter_cell(j, fy, a, Cj, w);
              scatter_node(i, fx, b, Ci, w);
              const bool on = v_src(dc, c->bc, clampi(Cj, 0, dc.ny - 2), clampi(Ci, 0, dc.nx - 1), js, is);
              tab[off + (size_t)(kTabCols + k) * R + r] = on ? (uint16_t)dc.at(js, is) : (uint16_t)Pc;
            }
        }
        for (; k < kTabProlong; ++k) tab[off + (size_t)(kTabCols + k) * R + r] = (uint16_t)Pc;
      }
      ++r;
    };
    for (int p = 0; p < 4; ++p) {
      c->sub_cls[l][p] = r;
      const bool urow = p < 2;
      for (int i = 0; i < d.nx; ++i)
        for (int j = 0; j < d.ny; ++j)
          if (((i + j) & 1) == (p & 1) && (urow ? u_int(d, j, i) : v_int(d, j, i))) put(j, i, urow);
    }
    c->sub_cls[l][4] = r;
    if (r != R) return set_error(c, DIVA_CUDA_ERROR, "sub-cycle row table size");
    off += level_tab_entries(c->lv[l].d);
  }
  if (!tab.empty())
    DIVA_CUDA(c, cudaMemcpy(c->sub_tab, tab.data(), tab.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
  return DIVA_OK;
}

size_t solver_table_entries(const Ctx* c) { return sub_tab_entries(c, sub_first_fit(c)); }

// dynamic shared memory of the four tile kernels (down/up, with/without front rows) of one shape
template <int TJ, int TI, bool S, class R, int H>
static int tile_attrs(Ctx* c) {
  using G = TileGeom<TJ, TI, S, R, H>;
  const void* k[4] = {(const void*)k_smooth_down<TJ, TI, S, false, R, H>, (const void*)k_smooth_down<TJ, TI, S, true, R, H>,
                      (const void*)k_smooth_up<TJ, TI, S, false, R, H>, (const void*)k_smooth_up<TJ, TI, S, true, R, H>};
  for (int q = 0; q < 4; ++q)   // the up kernels (2, 3) also stage the coarse correction
    DIVA_CUDA(c, cudaFuncSetAttribute(k[q], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(q < 2 ? G::smem : G::smem_up)));
  return DIVA_OK;
}
// every tile shape (square, and 1.5x wider along i) of both edges, both types, both halos
template <int TJ, int TI>
static int tile_attrs_shape(Ctx* c) {
  constexpr bool S = TJ == 16 ? kStage16 : kStage32;
  if (int st = tile_attrs<TJ, TI, S, double, kHalo>(c)) return st;
  if (int st = tile_attrs<TJ, TI, true, float, kHalo>(c)) return st;
  if (int st = tile_attrs<TJ, TI, S, double, kHaloOne>(c)) return st;
  if (int st = tile_attrs<TJ, TI, true, float, kHaloOne>(c)) return st;
  return DIVA_OK;
}

int solver_init(Ctx* c) {
  if (sub_bytes(c, c->nlev - 1) > kSubSmemBudget)
    return set_error(c, DIVA_UNSUPPORTED, "coarsest multigrid level too large for the one-block sub-cycle");
  if (int st = build_sub_tables(c)) return st;
  DIVA_CUDA(c, cudaFuncSetAttribute(k_small_setup, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInvSmem));
  DIVA_CUDA(c, cudaFuncSetAttribute(k_subcycle, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kSubSmemBudget));
  if (int st = tile_attrs_shape<32, 32>(c)) return st;
  if (int st = tile_attrs_shape<16, 16>(c)) return st;
  if (int st = tile_attrs_shape<32, 48>(c)) return st;
  if (int st = tile_attrs_shape<16, 24>(c)) return st;
  const BCs& b = c->bc;
  const int all[8] = {b.uW, b.uE, b.uS, b.uN, b.vW, b.vE, b.vS, b.vN};
  bool periodic = false;
  for (int q = 0; q < 8; ++q) periodic = periodic || all[q] == DIVA_BC_PERIODIC;
  c->tiled = !periodic && !c->tiles_disabled;
  return DIVA_OK;
}

// One V-cycle from level l down, entered with x = 0.  b is given in bu/bv, or (rs.on)
// restricted from the finer level's residual by the level's first kernel.
// Gauss-Seidel sweeps before and after the coarse correction.  The finest level and every
// coarser level of at least DIVA_MG_NU2_POINTS points take two (V(2,2)); smaller levels,
// whose kernels are bound by the latency of their barrier-separated colour passes rather
// than by their points, take one (V(1,1)), and so does the one-block sub-cycle.  Measured
// on one B200, solves to rel-res 1e-6: on the 321 x 561 ice cap one sweep below the finest
// level keeps the V-cycle count of V(2,2) everywhere (79 relaxed, 43 with Anderson mixing)
// at 8-13 % less time per solve; on the 1501 x 1501 sheet one sweep on its large coarse
// levels (751 x 751, 376 x 376) doubled the V-cycles per viscosity iteration.
#ifndef DIVA_MG_NU2_POINTS
#define DIVA_MG_NU2_POINTS 100000
#endif
static int level_nu(const Ctx* c, int l) {
  return (l == 0 || (long long)c->lv[l].d.nx * c->lv[l].d.ny >= DIVA_MG_NU2_POINTS) ? 2 : 1;
}
static int vcycle(Ctx* c, int l, double* xu, double* xv, const double* bu, const double* bv,
                  const Restriction& rs) {
  const int nu1 = level_nu(c, l), nu2 = nu1, coarse_sweeps = 64;
  if (l == sub_first_level(c)) {
    SubCycle sc;
    sc.first = l;
    sc.last = c->nlev - 1;
    sc.nu1 = nu1;
    sc.nu2 = nu2;
    sc.coarse_sweeps = coarse_sweeps;
    sc.direct = c->coarse_direct ? 1 : 0;
    sc.map = coarse_map(c);
    sc.Ainv = c->coarse_inv;
    sc.singular = c->coarse_singular;
    int soff = 0, toff = 0;
    for (int q = l; q < c->nlev; ++q) {
      const Level& L = c->lv[q];
      SubLevel& S = sc.L[q];
      S.o = make_op(c, q);
      S.idu = L.idu; S.idv = L.idv;
      S.fx = 1; S.fy = 1;
      if (q + 1 < c->nlev) factors(c, q, &S.fx, &S.fy);
      S.soff = soff;
      soff += kSubArrays * (L.d.nx * L.d.ny + 1);
      S.rows = level_rows(L.d);
      for (int k = 0; k < 5; ++k) S.cls[k] = c->sub_cls[q][k];
      S.toff = toff;
      S.gtab = c->sub_tab + c->sub_tab_off[q];
      toff += (int)level_tab_entries(L.d);
    }
    sc.dbl = soff;
    sc.ainv_off = soff + (int)sub_tab_dbl(c, l);
    sc.tab16 = toff / 8;
    sc.rs = rs;
    k_subcycle<<<1, kSubThreads, sub_bytes(c, l), c->stream>>>(sc, xu, xv, bu, bv); c->launches++;
    DIVA_LAUNCHED(c, "k_subcycle");
    for (int q = l; q < c->nlev; ++q) c->fine_passes += 8.0 * (double)c->lv[q].d.plane / (double)c->d.plane;
    return DIVA_OK;
  }
  if (l == c->nlev - 1) {
    k_coarse_solve<<<1, 256, 0, c->stream>>>(make_op(c, l), xu, xv, bu, bv, c->lv[l].idu, c->lv[l].idv,
                                             coarse_sweeps); c->launches++;
    DIVA_LAUNCHED(c, "k_coarse_solve");
    return DIVA_OK;
  }
  const Level& L = c->lv[l];
  const Level& K = c->lv[l + 1];
  int st;
  if (c->tiled) return vcycle_tiled(c, l, xu, xv, bu, bv, rs, nu1, nu2);
  for (int s = 0; s < nu1; ++s)
    if ((st = gs_sweep(c, l, xu, xv, bu, bv, true))) return st;
  k_residual<<<GL(l)>>>(make_op(c, l), xu, xv, bu, bv, L.ru, L.rv); c->launches++;
  DIVA_LAUNCHED(c, "k_residual");
  int fx, fy;
  factors(c, l, &fx, &fy);
  k_restrict<<<GL(l + 1)>>>(L.d, K.d, fx, fy, L.ru, L.rv, K.bu, K.bv, K.xu, K.xv); c->launches++;
  DIVA_LAUNCHED(c, "k_restrict");
  if ((st = vcycle(c, l + 1, K.xu, K.xv, K.bu, K.bv, Restriction{}))) return st;
  k_prolong<<<GL(l)>>>(make_op(c, l + 1), L.d, fx, fy, K.xu, K.xv, xu, xv); c->launches++;
  DIVA_LAUNCHED(c, "k_prolong");
  for (int s = 0; s < nu2; ++s)
    if ((st = gs_sweep(c, l, xu, xv, bu, bv, false))) return st;
  return DIVA_OK;
}

// z = M^{-1} r: one V-cycle from zero
static int precond(Ctx* c, const double* ru, const double* rv, double* zu, double* zv) {
  // the tiled kernels and the sub-cycle start from x = 0 themselves and write every
  // point of z; the per-colour sweeps read x
  if (!c->tiled && sub_first_level(c) > 0) {
    DIVA_CUDA(c, cudaMemsetAsync(zu, 0, sizeof(double) * c->d.plane, c->stream));
    DIVA_CUDA(c, cudaMemsetAsync(zv, 0, sizeof(double) * c->d.plane, c->stream));
  }
  c->mg_cycles++;
  return vcycle(c, 0, zu, zv, ru, rv, Restriction{});
}

static int read_scalars(Ctx* c) {
  DIVA_CUDA(c, cudaMemcpyAsync(c->h_scal, c->scal, sizeof(double) * SC_COUNT, cudaMemcpyDeviceToHost, c->stream));
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int solver_solve(Ctx* c, const double* u0, const double* v0, double rtol, int maxit, int* iters, double* relres0) {
  const Dims d = c->d;
  const Op o = make_op(c, 0);
  auto U_ = [&](int k) { return c->kv[k][0]; };
  auto V_ = [&](int k) { return c->kv[k][1]; };
  dim3 g = grid2d(d.ny, d.nx);
  const int nb = g.x * g.y;
  DIVA_CUDA(c, cudaMemcpyAsync(U_(KV_X), u0, sizeof(double) * d.plane, cudaMemcpyDeviceToDevice, c->stream));
  DIVA_CUDA(c, cudaMemcpyAsync(V_(KV_X), v0, sizeof(double) * d.plane, cudaMemcpyDeviceToDevice, c->stream));
  k_init_residual<<<g, block2d(), 0, c->stream>>>(o, U_(KV_X), V_(KV_X), U_(KV_B), V_(KV_B), U_(KV_R), V_(KV_R),
                                                  U_(KV_RHAT), V_(KV_RHAT), U_(KV_P), V_(KV_P), c->partials, g.x); c->launches++;
  k_reduce<<<1, 256, 0, c->stream>>>(c->partials, nb, c->scal, ST_INIT); c->launches++;
  DIVA_LAUNCHED(c, "k_init_residual");
  c->fine_passes += 1.0;
  int st = read_scalars(c);
  if (st) return st;
  const double bnorm = sqrt(c->h_scal[SC_BNORM2]);
  double rnorm = sqrt(c->h_scal[SC_RNORM2]);
  if (relres0) *relres0 = bnorm > 0.0 ? rnorm / bnorm : rnorm;
  const double target = rtol * (bnorm > 0.0 ? bnorm : 1.0);
  int it = 0;
  bool done = rnorm <= target;
  while (!done && it < maxit) {
    ++it;
    if ((st = precond(c, U_(KV_P), V_(KV_P), U_(KV_PHAT), V_(KV_PHAT)))) return st;
    k_matvec<<<g, block2d(), 0, c->stream>>>(o, U_(KV_PHAT), V_(KV_PHAT), U_(KV_V), V_(KV_V), U_(KV_RHAT),
                                             V_(KV_RHAT), nullptr, nullptr, c->partials, g.x); c->launches++;
    k_reduce<<<1, 256, 0, c->stream>>>(c->partials, nb, c->scal, ST_ALPHA); c->launches++;
    k_update_s<<<g, block2d(), 0, c->stream>>>(d, c->scal, U_(KV_R), V_(KV_R), U_(KV_V), V_(KV_V), U_(KV_S),
                                               V_(KV_S), c->partials, g.x); c->launches++;
    k_reduce<<<1, 256, 0, c->stream>>>(c->partials, nb, c->scal, ST_SNORM); c->launches++;
    DIVA_LAUNCHED(c, "bicgstab half step");
    if ((st = read_scalars(c))) return st;
    if (sqrt(c->h_scal[SC_SNORM2]) <= target) {
      k_update_x_half<<<g, block2d(), 0, c->stream>>>(d, c->scal, U_(KV_X), V_(KV_X), U_(KV_PHAT), V_(KV_PHAT)); c->launches++;
      DIVA_LAUNCHED(c, "k_update_x_half");
      rnorm = sqrt(c->h_scal[SC_SNORM2]);
      done = true;
      break;
    }
    if ((st = precond(c, U_(KV_S), V_(KV_S), U_(KV_SHAT), V_(KV_SHAT)))) return st;
    k_matvec<<<g, block2d(), 0, c->stream>>>(o, U_(KV_SHAT), V_(KV_SHAT), U_(KV_T), V_(KV_T), U_(KV_S), V_(KV_S),
                                             nullptr, nullptr, c->partials, g.x); c->launches++;
    k_reduce<<<1, 256, 0, c->stream>>>(c->partials, nb, c->scal, ST_OMEGA); c->launches++;
    k_update_xr<<<g, block2d(), 0, c->stream>>>(d, c->scal, U_(KV_X), V_(KV_X), U_(KV_PHAT), V_(KV_PHAT),
                                                U_(KV_SHAT), V_(KV_SHAT), U_(KV_S), V_(KV_S), U_(KV_T), V_(KV_T),
                                                U_(KV_R), V_(KV_R), U_(KV_RHAT), V_(KV_RHAT), c->partials, g.x); c->launches++;
    k_reduce<<<1, 256, 0, c->stream>>>(c->partials, nb, c->scal, ST_RHO); c->launches++;
    k_update_p<<<g, block2d(), 0, c->stream>>>(d, c->scal, U_(KV_R), V_(KV_R), U_(KV_V), V_(KV_V), U_(KV_P),
                                               V_(KV_P)); c->launches++;
    DIVA_LAUNCHED(c, "bicgstab full step");
    c->fine_passes += 6.0;
    if ((st = read_scalars(c))) return st;
    rnorm = sqrt(c->h_scal[SC_RNORM2]);
    if (!std::isfinite(rnorm)) return set_error(c, DIVA_NAN_DETECTED, "NaN in the linear solve");
    done = rnorm <= target;
  }
  k_fill_boundary<<<g, block2d(), 0, c->stream>>>(d, c->bc, U_(KV_X), V_(KV_X)); c->launches++;
  DIVA_LAUNCHED(c, "k_fill_boundary");
  *iters = it;
  c->lin_iters += it;
  if (!done) {
    char buf[160];
    snprintf(buf, sizeof(buf), "linear solve reached %d iterations at relative residual %.3e (target %.1e)", it,
             bnorm > 0 ? rnorm / bnorm : rnorm, rtol);
    c->err = buf;
    return DIVA_LINEAR_NOT_CONVERGED;
  }
  return DIVA_OK;
}

int solver_relres(Ctx* c, const double* u, const double* v, double* relres) {
  const Dims d = c->d;
  dim3 g = grid2d(d.ny, d.nx);
  k_relres<<<g, block2d(), 0, c->stream>>>(make_op(c, 0), u, v, c->kv[KV_B][0], c->kv[KV_B][1], c->partials, g.x); c->launches++;
  k_reduce<<<1, 256, 0, c->stream>>>(c->partials, g.x * g.y, c->scal, ST_INIT); c->launches++;
  DIVA_LAUNCHED(c, "k_relres");
  c->fine_passes += 1.0;
  int st = read_scalars(c);
  if (st) return st;
  const double bb = c->h_scal[SC_BNORM2], rr = c->h_scal[SC_RNORM2];
  *relres = bb > 0.0 ? sqrt(rr / bb) : sqrt(rr);
  return DIVA_OK;
}

// Fine-level smoothing as the V-cycle runs it (used to time the smoother): the tiled
// pre- and post-smoothing kernels (V(2,2), residual included) when the grid is tiled,
// else `sweeps` per-colour sweeps.  x, b and the coarse correction are the solver's
// scratch vectors.
int solver_smooth_fine(Ctx* c, int sweeps) {
  if (c->tiled && c->nlev > 1 && sub_first_level(c) > 0) {
    const int nu = 2;
    int fx, fy;
    factors(c, 0, &fx, &fy);
    double *xu = c->kv[KV_X][0], *xv = c->kv[KV_X][1];
    double *bu = c->kv[KV_B][0], *bv = c->kv[KV_B][1];   // not written: the restriction is off
    int st = tile_down(c, 0, Restriction{}, bu, bv, xu, xv, nu);
    if (!st) st = tile_up(c, 0, fx, fy, bu, bv, xu, xv, nu);
    return st;
  }
  for (int s = 0; s < sweeps; ++s) {
    int st = gs_sweep(c, 0, c->kv[KV_X][0], c->kv[KV_X][1], c->kv[KV_B][0], c->kv[KV_B][1], true);
    if (st) return st;
  }
  return DIVA_OK;
}

// compulsory FP64 values per fine-level point moved by one solver_smooth_fine(c, 1)
int solver_smooth_fine_values(const Ctx* c) {
  // tiled, per point and component pair: pre reads b_u, b_v and N_a, N_b, beta_x, beta_y
  // and the two inverse diagonals (8) and writes x_u, x_v, r_u, r_v (4); post reads x_u,
  // x_v, b_u, b_v and the same 6 coefficients (10) and writes x_u, x_v (2)
  return (c->tiled && c->nlev > 1 && sub_first_level(c) > 0) ? 24 : 10;
}

int solver_matvec_fine(Ctx* c, int reps) {
  const Dims d = c->d;
  dim3 g = grid2d(d.ny, d.nx);
  const Op o = make_op(c, 0);
  for (int r = 0; r < reps; ++r) {
    k_matvec<<<g, block2d(), 0, c->stream>>>(o, c->kv[KV_X][0], c->kv[KV_X][1], c->kv[KV_T][0], c->kv[KV_T][1],
                                             c->kv[KV_RHAT][0], c->kv[KV_RHAT][1], nullptr, nullptr, c->partials, g.x); c->launches++;
  }
  DIVA_LAUNCHED(c, "k_matvec");
  return DIVA_OK;
}

// one preconditioner application (V-cycle from zero) on the current Krylov residual
int solver_vcycle_fine(Ctx* c, int reps) {
  for (int r = 0; r < reps; ++r) {
    int st = precond(c, c->kv[KV_R][0], c->kv[KV_R][1], c->kv[KV_PHAT][0], c->kv[KV_PHAT][1]);
    if (st) return st;
  }
  return DIVA_OK;
}

// the one-block part of the V-cycle alone, on the arrays of its first level
int solver_subcycle(Ctx* c, int reps) {
  const int l = sub_first_level(c);
  const Level& L = c->lv[l];
  for (int r = 0; r < reps; ++r) {
    int st = vcycle(c, l, L.xu, L.xv, L.bu, L.bv, Restriction{});
    if (st) return st;
  }
  return DIVA_OK;
}

// algorithmic bytes of one V-cycle (FP64, compulsory traffic per point and level):
// each sweep 10 values, the residual 8, the transfers 6, weighted by the level's points
double solver_vcycle_bytes(const Ctx* c) {
  double b = 0.0;
  for (int l = 0; l < c->nlev; ++l)
    b += (double)c->lv[l].d.nx * c->lv[l].d.ny * sizeof(double) * (4 * 10 + 8 + 6);
  return b;
}

// row types of the finest level (choice_ice_margin 'BC'), from the SICO masks of this solve
int solver_row_types(Ctx* c) {
  if (c->c.choice_ice_margin != DIVA_MARGIN_BC) return DIVA_OK;
  k_row_types<<<GL(0)>>>(c->d, c->I(DIVA_F_DIVA_MASK_COMBI), c->I(DIVA_F_DIVA_ISFRONT_INNER),
                         c->I(DIVA_F_DIVA_ISFRONT_OUTER), c->rtu, c->rtv); c->launches++;
  DIVA_LAUNCHED(c, "k_row_types");
  return DIVA_OK;
}

int solver_fill_boundary(Ctx* c, double* u, double* v) {
  k_fill_boundary<<<grid2d(c->d.ny, c->d.nx), block2d(), 0, c->stream>>>(c->d, c->bc, u, v); c->launches++;
  DIVA_LAUNCHED(c, "k_fill_boundary");
  return DIVA_OK;
}

// ---- the viscosity iteration loop as one CUDA graph -------------------------------
//
// One viscosity iteration (ITER):
//   pre   : k_ctl_begin, coefficients (K1 + faces), operator set-up of all levels,
//           [relres stop rule] nonlinear residual -> k_ctl_relres sets IF(solve)
//   IF(solve):
//     head  : x <- (u,v), initial residual, k_ctl_lin_init sets WHILE(krylov)
//     WHILE(krylov):
//       first : V-cycle p -> phat, v = A phat, alpha, s, k_ctl_half sets IF(second)
//               and may end the loop; x += alpha phat if it did
//       IF(second): V-cycle s -> shat, t = A shat, omega, x and r, k_ctl_full
//                   sets WHILE(krylov), p update
//     tail  : boundary fill, Picard update (limits, relaxation, step norm, basal
//             stress and velocity), stop test, DIVA_err commit
//   post  : [DIVA] basal stress/velocity when the residual stopped the iteration;
//           k_ctl_loop: continue unless the iteration converged, the residual met
//           its tolerance, a NaN appeared or the iteration budget is spent
//
// The whole loop: WHILE(picard) { ITER(parity p); IF(odd) { ITER(parity 1 - p) } }.
// The viscosity is double-buffered (each iteration reads one buffer and writes the
// other), and captured kernel arguments are fixed pointers, so the body holds two
// iterations, one per buffer order; the first sets IF(odd) to its continue flag.
// Two instances are built, one per starting buffer; one launch runs a whole solve
// with no host round trip between iterations.
namespace {

struct CaptureCtx {
  Ctx* c;
  cudaStream_t s[6] = {};
  bool capturing[6] = {};
  long long l0 = 0;
  double p0 = 0.0;
  void mark() { l0 = c->launches; p0 = c->fine_passes; }
  long long dl() const { return c->launches - l0; }
  double dp() const { return c->fine_passes - p0; }
};

int add_conditional(Ctx* c, cudaStream_t s, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                    cudaGraph_t* body) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  DIVA_CUDA(c, cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
  if (st != cudaStreamCaptureStatusActive) return set_error(c, DIVA_CUDA_ERROR, "stream is not capturing");
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = type;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  DIVA_CUDA(c, cudaGraphAddNode(&node, g, deps, nd, &p));
  *body = p.conditional.phGraph_out[0];
  DIVA_CUDA(c, cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  return DIVA_OK;
}

// the graph a capturing stream records into
int capture_graph(Ctx* c, cudaStream_t s, cudaGraph_t* g) {
  cudaStreamCaptureStatus st;
  DIVA_CUDA(c, cudaStreamGetCaptureInfo(s, &st, nullptr, g, nullptr, nullptr));
  if (st != cudaStreamCaptureStatusActive) return set_error(c, DIVA_CUDA_ERROR, "stream is not capturing");
  return DIVA_OK;
}

// end of an iteration: totals of the loop, and whether it goes on (sets h_a, and h_b if given)
__global__ void k_ctl_loop(double* sc, cudaGraphConditionalHandle h_a, cudaGraphConditionalHandle h_b, int has_b,
                           int nit) {
  sc[SC_SUM_LIN] += sc[SC_LIN_IT];
  sc[SC_SUM_FULL] += sc[SC_LIN_FULL];
  sc[SC_N_SOLVED] += sc[SC_SOLVED];
  const bool stop = sc[SC_CONVERGED] != 0.0 || sc[SC_EXIT_RELRES] != 0.0 || sc[SC_NAN] != 0.0 ||
                    sc[SC_PIC_IT] > (double)nit;
  cudaGraphSetConditional(h_a, stop ? 0u : 1u);
  if (has_b) cudaGraphSetConditional(h_b, stop ? 0u : 1u);
}

// One viscosity iteration recorded into the graph that stream `top` is capturing; its
// conditional bodies use cc.s[3..5].  `count`: record the launches and passes of its parts.
int capture_iteration(Ctx* c, CaptureCtx& cc, cudaStream_t top, bool diva, PicardGraphs& G, bool count,
                      cudaGraphConditionalHandle h_a, cudaGraphConditionalHandle h_b, int has_b) {
  const diva_config_t& C = c->c;
  const bool relmode = C.picard_stop == DIVA_STOP_RELRES;
  const Dims d = c->d;
  const Op o = make_op(c, 0);
  dim3 g2 = grid2d(d.ny, d.nx);
  const int nb = g2.x * g2.y;
  auto U_ = [&](int k) { return c->kv[k][0]; };
  auto V_ = [&](int k) { return c->kv[k][1]; };
  double* u = c->D(diva ? DIVA_F_U_VAV_CX : DIVA_F_U_SSA_CX);
  double* v = c->D(diva ? DIVA_F_V_VAV_CY : DIVA_F_V_SSA_CY);
  int st;
  cudaGraph_t graph;
  if ((st = capture_graph(c, top, &graph))) return st;
  cudaGraphConditionalHandle h_solve;
  DIVA_CUDA(c, cudaGraphConditionalHandleCreate(&h_solve, graph, 1, cudaGraphCondAssignDefault));
  c->stream = top;
  // ---- pre
  cc.mark();
  k_ctl_begin<<<1, 1, 0, c->stream>>>(c->scal); c->launches++;
  if ((st = launch_diva_coefficients(c, u, v, diva, K1_LOOP))) return st;   // swaps the viscosity buffers
  if ((st = solver_setup(c, 1))) return st;
  if (relmode) {
    k_relres<<<g2, block2d(), 0, c->stream>>>(o, u, v, U_(KV_B), V_(KV_B), c->partials, g2.x); c->launches++;
    k_ctl_relres<<<1, 256, 0, c->stream>>>(c->partials, nb, c->scal, h_solve, C.picard_relres_tol,
                                           C.picard_stall_its); c->launches++;
    c->fine_passes += 1.0;
  }
  DIVA_LAUNCHED(c, "graph pre");
  if (count) { G.n_pre = cc.dl(); G.p_pre = cc.dp(); }
  // ---- IF(solve)
  cudaGraph_t body_solve;
  if ((st = add_conditional(c, top, h_solve, cudaGraphCondTypeIf, &body_solve))) return st;
  cudaGraphConditionalHandle h_while;
  DIVA_CUDA(c, cudaGraphConditionalHandleCreate(&h_while, body_solve, 0, cudaGraphCondAssignDefault));
  DIVA_CUDA(c, cudaStreamBeginCaptureToGraph(cc.s[3], body_solve, nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal));
  cc.capturing[3] = true;
  c->stream = cc.s[3];
  cc.mark();
  DIVA_CUDA(c, cudaMemcpyAsync(U_(KV_X), u, sizeof(double) * d.plane, cudaMemcpyDeviceToDevice, c->stream));
  DIVA_CUDA(c, cudaMemcpyAsync(V_(KV_X), v, sizeof(double) * d.plane, cudaMemcpyDeviceToDevice, c->stream));
  k_init_residual<<<g2, block2d(), 0, c->stream>>>(o, U_(KV_X), V_(KV_X), U_(KV_B), V_(KV_B), U_(KV_R), V_(KV_R),
                                                   U_(KV_RHAT), V_(KV_RHAT), U_(KV_P), V_(KV_P), c->partials, g2.x); c->launches++;
  k_ctl_lin_init<<<1, 256, 0, c->stream>>>(c->partials, nb, c->scal, h_while, relmode && C.lin_adaptive, C.lin_rtol,
                                           C.lin_maxit); c->launches++;
  c->fine_passes += 1.0;
  DIVA_LAUNCHED(c, "graph head");
  if (count) { G.n_head = cc.dl(); G.p_head = cc.dp(); }
  // ---- WHILE(krylov)
  cudaGraph_t body_while;
  if ((st = add_conditional(c, cc.s[3], h_while, cudaGraphCondTypeWhile, &body_while))) return st;
  cudaGraphConditionalHandle h_half;
  DIVA_CUDA(c, cudaGraphConditionalHandleCreate(&h_half, body_while, 1, cudaGraphCondAssignDefault));
  DIVA_CUDA(c, cudaStreamBeginCaptureToGraph(cc.s[4], body_while, nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal));
  cc.capturing[4] = true;
  c->stream = cc.s[4];
  cc.mark();
  if ((st = precond(c, U_(KV_P), V_(KV_P), U_(KV_PHAT), V_(KV_PHAT)))) return st;
  k_matvec<<<g2, block2d(), 0, c->stream>>>(o, U_(KV_PHAT), V_(KV_PHAT), U_(KV_V), V_(KV_V), U_(KV_RHAT), V_(KV_RHAT),
                                            nullptr, nullptr, c->partials, g2.x); c->launches++;
  k_reduce<<<1, 256, 0, c->stream>>>(c->partials, nb, c->scal, ST_ALPHA); c->launches++;
  k_update_s<<<g2, block2d(), 0, c->stream>>>(d, c->scal, U_(KV_R), V_(KV_R), U_(KV_V), V_(KV_V), U_(KV_S), V_(KV_S),
                                              c->partials, g2.x); c->launches++;
  k_ctl_half<<<1, 256, 0, c->stream>>>(c->partials, nb, c->scal, h_while, h_half); c->launches++;
  k_x_half_pred<<<g2, block2d(), 0, c->stream>>>(d, c->scal, U_(KV_X), V_(KV_X), U_(KV_PHAT), V_(KV_PHAT)); c->launches++;
  c->fine_passes += 3.0;
  DIVA_LAUNCHED(c, "graph first half");
  if (count) { G.n_first = cc.dl(); G.p_first = cc.dp(); }
  // ---- IF(second half)
  cudaGraph_t body_half;
  if ((st = add_conditional(c, cc.s[4], h_half, cudaGraphCondTypeIf, &body_half))) return st;
  DIVA_CUDA(c, cudaStreamBeginCaptureToGraph(cc.s[5], body_half, nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal));
  cc.capturing[5] = true;
  c->stream = cc.s[5];
  cc.mark();
  if ((st = precond(c, U_(KV_S), V_(KV_S), U_(KV_SHAT), V_(KV_SHAT)))) return st;
  k_matvec<<<g2, block2d(), 0, c->stream>>>(o, U_(KV_SHAT), V_(KV_SHAT), U_(KV_T), V_(KV_T), U_(KV_S), V_(KV_S),
                                            nullptr, nullptr, c->partials, g2.x); c->launches++;
  k_reduce<<<1, 256, 0, c->stream>>>(c->partials, nb, c->scal, ST_OMEGA); c->launches++;
  k_update_xr<<<g2, block2d(), 0, c->stream>>>(d, c->scal, U_(KV_X), V_(KV_X), U_(KV_PHAT), V_(KV_PHAT), U_(KV_SHAT),
                                               V_(KV_SHAT), U_(KV_S), V_(KV_S), U_(KV_T), V_(KV_T), U_(KV_R),
                                               V_(KV_R), U_(KV_RHAT), V_(KV_RHAT), c->partials, g2.x); c->launches++;
  k_ctl_full<<<1, 256, 0, c->stream>>>(c->partials, nb, c->scal, h_while, C.lin_maxit); c->launches++;
  k_update_p<<<g2, block2d(), 0, c->stream>>>(d, c->scal, U_(KV_R), V_(KV_R), U_(KV_V), V_(KV_V), U_(KV_P), V_(KV_P)); c->launches++;
  c->fine_passes += 3.0;
  DIVA_LAUNCHED(c, "graph second half");
  if (count) { G.n_second = cc.dl(); G.p_second = cc.dp(); }
  DIVA_CUDA(c, cudaStreamEndCapture(cc.s[5], &body_half));
  cc.capturing[5] = false;
  DIVA_CUDA(c, cudaStreamEndCapture(cc.s[4], &body_while));
  cc.capturing[4] = false;
  // ---- tail
  c->stream = cc.s[3];
  cc.mark();
  k_ctl_lin_finish<<<1, 1, 0, c->stream>>>(c->scal); c->launches++;
  k_fill_boundary<<<g2, block2d(), 0, c->stream>>>(d, c->bc, U_(KV_X), V_(KV_X)); c->launches++;
  DIVA_LAUNCHED(c, "graph tail");
  if (C.picard_anderson_m > 0 && (st = launch_anderson_prepare(c, u, v, U_(KV_X), V_(KV_X)))) return st;
  if ((st = launch_picard_update(c, u, v, U_(KV_X), V_(KV_X), diva))) return st;
  if ((st = launch_ctl_end(c, relmode))) return st;
  if ((st = launch_err_commit_pred(c))) return st;
  if (count) { G.n_tail = cc.dl(); G.p_tail = cc.dp(); }
  DIVA_CUDA(c, cudaStreamEndCapture(cc.s[3], &body_solve));
  cc.capturing[3] = false;
  // ---- post
  c->stream = top;
  cc.mark();
  if (diva && relmode && (st = launch_basal_pred(c))) return st;
  k_ctl_loop<<<1, 1, 0, c->stream>>>(c->scal, h_a, h_b, has_b, C.DIVA_visc_it_nit); c->launches++;
  DIVA_LAUNCHED(c, "k_ctl_loop");
  if (count) G.n_post = cc.dl();
  return DIVA_OK;
}

// The whole viscosity loop of one context, WHILE(picard) { ITER(parity); IF(odd) { ITER(1 -
// parity) } }, appended to `graph` as a root node (no dependencies): on its own the graph of
// build_one, several of them side by side the graph of a batch (solver_build_batch_graph).
int capture_loop(Ctx* c, CaptureCtx& cc, bool diva, PicardGraphs& G, int parity, cudaGraph_t graph, bool count) {
  cudaGraphConditionalHandle h_pic;
  DIVA_CUDA(c, cudaGraphConditionalHandleCreate(&h_pic, graph, 1, cudaGraphCondAssignDefault));
  DIVA_CUDA(c, cudaStreamBeginCaptureToGraph(cc.s[0], graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  cc.capturing[0] = true;
  G.visc_buf[parity] = c->f[DIVA_F_VISC_EFF_3D_A];
  int st;
  cudaGraph_t body_pic;
  if ((st = add_conditional(c, cc.s[0], h_pic, cudaGraphCondTypeWhile, &body_pic))) return st;
  DIVA_CUDA(c, cudaStreamBeginCaptureToGraph(cc.s[1], body_pic, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  cc.capturing[1] = true;
  cudaGraphConditionalHandle h_odd;
  DIVA_CUDA(c, cudaGraphConditionalHandleCreate(&h_odd, body_pic, 0, cudaGraphCondAssignDefault));
  // the first iteration of the pair (its buffer order is this graph's parity)
  if ((st = capture_iteration(c, cc, cc.s[1], diva, G, count, h_pic, h_odd, 1))) return st;
  cudaGraph_t body_odd;
  if ((st = add_conditional(c, cc.s[1], h_odd, cudaGraphCondTypeIf, &body_odd))) return st;
  DIVA_CUDA(c, cudaStreamBeginCaptureToGraph(cc.s[2], body_odd, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  cc.capturing[2] = true;
  if ((st = capture_iteration(c, cc, cc.s[2], diva, G, false, h_pic, h_pic, 0))) return st;
  DIVA_CUDA(c, cudaStreamEndCapture(cc.s[2], &body_odd));
  cc.capturing[2] = false;
  DIVA_CUDA(c, cudaStreamEndCapture(cc.s[1], &body_pic));
  cc.capturing[1] = false;
  cudaGraph_t top = nullptr;
  DIVA_CUDA(c, cudaStreamEndCapture(cc.s[0], &top));
  cc.capturing[0] = false;
  return DIVA_OK;
}

// the loop graph starting from the viscosity buffer `parity`
int build_one(Ctx* c, CaptureCtx& cc, bool diva, PicardGraphs& G, int parity) {
  cudaGraph_t graph;
  DIVA_CUDA(c, cudaGraphCreate(&graph, 0));
  int st = capture_loop(c, cc, diva, G, parity, graph, parity == 0);
  if (st) {
    cudaGraphDestroy(graph);
    return st;
  }
  cudaGraphExec_t exec = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  DIVA_CUDA(c, e);
  G.exec[parity] = exec;
  return DIVA_OK;
}

// end every capture a failed build left open, and forget the error it left behind
void close_captures(CaptureCtx& cc) {
  for (int q = 5; q >= 0; --q) {
    if (cc.capturing[q]) {
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(cc.s[q], &junk);
      if (junk) cudaGraphDestroy(junk);
      cc.capturing[q] = false;
    }
  }
  cudaGetLastError();
}

}  // namespace

int solver_tile_edges(const Ctx* c, int32_t* edges, int n) {
  const int first = sub_first_level(c);
  for (int l = 0; l < n; ++l)
    edges[l] = (l < c->nlev && c->tiled && c->nlev > 1 && l < first) ? tile_edge(c, l) : 0;
  return c->nlev;
}

void solver_destroy_graphs(Ctx* c) {
  for (auto& G : c->graphs) {
    for (auto& e : G.exec)
      if (e) cudaGraphExecDestroy(e), e = nullptr;
    G.valid = false;
  }
}

int solver_build_picard_graphs(Ctx* c, bool diva) {
  PicardGraphs& G = c->graphs[diva ? 1 : 0];
  if (G.valid) return DIVA_OK;
  CaptureCtx cc;
  cc.c = c;
  cudaStream_t user = c->stream;
  const long long launches0 = c->launches;
  const double passes0 = c->fine_passes;
  const long mg0 = c->mg_cycles;
  void* visc0 = c->f[DIVA_F_VISC_EFF_3D_A];
  double* prev0 = c->visc_prev;
  int st = DIVA_OK;
  for (int q = 0; q < 6 && !st; ++q)
    if (cudaStreamCreateWithFlags(&cc.s[q], cudaStreamNonBlocking) != cudaSuccess) st = DIVA_CUDA_ERROR;
  // parity 0 starts from the current buffer, parity 1 from the other; each graph
  // captures two iterations, which swap the viscosity buffers twice
  for (int parity = 0; parity < 2 && !st; ++parity) {
    if (parity == 1) std::swap(c->f[DIVA_F_VISC_EFF_3D_A], *reinterpret_cast<void**>(&c->visc_prev));
    st = build_one(c, cc, diva, G, parity);
  }
  close_captures(cc);   // and clear any capture error so the host path can proceed
  for (int q = 0; q < 6; ++q)
    if (cc.s[q]) cudaStreamDestroy(cc.s[q]);
  c->stream = user;
  c->launches = launches0;
  c->fine_passes = passes0;
  c->mg_cycles = mg0;
  c->f[DIVA_F_VISC_EFF_3D_A] = visc0;   // the captures swap these without running anything
  c->visc_prev = prev0;
  if (st) {
    for (auto& e : G.exec)
      if (e) cudaGraphExecDestroy(e), e = nullptr;
    return st;
  }
  G.valid = true;
  return DIVA_OK;
}

// One graph holding the viscosity loops of n contexts side by side (a batch, diva_batch_create):
// each member's loop is captured as it stands now (its viscosity buffer order, its
// configuration) into one parent graph, instantiated once.  bufs[k] receives the buffer
// member k's loop starts from.  Every member's own loop graphs must exist already (their
// launch and pass counts account for the batch's iterations).
int solver_build_batch_graph(Ctx* const* cs, int n, cudaGraphExec_t* exec, void** bufs) {
  Ctx* c0 = cs[0];
  *exec = nullptr;
  cudaGraph_t parent = nullptr;
  DIVA_CUDA(c0, cudaGraphCreate(&parent, 0));
  CaptureCtx cc;
  int st = DIVA_OK;
  for (int q = 0; q < 6 && !st; ++q)
    if (cudaStreamCreateWithFlags(&cc.s[q], cudaStreamNonBlocking) != cudaSuccess) st = DIVA_CUDA_ERROR;
  for (int k = 0; k < n && !st; ++k) {
    Ctx* c = cs[k];
    cc.c = c;
    PicardGraphs scratch;   // the loop's counts are the member's own graphs'
    cudaStream_t user = c->stream;
    const long long launches0 = c->launches;
    const double passes0 = c->fine_passes;
    const long mg0 = c->mg_cycles;
    void* visc0 = c->f[DIVA_F_VISC_EFF_3D_A];
    double* prev0 = c->visc_prev;
    bufs[k] = visc0;
    st = capture_loop(c, cc, true, scratch, 0, parent, false);
    c->stream = user;
    c->launches = launches0;
    c->fine_passes = passes0;
    c->mg_cycles = mg0;
    c->f[DIVA_F_VISC_EFF_3D_A] = visc0;   // the capture swaps these without running anything
    c->visc_prev = prev0;
    if (st) set_error(c0, st, "batch graph: capture of member " + std::to_string(k) + " failed: " + c->err);
  }
  close_captures(cc);
  for (int q = 0; q < 6; ++q)
    if (cc.s[q]) cudaStreamDestroy(cc.s[q]);
  if (!st && cudaGraphInstantiate(exec, parent, 0) != cudaSuccess) {
    *exec = nullptr;
    cudaGetLastError();
    st = set_error(c0, DIVA_CUDA_ERROR, "batch graph: instantiation failed");
  }
  cudaGraphDestroy(parent);
  return st;
}

}  // namespace diva
