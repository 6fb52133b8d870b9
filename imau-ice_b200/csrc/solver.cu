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
//   * the coarsest level is relaxed by one thread block with many sweeps.
// All reductions are two-stage (block partials, then one fixed-order sum) so
// results are bit-reproducible from run to run.
#include <cmath>
#include <cstdio>
#include "ctx.hpp"

namespace diva {
namespace {

struct Op {
  Dims d;
  BCs bc;
  double ax, ay;   // hy/hx and hx/hy of the level's cells (1 on the fine grid)
  const double *Na, *Nb, *Bx, *By;
};

__device__ __forceinline__ bool u_int(const Dims& d, int j, int i) {
  return i >= 1 && i <= d.nx - 3 && j >= 1 && j <= d.ny - 2;
}
__device__ __forceinline__ bool v_int(const Dims& d, int j, int i) {
  return i >= 1 && i <= d.nx - 2 && j >= 1 && j <= d.ny - 3;
}
__device__ __forceinline__ int bc_pick(int a, int b) {
  if (a == DIVA_BC_ZERO || b == DIVA_BC_ZERO) return DIVA_BC_ZERO;
  if (a == DIVA_BC_INFINITE || b == DIVA_BC_INFINITE) return DIVA_BC_INFINITE;
  return DIVA_BC_PERIODIC;
}
// Source of u(j,i) (list_DIVA_matrix_coefficients_eq_1_boundary :1932-2061); false = zero.
__device__ __forceinline__ bool u_src(const Dims& d, const BCs& b, int j, int i, int& js, int& is) {
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
__device__ __forceinline__ bool v_src(const Dims& d, const BCs& b, int j, int i, int& js, int& is) {
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
// Read a u (v) value through the boundary elimination (RAW = false), or as
// stored (RAW = true: the reference's assembled rows reference stored values).
template <bool RAW = false>
__device__ __forceinline__ double LU(const Op& o, const double* x, int j, int i) {
  if (RAW) return x[o.d.at(j, i)];
  int js, is;
  return u_src(o.d, o.bc, j, i, js, is) ? x[o.d.at(js, is)] : 0.0;
}
template <bool RAW = false>
__device__ __forceinline__ double LV(const Op& o, const double* x, int j, int i) {
  if (RAW) return x[o.d.at(j, i)];
  int js, is;
  return v_src(o.d, o.bc, j, i, js, is) ? x[o.d.at(js, is)] : 0.0;
}

// (A x) of the u row at interior (j,i) (list_DIVA_matrix_coefficients_eq_1_free :2342-2404)
template <bool RAW = false>
__device__ __forceinline__ double Au(const Op& o, const double* xu, const double* xv, int j, int i) {
  const Dims& d = o.d;
  const double Ae = o.Na[d.at(j, i + 1)], Aw = o.Na[d.at(j, i)], Bn = o.Nb[d.at(j, i)], Bs = o.Nb[d.at(j - 1, i)];
  const double cE = 4.0 * o.ax * Ae, cW = 4.0 * o.ax * Aw, cN = o.ay * Bn, cS = o.ay * Bs;
  const double diag = -(cE + cW + cN + cS) - o.Bx[d.at(j, i)];
  return cE * LU<RAW>(o, xu, j, i + 1) + cW * LU<RAW>(o, xu, j, i - 1) + cN * LU<RAW>(o, xu, j + 1, i) +
         cS * LU<RAW>(o, xu, j - 1, i) + diag * xu[d.at(j, i)] + (-2.0 * Aw - Bn) * LV<RAW>(o, xv, j, i) +
         (2.0 * Ae + Bn) * LV<RAW>(o, xv, j, i + 1) + (2.0 * Aw + Bs) * LV<RAW>(o, xv, j - 1, i) +
         (-2.0 * Ae - Bs) * LV<RAW>(o, xv, j - 1, i + 1);
}
// (A x) of the v row at interior (j,i) (list_DIVA_matrix_coefficients_eq_2_free :2405-2467)
template <bool RAW = false>
__device__ __forceinline__ double Av(const Op& o, const double* xu, const double* xv, int j, int i) {
  const Dims& d = o.d;
  const double An = o.Na[d.at(j + 1, i)], As = o.Na[d.at(j, i)], Be = o.Nb[d.at(j, i)], Bw = o.Nb[d.at(j, i - 1)];
  const double cN = 4.0 * o.ay * An, cS = 4.0 * o.ay * As, cE = o.ax * Be, cW = o.ax * Bw;
  const double diag = -(cN + cS + cE + cW) - o.By[d.at(j, i)];
  return cN * LV<RAW>(o, xv, j + 1, i) + cS * LV<RAW>(o, xv, j - 1, i) + cE * LV<RAW>(o, xv, j, i + 1) +
         cW * LV<RAW>(o, xv, j, i - 1) + diag * xv[d.at(j, i)] + (-2.0 * An - Bw) * LU<RAW>(o, xu, j + 1, i - 1) +
         (2.0 * An + Be) * LU<RAW>(o, xu, j + 1, i) + (2.0 * As + Bw) * LU<RAW>(o, xu, j, i - 1) +
         (-2.0 * As - Be) * LU<RAW>(o, xu, j, i);
}
// effective diagonal of the reduced system: couplings to boundary unknowns whose source is the row itself fold in
__device__ __forceinline__ double diag_u(const Op& o, int j, int i) {
  const Dims& d = o.d;
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

__global__ void k_diag(Op o, double* idu, double* idv) {
  IDX2D
  if (j >= o.d.ny || i >= o.d.nx) return;
  const long long q = o.d.at(j, i);
  idu[q] = u_int(o.d, j, i) ? 1.0 / diag_u(o, j, i) : 0.0;
  idv[q] = v_int(o.d, j, i) ? 1.0 / diag_v(o, j, i) : 0.0;
}

// rhs of the free rows: b = -taud * dx^2 (divided by N_cx/N_cy without cross terms)
__global__ void k_rhs(Dims d, int crossterms, const double* tdx, const double* tdy, const double* Ncx,
                      const double* Ncy, double* bu, double* bv) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  const double dx2 = d.dx * d.dx;
  bu[q] = u_int(d, j, i) ? (crossterms ? -tdx[q] * dx2 : -tdx[q] * dx2 / Ncx[q]) : 0.0;
  bv[q] = v_int(d, j, i) ? (crossterms ? -tdy[q] * dx2 : -tdy[q] * dx2 / Ncy[q]) : 0.0;
}

// one colour of Gauss-Seidel: comp 0 = u, 1 = v; colour = (i+j) parity
__global__ void k_gs(Op o, double* xu, double* xv, const double* bu, const double* bv, const double* idu,
                     const double* idv, int comp, int color) {
  const int jj = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  const int j = 2 * jj + ((i + color) & 1);
  if (j >= o.d.ny || i >= o.d.nx) return;
  const long long q = o.d.at(j, i);
  if (comp == 0) {
    if (!u_int(o.d, j, i)) return;
    xu[q] += (bu[q] - Au(o, xu, xv, j, i)) * idu[q];
  } else {
    if (!v_int(o.d, j, i)) return;
    xv[q] += (bv[q] - Av(o, xu, xv, j, i)) * idv[q];
  }
}

// relaxation of the coarsest level by one block (bounded number of sweeps)
__global__ void k_coarse_solve(Op o, double* xu, double* xv, const double* bu, const double* bv, const double* idu,
                               const double* idv, int sweeps) {
  const Dims& d = o.d;
  const int n = d.nx * d.ny;
  for (int s = 0; s < sweeps; ++s) {
    for (int pass = 0; pass < 8; ++pass) {
      // symmetric order: u0 u1 v0 v1 | v1 v0 u1 u0
      const int p = pass < 4 ? pass : 7 - pass;
      const int comp = p >> 1, color = p & 1;
      for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int j = t % d.ny, i = t / d.ny;
        if (((i + j) & 1) != color) continue;
        const long long q = d.at(j, i);
        if (comp == 0) {
          if (u_int(d, j, i)) xu[q] += (bu[q] - Au(o, xu, xv, j, i)) * idu[q];
        } else {
          if (v_int(d, j, i)) xv[q] += (bv[q] - Av(o, xu, xv, j, i)) * idv[q];
        }
      }
      __syncthreads();
    }
  }
}

// r = b - A x on the interior (zero elsewhere)
__global__ void k_residual(Op o, const double* xu, const double* xv, const double* bu, const double* bv, double* ru,
                           double* rv) {
  IDX2D
  if (j >= o.d.ny || i >= o.d.nx) return;
  const long long q = o.d.at(j, i);
  ru[q] = u_int(o.d, j, i) ? bu[q] - Au(o, xu, xv, j, i) : 0.0;
  rv[q] = v_int(o.d, j, i) ? bv[q] - Av(o, xu, xv, j, i) : 0.0;
}

// 1D transfer weights.  "cell" direction: u along x, v along y; "node": u along y, v along x.
// Gather form of the restriction: coarse C collects fine f with weight w.
__device__ __forceinline__ int gather_cell(int C, int f2, int* f, double* w) {
  if (f2 == 1) { f[0] = C; w[0] = 1.0; return 1; }
  f[0] = 2 * C - 1; w[0] = 0.25; f[1] = 2 * C; w[1] = 0.75; f[2] = 2 * C + 1; w[2] = 0.75; f[3] = 2 * C + 2; w[3] = 0.25;
  return 4;
}
__device__ __forceinline__ int gather_node(int C, int f2, int* f, double* w) {
  if (f2 == 1) { f[0] = C; w[0] = 1.0; return 1; }
  f[0] = 2 * C - 1; w[0] = 0.5; f[1] = 2 * C; w[1] = 1.0; f[2] = 2 * C + 1; w[2] = 0.5;
  return 3;
}
// Scatter form (prolongation): fine f takes coarse C with weight w.
__device__ __forceinline__ int scatter_cell(int f, int f2, int* C, double* w) {
  if (f2 == 1) { C[0] = f; w[0] = 1.0; return 1; }
  const int c = f >> 1;
  if ((f & 1) == 0) { C[0] = c; w[0] = 0.75; C[1] = c - 1; w[1] = 0.25; }
  else { C[0] = c; w[0] = 0.75; C[1] = c + 1; w[1] = 0.25; }
  return 2;
}
__device__ __forceinline__ int scatter_node(int f, int f2, int* C, double* w) {
  if (f2 == 1) { C[0] = f; w[0] = 1.0; return 1; }
  const int c = f >> 1;
  if ((f & 1) == 0) { C[0] = c; w[0] = 1.0; return 1; }
  C[0] = c; w[0] = 0.5; C[1] = c + 1; w[1] = 0.5;
  return 2;
}

// b_c = P^T r_f on coarse interior points; x_c = 0
__global__ void k_restrict(Dims df, Dims dc, int fx, int fy, const double* ru, const double* rv, double* bu,
                           double* bv, double* xu, double* xv) {
  IDX2D
  if (j >= dc.ny || i >= dc.nx) return;
  const long long q = dc.at(j, i);
  int fi[4], fj[4];
  double wi[4], wj[4];
  double s = 0.0;
  if (u_int(dc, j, i)) {
    const int ni = gather_cell(i, fx, fi, wi), nj = gather_node(j, fy, fj, wj);
    for (int a = 0; a < nj; ++a)
      for (int b = 0; b < ni; ++b)
        if (u_int(df, fj[a], fi[b])) s += wj[a] * wi[b] * ru[df.at(fj[a], fi[b])];
  }
  bu[q] = s;
  s = 0.0;
  if (v_int(dc, j, i)) {
    const int ni = gather_node(i, fx, fi, wi), nj = gather_cell(j, fy, fj, wj);
    for (int a = 0; a < nj; ++a)
      for (int b = 0; b < ni; ++b)
        if (v_int(df, fj[a], fi[b])) s += wj[a] * wi[b] * rv[df.at(fj[a], fi[b])];
  }
  bv[q] = s;
  xu[q] = 0.0;
  xv[q] = 0.0;
}

// x_f += P x_c on fine interior points (coarse values read through the coarse boundary mapping)
__global__ void k_prolong(Op oc, Dims df, int fx, int fy, const double* xcu, const double* xcv, double* xu,
                          double* xv) {
  IDX2D
  if (j >= df.ny || i >= df.nx) return;
  const long long q = df.at(j, i);
  int Ci[2], Cj[2];
  double wi[2], wj[2];
  const Dims& dc = oc.d;
  if (u_int(df, j, i)) {
    const int ni = scatter_cell(i, fx, Ci, wi), nj = scatter_node(j, fy, Cj, wj);
    double s = 0.0;
    for (int a = 0; a < nj; ++a)
      for (int b = 0; b < ni; ++b) {
        const int J = min(max(Cj[a], 0), dc.ny - 1), I = min(max(Ci[b], 0), dc.nx - 2);
        s += wj[a] * wi[b] * LU(oc, xcu, J, I);
      }
    xu[q] += s;
  }
  if (v_int(df, j, i)) {
    const int ni = scatter_node(i, fx, Ci, wi), nj = scatter_cell(j, fy, Cj, wj);
    double s = 0.0;
    for (int a = 0; a < nj; ++a)
      for (int b = 0; b < ni; ++b) {
        const int J = min(max(Cj[a], 0), dc.ny - 2), I = min(max(Ci[b], 0), dc.nx - 1);
        s += wj[a] * wi[b] * LV(oc, xcv, J, I);
      }
    xv[q] += s;
  }
}

// rediscretised coarse coefficients (averages of the fine ones; B scales with the cell area)
__global__ void k_coarsen(Dims df, Dims dc, int fx, int fy, const double* Na, const double* Nb, const double* Bx,
                          const double* By, double* cNa, double* cNb, double* cBx, double* cBy) {
  IDX2D
  if (j >= dc.ny || i >= dc.nx) return;
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

// ---- host side --------------------------------------------------------------------
Op op_of(const Ctx* c, int l) {
  Op o;
  o.d = c->lv[l].d;
  o.bc = c->bc;
  o.ax = c->lv[l].d.dx;   // placeholders, set below
  o.ay = 1.0;
  o.Na = c->lv[l].Na; o.Nb = c->lv[l].Nb; o.Bx = c->lv[l].Bx; o.By = c->lv[l].By;
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
static void factors(const Ctx* c, int l, int* fx, int* fy) {
  *fx = (c->lv[l + 1].d.nx != c->lv[l].d.nx) ? 2 : 1;
  *fy = (c->lv[l + 1].d.ny != c->lv[l].d.ny) ? 2 : 1;
}

#define GL(l) grid2d(c->lv[l].d.ny, c->lv[l].d.nx), block2d(), 0, c->stream

int solver_setup(Ctx* c) {
  const diva_config_t& C = c->c;
  if (C.choice_ice_margin == DIVA_MARGIN_BC)
    return set_error(c, DIVA_UNSUPPORTED, "choice_ice_margin 'BC' is not implemented by the GPU solver");
  k_rhs<<<GL(0)>>>(c->d, C.include_SSADIVA_crossterms, c->D(DIVA_F_TAUDX_CX), c->D(DIVA_F_TAUDY_CY),
                   c->D(DIVA_F_N_CX), c->D(DIVA_F_N_CY), c->kv[KV_B][0], c->kv[KV_B][1]); c->launches++;
  DIVA_LAUNCHED(c, "k_rhs");
  for (int l = 0; l + 1 < c->nlev; ++l) {
    int fx, fy;
    factors(c, l, &fx, &fy);
    const Level& F = c->lv[l];
    const Level& K = c->lv[l + 1];
    k_coarsen<<<GL(l + 1)>>>(F.d, K.d, fx, fy, F.Na, F.Nb, F.Bx, F.By, K.Na, K.Nb, K.Bx, K.By); c->launches++;
    DIVA_LAUNCHED(c, "k_coarsen");
  }
  for (int l = 0; l < c->nlev; ++l) {
    k_diag<<<GL(l)>>>(make_op(c, l), c->lv[l].idu, c->lv[l].idv); c->launches++;
    DIVA_LAUNCHED(c, "k_diag");
  }
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

static int vcycle(Ctx* c, int l, double* xu, double* xv, const double* bu, const double* bv) {
  const int nu1 = 2, nu2 = 2, coarse_sweeps = 64;
  if (l == c->nlev - 1) {
    k_coarse_solve<<<1, 256, 0, c->stream>>>(make_op(c, l), xu, xv, bu, bv, c->lv[l].idu, c->lv[l].idv,
                                             coarse_sweeps); c->launches++;
    DIVA_LAUNCHED(c, "k_coarse_solve");
    return DIVA_OK;
  }
  const Level& L = c->lv[l];
  const Level& K = c->lv[l + 1];
  int st;
  for (int s = 0; s < nu1; ++s)
    if ((st = gs_sweep(c, l, xu, xv, bu, bv, true))) return st;
  k_residual<<<GL(l)>>>(make_op(c, l), xu, xv, bu, bv, L.ru, L.rv); c->launches++;
  DIVA_LAUNCHED(c, "k_residual");
  int fx, fy;
  factors(c, l, &fx, &fy);
  k_restrict<<<GL(l + 1)>>>(L.d, K.d, fx, fy, L.ru, L.rv, K.bu, K.bv, K.xu, K.xv); c->launches++;
  DIVA_LAUNCHED(c, "k_restrict");
  if ((st = vcycle(c, l + 1, K.xu, K.xv, K.bu, K.bv))) return st;
  k_prolong<<<GL(l)>>>(make_op(c, l + 1), L.d, fx, fy, K.xu, K.xv, xu, xv); c->launches++;
  DIVA_LAUNCHED(c, "k_prolong");
  for (int s = 0; s < nu2; ++s)
    if ((st = gs_sweep(c, l, xu, xv, bu, bv, false))) return st;
  return DIVA_OK;
}

// z = M^{-1} r: one V-cycle from zero
static int precond(Ctx* c, const double* ru, const double* rv, double* zu, double* zv) {
  DIVA_CUDA(c, cudaMemsetAsync(zu, 0, sizeof(double) * c->d.plane, c->stream));
  DIVA_CUDA(c, cudaMemsetAsync(zv, 0, sizeof(double) * c->d.plane, c->stream));
  c->mg_cycles++;
  return vcycle(c, 0, zu, zv, ru, rv);
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

// fine-level smoothing sweeps on the Krylov solution vector (used to time the smoother)
int solver_smooth_fine(Ctx* c, int sweeps) {
  for (int s = 0; s < sweeps; ++s) {
    int st = gs_sweep(c, 0, c->kv[KV_X][0], c->kv[KV_X][1], c->kv[KV_B][0], c->kv[KV_B][1], true);
    if (st) return st;
  }
  return DIVA_OK;
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

int solver_fill_boundary(Ctx* c, double* u, double* v) {
  k_fill_boundary<<<grid2d(c->d.ny, c->d.nx), block2d(), 0, c->stream>>>(c->d, c->bc, u, v); c->launches++;
  DIVA_LAUNCHED(c, "k_fill_boundary");
  return DIVA_OK;
}

}  // namespace diva
