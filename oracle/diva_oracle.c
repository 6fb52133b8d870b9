/*
 * diva_oracle.c -- CPU restatement of IMAU-ICE's ice-velocity hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker of the B200
 * library (libdiva_b200.so); only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load it.  The product path never
 * calls it and never falls back to it.
 *
 * It restates, routine by routine and in the reference's loop order
 * (i outer, j inner, k innermost), the Fortran of IMAU-ICE v2.0:
 *   src/ice_velocity_module.f90            solve_SIA/SSA/DIVA and helpers
 *   src/utilities_module.f90               column quadratures, flotation, SOR
 *   src/derivatives_and_grids_module.f90   staggering and derivatives
 *   src/general_ice_model_data_module.f90  masks, flood-fill, grounded fractions
 *   src/basal_conditions_and_sliding_module.f90  hydrology, sliding laws
 *   src/thermodynamics_module.f90          pressure melting point, rheology
 *   src/petsc_module.F90                   PETSc KSP call (restated as GMRES(30)+ILU(0))
 * Each function cites the lines it follows.
 *
 * Parity pinning: the reference cannot be compiled here (no Fortran compiler,
 * MPI, PETSc or NetCDF) and ships no tests or golden vectors, so this oracle is
 * pinned only by known-answer checks written from the reference's own code:
 * the Schoof (2006) SSA ice-stream solution (utilities_module.f90:836-878),
 * exact quadratures on the zeta grid, hand-built grounded-fraction quads and
 * operator identities.  Against reference outputs, parity is unpinned.
 *
 * Conventions: Fortran MAX/MIN with a NaN argument are taken as C fmax/fmin
 * (the non-NaN argument wins), which is what gfortran's expansion of MAX/MIN
 * yields for the calls on this path; e.g. MAX(NaN, visc_eff_min) = visc_eff_min
 * on the first Picard iteration of a cold start (0/0 in du/dz).
 * Build with -ffp-contract=off: no fused multiply-adds, as in the reference.
 */
#define _POSIX_C_SOURCE 200809L   /* pthread barriers under -std=c11 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <time.h>
#include <pthread.h>

#include "../include/diva.h"

/* parameters_module.f90:10-23 */
#define PI_C          3.141592653589793
#define T0_C          273.16
#define CC_C          8.7E-04
#define GRAV          9.81
#define ICE_DENSITY   910.0
#define SW_DENSITY    1028.0
#define R_GAS         8.314

/* mask type codes, configuration_module.f90:3171-3179 */
enum { TYPE_LAND = 0, TYPE_OCEAN = 1, TYPE_LAKE = 2, TYPE_SHEET = 3, TYPE_SHELF = 4,
       TYPE_COAST = 5, TYPE_MARGIN = 6, TYPE_GL = 7, TYPE_CF = 8 };

/* linear solvers of the oracle */
#define ORC_MAX_THREADS 64
struct orc_pool;
enum { ORC_LIN_DIRECT = 0, ORC_LIN_SOR = 1, ORC_LIN_GMRES_ILU = 2, ORC_LIN_GMRES_WARM = 3 };

typedef struct {
  int m, nnz_max, nnz;
  int *ptr, *idx;
  double *val, *b, *x;
} csr_t;

typedef struct orc_ctx {
  diva_grid_t g;
  diva_config_t c;
  int nx, ny, nz;
  double dx;
  void* F[DIVA_NUM_FIELDS];
  void* S[DIVA_NUM_FIELDS];          /* saved state (diva_state_save) */
  /* solution matrix bookkeeping, initialise_SSADIVA_solution_matrix */
  int neq;
  int *ij2n_u, *ij2n_v;              /* (ny,nx-1), (ny-1,nx), 0-based row numbers */
  int *n2ij;                         /* neq x 4: i_u, j_u, i_v, j_v (0-based, -1 unused) */
  csr_t m;
  /* linear solver choice and settings */
  int lin_solver;
  int SOR_nit; double SOR_tol, SOR_omega;
  double petsc_rtol, petsc_abstol;
  int lin_iters_last;
  int true_residual;        /* GMRES tests the true residual (right preconditioning) */
  int threads;              /* threads of the timed CPU baseline (1: the sequential algorithm) */
  struct orc_pool* pool;    /* their workers (NULL with one thread) */
  long lin_iters_total;
  /* Anderson mixing of the viscosity iteration (picard_anderson_m > 0): history columns of
   * residual differences dF and map differences dG (u on cx points then v on cy points),
   * the previous residual f and map value g, and the small least-squares state */
  double *aa_dF[5], *aa_dG[5], *aa_f, *aa_g;
  int aa_have, aa_n, aa_head, aa_restarts, aa_off, aa_since;
  double aa_G[25], aa_rhs[5], aa_gamma[5], aa_rprev, aa_best;
  char err[512];
} orc_ctx;

/* ------------------------------------------------------------------------ */
/* field table                                                               */
static const diva_field_info_t g_info[DIVA_NUM_FIELDS] = {
#define X(ID, name, grid, type) { #name, DIVA_GRID_##grid, DIVA_DTYPE_##type },
  DIVA_FIELD_LIST(X)
#undef X
};

static int64_t numel_kind(int nx, int ny, int nz, int kind) {
  switch (kind) {
    case DIVA_GRID_A:   return (int64_t)ny * nx;
    case DIVA_GRID_CX:  return (int64_t)ny * (nx - 1);
    case DIVA_GRID_CY:  return (int64_t)(ny - 1) * nx;
    case DIVA_GRID_B:   return (int64_t)(ny - 1) * (nx - 1);
    case DIVA_GRID_A3:  return (int64_t)nz * ny * nx;
    case DIVA_GRID_CX3: return (int64_t)nz * ny * (nx - 1);
    case DIVA_GRID_CY3: return (int64_t)nz * (ny - 1) * nx;
    case DIVA_GRID_B3:  return (int64_t)nz * (ny - 1) * (nx - 1);
  }
  return 0;
}

/* index helpers, 0-based, Fortran column-major storage */
#define IA(j, i)      ((size_t)(i) * ny + (j))
#define ICX(j, i)     ((size_t)(i) * ny + (j))
#define ICY(j, i)     ((size_t)(i) * (ny - 1) + (j))
#define IB(j, i)      ((size_t)(i) * (ny - 1) + (j))
#define IA3(k, j, i)  (((size_t)(i) * ny + (j)) * nz + (k))
#define ICX3(k, j, i) (((size_t)(i) * ny + (j)) * nz + (k))
#define ICY3(k, j, i) (((size_t)(i) * (ny - 1) + (j)) * nz + (k))
#define IB3(k, j, i)  (((size_t)(i) * (ny - 1) + (j)) * nz + (k))

#define FD(ctx, ID) ((double*)(ctx)->F[DIVA_F_##ID])
#define FI(ctx, ID) ((int32_t*)(ctx)->F[DIVA_F_##ID])
#define DECL_DIMS(ctx) const int nx = (ctx)->nx, ny = (ctx)->ny, nz = (ctx)->nz; (void)nx; (void)ny; (void)nz

static int fail(orc_ctx* c, int code, const char* msg) {
  if (c) snprintf(c->err, sizeof(c->err), "%s", msg);
  return code;
}

/* ------------------------------------------------------------------------ */
/* column quadratures, utilities_module.f90:21-124                           */

/* vertical_integration_from_bottom_to_zeta, utilities_module.f90:21-46 */
static void vint_bottom_to_zeta(const double* zeta, int nz, const double* f, double* out) {
  out[nz - 1] = 0.0;
  for (int k = nz - 2; k >= 0; --k)
    out[k] = out[k + 1] - 0.5 * (f[k + 1] + f[k]) * (zeta[k + 1] - zeta[k]);
}
/* vertical_integrate, utilities_module.f90:70-95 */
static double vint(const double* zeta, int nz, const double* f) {
  double s = 0.0;
  for (int k = 1; k < nz; ++k) s = s + 0.5 * (f[k] + f[k - 1]) * (zeta[k] - zeta[k - 1]);
  return s;
}
/* vertical_average, utilities_module.f90:96-124 */
static double vavg(const double* zeta, int nz, const double* f) {
  double s = 0.0;
  for (int k = 0; k < nz - 1; ++k) s = s + 0.5 * (f[k + 1] + f[k]) * (zeta[k + 1] - zeta[k]);
  return s;
}

/* flotation functions, utilities_module.f90:126-159 */
static int is_floating(double Hi, double Hb, double SL) {
  return Hi < (SL - Hb) * SW_DENSITY / ICE_DENSITY;
}
static double surface_elevation(double Hi, double Hb, double SL) {
  return Hi + fmax(SL - ICE_DENSITY / SW_DENSITY * Hi, Hb);
}
static double thickness_above_floatation(double Hi, double Hb, double SL) {
  return Hi - fmax(0.0, (SL - Hb) * (SW_DENSITY / ICE_DENSITY));
}

/* calc_staggered_margin, ice_velocity_module.f90:1300-1319 */
static double stag_margin(double v0, double v1, double H0, double H1) {
  if (H0 > 0.0 && H1 == 0.0) return v0;
  if (H0 == 0.0 && H1 > 0.0) return v1;
  return 0.5 * (v0 + v1);
}

/* ------------------------------------------------------------------------ */
/* grid operators, derivatives_and_grids_module.f90                           */

/* ddx_a_to_a_2D :24-58 */
static void ddx_a_to_a(int nx, int ny, double dx, const double* d, double* o) {
  for (int i = 1; i < nx - 1; ++i)
    for (int j = 0; j < ny; ++j) o[IA(j, i)] = (d[IA(j, i + 1)] - d[IA(j, i - 1)]) / (2 * dx);
  for (int j = 0; j < ny; ++j) {
    o[IA(j, 0)] = (d[IA(j, 1)] - d[IA(j, 0)]) / dx;
    o[IA(j, nx - 1)] = (d[IA(j, nx - 1)] - d[IA(j, nx - 2)]) / dx;
  }
}
/* ddy_a_to_a_2D :59-93 */
static void ddy_a_to_a(int nx, int ny, double dx, const double* d, double* o) {
  for (int i = 0; i < nx; ++i)
    for (int j = 1; j < ny - 1; ++j) o[IA(j, i)] = (d[IA(j + 1, i)] - d[IA(j - 1, i)]) / (2 * dx);
  for (int i = 0; i < nx; ++i) {
    o[IA(0, i)] = (d[IA(1, i)] - d[IA(0, i)]) / dx;
    o[IA(ny - 1, i)] = (d[IA(ny - 1, i)] - d[IA(ny - 2, i)]) / dx;
  }
}
/* ddx_a_to_cx_2D :478-506 */
static void ddx_a_to_cx(int nx, int ny, double dx, const double* d, double* o) {
  for (int i = 0; i < nx - 1; ++i)
    for (int j = 0; j < ny; ++j) o[ICX(j, i)] = (d[IA(j, i + 1)] - d[IA(j, i)]) / dx;
}
/* ddy_a_to_cy_2D :507-535 */
static void ddy_a_to_cy(int nx, int ny, double dx, const double* d, double* o) {
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny - 1; ++j) o[ICY(j, i)] = (d[IA(j + 1, i)] - d[IA(j, i)]) / dx;
}
/* ddx_a_to_cy_2D :536-572 */
static void ddx_a_to_cy(int nx, int ny, double dx, const double* d, double* o) {
  for (int i = 1; i < nx - 1; ++i)
    for (int j = 0; j < ny - 1; ++j)
      o[ICY(j, i)] = (d[IA(j, i + 1)] + d[IA(j + 1, i + 1)] - d[IA(j, i - 1)] - d[IA(j + 1, i - 1)]) / (4.0 * dx);
  for (int j = 0; j < ny - 1; ++j) {
    o[ICY(j, 0)] = (d[IA(j, 1)] + d[IA(j + 1, 1)] - d[IA(j, 0)] - d[IA(j + 1, 0)]) / (2.0 * dx);
    o[ICY(j, nx - 1)] = (d[IA(j, nx - 1)] + d[IA(j + 1, nx - 1)] - d[IA(j, nx - 2)] - d[IA(j + 1, nx - 2)]) / (2.0 * dx);
  }
}
/* ddy_a_to_cx_2D :573-610 */
static void ddy_a_to_cx(int nx, int ny, double dx, const double* d, double* o) {
  for (int i = 0; i < nx - 1; ++i)
    for (int j = 1; j < ny - 1; ++j)
      o[ICX(j, i)] = (d[IA(j + 1, i)] + d[IA(j + 1, i + 1)] - d[IA(j - 1, i)] - d[IA(j - 1, i + 1)]) / (4.0 * dx);
  for (int i = 0; i < nx - 1; ++i) {
    o[ICX(0, i)] = (d[IA(1, i)] + d[IA(1, i + 1)] - d[IA(0, i)] - d[IA(0, i + 1)]) / (2.0 * dx);
    o[ICX(ny - 1, i)] = (d[IA(ny - 1, i)] + d[IA(ny - 1, i + 1)] - d[IA(ny - 2, i)] - d[IA(ny - 2, i + 1)]) / (2.0 * dx);
  }
}
/* ddx_cx_to_a_2D :755-787 */
static void ddx_cx_to_a(int nx, int ny, double dx, const double* d, double* o) {
  for (int i = 1; i < nx - 1; ++i)
    for (int j = 0; j < ny; ++j) o[IA(j, i)] = (d[ICX(j, i)] - d[ICX(j, i - 1)]) / dx;
  for (int j = 0; j < ny; ++j) {
    o[IA(j, 0)] = o[IA(j, 1)];
    o[IA(j, nx - 1)] = o[IA(j, nx - 2)];
  }
}
/* ddy_cy_to_a_2D :788-820 */
static void ddy_cy_to_a(int nx, int ny, double dx, const double* d, double* o) {
  for (int i = 0; i < nx; ++i)
    for (int j = 1; j < ny - 1; ++j) o[IA(j, i)] = (d[ICY(j, i)] - d[ICY(j - 1, i)]) / dx;
  for (int i = 0; i < nx; ++i) {
    o[IA(0, i)] = o[IA(1, i)];
    o[IA(ny - 1, i)] = o[IA(ny - 2, i)];
  }
}
/* ddy_cx_to_a_2D :821-879 (the reference's 4dx denominators on the edges are kept) */
static void ddy_cx_to_a(int nx, int ny, double dx, const double* d, double* o) {
  for (int i = 1; i < nx - 1; ++i)
    for (int j = 1; j < ny - 1; ++j)
      o[IA(j, i)] = (d[ICX(j + 1, i - 1)] + d[ICX(j + 1, i)] - d[ICX(j - 1, i - 1)] - d[ICX(j - 1, i)]) / (4.0 * dx);
  for (int i = 1; i < nx - 1; ++i) {
    int j = 0;
    o[IA(j, i)] = (d[ICX(j + 1, i - 1)] + d[ICX(j + 1, i)] - d[ICX(j, i - 1)] - d[ICX(j, i)]) / (4.0 * dx);
    j = ny - 1;
    o[IA(j, i)] = (d[ICX(j, i - 1)] + d[ICX(j, i)] - d[ICX(j - 1, i - 1)] - d[ICX(j - 1, i)]) / (4.0 * dx);
  }
  for (int j = 1; j < ny - 1; ++j) {
    int i = 0;
    o[IA(j, i)] = (d[ICX(j + 1, i)] - d[ICX(j - 1, i)]) / (2.0 * dx);
    i = nx - 1;
    o[IA(j, i)] = (d[ICX(j + 1, i - 1)] - d[ICX(j - 1, i - 1)]) / (2.0 * dx);
  }
  o[IA(0, 0)] = (d[ICX(1, 0)] - d[ICX(0, 0)]) / dx;
  o[IA(0, nx - 1)] = (d[ICX(1, nx - 2)] - d[ICX(0, nx - 2)]) / dx;
  o[IA(ny - 1, 0)] = (d[ICX(ny - 1, 0)] - d[ICX(ny - 2, 0)]) / dx;
  o[IA(ny - 1, nx - 1)] = (d[ICX(ny - 1, nx - 2)] - d[ICX(ny - 2, nx - 2)]) / dx;
}
/* ddx_cy_to_a_2D :880-939 */
static void ddx_cy_to_a(int nx, int ny, double dx, const double* d, double* o) {
  for (int i = 1; i < nx - 1; ++i)
    for (int j = 1; j < ny - 1; ++j)
      o[IA(j, i)] = (d[ICY(j - 1, i + 1)] + d[ICY(j, i + 1)] - d[ICY(j - 1, i - 1)] - d[ICY(j, i - 1)]) / (4.0 * dx);
  for (int j = 1; j < ny - 1; ++j) {
    int i = 0;
    o[IA(j, i)] = (d[ICY(j - 1, i + 1)] + d[ICY(j, i + 1)] - d[ICY(j - 1, i)] - d[ICY(j, i)]) / (4.0 * dx);
    i = nx - 1;
    o[IA(j, i)] = (d[ICY(j - 1, i)] + d[ICY(j, i)] - d[ICY(j - 1, i - 1)] - d[ICY(j, i - 1)]) / (4.0 * dx);
  }
  for (int i = 1; i < nx - 1; ++i) {
    int j = 0;
    o[IA(j, i)] = (d[ICY(j, i + 1)] - d[ICY(j, i - 1)]) / (2.0 * dx);
    j = ny - 1;
    o[IA(j, i)] = (d[ICY(j - 1, i + 1)] - d[ICY(j - 1, i - 1)]) / (2.0 * dx);
  }
  o[IA(0, 0)] = (d[ICY(0, 1)] - d[ICY(0, 0)]) / dx;
  o[IA(0, nx - 1)] = (d[ICY(0, nx - 1)] - d[ICY(0, nx - 2)]) / dx;
  o[IA(ny - 1, 0)] = (d[ICY(ny - 2, 1)] - d[ICY(ny - 2, 0)]) / dx;
  o[IA(ny - 1, nx - 1)] = (d[ICY(ny - 2, nx - 1)] - d[ICY(ny - 2, nx - 2)]) / dx;
}
/* map_a_to_cx_2D :1454-1482 */
static void map_a_to_cx(int nx, int ny, const double* d, double* o) {
  for (int i = 0; i < nx - 1; ++i)
    for (int j = 0; j < ny; ++j) o[ICX(j, i)] = (d[IA(j, i)] + d[IA(j, i + 1)]) / 2.0;
}
/* map_a_to_cy_2D :1483-1512 */
static void map_a_to_cy(int nx, int ny, const double* d, double* o) {
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny - 1; ++j) o[ICY(j, i)] = (d[IA(j, i)] + d[IA(j + 1, i)]) / 2.0;
}
/* map_a_to_cx_3D / map_a_to_cy_3D :1513-1578 */
static void map_a_to_cx_3d(int nx, int ny, int nz, const double* d, double* o) {
  for (int i = 0; i < nx - 1; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) o[ICX3(k, j, i)] = (d[IA3(k, j, i)] + d[IA3(k, j, i + 1)]) / 2.0;
}
static void map_a_to_cy_3d(int nx, int ny, int nz, const double* d, double* o) {
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny - 1; ++j)
      for (int k = 0; k < nz; ++k) o[ICY3(k, j, i)] = (d[IA3(k, j, i)] + d[IA3(k, j + 1, i)]) / 2.0;
}
/* map_cx_to_a_2D :1579-1611 */
static void map_cx_to_a(int nx, int ny, const double* d, double* o) {
  for (int i = 1; i < nx - 1; ++i)
    for (int j = 0; j < ny; ++j) o[IA(j, i)] = (d[ICX(j, i - 1)] + d[ICX(j, i)]) / 2.0;
  for (int j = 0; j < ny; ++j) {
    o[IA(j, 0)] = d[ICX(j, 0)];
    o[IA(j, nx - 1)] = d[ICX(j, nx - 2)];
  }
}
/* map_cy_to_a_2D :1612-1645 */
static void map_cy_to_a(int nx, int ny, const double* d, double* o) {
  for (int i = 0; i < nx; ++i)
    for (int j = 1; j < ny - 1; ++j) o[IA(j, i)] = (d[ICY(j - 1, i)] + d[ICY(j, i)]) / 2.0;
  for (int i = 0; i < nx; ++i) {
    o[IA(0, i)] = d[ICY(0, i)];
    o[IA(ny - 1, i)] = d[ICY(ny - 2, i)];
  }
}
/* map_cx_to_cy_2D :1718-1756 */
static void map_cx_to_cy(int nx, int ny, const double* d, double* o) {
  for (int i = 1; i < nx - 1; ++i)
    for (int j = 0; j < ny - 1; ++j)
      o[ICY(j, i)] = (d[ICX(j, i - 1)] + d[ICX(j, i)] + d[ICX(j + 1, i - 1)] + d[ICX(j + 1, i)]) / 4.0;
  for (int j = 0; j < ny - 1; ++j) {
    o[ICY(j, 0)] = (d[ICX(j, 0)] + d[ICX(j + 1, 0)]) / 2.0;
    o[ICY(j, nx - 1)] = (d[ICX(j, nx - 2)] + d[ICX(j + 1, nx - 2)]) / 2.0;
  }
}
/* map_cy_to_cx_2D :1757-1797 */
static void map_cy_to_cx(int nx, int ny, const double* d, double* o) {
  for (int i = 0; i < nx - 1; ++i)
    for (int j = 1; j < ny - 1; ++j)
      o[ICX(j, i)] = (d[ICY(j - 1, i)] + d[ICY(j - 1, i + 1)] + d[ICY(j, i)] + d[ICY(j, i + 1)]) / 4.0;
  for (int i = 0; i < nx - 1; ++i) {
    o[ICX(0, i)] = (d[ICY(0, i)] + d[ICY(0, i + 1)]) / 2.0;
    o[ICX(ny - 1, i)] = (d[ICY(ny - 2, i)] + d[ICY(ny - 2, i + 1)]) / 2.0;
  }
}
/* map_a_to_b_2D :1798-1827 */
static void map_a_to_b(int nx, int ny, const double* d, double* o) {
  for (int i = 0; i < nx - 1; ++i)
    for (int j = 0; j < ny - 1; ++j)
      o[IB(j, i)] = (d[IA(j, i)] + d[IA(j, i + 1)] + d[IA(j + 1, i)] + d[IA(j + 1, i + 1)]) / 4.0;
}

/* ------------------------------------------------------------------------ */
/* masks, general_ice_model_data_module.f90                                  */

/* ocean_floodfill :868-988 (stack flood-fill from all domain edges, 8-connectivity) */
static void ocean_floodfill(orc_ctx* c) {
  DECL_DIMS(c);
  const double *Hi = FD(c, HI_A), *Hb = FD(c, HB_A), *SL = FD(c, SL_A);
  int32_t *land = FI(c, MASK_LAND_A), *ocean = FI(c, MASK_OCEAN_A), *mask = FI(c, MASK_A);
  int32_t* map = (int32_t*)calloc((size_t)nx * ny, sizeof(int32_t));
  int32_t* stack = (int32_t*)malloc(sizeof(int32_t) * 2 * ((size_t)nx * ny + 2 * (nx + ny) + 8));
  int n = 0;
  for (size_t q = 0; q < (size_t)nx * ny; ++q) { land[q] = 1; ocean[q] = 0; mask[q] = TYPE_LAND; }
  for (int i = 0; i < nx; ++i) {
    int j = 0;      stack[2 * n] = i; stack[2 * n + 1] = j; ++n; map[IA(j, i)] = 1;
    j = ny - 1;     stack[2 * n] = i; stack[2 * n + 1] = j; ++n; map[IA(j, i)] = 1;
  }
  for (int j = 0; j < ny; ++j) {
    int i = 0;      stack[2 * n] = i; stack[2 * n + 1] = j; ++n; map[IA(j, i)] = 1;
    i = nx - 1;     stack[2 * n] = i; stack[2 * n + 1] = j; ++n; map[IA(j, i)] = 1;
  }
  while (n > 0) {
    --n;
    int i = stack[2 * n], j = stack[2 * n + 1];
    if (is_floating(Hi[IA(j, i)], Hb[IA(j, i)], SL[IA(j, i)])) {
      map[IA(j, i)] = 2;
      ocean[IA(j, i)] = 1; land[IA(j, i)] = 0; mask[IA(j, i)] = TYPE_OCEAN;
      for (int ii = i - 1; ii <= i + 1; ++ii)
        for (int jj = j - 1; jj <= j + 1; ++jj) {
          if (ii >= 0 && ii < nx && jj >= 0 && jj < ny && !(ii == i && jj == j)) {
            if (map[IA(jj, ii)] == 0) {
              map[IA(jj, ii)] = 1;
              stack[2 * n] = ii; stack[2 * n + 1] = jj; ++n;
            }
          }
        }
    }
  }
  free(map); free(stack);
}

/* determine_masks_landocean :110-158 */
static void determine_masks_landocean(orc_ctx* c) {
  DECL_DIMS(c);
  int32_t *land = FI(c, MASK_LAND_A), *ocean = FI(c, MASK_OCEAN_A);
  for (size_t q = 0; q < (size_t)nx * ny; ++q) { land[q] = 1; ocean[q] = 0; }
  if (c->c.do_ocean_floodfill) {
    ocean_floodfill(c);
  } else {
    const double *Hi = FD(c, HI_A), *Hb = FD(c, HB_A), *SL = FD(c, SL_A);
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j)
        if (is_floating(Hi[IA(j, i)], Hb[IA(j, i)], SL[IA(j, i)])) { land[IA(j, i)] = 0; ocean[IA(j, i)] = 1; }
  }
}

/* determine_masks_ice :159-207 */
static void determine_masks_ice(orc_ctx* c) {
  DECL_DIMS(c);
  determine_masks_landocean(c);
  const double* Hi = FD(c, HI_A);
  int32_t *land = FI(c, MASK_LAND_A), *ocean = FI(c, MASK_OCEAN_A);
  int32_t *ice = FI(c, MASK_ICE_A), *sheet = FI(c, MASK_SHEET_A), *shelf = FI(c, MASK_SHELF_A);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      size_t q = IA(j, i);
      ice[q] = 0; sheet[q] = 0; shelf[q] = 0;
      if (Hi[q] > DBL_MIN) ice[q] = 1;                       /* TINY(1._dp) */
      if (ice[q] == 1 && land[q] == 1) sheet[q] = 1;
      if (ice[q] == 1 && ocean[q] == 1) shelf[q] = 1;
    }
}

/* determine_masks_transitions :208-285 (interior only) */
static void determine_masks_transitions(orc_ctx* c) {
  DECL_DIMS(c);
  determine_masks_landocean(c);
  int32_t *land = FI(c, MASK_LAND_A), *ocean = FI(c, MASK_OCEAN_A), *ice = FI(c, MASK_ICE_A);
  int32_t *sheet = FI(c, MASK_SHEET_A), *shelf = FI(c, MASK_SHELF_A);
  int32_t *coast = FI(c, MASK_COAST_A), *margin = FI(c, MASK_MARGIN_A), *gl = FI(c, MASK_GL_A), *cf = FI(c, MASK_CF_A);
  for (size_t q = 0; q < (size_t)nx * ny; ++q) { coast[q] = 0; margin[q] = 0; gl[q] = 0; cf[q] = 0; }
  for (int i = 1; i < nx - 1; ++i)
    for (int j = 1; j < ny - 1; ++j) {
      size_t q = IA(j, i), s = IA(j - 1, i), n = IA(j + 1, i), w = IA(j, i - 1), e = IA(j, i + 1);
      if (land[q] == 1 && ice[q] == 0)
        if (ocean[s] == 1 || ocean[n] == 1 || ocean[w] == 1 || ocean[e] == 1) coast[q] = 1;
      if (ice[q] == 1)
        if (ice[s] == 0 || ice[n] == 0 || ice[w] == 0 || ice[e] == 0) margin[q] = 1;
      if (sheet[q] == 1)
        if (shelf[s] == 1 || shelf[n] == 1 || shelf[w] == 1 || shelf[e] == 1) gl[q] = 1;
      if (ice[q] == 1)
        if ((ocean[s] == 1 && ice[s] == 0) || (ocean[n] == 1 && ice[n] == 0) ||
            (ocean[w] == 1 && ice[w] == 0) || (ocean[e] == 1 && ice[e] == 0)) cf[q] = 1;
    }
}

/* determine_masks_total :286-347 */
static void determine_masks_total(orc_ctx* c) {
  DECL_DIMS(c);
  int32_t *land = FI(c, MASK_LAND_A), *coast = FI(c, MASK_COAST_A), *sheet = FI(c, MASK_SHEET_A);
  int32_t *shelf = FI(c, MASK_SHELF_A), *margin = FI(c, MASK_MARGIN_A), *gl = FI(c, MASK_GL_A);
  int32_t *cf = FI(c, MASK_CF_A), *mask = FI(c, MASK_A);
  for (size_t q = 0; q < (size_t)nx * ny; ++q) {
    mask[q] = (land[q] == 1) ? TYPE_LAND : TYPE_OCEAN;
    if (coast[q] == 1) mask[q] = TYPE_COAST;
    if (sheet[q] == 1) mask[q] = TYPE_SHEET;
    else if (shelf[q] == 1) mask[q] = TYPE_SHELF;
    if (margin[q] == 1) mask[q] = TYPE_MARGIN;
    if (gl[q] == 1) mask[q] = TYPE_GL;
    if (cf[q] == 1) mask[q] = TYPE_CF;
  }
}

/* update_general_ice_model_data :30-86 */
int orc_update_general_ice_model_data(orc_ctx* c) {
  DECL_DIMS(c);
  const double dx = c->dx;
  const double *Hi = FD(c, HI_A), *Hb = FD(c, HB_A), *SL = FD(c, SL_A);
  double *Hs = FD(c, HS_A), *TAF = FD(c, TAF_A);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      size_t q = IA(j, i);
      Hs[q] = surface_elevation(Hi[q], Hb[q], SL[q]);
      TAF[q] = thickness_above_floatation(Hi[q], Hb[q], SL[q]);
    }
  /* determine_masks :87-109 */
  determine_masks_landocean(c);
  determine_masks_ice(c);
  determine_masks_transitions(c);
  determine_masks_total(c);

  map_a_to_cx(nx, ny, Hi, FD(c, HI_CX));
  map_a_to_cy(nx, ny, Hi, FD(c, HI_CY));
  map_a_to_b(nx, ny, Hi, FD(c, HI_B));
  map_a_to_cx_3d(nx, ny, nz, FD(c, A_FLOW_3D_A), FD(c, A_FLOW_3D_CX));
  map_a_to_cy_3d(nx, ny, nz, FD(c, A_FLOW_3D_A), FD(c, A_FLOW_3D_CY));
  map_a_to_cx(nx, ny, FD(c, A_FLOW_VAV_A), FD(c, A_FLOW_VAV_CX));
  map_a_to_cy(nx, ny, FD(c, A_FLOW_VAV_A), FD(c, A_FLOW_VAV_CY));
  ddx_a_to_a(nx, ny, dx, Hi, FD(c, DHI_DX_A));
  ddy_a_to_a(nx, ny, dx, Hi, FD(c, DHI_DY_A));
  ddx_a_to_a(nx, ny, dx, Hs, FD(c, DHS_DX_A));
  ddy_a_to_a(nx, ny, dx, Hs, FD(c, DHS_DY_A));
  ddx_a_to_cx(nx, ny, dx, Hs, FD(c, DHS_DX_CX));
  ddy_a_to_cx(nx, ny, dx, Hs, FD(c, DHS_DY_CX));
  ddx_a_to_cy(nx, ny, dx, Hs, FD(c, DHS_DX_CY));
  ddy_a_to_cy(nx, ny, dx, Hs, FD(c, DHS_DY_CY));
  return DIVA_OK;
}

/* ------------------------------------------------------------------------ */
/* grounded fractions, general_ice_model_data_module.f90:349-783             */

/* rotate_quad :767-783 (anticlockwise by 90 degrees) */
static void rotate_quad(double* NW, double* NE, double* SW, double* SE) {
  double f1 = *NW, f2 = *NE, f3 = *SE, f4 = *SW;
  *NW = f2; *NE = f3; *SE = f4; *SW = f1;
}
/* rotate_quad_until_match :712-766; returns scenario 1..4, or 0 if none after 4 turns */
static int rotate_quad_until_match(double* NW, double* NE, double* SW, double* SE) {
  for (int nit = 1; nit <= 4; ++nit) {
    rotate_quad(NW, NE, SW, SE);
    if (*SW > 0.0 && *SE < 0.0 && *NE < 0.0 && *NW < 0.0) return 1;
    if (*SW < 0.0 && *SE > 0.0 && *NE > 0.0 && *NW > 0.0) return 2;
    if (*SW > 0.0 && *SE > 0.0 && *NE < 0.0 && *NW < 0.0) return 3;
    if (*SW > 0.0 && *SE < 0.0 && *NE > 0.0 && *NW < 0.0) return 4;
  }
  return 0;
}
static double nudge(double f, double t) {
  if (f == 0.0) return t;
  if (f > 0.0) return fmax(t, f);
  if (f < 0.0) return fmin(-t, f);
  return f;
}
/* calc_fraction_above_zero :521-711 */
double orc_calc_fraction_above_zero(double f_NW, double f_NE, double f_SW, double f_SE) {
  const double ftol = 1E-4;
  double NW = nudge(f_NW, ftol * 1.1), NE = nudge(f_NE, ftol * 1.21);
  double SW = nudge(f_SW, ftol * 1.13), SE = nudge(f_SE, ftol * 0.97);
  double phi, aa, bb, cc, dd, x, f1, f2;
  if (NW >= 0.0 && NE >= 0.0 && SW >= 0.0 && SE >= 0.0) {
    phi = 1.0;
  } else if (NW <= 0.0 && NE <= 0.0 && SW <= 0.0 && SE <= 0.0) {
    phi = 0.0;
  } else {
    int scen = rotate_quad_until_match(&NW, &NE, &SW, &SE);
    if (scen == 1) {
      aa = SW; bb = SE - SW; cc = NW - SW; dd = NE + SW - NW - SE;
      phi = ((bb * cc - aa * dd) * log(fabs(1.0 - (aa * dd) / (bb * cc))) + aa * dd) / (dd * dd);
      if (fabs(dd) < 1E-4) {
        if (SW > 0.0) SW = SW + 0.1; else SW = SW - 0.1;
        aa = SW; bb = SE - SW; cc = NW - SW; dd = NE + SW - NW - SE;
        phi = ((bb * cc - aa * dd) * log(fabs(1.0 - (aa * dd) / (bb * cc))) + aa * dd) / (dd * dd);
      }
    } else if (scen == 2) {
      aa = -(SW); bb = -(SE - SW); cc = -(NW - SW); dd = -(NE + SW - NW - SE);
      phi = 1.0 - ((bb * cc - aa * dd) * log(fabs(1.0 - (aa * dd) / (bb * cc))) + aa * dd) / (dd * dd);
      if (fabs(dd) < 1E-4) {
        if (SW > 0.0) SW = SW + 0.1; else SW = SW - 0.1;
        aa = -(SW); bb = -(SE - SW); cc = -(NW - SW); dd = -(NE + SW - NW - SE);
        phi = 1.0 - ((bb * cc - aa * dd) * log(fabs(1.0 - (aa * dd) / (bb * cc))) + aa * dd) / (dd * dd);
      }
    } else if (scen == 3) {
      if (fabs(1.0 - NW / NE) < 1E-6 && fabs(1.0 - SW / SE) < 1E-6) {
        phi = SW / (SW - NW);
      } else {
        aa = SW; bb = SE - SW; cc = NW - SW; dd = NE + SW - NW - SE;
        x = 0.0; f1 = ((bb * cc - aa * dd) * log(fabs(cc + dd * x)) - bb * dd * x) / (dd * dd);
        x = 1.0; f2 = ((bb * cc - aa * dd) * log(fabs(cc + dd * x)) - bb * dd * x) / (dd * dd);
        phi = f2 - f1;
        if (fabs(dd) < 1E-4) {
          if (SW > 0.0) SW = SW + 0.1; else SW = SW - 0.1;
          aa = SW; bb = SE - SW; cc = NW - SW; dd = NE + SW - NW - SE;
          x = 0.0; f1 = ((bb * cc - aa * dd) * log(fabs(cc + dd * x)) - bb * dd * x) / (dd * dd);
          x = 1.0; f2 = ((bb * cc - aa * dd) * log(fabs(cc + dd * x)) - bb * dd * x) / (dd * dd);
          phi = f2 - f1;
        }
      }
    } else if (scen == 4) {
      aa = SW; bb = SE - SW; cc = NW - SW; dd = NE + SW - NW - SE;
      phi = ((bb * cc - aa * dd) * log(fabs(1.0 - (aa * dd) / (bb * cc))) + aa * dd) / (dd * dd);
      rotate_quad(&NW, &NE, &SW, &SE);
      rotate_quad(&NW, &NE, &SW, &SE);
      aa = SW; bb = SE - SW; cc = NW - SW; dd = NE + SW - NW - SE;
      phi = phi + ((bb * cc - aa * dd) * log(fabs(1.0 - (aa * dd) / (bb * cc))) + aa * dd) / (dd * dd);
    } else {
      phi = NAN;  /* the reference crashes ('couldnt find matching scenario') */
    }
  }
  return fmax(0.0, fmin(1.0, phi));
}

/* determine_grounded_fractions :349-419 with ..._CISM_quads :420-520 */
static void determine_grounded_fractions(orc_ctx* c) {
  DECL_DIMS(c);
  const double* TAF = FD(c, TAF_A);
  const int ex = ny + 2;
  double* T = (double*)malloc(sizeof(double) * (size_t)(nx + 2) * ex);
  double *qNW = (double*)malloc(sizeof(double) * (size_t)nx * ny), *qNE = (double*)malloc(sizeof(double) * (size_t)nx * ny);
  double *qSW = (double*)malloc(sizeof(double) * (size_t)nx * ny), *qSE = (double*)malloc(sizeof(double) * (size_t)nx * ny);
#define TE(jj, ii) T[(size_t)(ii) * ex + (jj)]
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) TE(j + 1, i + 1) = TAF[IA(j, i)];
  for (int j = 0; j < ny; ++j) { TE(j + 1, 0) = TAF[IA(j, 0)]; TE(j + 1, nx + 1) = TAF[IA(j, nx - 1)]; }
  for (int i = 0; i < nx; ++i) { TE(0, i + 1) = TAF[IA(0, i)]; TE(ny + 1, i + 1) = TAF[IA(ny - 1, i)]; }
  TE(0, 0) = TAF[IA(0, 0)];
  TE(0, nx + 1) = TAF[IA(0, nx - 1)];
  TE(ny + 1, 0) = TAF[IA(ny - 1, 0)];
  TE(ny + 1, nx + 1) = TAF[IA(ny - 1, nx - 1)];
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      int ii = i + 1, jj = j + 1;
      double f_NW = 0.25 * (TE(jj + 1, ii - 1) + TE(jj + 1, ii) + TE(jj, ii - 1) + TE(jj, ii));
      double f_N  = 0.5  * (TE(jj + 1, ii) + TE(jj, ii));
      double f_NE = 0.25 * (TE(jj + 1, ii) + TE(jj + 1, ii + 1) + TE(jj, ii) + TE(jj, ii + 1));
      double f_W  = 0.5  * (TE(jj, ii - 1) + TE(jj, ii));
      double f_m  = TE(jj, ii);
      double f_E  = 0.5  * (TE(jj, ii) + TE(jj, ii + 1));
      double f_SW = 0.25 * (TE(jj, ii - 1) + TE(jj, ii) + TE(jj - 1, ii - 1) + TE(jj - 1, ii));
      double f_S  = 0.5  * (TE(jj, ii) + TE(jj - 1, ii));
      double f_SE = 0.25 * (TE(jj, ii) + TE(jj, ii + 1) + TE(jj - 1, ii) + TE(jj - 1, ii + 1));
      qNW[IA(j, i)] = orc_calc_fraction_above_zero(f_NW, f_N, f_W, f_m);
      qNE[IA(j, i)] = orc_calc_fraction_above_zero(f_N, f_NE, f_m, f_E);
      qSW[IA(j, i)] = orc_calc_fraction_above_zero(f_W, f_m, f_SW, f_S);
      qSE[IA(j, i)] = orc_calc_fraction_above_zero(f_m, f_E, f_S, f_SE);
    }
#undef TE
  double *fa = FD(c, F_GRND_A), *fcx = FD(c, F_GRND_CX), *fcy = FD(c, F_GRND_CY), *fb = FD(c, F_GRND_B);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      fa[IA(j, i)] = 0.25 * (qNW[IA(j, i)] + qNE[IA(j, i)] + qSW[IA(j, i)] + qSE[IA(j, i)]);
      if (i < nx - 1) fcx[ICX(j, i)] = 0.25 * (qNE[IA(j, i)] + qSE[IA(j, i)] + qNW[IA(j, i + 1)] + qSW[IA(j, i + 1)]);
      if (j < ny - 1) fcy[ICY(j, i)] = 0.25 * (qNE[IA(j, i)] + qNW[IA(j, i)] + qSE[IA(j + 1, i)] + qSW[IA(j + 1, i)]);
      if (i < nx - 1 && j < ny - 1)
        fb[IB(j, i)] = 0.25 * (qNE[IA(j, i)] + qNW[IA(j, i + 1)] + qSE[IA(j + 1, i)] + qSW[IA(j + 1, i + 1)]);
    }
  free(T); free(qNW); free(qNE); free(qSW); free(qSE);
}

/* ------------------------------------------------------------------------ */
/* thermodynamics_module.f90                                                 */

/* calc_pressure_melting_point :609-640 */
int orc_calc_pressure_melting_point(orc_ctx* c) {
  DECL_DIMS(c);
  const double* Hi = FD(c, HI_A);
  double* Tp = FD(c, TI_PMP_A);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) Tp[IA3(k, j, i)] = T0_C - CC_C * Hi[IA(j, i)] * c->g.zeta[k];
  return DIVA_OK;
}

/* calc_ice_rheology :641-753 ('uniform' and 'Huybrechts1992') */
int orc_calc_ice_rheology(orc_ctx* c) {
  DECL_DIMS(c);
  const double A_low = 1.14E-05, A_high = 5.47E+10, Q_low = 6.0E+04, Q_high = 13.9E+04;
  const double* Ti = FD(c, TI_A);
  double* A = FD(c, A_FLOW_3D_A);
  const int32_t *ice = FI(c, MASK_ICE_A), *sheet = FI(c, MASK_SHEET_A), *shelf = FI(c, MASK_SHELF_A);
  if (c->c.choice_ice_rheology == DIVA_RHEO_UNIFORM) {
    for (size_t q = 0; q < (size_t)nx * ny * nz; ++q) A[q] = c->c.uniform_flow_factor;
  } else if (c->c.choice_ice_rheology == DIVA_RHEO_HUYBRECHTS1992) {
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) {
          size_t q = IA3(k, j, i);
          if (ice[IA(j, i)] == 1) {
            if (Ti[q] < 263.15) A[q] = A_low * exp(-Q_low / (R_GAS * Ti[q]));
            else                A[q] = A_high * exp(-Q_high / (R_GAS * Ti[q]));
          } else {
            if (c->c.choice_ice_margin == DIVA_MARGIN_BC) A[q] = 0.0;
            else A[q] = A_low * exp(-Q_low / (R_GAS * 263.15));
          }
        }
  } else {
    return fail(c, DIVA_BAD_INPUT, "unknown choice_ice_rheology");
  }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      double m = 1.0; int apply = 0;
      if (sheet[IA(j, i)] == 1) { m = c->c.m_enh_sheet; apply = 1; }
      else if (shelf[IA(j, i)] == 1) { m = c->c.m_enh_shelf; apply = 1; }
      if (apply) for (int k = 0; k < nz; ++k) A[IA3(k, j, i)] = A[IA3(k, j, i)] * m;
    }
  double* Av = FD(c, A_FLOW_VAV_A);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) Av[IA(j, i)] = vavg(c->g.zeta, nz, &A[IA3(0, j, i)]);
  map_a_to_cx_3d(nx, ny, nz, A, FD(c, A_FLOW_3D_CX));
  map_a_to_cy_3d(nx, ny, nz, A, FD(c, A_FLOW_3D_CY));
  map_a_to_cx(nx, ny, Av, FD(c, A_FLOW_VAV_CX));
  map_a_to_cy(nx, ny, Av, FD(c, A_FLOW_VAV_CY));
  return DIVA_OK;
}

/* ------------------------------------------------------------------------ */
/* basal conditions, basal_conditions_and_sliding_module.f90                 */

/* calc_basal_hydrology :90-143 (+ :173-227); calc_bed_roughness is 'prescribed' here */
static int calc_basal_conditions(orc_ctx* c) {
  DECL_DIMS(c);
  const double *Hi = FD(c, HI_A), *Hb = FD(c, HB_A), *SL = FD(c, SL_A);
  double *pwp = FD(c, PORE_WATER_PRESSURE_A), *ob = FD(c, OVERBURDEN_PRESSURE_A), *Neff = FD(c, NEFF_A);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      size_t q = IA(j, i);
      if (c->c.choice_basal_hydrology == DIVA_HYDRO_DRY) {
        pwp[q] = 0.0;
      } else if (c->c.choice_basal_hydrology == DIVA_HYDRO_SATURATED) {
        pwp[q] = -SW_DENSITY * GRAV * (SL[q] - Hb[q]);
      } else {
        double lambda_p = fmin(1.0, fmax(0.0, 1.0 - (Hb[q] - SL[q] - c->c.Martin2011_hydro_Hb_min) /
                                              (c->c.Martin2011_hydro_Hb_max - c->c.Martin2011_hydro_Hb_min)));
        pwp[q] = 0.96 * ICE_DENSITY * GRAV * Hi[q] * lambda_p;
      }
    }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      size_t q = IA(j, i);
      ob[q] = ICE_DENSITY * GRAV * Hi[q];
      Neff[q] = fmax(0.0, ob[q] - pwp[q]);
    }
  return DIVA_OK;
}

/* calc_sliding_law :908-957 and the laws :958-1236 */
static void calc_sliding_law(orc_ctx* c, const double* u_a, const double* v_a, double* beta_a) {
  DECL_DIMS(c);
  const diva_config_t* C = &c->c;
  const double *bsq = FD(c, BETA_SQ_A), *phi = FD(c, PHI_FRIC_A), *asq = FD(c, ALPHA_SQ_A), *Neff = FD(c, NEFF_A);
  double* tauc = FD(c, TAUC_A);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      size_t q = IA(j, i);
      double uabs = sqrt(C->slid_delta_v * C->slid_delta_v + u_a[q] * u_a[q] + v_a[q] * v_a[q]);
      switch (C->choice_sliding_law) {
        case DIVA_SLIDING_NONE: beta_a[q] = 0.0; break;
        case DIVA_SLIDING_WEERTMAN:
          beta_a[q] = bsq[q] * pow(uabs, 1.0 / C->slid_Weertman_m - 1.0); break;
        case DIVA_SLIDING_COULOMB:
          if (!C->prescribed_tauc) tauc[q] = tan((PI_C / 180.0) * phi[q]) * Neff[q];
          beta_a[q] = tauc[q] / uabs; break;
        case DIVA_SLIDING_COULOMB_REGULARISED:
          tauc[q] = tan((PI_C / 180.0) * phi[q]) * Neff[q];
          beta_a[q] = tauc[q] * pow(uabs, C->slid_Coulomb_reg_q_plastic - 1.0) /
                      pow(C->slid_Coulomb_reg_u_threshold, C->slid_Coulomb_reg_q_plastic); break;
        case DIVA_SLIDING_TSAI2015:
          beta_a[q] = fmin(asq[q] * Neff[q], bsq[q] * pow(uabs, 1.0 / C->slid_Weertman_m)) * pow(uabs, -1.0); break;
        case DIVA_SLIDING_SCHOOF2005: {
          double a2 = asq[q], b2 = bsq[q], m = C->slid_Weertman_m;
          beta_a[q] = ((b2 * pow(uabs, 1.0 / m) * a2 * Neff[q]) /
                       (pow(pow(b2, m) * uabs + pow(a2 * Neff[q], m), 1.0 / m))) * pow(uabs, -1.0);
          break;
        }
        case DIVA_SLIDING_ZOET_IVERSON:
          beta_a[q] = Neff[q] * tan((PI_C / 180.0) * phi[q]) * (pow(uabs, 1.0 / C->slid_ZI_p - 1.0)) *
                      (pow(uabs + C->slid_ZI_ut, -1.0 / C->slid_ZI_p)); break;
        default: beta_a[q] = NAN;
      }
    }
}

/* ------------------------------------------------------------------------ */
/* ice_velocity_module.f90: viscosity, friction, F-integrals                 */

/* calc_vertical_shear_strain_rates :664-721 */
static void calc_vertical_shear_strain_rates(orc_ctx* c) {
  DECL_DIMS(c);
  const double* zeta = c->g.zeta;
  const int32_t* ice = FI(c, MASK_ICE_A);
  const double *visc = FD(c, VISC_EFF_3D_A), *Hi = FD(c, HI_A), *tbx = FD(c, TAUB_CX), *tby = FD(c, TAUB_CY);
  double *dudz = FD(c, DU_DZ_3D_CX), *dvdz = FD(c, DV_DZ_3D_CY);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (i < nx - 1) {
        if (ice[IA(j, i)] == 0 && ice[IA(j, i + 1)] == 0) {
          for (int k = 0; k < nz; ++k) dudz[ICX3(k, j, i)] = 0.0;
        } else {
          for (int k = 0; k < nz; ++k) {
            double vcx = stag_margin(visc[IA3(k, j, i)], visc[IA3(k, j, i + 1)], Hi[IA(j, i)], Hi[IA(j, i + 1)]);
            dudz[ICX3(k, j, i)] = (tbx[ICX(j, i)] / vcx) * zeta[k];
          }
        }
      }
      if (j < ny - 1) {
        if (ice[IA(j, i)] == 0 && ice[IA(j + 1, i)] == 0) {
          for (int k = 0; k < nz; ++k) dvdz[ICY3(k, j, i)] = 0.0;
        } else {
          for (int k = 0; k < nz; ++k) {
            double vcy = stag_margin(visc[IA3(k, j, i)], visc[IA3(k, j + 1, i)], Hi[IA(j, i)], Hi[IA(j + 1, i)]);
            dvdz[ICY3(k, j, i)] = (tby[ICY(j, i)] / vcy) * zeta[k];
          }
        }
      }
    }
}

/* calc_effective_viscosity :722-899 */
/* rows of block b of nb (contiguous, balanced by row count) */
static void block_rows(int n, int nb, int b, int* lo, int* hi) {
  *lo = (int)((long long)n * b / nb);
  *hi = (int)((long long)n * (b + 1) / nb);
}

/* ---- worker pool of the timed CPU baseline (pthreads; one per context with threads > 1) ----
 * pool_run(P, fn, arg) runs fn(arg, t, T) on T threads (the caller is thread 0) and returns
 * when all have finished; with T = 1 it is a plain call. */
typedef void (*task_fn)(void* arg, int t, int T);
struct worker_arg { struct orc_pool* P; int t; };
struct orc_pool {
  int T, quit;
  pthread_t th[ORC_MAX_THREADS];
  struct worker_arg wa[ORC_MAX_THREADS];
  pthread_barrier_t start, done;
  task_fn fn;
  void* arg;
};
static void* pool_worker(void* wa) {
  struct orc_pool* P = ((struct worker_arg*)wa)->P;
  const int t = ((struct worker_arg*)wa)->t;
  for (;;) {
    pthread_barrier_wait(&P->start);
    if (P->quit) break;
    P->fn(P->arg, t, P->T);
    pthread_barrier_wait(&P->done);
  }
  return NULL;
}
static void pool_run(struct orc_pool* P, task_fn fn, void* arg) {
  if (!P || P->T <= 1) { fn(arg, 0, 1); return; }
  P->fn = fn;
  P->arg = arg;
  pthread_barrier_wait(&P->start);
  fn(arg, 0, P->T);
  pthread_barrier_wait(&P->done);
}
static struct orc_pool* pool_create(int T) {
  struct orc_pool* P = (struct orc_pool*)calloc(1, sizeof(struct orc_pool));
  P->T = T;
  pthread_barrier_init(&P->start, NULL, (unsigned)T);
  pthread_barrier_init(&P->done, NULL, (unsigned)T);
  for (int t = 1; t < T; ++t) {
    P->wa[t].P = P;
    P->wa[t].t = t;
    pthread_create(&P->th[t], NULL, pool_worker, &P->wa[t]);
  }
  return P;
}
static void pool_destroy(struct orc_pool* P) {
  if (!P) return;
  if (P->T > 1) {
    P->quit = 1;
    pthread_barrier_wait(&P->start);
    for (int t = 1; t < P->T; ++t) pthread_join(P->th[t], NULL);
  }
  pthread_barrier_destroy(&P->start);
  pthread_barrier_destroy(&P->done);
  free(P);
}

/* the columns [i0, i1) of calc_effective_viscosity (one slice per baseline thread) */
static void visc_columns_range(orc_ctx* c, const double* du_dx, const double* du_dy, const double* dv_dx,
                               const double* dv_dy, int i0, int i1) {
  DECL_DIMS(c);
  const diva_config_t* C = &c->c;
  const double* zeta = c->g.zeta;
  const int32_t* ice = FI(c, MASK_ICE_A);
  const double *Hi = FD(c, HI_A), *A = FD(c, A_FLOW_3D_A), *dudz = FD(c, DU_DZ_3D_CX), *dvdz = FD(c, DV_DZ_3D_CY);
  double *visc = FD(c, VISC_EFF_3D_A), *vint_a = FD(c, VISC_EFF_INT_A), *Na = FD(c, N_A);
  const double e_A = -1.0 / C->n_flow, e_eps = (1.0 - C->n_flow) / (2.0 * C->n_flow);
  const int bc = (C->choice_ice_margin == DIVA_MARGIN_BC);
  for (int i = i0; i < i1; ++i)
    for (int j = 0; j < ny; ++j) {
      if (bc && ice[IA(j, i)] == 0) {
        for (int k = 0; k < nz; ++k) visc[IA3(k, j, i)] = 0.0;
        continue;
      }
      for (int k = 0; k < nz; ++k) {
        double du_dz_a, dv_dz_a;
        if (i == 0) du_dz_a = dudz[ICX3(k, j, 0)];
        else if (i == nx - 1) du_dz_a = dudz[ICX3(k, j, nx - 2)];
        else du_dz_a = stag_margin(dudz[ICX3(k, j, i - 1)], dudz[ICX3(k, j, i)], Hi[IA(j, i - 1)], Hi[IA(j, i)]);
        if (j == 0) dv_dz_a = dvdz[ICY3(k, 0, i)];
        else if (j == ny - 1) dv_dz_a = dvdz[ICY3(k, ny - 2, i)];
        else dv_dz_a = stag_margin(dvdz[ICY3(k, j - 1, i)], dvdz[ICY3(k, j, i)], Hi[IA(j - 1, i)], Hi[IA(j, i)]);
        size_t q = IA(j, i);
        double eps_sq = du_dx[q] * du_dx[q] + dv_dy[q] * dv_dy[q] + du_dx[q] * dv_dy[q] +
                        0.25 * ((du_dy[q] + dv_dx[q]) * (du_dy[q] + dv_dx[q])) +
                        0.25 * (du_dz_a * du_dz_a + dv_dz_a * dv_dz_a) + C->DIVA_epsilon_sq_0;
        double v = 0.5 * pow(A[IA3(k, j, i)], e_A) * pow(eps_sq, e_eps);
        visc[IA3(k, j, i)] = fmax(v, C->DIVA_visc_eff_min);
      }
      vint_a[IA(j, i)] = vint(zeta, nz, &visc[IA3(0, j, i)]);
      Na[IA(j, i)] = bc ? vint_a[IA(j, i)] * Hi[IA(j, i)] : vint_a[IA(j, i)] * fmax(0.1, Hi[IA(j, i)]);
    }
}

struct visc_cols { orc_ctx* c; const double *du_dx, *du_dy, *dv_dx, *dv_dy; };
static void visc_b_range(orc_ctx* c, int i0, int i1);
static void visc_b_columns(void* arg, int t, int T) {
  struct visc_cols* v = (struct visc_cols*)arg;
  int i0, i1;
  block_rows(v->c->nx - 1, T, t, &i0, &i1);
  visc_b_range(v->c, i0, i1);
}
static void visc_columns(void* arg, int t, int T) {
  struct visc_cols* v = (struct visc_cols*)arg;
  int i0, i1;
  block_rows(v->c->nx, T, t, &i0, &i1);
  visc_columns_range(v->c, v->du_dx, v->du_dy, v->dv_dx, v->dv_dy, i0, i1);
}

static void calc_effective_viscosity(orc_ctx* c, const double* u_cx, const double* v_cy) {
  DECL_DIMS(c);
  const diva_config_t* C = &c->c;
  const double dx = c->dx;
  const size_t na = (size_t)nx * ny;
  double *du_dx = (double*)malloc(na * sizeof(double)), *du_dy = (double*)malloc(na * sizeof(double));
  double *dv_dx = (double*)malloc(na * sizeof(double)), *dv_dy = (double*)malloc(na * sizeof(double));
  ddx_cx_to_a(nx, ny, dx, u_cx, du_dx);
  ddy_cx_to_a(nx, ny, dx, u_cx, du_dy);
  ddx_cy_to_a(nx, ny, dx, v_cy, dv_dx);
  ddy_cy_to_a(nx, ny, dx, v_cy, dv_dy);
  double* Na = FD(c, N_A);
  /* the a-grid columns, in column strips over the baseline's threads */
  struct visc_cols a = {c, du_dx, du_dy, dv_dx, dv_dy};
  pool_run(c->pool, visc_columns, &a);
  struct visc_cols bb = {c, NULL, NULL, NULL, NULL};
  pool_run(c->pool, visc_b_columns, &bb);
  if (!C->include_SSADIVA_crossterms) {
    map_a_to_cx(nx, ny, Na, FD(c, N_CX));
    map_a_to_cy(nx, ny, Na, FD(c, N_CY));
  }
  free(du_dx); free(du_dy); free(dv_dx); free(dv_dy);
}

/* the b-grid columns [i0, i1) of calc_effective_viscosity (:820-874) */
static void visc_b_range(orc_ctx* c, int i0, int i1) {
  DECL_DIMS(c);
  const diva_config_t* C = &c->c;
  const double* zeta = c->g.zeta;
  const int32_t* ice = FI(c, MASK_ICE_A);
  const double* visc = FD(c, VISC_EFF_3D_A);
  const int bc = (C->choice_ice_margin == DIVA_MARGIN_BC);
  double *visc_b = FD(c, VISC_EFF_3D_B), *vint_b = FD(c, VISC_EFF_INT_B), *Nb = FD(c, N_B);
  const double* Hi_b = FD(c, HI_B);
  for (int i = i0; i < i1; ++i)
    for (int j = 0; j < ny - 1; ++j) {
      double* vb = &visc_b[IB3(0, j, i)];
      if (bc) {
        double w = 0.0;
        for (int k = 0; k < nz; ++k) vb[k] = 0.0;
        if (ice[IA(j, i)] == 1)         { for (int k = 0; k < nz; ++k) vb[k] = vb[k] + visc[IA3(k, j, i)];         w = w + 1.0; }
        if (ice[IA(j, i + 1)] == 1)     { for (int k = 0; k < nz; ++k) vb[k] = vb[k] + visc[IA3(k, j, i + 1)];     w = w + 1.0; }
        if (ice[IA(j + 1, i)] == 1)     { for (int k = 0; k < nz; ++k) vb[k] = vb[k] + visc[IA3(k, j + 1, i)];     w = w + 1.0; }
        if (ice[IA(j + 1, i + 1)] == 1) { for (int k = 0; k < nz; ++k) vb[k] = vb[k] + visc[IA3(k, j + 1, i + 1)]; w = w + 1.0; }
        if (w > 0.0) for (int k = 0; k < nz; ++k) vb[k] = vb[k] / w;
      } else {
        for (int k = 0; k < nz; ++k)
          vb[k] = (visc[IA3(k, j, i)] + visc[IA3(k, j, i + 1)] + visc[IA3(k, j + 1, i)] + visc[IA3(k, j + 1, i + 1)]) / 4.0;
      }
      vint_b[IB(j, i)] = vint(zeta, nz, vb);
      Nb[IB(j, i)] = bc ? vint_b[IB(j, i)] * Hi_b[IB(j, i)] : vint_b[IB(j, i)] * fmax(0.1, Hi_b[IB(j, i)]);
    }
}

/* calc_sliding_term_beta :900-959 */
static void calc_sliding_term_beta(orc_ctx* c, const double* u_cx, const double* v_cy) {
  DECL_DIMS(c);
  const size_t na = (size_t)nx * ny;
  double *u_a = (double*)malloc(na * sizeof(double)), *v_a = (double*)malloc(na * sizeof(double));
  map_cx_to_a(nx, ny, u_cx, u_a);
  map_cy_to_a(nx, ny, v_cy, v_a);
  double* beta = FD(c, BETA_A);
  calc_sliding_law(c, u_a, v_a, beta);
  for (size_t q = 0; q < na; ++q) beta[q] = fmin(beta[q], c->c.DIVA_beta_max);
  if (!c->c.do_GL_subgrid_friction) {
    const int32_t* ocean = FI(c, MASK_OCEAN_A);
    for (size_t q = 0; q < na; ++q) if (ocean[q] == 1) beta[q] = 0.0;
  }
  free(u_a); free(v_a);
}

/* calc_F_integral( n = 2) :960-1013 */
static void calc_F_integral(orc_ctx* c) {
  DECL_DIMS(c);
  const double* zeta = c->g.zeta;
  double tmp[64];
  for (int k = 0; k < nz; ++k) tmp[k] = (1.0 / c->c.DIVA_visc_eff_min) * pow(zeta[k], 2.0);
  const double Fmin = vint(zeta, nz, tmp);
  const int32_t* ice = FI(c, MASK_ICE_A);
  const double *Hi = FD(c, HI_A), *visc = FD(c, VISC_EFF_3D_A);
  double* F2 = FD(c, F2_A);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      size_t q = IA(j, i);
      if (ice[q] == 1) {
        for (int k = 0; k < nz; ++k) tmp[k] = (Hi[q] / visc[IA3(k, j, i)]) * pow(zeta[k], 2.0);
        F2[q] = fmax(Fmin, vint(zeta, nz, tmp));
      } else {
        F2[q] = (c->c.choice_ice_margin == DIVA_MARGIN_BC) ? 0.0 : Fmin;
      }
    }
}

/* calc_beta_eff :1014-1086 */
static void calc_beta_eff(orc_ctx* c) {
  DECL_DIMS(c);
  const double *beta = FD(c, BETA_A), *F2 = FD(c, F2_A), *Ti = FD(c, TI_A), *Tp = FD(c, TI_PMP_A);
  double* be = FD(c, BETA_EFF_A);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      size_t q = IA(j, i);
      if (c->c.choice_sliding_law == DIVA_SLIDING_NONE) {
        be[q] = 1.0 / F2[q];
      } else {
        be[q] = beta[q] / (1.0 + beta[q] * F2[q]);
        if (c->c.include_basal_freezing)
          if (Tp[IA3(nz - 1, j, i)] - Ti[IA3(nz - 1, j, i)] > c->c.deltaT_basal_freezing) be[q] = 1.0 / F2[q];
      }
    }
  double *bcx = FD(c, BETA_EFF_CX), *bcy = FD(c, BETA_EFF_CY);
  map_a_to_cx(nx, ny, be, bcx);
  map_a_to_cy(nx, ny, be, bcy);
  if (c->c.do_GL_subgrid_friction) {
    const double *fcx = FD(c, F_GRND_CX), *fcy = FD(c, F_GRND_CY);
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j) {
        if (i < nx - 1) bcx[ICX(j, i)] = bcx[ICX(j, i)] * (fcx[ICX(j, i)] * fcx[ICX(j, i)]);
        if (j < ny - 1) bcy[ICY(j, i)] = bcy[ICY(j, i)] * (fcy[ICY(j, i)] * fcy[ICY(j, i)]);
      }
  }
}

/* calc_basal_stress :1087-1120 */
static void calc_basal_stress(orc_ctx* c) {
  DECL_DIMS(c);
  const double *bcx = FD(c, BETA_EFF_CX), *bcy = FD(c, BETA_EFF_CY), *u = FD(c, U_VAV_CX), *v = FD(c, V_VAV_CY);
  double *tbx = FD(c, TAUB_CX), *tby = FD(c, TAUB_CY);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (i < nx - 1) tbx[ICX(j, i)] = bcx[ICX(j, i)] * u[ICX(j, i)];
      if (j < ny - 1) tby[ICY(j, i)] = bcy[ICY(j, i)] * v[ICY(j, i)];
    }
}

/* calc_basal_velocities :1121-1199 */
static void calc_basal_velocities(orc_ctx* c) {
  DECL_DIMS(c);
  double *ub = FD(c, U_BASE_CX), *vb = FD(c, V_BASE_CY);
  if (c->c.choice_sliding_law == DIVA_SLIDING_NONE) {
    memset(ub, 0, sizeof(double) * (size_t)ny * (nx - 1));
    memset(vb, 0, sizeof(double) * (size_t)(ny - 1) * nx);
    return;
  }
  const double *F2 = FD(c, F2_A), *Hi = FD(c, HI_A), *u = FD(c, U_VAV_CX), *v = FD(c, V_VAV_CY);
  const double *tbx = FD(c, TAUB_CX), *tby = FD(c, TAUB_CY), *Ti = FD(c, TI_A), *Tp = FD(c, TI_PMP_A);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      int frozen = c->c.include_basal_freezing &&
                   (Tp[IA3(nz - 1, j, i)] - Ti[IA3(nz - 1, j, i)] > c->c.deltaT_basal_freezing);
      if (i < nx - 1) {
        double F2s = stag_margin(F2[IA(j, i)], F2[IA(j, i + 1)], Hi[IA(j, i)], Hi[IA(j, i + 1)]);
        ub[ICX(j, i)] = u[ICX(j, i)] - tbx[ICX(j, i)] * F2s;
        if (frozen) ub[ICX(j, i)] = 0.0;
      }
      if (j < ny - 1) {
        double F2s = stag_margin(F2[IA(j, i)], F2[IA(j + 1, i)], Hi[IA(j, i)], Hi[IA(j + 1, i)]);
        vb[ICY(j, i)] = v[ICY(j, i)] - tby[ICY(j, i)] * F2s;
        if (frozen) vb[ICY(j, i)] = 0.0;
      }
    }
}

/* calc_3D_horizontal_velocities_DIVA :1200-1298 */
static void calc_3D_horizontal_velocities_DIVA(orc_ctx* c) {
  DECL_DIMS(c);
  const double* zeta = c->g.zeta;
  const double *Hi = FD(c, HI_A), *visc = FD(c, VISC_EFF_3D_A);
  double* F1 = FD(c, F1_3D_A);
  double tmp[64];
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      for (int k = 0; k < nz; ++k) tmp[k] = (-Hi[IA(j, i)] / visc[IA3(k, j, i)]) * zeta[k];
      vint_bottom_to_zeta(zeta, nz, tmp, &F1[IA3(0, j, i)]);
    }
  const int bc = (c->c.choice_ice_margin == DIVA_MARGIN_BC);
  const double *ub = FD(c, U_BASE_CX), *vb = FD(c, V_BASE_CY), *tbx = FD(c, TAUB_CX), *tby = FD(c, TAUB_CY);
  double *u3 = FD(c, U_3D_CX), *v3 = FD(c, V_3D_CY);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (i < nx - 1) {
        double H0 = Hi[IA(j, i)], H1 = Hi[IA(j, i + 1)];
        for (int k = 0; k < nz; ++k) {
          double a = F1[IA3(k, j, i)], b = F1[IA3(k, j, i + 1)], s;
          if (bc) {
            if (H0 > 0.0 && H1 == 0.0) s = a;
            else if (H0 == 0.0 && H1 > 0.0) s = b;
            else if (H0 > 0.0 && H1 > 0.0) s = 0.5 * (a + b);
            else s = 0.0;
          } else s = 0.5 * (a + b);
          u3[ICX3(k, j, i)] = ub[ICX(j, i)] + tbx[ICX(j, i)] * s;
        }
      }
      if (j < ny - 1) {
        double H0 = Hi[IA(j, i)], H1 = Hi[IA(j + 1, i)];
        for (int k = 0; k < nz; ++k) {
          double a = F1[IA3(k, j, i)], b = F1[IA3(k, j + 1, i)], s;
          if (bc) {
            if (H0 > 0.0 && H1 == 0.0) s = a;
            else if (H0 == 0.0 && H1 > 0.0) s = b;
            else if (H0 > 0.0 && H1 > 0.0) s = 0.5 * (a + b);
            else s = 0.0;
          } else s = 0.5 * (a + b);
          v3[ICY3(k, j, i)] = vb[ICY(j, i)] + tby[ICY(j, i)] * s;
        }
      }
    }
}

/* ------------------------------------------------------------------------ */
/* Picard bookkeeping, ice_velocity_module.f90:1322-1652                     */

/* set_sico_masks :1322-1431, including the column range of the inner-front reset
 * (:1384 uses ny where nx is meant; kept as written) */
static void set_sico_masks(orc_ctx* c) {
  DECL_DIMS(c);
  const double *TAF = FD(c, TAF_A), *Hi = FD(c, HI_A);
  int32_t *combi = FI(c, DIVA_MASK_COMBI), *inner = FI(c, DIVA_ISFRONT_INNER), *outer = FI(c, DIVA_ISFRONT_OUTER);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      size_t q = IA(j, i);
      int is_float = TAF[q] < 0.0;
      if (Hi[q] == 0.0) combi[q] = is_float ? 2 : 1;
      else combi[q] = is_float ? 3 : 0;
    }
  const int ireset = (ny - 1 < nx) ? ny - 1 : nx;
  for (int i = 0; i < ireset; ++i)
    for (int j = 0; j < ny; ++j) inner[IA(j, i)] = 0;
  for (size_t q = 0; q < (size_t)nx * ny; ++q) outer[q] = 0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      int i1 = i - 1 < 0 ? 0 : i - 1, i2 = i + 1 > nx - 1 ? nx - 1 : i + 1;
      int j1 = j - 1 < 0 ? 0 : j - 1, j2 = j + 1 > ny - 1 ? ny - 1 : j + 1;
      size_t q = IA(j, i);
      if (Hi[q] > 0.0 && (Hi[IA(j, i1)] == 0.0 || Hi[IA(j, i2)] == 0.0 || Hi[IA(j1, i)] == 0.0 || Hi[IA(j2, i)] == 0.0))
        inner[q] = 1;
      if (Hi[q] == 0.0 && (Hi[IA(j, i1)] > 0.0 || Hi[IA(j, i2)] > 0.0 || Hi[IA(j1, i)] > 0.0 || Hi[IA(j2, i)] > 0.0))
        outer[q] = 1;
      if (inner[q] == 1 && combi[q] == 0) inner[q] = 0;   /* disable_grounded_fronts */
    }
}

/* apply_velocity_limits :1432-1498 */
static void apply_velocity_limits(orc_ctx* c, double* u_cx, double* v_cy) {
  DECL_DIMS(c);
  const size_t ncx = (size_t)ny * (nx - 1), ncy = (size_t)(ny - 1) * nx;
  double *v_cx = (double*)malloc(ncx * sizeof(double)), *u_cy = (double*)malloc(ncy * sizeof(double));
  double *ab_cx = (double*)malloc(ncx * sizeof(double)), *ab_cy = (double*)malloc(ncy * sizeof(double));
  map_cx_to_cy(nx, ny, u_cx, u_cy);
  map_cy_to_cx(nx, ny, v_cy, v_cx);
  for (size_t q = 0; q < ncx; ++q) ab_cx[q] = sqrt(u_cx[q] * u_cx[q] + v_cx[q] * v_cx[q]);
  for (size_t q = 0; q < ncy; ++q) ab_cy[q] = sqrt(u_cy[q] * u_cy[q] + v_cy[q] * v_cy[q]);
  const double vmax = c->c.DIVA_vel_max;
  for (size_t q = 0; q < ncx; ++q) if (ab_cx[q] > vmax) u_cx[q] = u_cx[q] * vmax / ab_cx[q];
  for (size_t q = 0; q < ncy; ++q) if (ab_cy[q] > vmax) v_cy[q] = v_cy[q] * vmax / ab_cy[q];
  free(v_cx); free(u_cy); free(ab_cx); free(ab_cy);
}

/* relax_DIVA_visc_iterations :1499-1529 */
static void relax_visc_iterations(orc_ctx* c, double* u_cx, double* v_cy, double rel) {
  DECL_DIMS(c);
  const double *up = FD(c, U_CX_PREV), *vp = FD(c, V_CY_PREV);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (i < nx - 1) u_cx[ICX(j, i)] = rel * u_cx[ICX(j, i)] + (1.0 - rel) * up[ICX(j, i)];
      if (j < ny - 1) v_cy[ICY(j, i)] = rel * v_cy[ICY(j, i)] + (1.0 - rel) * vp[ICY(j, i)];
    }
}

/* DIVA_vel_tolerance = 1e-6 is a default-REAL literal in the reference (:1547, :1617) */
#define DIVA_VEL_TOLERANCE ((double)1e-6f)

/* calc_visc_iter_UV_resid :1530-1601 */
static double calc_visc_iter_UV_resid(orc_ctx* c, const double* u_cx, const double* v_cy) {
  DECL_DIMS(c);
  const double *up = FD(c, U_CX_PREV), *vp = FD(c, V_CY_PREV);
  long ncx = 0, ncy = 0;
  double r1 = 0.0, r2 = 0.0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (i < nx - 1) {
        double u = u_cx[ICX(j, i)], p = up[ICX(j, i)];
        if (fabs(u) > DIVA_VEL_TOLERANCE) { ++ncx; r1 = r1 + (u - p) * (u - p); r2 = r2 + (u + p) * (u + p); }
      }
      if (j < ny - 1) {
        double v = v_cy[ICY(j, i)], p = vp[ICY(j, i)];
        if (fabs(v) > DIVA_VEL_TOLERANCE) { ++ncy; r1 = r1 + (v - p) * (v - p); r2 = r2 + (v + p) * (v + p); }
      }
    }
  if (ncx + ncy > 0) {
    r1 = sqrt(r1);
    r2 = fmax(sqrt(r2), 1E-8);
    return 2.0 * r1 / r2;
  }
  return 0.0;
}

/* estimate_visc_iter_UV_errors :1602-1652 */
static void estimate_visc_iter_UV_errors(orc_ctx* c, const double* u_cx, const double* v_cy) {
  DECL_DIMS(c);
  const double *up = FD(c, U_CX_PREV), *vp = FD(c, V_CY_PREV), *uv = FD(c, U_VAV_CX), *vv = FD(c, V_VAV_CY);
  double *ex = FD(c, DIVA_ERR_CX), *ey = FD(c, DIVA_ERR_CY);
  const double tol = 1E-5;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (i < nx - 1) {
        size_t q = ICX(j, i);
        ex[q] = (fabs(uv[q]) > DIVA_VEL_TOLERANCE) ? 2.0 * fabs(u_cx[q] - up[q]) / fabs(u_cx[q] + up[q] + tol) : 0.0;
      }
      if (j < ny - 1) {
        size_t q = ICY(j, i);
        ey[q] = (fabs(vv[q]) > DIVA_VEL_TOLERANCE) ? 2.0 * fabs(v_cy[q] - vp[q]) / fabs(v_cy[q] + vp[q] + tol) : 0.0;
      }
    }
}

/* ------------------------------------------------------------------------ */
/* stiffness matrix assembly, ice_velocity_module.f90:1656-2589              */

#define ADD(col, v) do { m->idx[m->nnz] = (col); m->val[m->nnz] = (v); m->nnz++; } while (0)

static int bc_pick(int a, int b) {
  if (a == DIVA_BC_ZERO || b == DIVA_BC_ZERO) return DIVA_BC_ZERO;
  if (a == DIVA_BC_INFINITE || b == DIVA_BC_INFINITE) return DIVA_BC_INFINITE;
  return DIVA_BC_PERIODIC;
}

/* list_DIVA_matrix_coefficients_eq_1_boundary :1932-2061 */
static void row_u_boundary(orc_ctx* c, const double* u, int n, int i, int j) {
  DECL_DIMS(c);
  csr_t* m = &c->m;
  const diva_config_t* C = &c->c;
  int BC;
  if (i == 0 && j == 0) BC = bc_pick(C->BC_u_south, C->BC_u_west);
  else if (i == nx - 2 && j == 0) BC = bc_pick(C->BC_u_south, C->BC_u_east);
  else if (i == 0 && j == ny - 1) BC = bc_pick(C->BC_u_north, C->BC_u_west);
  else if (i == nx - 2 && j == ny - 1) BC = bc_pick(C->BC_u_north, C->BC_u_east);
  else if (i == 0) BC = C->BC_u_west;
  else if (i == nx - 2) BC = C->BC_u_east;
  else if (j == 0) BC = C->BC_u_south;
  else BC = C->BC_u_north;
  int i_in = i, i_opp = i, j_in = j, j_opp = j;
  if (i == 0) { i_in = 1; i_opp = nx - 3; } else if (i == nx - 2) { i_in = nx - 3; i_opp = 1; }
  if (j == 0) { j_in = 1; j_opp = ny - 2; } else if (j == ny - 1) { j_in = ny - 2; j_opp = 1; }
  int nu = c->ij2n_u[ICX(j, i)], nu_in = c->ij2n_u[ICX(j_in, i_in)], nu_opp = c->ij2n_u[ICX(j_opp, i_opp)];
  if (BC == DIVA_BC_INFINITE) { ADD(nu, 1.0); ADD(nu_in, -1.0); m->b[n] = 0.0; m->x[n] = u[ICX(j, i)]; }
  else if (BC == DIVA_BC_ZERO) { ADD(nu, 1.0); m->b[n] = 0.0; m->x[n] = 0.0; }
  else { ADD(nu, 1.0); ADD(nu_opp, -1.0); m->b[n] = 0.0; m->x[n] = u[ICX(j, i)]; }
}
/* list_DIVA_matrix_coefficients_eq_2_boundary :2062-2191 */
static void row_v_boundary(orc_ctx* c, const double* v, int n, int i, int j) {
  DECL_DIMS(c);
  csr_t* m = &c->m;
  const diva_config_t* C = &c->c;
  int BC;
  if (i == 0 && j == 0) BC = bc_pick(C->BC_v_south, C->BC_v_west);
  else if (i == nx - 1 && j == 0) BC = bc_pick(C->BC_v_south, C->BC_v_east);
  else if (i == 0 && j == ny - 2) BC = bc_pick(C->BC_v_north, C->BC_v_west);
  else if (i == nx - 1 && j == ny - 2) BC = bc_pick(C->BC_v_north, C->BC_v_east);
  else if (i == 0) BC = C->BC_v_west;
  else if (i == nx - 1) BC = C->BC_v_east;
  else if (j == 0) BC = C->BC_v_south;
  else BC = C->BC_v_north;
  int i_in = i, i_opp = i, j_in = j, j_opp = j;
  if (i == 0) { i_in = 1; i_opp = nx - 2; } else if (i == nx - 1) { i_in = nx - 2; i_opp = 1; }
  if (j == 0) { j_in = 1; j_opp = ny - 3; } else if (j == ny - 2) { j_in = ny - 3; j_opp = 1; }
  int nv = c->ij2n_v[ICY(j, i)], nv_in = c->ij2n_v[ICY(j_in, i_in)], nv_opp = c->ij2n_v[ICY(j_opp, i_opp)];
  if (BC == DIVA_BC_INFINITE) { ADD(nv, 1.0); ADD(nv_in, -1.0); m->b[n] = 0.0; m->x[n] = v[ICY(j, i)]; }
  else if (BC == DIVA_BC_ZERO) { ADD(nv, 1.0); m->b[n] = 0.0; m->x[n] = 0.0; }
  else { ADD(nv, 1.0); ADD(nv_opp, -1.0); m->b[n] = 0.0; m->x[n] = v[ICY(j, i)]; }
}

/* list_DIVA_matrix_coefficients_eq_1_free :2342-2404 and _free_sans :2468-2528 */
static void row_u_free(orc_ctx* c, const double* u, int n, int i, int j) {
  DECL_DIMS(c);
  csr_t* m = &c->m;
  const double *Na = FD(c, N_A), *Nb = FD(c, N_B), *bcx = FD(c, BETA_EFF_CX), *tdx = FD(c, TAUDX_CX);
  const double dx = c->dx;
  const int* U = c->ij2n_u; const int* V = c->ij2n_v;
  if (c->c.include_SSADIVA_crossterms) {
    ADD(U[ICX(j, i + 1)], 4.0 * Na[IA(j, i + 1)]);
    ADD(U[ICX(j, i - 1)], 4.0 * Na[IA(j, i)]);
    ADD(U[ICX(j + 1, i)], Nb[IB(j, i)]);
    ADD(U[ICX(j - 1, i)], Nb[IB(j - 1, i)]);
    ADD(U[ICX(j, i)], -4.0 * (Na[IA(j, i + 1)] + Na[IA(j, i)]) + -1.0 * (Nb[IB(j, i)] + Nb[IB(j - 1, i)]) -
                      bcx[ICX(j, i)] * (dx * dx));
    ADD(V[ICY(j, i)], -2.0 * Na[IA(j, i)] - Nb[IB(j, i)]);
    ADD(V[ICY(j, i + 1)], 2.0 * Na[IA(j, i + 1)] + Nb[IB(j, i)]);
    ADD(V[ICY(j - 1, i)], 2.0 * Na[IA(j, i)] + Nb[IB(j - 1, i)]);
    ADD(V[ICY(j - 1, i + 1)], -2.0 * Na[IA(j, i + 1)] - Nb[IB(j - 1, i)]);
    m->b[n] = -tdx[ICX(j, i)] * (dx * dx);
  } else {
    const double* Ncx = FD(c, N_CX);
    ADD(U[ICX(j, i + 1)], 4.0);
    ADD(U[ICX(j, i - 1)], 4.0);
    ADD(U[ICX(j + 1, i)], 1.0);
    ADD(U[ICX(j - 1, i)], 1.0);
    ADD(U[ICX(j, i)], -10.0 - (dx * dx) * bcx[ICX(j, i)] / Ncx[ICX(j, i)]);
    ADD(V[ICY(j, i)], -3.0);
    ADD(V[ICY(j, i + 1)], 3.0);
    ADD(V[ICY(j - 1, i)], 3.0);
    ADD(V[ICY(j - 1, i + 1)], -3.0);
    m->b[n] = -tdx[ICX(j, i)] * (dx * dx) / Ncx[ICX(j, i)];
  }
  m->x[n] = u[ICX(j, i)];
}
/* list_DIVA_matrix_coefficients_eq_2_free :2405-2467 and _free_sans :2529-2589 */
static void row_v_free(orc_ctx* c, const double* v, int n, int i, int j) {
  DECL_DIMS(c);
  csr_t* m = &c->m;
  const double *Na = FD(c, N_A), *Nb = FD(c, N_B), *bcy = FD(c, BETA_EFF_CY), *tdy = FD(c, TAUDY_CY);
  const double dx = c->dx;
  const int* U = c->ij2n_u; const int* V = c->ij2n_v;
  if (c->c.include_SSADIVA_crossterms) {
    ADD(V[ICY(j + 1, i)], 4.0 * Na[IA(j + 1, i)]);
    ADD(V[ICY(j - 1, i)], 4.0 * Na[IA(j, i)]);
    ADD(V[ICY(j, i + 1)], Nb[IB(j, i)]);
    ADD(V[ICY(j, i - 1)], Nb[IB(j, i - 1)]);
    ADD(V[ICY(j, i)], -4.0 * (Na[IA(j + 1, i)] + Na[IA(j, i)]) + -1.0 * (Nb[IB(j, i)] + Nb[IB(j, i - 1)]) -
                      bcy[ICY(j, i)] * (dx * dx));
    ADD(U[ICX(j + 1, i - 1)], -2.0 * Na[IA(j + 1, i)] - Nb[IB(j, i - 1)]);
    ADD(U[ICX(j + 1, i)], 2.0 * Na[IA(j + 1, i)] + Nb[IB(j, i)]);
    ADD(U[ICX(j, i - 1)], 2.0 * Na[IA(j, i)] + Nb[IB(j, i - 1)]);
    ADD(U[ICX(j, i)], -2.0 * Na[IA(j, i)] - Nb[IB(j, i)]);
    m->b[n] = -tdy[ICY(j, i)] * (dx * dx);
  } else {
    const double* Ncy = FD(c, N_CY);
    ADD(V[ICY(j + 1, i)], 4.0);
    ADD(V[ICY(j - 1, i)], 4.0);
    ADD(V[ICY(j, i + 1)], 1.0);
    ADD(V[ICY(j, i - 1)], 1.0);
    ADD(V[ICY(j, i)], -10.0 - (dx * dx) * bcy[ICY(j, i)] / Ncy[ICY(j, i)]);
    ADD(U[ICX(j + 1, i - 1)], -3.0);
    ADD(U[ICX(j + 1, i)], 3.0);
    ADD(U[ICX(j, i - 1)], 3.0);
    ADD(U[ICX(j, i)], -3.0);
    m->b[n] = -tdy[ICY(j, i)] * (dx * dx) / Ncy[ICY(j, i)];
  }
  m->x[n] = v[ICY(j, i)];
}

/* list_DIVA_matrix_coefficients_eq_1_margin :2192-2266 */
static void row_u_margin(orc_ctx* c, const double* u, int n, int i, int j) {
  DECL_DIMS(c);
  csr_t* m = &c->m;
  const int32_t *inner = FI(c, DIVA_ISFRONT_INNER), *outer = FI(c, DIVA_ISFRONT_OUTER);
  const double *Na = FD(c, N_A), *Hi = FD(c, HI_A), *SL = FD(c, SL_A), *Hb = FD(c, HB_A);
  const double inv_dx = 1.0 / c->dx;
  int i1 = (inner[IA(j, i)] == 1) ? i : i + 1;
  if (outer[IA(j, i1 - 1)] == 1 && outer[IA(j, i1 + 1)] == 1) {
    ADD(n, 1.0); m->b[n] = 0.0; m->x[n] = 0.0;
    return;
  }
  ADD(c->ij2n_u[ICX(j, i1 - 1)], -4.0 * inv_dx * Na[IA(j, i1)]);
  ADD(c->ij2n_u[ICX(j, i1)], 4.0 * inv_dx * Na[IA(j, i1)]);
  ADD(c->ij2n_v[ICY(j - 1, i1)], -2.0 * inv_dx * Na[IA(j, i1)]);
  ADD(c->ij2n_v[ICY(j, i1)], 2.0 * inv_dx * Na[IA(j, i1)]);
  double H_ice = Hi[IA(j, i1)], H_ocn;
  if (SL[IA(j, i1)] > Hb[IA(j, i1)]) H_ocn = fmin(ICE_DENSITY / SW_DENSITY * Hi[IA(j, i1)], SL[IA(j, i1)] - Hb[IA(j, i1)]);
  else H_ocn = 0.0;
  m->b[n] = 0.5 * ICE_DENSITY * GRAV * H_ice * H_ice - 0.5 * SW_DENSITY * GRAV * H_ocn * H_ocn;
  m->x[n] = u[ICX(j, i)];
}
/* list_DIVA_matrix_coefficients_eq_2_margin :2267-2341 */
static void row_v_margin(orc_ctx* c, const double* v, int n, int i, int j) {
  DECL_DIMS(c);
  csr_t* m = &c->m;
  const int32_t *inner = FI(c, DIVA_ISFRONT_INNER), *outer = FI(c, DIVA_ISFRONT_OUTER);
  const double *Na = FD(c, N_A), *Hi = FD(c, HI_A), *SL = FD(c, SL_A), *Hb = FD(c, HB_A);
  const double inv_dx = 1.0 / c->dx;
  int j1 = (inner[IA(j, i)] == 1) ? j : j + 1;
  if (outer[IA(j1 - 1, i)] == 1 && outer[IA(j1 + 1, i)] == 1) {
    ADD(n, 1.0); m->b[n] = 0.0; m->x[n] = 0.0;
    return;
  }
  ADD(c->ij2n_v[ICY(j1 - 1, i)], -4.0 * inv_dx * Na[IA(j1, i)]);
  ADD(c->ij2n_v[ICY(j1, i)], 4.0 * inv_dx * Na[IA(j1, i)]);
  ADD(c->ij2n_u[ICX(j1, i - 1)], -2.0 * inv_dx * Na[IA(j1, i)]);
  ADD(c->ij2n_u[ICX(j1, i)], 2.0 * inv_dx * Na[IA(j1, i)]);
  double H_ice = Hi[IA(j1, i)], H_ocn;
  if (SL[IA(j1, i)] > Hb[IA(j1, i)]) H_ocn = fmin(ICE_DENSITY / SW_DENSITY * Hi[IA(j1, i)], SL[IA(j1, i)] - Hb[IA(j1, i)]);
  else H_ocn = 0.0;
  m->b[n] = 0.5 * ICE_DENSITY * GRAV * H_ice * H_ice - 0.5 * SW_DENSITY * GRAV * H_ocn * H_ocn;
  m->x[n] = v[ICY(j, i)];
}

/* solve_DIVA_stag_linearised :1683-1727 (the assembly loop only) */
static void assemble(orc_ctx* c, const double* u, const double* v) {
  DECL_DIMS(c);
  csr_t* m = &c->m;
  const int bc = (c->c.choice_ice_margin == DIVA_MARGIN_BC);
  const int32_t* combi = FI(c, DIVA_MASK_COMBI);
  const int32_t *inner = FI(c, DIVA_ISFRONT_INNER), *outer = FI(c, DIVA_ISFRONT_OUTER);
  m->nnz = 0;
  m->ptr[0] = 0;
  for (int n = 0; n < c->neq; ++n) {
    if (c->n2ij[4 * n + 0] >= 0) {
      int i = c->n2ij[4 * n + 0], j = c->n2ij[4 * n + 1];
      if (i == 0 || i == nx - 2 || j == 0 || j == ny - 1) row_u_boundary(c, u, n, i, j);
      else if (bc && ((combi[IA(j, i)] == 3 && combi[IA(j, i + 1)] == 1) || (combi[IA(j, i)] == 1 && combi[IA(j, i + 1)] == 3))) {
        ADD(n, 1.0); m->b[n] = 0.0; m->x[n] = 0.0;
      } else if (bc && ((inner[IA(j, i)] == 1 && outer[IA(j, i + 1)] == 1) || (outer[IA(j, i)] == 1 && inner[IA(j, i + 1)] == 1))) {
        row_u_margin(c, u, n, i, j);
      } else row_u_free(c, u, n, i, j);
    } else {
      int i = c->n2ij[4 * n + 2], j = c->n2ij[4 * n + 3];
      if (i == 0 || i == nx - 1 || j == 0 || j == ny - 2) row_v_boundary(c, v, n, i, j);
      else if (bc && ((combi[IA(j, i)] == 3 && combi[IA(j + 1, i)] == 1) || (combi[IA(j, i)] == 1 && combi[IA(j + 1, i)] == 3))) {
        ADD(n, 1.0); m->b[n] = 0.0; m->x[n] = 0.0;
      } else if (bc && ((inner[IA(j, i)] == 1 && outer[IA(j + 1, i)] == 1) || (outer[IA(j, i)] == 1 && inner[IA(j + 1, i)] == 1))) {
        row_v_margin(c, v, n, i, j);
      } else row_v_free(c, v, n, i, j);
    }
    m->ptr[n + 1] = m->nnz;
  }
}
#undef ADD

/* ------------------------------------------------------------------------ */
/* linear solvers                                                            */

/* solve_matrix_equation_CSR_SOR, utilities_module.f90:644-718 (one rank) */
static int solve_sor(orc_ctx* c) {
  csr_t* m = &c->m;
  double omega = c->SOR_omega, res_max = c->SOR_tol * 2.0;
  int it = 0;
  while (res_max > c->SOR_tol && it < c->SOR_nit) {
    ++it;
    res_max = 0.0;
    for (int i = 0; i < m->m; ++i) {
      double lhs = 0.0, cij = 0.0;
      for (int k = m->ptr[i]; k < m->ptr[i + 1]; ++k) {
        int j = m->idx[k];
        lhs = lhs + m->val[k] * m->x[j];
        if (j == i) cij = m->val[k];
      }
      double res = (lhs - m->b[i]) / cij;
      res_max = fmax(res_max, fabs(res));
      m->x[i] = m->x[i] - omega * res;
    }
    if (it > 100 && res_max > 1E3) {
      omega = omega - 0.1;
      it = 0;
      for (int i = 0; i < m->m; ++i) m->x[i] = 0.0;
      if (omega <= 0.1) return fail(c, DIVA_LINEAR_NOT_CONVERGED, "SOR diverged even with extremely low relaxation");
    }
  }
  c->lin_iters_last = it;
  c->lin_iters_total += it;
  return DIVA_OK;
}

/* Banded LU with partial pivoting (a direct solve for exact linear parity).
 * Rows and columns are permuted symmetrically to the ordering with the smaller
 * bandwidth (the reference's i-outer interleave, or its j-outer transpose). */
static int solve_direct(orc_ctx* c) {
  DECL_DIMS(c);
  csr_t* m = &c->m;
  const int n = m->m;
  int* perm = (int*)malloc(sizeof(int) * n);   /* old row -> new row */
  if (ny <= nx) {
    for (int q = 0; q < n; ++q) perm[q] = q;
  } else {
    int r = 0;
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        if (i < nx - 1) perm[c->ij2n_u[ICX(j, i)]] = r++;
        if (j < ny - 1) perm[c->ij2n_v[ICY(j, i)]] = r++;
      }
  }
  int kl = 0, ku = 0;
  for (int r = 0; r < n; ++r)
    for (int k = m->ptr[r]; k < m->ptr[r + 1]; ++k) {
      int d = perm[m->idx[k]] - perm[r];
      if (d < 0 && -d > kl) kl = -d;
      if (d > 0 && d > ku) ku = d;
    }
  const int W = 2 * kl + ku + 1;  /* row r holds logical columns [r-kl, r+kl+ku] */
  double* Bm = (double*)calloc((size_t)n * W, sizeof(double));
  double* rhs = (double*)malloc(sizeof(double) * n);
  if (!Bm || !rhs) { free(perm); free(Bm); free(rhs); return fail(c, DIVA_BAD_INPUT, "direct solve: out of memory"); }
#define BM(r, col) Bm[(size_t)(r) * W + ((col) - (r) + kl)]
  for (int r = 0; r < n; ++r) {
    int pr = perm[r];
    for (int k = m->ptr[r]; k < m->ptr[r + 1]; ++k) BM(pr, perm[m->idx[k]]) += m->val[k];
    rhs[pr] = m->b[r];
  }
  for (int col = 0; col < n; ++col) {
    int last = col + kl < n - 1 ? col + kl : n - 1;
    int p = col; double best = fabs(BM(col, col));
    for (int r = col + 1; r <= last; ++r) if (fabs(BM(r, col)) > best) { best = fabs(BM(r, col)); p = r; }
    if (best == 0.0) { free(perm); free(Bm); free(rhs); return fail(c, DIVA_LINEAR_NOT_CONVERGED, "direct solve: singular matrix"); }
    int cmax = col + kl + ku < n - 1 ? col + kl + ku : n - 1;
    if (p != col) {
      for (int cc = col; cc <= cmax; ++cc) { double t = BM(col, cc); BM(col, cc) = BM(p, cc); BM(p, cc) = t; }
      double t = rhs[col]; rhs[col] = rhs[p]; rhs[p] = t;
    }
    double piv = BM(col, col);
    for (int r = col + 1; r <= last; ++r) {
      double f = BM(r, col);
      if (f == 0.0) continue;
      f = f / piv;
      BM(r, col) = 0.0;
      for (int cc = col + 1; cc <= cmax; ++cc) BM(r, cc) -= f * BM(col, cc);
      rhs[r] -= f * rhs[col];
    }
  }
  for (int r = n - 1; r >= 0; --r) {
    int cmax = r + kl + ku < n - 1 ? r + kl + ku : n - 1;
    double s = rhs[r];
    for (int cc = r + 1; cc <= cmax; ++cc) s -= BM(r, cc) * rhs[cc];
    rhs[r] = s / BM(r, r);
  }
#undef BM
  for (int q = 0; q < n; ++q) m->x[q] = rhs[perm[q]];
  free(perm); free(Bm); free(rhs);
  c->lin_iters_last = 1;
  c->lin_iters_total += 1;
  return DIVA_OK;
}

/* GMRES(30) with left ILU(0) preconditioning, zero initial guess and the
 * preconditioned-residual test ||B r|| <= max(rtol ||B b||, abstol): the
 * PETSc defaults that KSPSetFromOptions picks without options
 * (petsc_module.F90:49-69; PETSc is not vendored, this restates its
 * published algorithm).  Classical Gram-Schmidt, Givens rotations. */
/* ILU(0) of the rows [lo, hi) restricted to the columns [lo, hi): with one block this is
 * ILU(0) of the whole matrix; with T blocks it is block-Jacobi ILU(0), the
 * preconditioner PETSc's KSPSetFromOptions picks when the matrix is split over T
 * ranks.  Entries outside the block are kept in lu but never used. */
static void ilu0_factor_block(const csr_t* m, double* lu, int* diag, int* pos, int lo, int hi) {
  for (int i = lo; i < hi; ++i) {
    diag[i] = -1;
    for (int k = m->ptr[i]; k < m->ptr[i + 1]; ++k) {
      const int col = m->idx[k];
      if (col < lo || col >= hi) continue;
      pos[col] = k;
      if (col == i) diag[i] = k;
    }
    /* eliminate the row's lower entries in increasing column order (IKJ variant) */
    int cnt = 0, order[64];
    for (int k = m->ptr[i]; k < m->ptr[i + 1]; ++k)
      if (m->idx[k] >= lo && m->idx[k] < hi) order[cnt++] = k;
    for (int a = 1; a < cnt; ++a) { int v = order[a], b = a - 1; while (b >= 0 && m->idx[order[b]] > m->idx[v]) { order[b + 1] = order[b]; --b; } order[b + 1] = v; }
    for (int t = 0; t < cnt; ++t) {
      int kk = order[t], col = m->idx[kk];
      if (col >= i) break;
      lu[kk] = lu[kk] / lu[diag[col]];
      for (int k2 = m->ptr[col]; k2 < m->ptr[col + 1]; ++k2) {
        int c2 = m->idx[k2];
        if (c2 > col && c2 >= lo && c2 < hi && pos[c2] >= 0) lu[pos[c2]] -= lu[kk] * lu[k2];
      }
    }
    for (int k = m->ptr[i]; k < m->ptr[i + 1]; ++k)
      if (m->idx[k] >= lo && m->idx[k] < hi) pos[m->idx[k]] = -1;
  }
}
static void ilu0_apply_block(const csr_t* m, const double* lu, const int* diag, const double* r, double* z, int lo,
                             int hi) {
  for (int i = lo; i < hi; ++i) {
    double s = r[i];
    for (int k = m->ptr[i]; k < m->ptr[i + 1]; ++k) {
      const int col = m->idx[k];
      if (col < i && col >= lo) s -= lu[k] * z[col];
    }
    z[i] = s;
  }
  for (int i = hi - 1; i >= lo; --i) {
    double s = z[i];
    for (int k = m->ptr[i]; k < m->ptr[i + 1]; ++k) {
      const int col = m->idx[k];
      if (col > i && col < hi) s -= lu[k] * z[col];
    }
    z[i] = s / lu[diag[i]];
  }
}
/* the parallel pieces of GMRES: thread t of T takes the t-th contiguous slice of rows */
struct vec_task {
  const csr_t* m;
  const double *lu, *r, *x, *a, *b;
  const int* diag;
  double *z, *y, *out;
  double s;
  int n, op;
  double part[ORC_MAX_THREADS];
};
enum { VT_ILU_FACTOR, VT_ILU_APPLY, VT_SPMV, VT_DOT, VT_AXPY, VT_SCALE };
static void vec_task_run(void* arg, int t, int T) {
  struct vec_task* v = (struct vec_task*)arg;
  int lo, hi;
  block_rows(v->n, T, t, &lo, &hi);
  switch (v->op) {
    case VT_ILU_FACTOR: {
      int* pos = (int*)malloc(sizeof(int) * v->n);
      for (int q = lo; q < hi; ++q) pos[q] = -1;
      ilu0_factor_block(v->m, v->z, (int*)v->diag, pos, lo, hi);
      free(pos);
      break;
    }
    case VT_ILU_APPLY: ilu0_apply_block(v->m, v->lu, v->diag, v->r, v->z, lo, hi); break;
    case VT_SPMV:
      for (int i = lo; i < hi; ++i) {
        double s = 0.0;
        for (int k = v->m->ptr[i]; k < v->m->ptr[i + 1]; ++k) s += v->m->val[k] * v->x[v->m->idx[k]];
        v->y[i] = s;
      }
      break;
    case VT_DOT: { double s = 0.0; for (int q = lo; q < hi; ++q) s += v->a[q] * v->b[q]; v->part[t] = s; break; }
    case VT_AXPY: for (int q = lo; q < hi; ++q) v->out[q] += v->s * v->a[q]; break;         /* out += s a */
    case VT_SCALE: for (int q = lo; q < hi; ++q) v->out[q] = v->s != 0.0 ? v->a[q] / v->s : 0.0; break;
  }
}
/* ILU(0) over as many row blocks as the pool has threads (one block: plain ILU(0)) */
static void ilu0_factor(struct orc_pool* P, const csr_t* m, double* lu, int* diag) {
  memcpy(lu, m->val, sizeof(double) * m->nnz);
  struct vec_task v = {0};
  v.m = m; v.z = lu; v.diag = diag; v.n = m->m; v.op = VT_ILU_FACTOR;
  pool_run(P, vec_task_run, &v);
}
static void ilu0_apply(struct orc_pool* P, const csr_t* m, const double* lu, const int* diag, const double* r,
                       double* z) {
  struct vec_task v = {0};
  v.m = m; v.lu = lu; v.diag = diag; v.r = r; v.z = z; v.n = m->m; v.op = VT_ILU_APPLY;
  pool_run(P, vec_task_run, &v);
}
static void spmv_p(struct orc_pool* P, const csr_t* m, const double* x, double* y) {
  struct vec_task v = {0};
  v.m = m; v.x = x; v.y = y; v.n = m->m; v.op = VT_SPMV;
  pool_run(P, vec_task_run, &v);
}
static void spmv(const csr_t* m, const double* x, double* y) { spmv_p(NULL, m, x, y); }
/* sums of the per-thread slices in thread order: deterministic for a given thread count,
 * and with one thread the plain sequential sum */
static double dot_p(struct orc_pool* P, int n, const double* a, const double* b) {
  struct vec_task v = {0};
  v.a = a; v.b = b; v.n = n; v.op = VT_DOT;
  pool_run(P, vec_task_run, &v);
  const int T = (P && P->T > 1) ? P->T : 1;
  double s = v.part[0];
  for (int t = 1; t < T; ++t) s += v.part[t];
  return s;
}
static double nrm2(int n, const double* a) { double s = 0.0; for (int q = 0; q < n; ++q) s += a[q] * a[q]; return sqrt(s); }
static double nrm2_p(struct orc_pool* P, int n, const double* a) {
  return (P && P->T > 1) ? sqrt(dot_p(P, n, a, a)) : nrm2(n, a);
}
static void axpy_p(struct orc_pool* P, int n, double s, const double* a, double* out) {
  struct vec_task v = {0};
  v.a = a; v.out = out; v.s = s; v.n = n; v.op = VT_AXPY;
  pool_run(P, vec_task_run, &v);
}
static void scale_p(struct orc_pool* P, int n, const double* a, double s, double* out) {   /* out = a / s */
  struct vec_task v = {0};
  v.a = a; v.out = out; v.s = s; v.n = n; v.op = VT_SCALE;
  pool_run(P, vec_task_run, &v);
}

/* right = 1: right preconditioning, A M^-1 y = b, x = M^-1 y; the Arnoldi residual is
 * then the true residual ||b - A x||, tested against rtol ||b|| -- the test of the
 * adaptive tolerance rule (the GPU's BiCGStab measures the true residual too).
 * right = 0: left preconditioning with PETSc's default test on ||M^-1 (b - A x)||. */
static int solve_gmres(orc_ctx* c, double rtol, double abstol, int maxit, int zero_guess, int right) {
  csr_t* m = &c->m;
  struct orc_pool* P = c->pool;   /* NULL: one thread, the sequential algorithm */
  const int n = m->m, R = 30;
  double* lu = (double*)malloc(sizeof(double) * m->nnz);
  int* diag = (int*)calloc((size_t)n, sizeof(int));
  ilu0_factor(P, m, lu, diag);
  /* a zero pivot ends the solve, as PETSc's factorisation does ("zero pivot in LU
   * factorization"); it arises from empty rows, e.g. between ocean cells with 'BC' margins */
  for (int q = 0; q < n; ++q)
    if (diag[q] < 0 || !(fabs(lu[diag[q]]) > 0.0) || !isfinite(lu[diag[q]])) {
      free(lu); free(diag);
      snprintf(c->err, sizeof(c->err), "ILU(0): zero pivot in row %d", q);
      return DIVA_LINEAR_NOT_CONVERGED;
    }
  double* V = (double*)malloc(sizeof(double) * (size_t)n * (R + 1));
  double *w = (double*)malloc(sizeof(double) * n), *t = (double*)malloc(sizeof(double) * n);
  double H[31 * 30], cs[30], sn[30], g[31], y[30];
  double* x = m->x;
  double* z = right ? (double*)malloc(sizeof(double) * n) : NULL;
  if (zero_guess) memset(x, 0, sizeof(double) * n);
  double bnorm;
  if (right) bnorm = nrm2_p(P, n, m->b);
  else {
    ilu0_apply(P, m, lu, diag, m->b, t);
    bnorm = nrm2_p(P, n, t);
  }
  spmv_p(P, m, x, w);
  for (int q = 0; q < n; ++q) w[q] = m->b[q] - w[q];
  if (right) memcpy(t, w, sizeof(double) * n);
  else ilu0_apply(P, m, lu, diag, w, t);
  double rnorm = nrm2_p(P, n, t);
  /* PETSc's default test is relative to the initial residual, which is ||B b|| from a zero guess;
   * a warm start is measured against ||B b|| as well */
  double r0 = bnorm;
  double target = fmax(rtol * r0, abstol);
  int it = 0, status = DIVA_OK;
  while (rnorm > target && it < maxit) {
    scale_p(P, n, t, rnorm, V);
    memset(g, 0, sizeof(g));
    g[0] = rnorm;
    int kk = 0;
    for (; kk < R && it < maxit; ++kk) {
      ++it;
      if (right) {
        ilu0_apply(P, m, lu, diag, &V[(size_t)kk * n], z);
        spmv_p(P, m, z, t);
      } else {
        spmv_p(P, m, &V[(size_t)kk * n], w);
        ilu0_apply(P, m, lu, diag, w, t);
      }
      for (int l = 0; l <= kk; ++l) H[l * R + kk] = dot_p(P, n, t, &V[(size_t)l * n]);
      for (int l = 0; l <= kk; ++l) axpy_p(P, n, -H[l * R + kk], &V[(size_t)l * n], t);
      double hn = nrm2_p(P, n, t);
      H[(kk + 1) * R + kk] = hn;
      scale_p(P, n, t, hn, &V[(size_t)(kk + 1) * n]);
      for (int l = 0; l < kk; ++l) {
        double a = H[l * R + kk], b = H[(l + 1) * R + kk];
        H[l * R + kk] = cs[l] * a + sn[l] * b;
        H[(l + 1) * R + kk] = -sn[l] * a + cs[l] * b;
      }
      double a = H[kk * R + kk], b = H[(kk + 1) * R + kk], d = sqrt(a * a + b * b);
      cs[kk] = (d == 0.0) ? 1.0 : a / d; sn[kk] = (d == 0.0) ? 0.0 : b / d;
      H[kk * R + kk] = d; H[(kk + 1) * R + kk] = 0.0;
      g[kk + 1] = -sn[kk] * g[kk]; g[kk] = cs[kk] * g[kk];
      rnorm = fabs(g[kk + 1]);
      if (rnorm <= target) { ++kk; break; }
    }
    for (int l = kk - 1; l >= 0; --l) {
      double s = g[l];
      for (int q = l + 1; q < kk; ++q) s -= H[l * R + q] * y[q];
      y[l] = s / H[l * R + l];
    }
    if (right) {   /* x += M^-1 (V y) */
      memset(w, 0, sizeof(double) * n);
      for (int l = 0; l < kk; ++l) axpy_p(P, n, y[l], &V[(size_t)l * n], w);
      ilu0_apply(P, m, lu, diag, w, z);
      axpy_p(P, n, 1.0, z, x);
    } else {
      for (int l = 0; l < kk; ++l) axpy_p(P, n, y[l], &V[(size_t)l * n], x);
    }
    spmv_p(P, m, x, w);
    for (int q = 0; q < n; ++q) w[q] = m->b[q] - w[q];
    if (right) memcpy(t, w, sizeof(double) * n);
    else ilu0_apply(P, m, lu, diag, w, t);
    rnorm = nrm2_p(P, n, t);
  }
  if (!(rnorm <= target)) status = DIVA_LINEAR_NOT_CONVERGED;   /* NaN included */
  c->lin_iters_last = it;
  c->lin_iters_total += it;
  free(lu); free(diag); free(V); free(w); free(t); free(z);
  return status;
}

static int linear_solve(orc_ctx* c) {
  switch (c->lin_solver) {
    case ORC_LIN_SOR: return solve_sor(c);
    case ORC_LIN_GMRES_ILU: return solve_gmres(c, c->petsc_rtol, c->petsc_abstol, 100000, 1, c->true_residual);
    case ORC_LIN_GMRES_WARM: return solve_gmres(c, c->petsc_rtol, c->petsc_abstol, 100000, 0, c->true_residual);
    default: return solve_direct(c);
  }
}

/* relative residual ||b - A x|| / ||b|| of the assembled system at the current (u,v) */
static double relres_current(orc_ctx* c, const double* u, const double* v) {
  DECL_DIMS(c);
  csr_t* m = &c->m;
  double* xv = (double*)malloc(sizeof(double) * m->m);
  for (int n = 0; n < m->m; ++n) {
    if (c->n2ij[4 * n] >= 0) xv[n] = u[ICX(c->n2ij[4 * n + 1], c->n2ij[4 * n])];
    else xv[n] = v[ICY(c->n2ij[4 * n + 3], c->n2ij[4 * n + 2])];
  }
  double rr = 0.0, bb = 0.0;
  for (int i = 0; i < m->m; ++i) {
    double s = 0.0;
    for (int k = m->ptr[i]; k < m->ptr[i + 1]; ++k) s += m->val[k] * xv[m->idx[k]];
    double r = m->b[i] - s;
    rr += r * r; bb += m->b[i] * m->b[i];
  }
  free(xv);
  return bb > 0.0 ? sqrt(rr / bb) : sqrt(rr);
}

/* solve_DIVA_stag_linearised :1656-1761 */
static int solve_stag_linearised(orc_ctx* c, double* u, double* v) {
  DECL_DIMS(c);
  set_sico_masks(c);
  assemble(c, u, v);
  int st = linear_solve(c);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (i < nx - 1) u[ICX(j, i)] = c->m.x[c->ij2n_u[ICX(j, i)]];
      if (j < ny - 1) v[ICY(j, i)] = c->m.x[c->ij2n_v[ICY(j, i)]];
    }
  return st;
}

/* ------------------------------------------------------------------------ */
/* secondary velocities, ice_velocity_module.f90:377-661, 2592-2811          */

/* map_velocity_from_cx_to_a_3D :2647-2701 (nzl = nz) and _2D :2592-2646 (nzl = 1) */
static void map_vel_cx_to_a(orc_ctx* c, const double* ucx, double* ua, int nzl) {
  DECL_DIMS(c);
  const int32_t* ice = FI(c, MASK_ICE_A);
#define CXI(k, j, i) (((size_t)(i) * ny + (j)) * nzl + (k))
#define AI(k, j, i) (((size_t)(i) * ny + (j)) * nzl + (k))
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nzl; ++k) {
        double r;
        if (i == 0) r = (ice[IA(j, i)] == 1) ? ucx[CXI(k, j, i)] : 0.0;
        else if (i == nx - 1) r = (ice[IA(j, i)] == 1) ? ucx[CXI(k, j, i - 1)] : 0.0;
        else {
          int m0 = ice[IA(j, i - 1)], m1 = ice[IA(j, i)], m2 = ice[IA(j, i + 1)];
          if (m0 == 1 && m1 == 1 && m2 == 1) r = 0.5 * (ucx[CXI(k, j, i - 1)] + ucx[CXI(k, j, i)]);
          else if (m0 == 0 && m1 == 1 && m2 == 1) r = ucx[CXI(k, j, i)];
          else if (m0 == 1 && m1 == 1 && m2 == 0) r = ucx[CXI(k, j, i - 1)];
          else r = 0.0;
        }
        ua[AI(k, j, i)] = r;
      }
#undef CXI
#undef AI
}
/* map_velocity_from_cy_to_a_3D :2757-2811 and _2D :2702-2756 */
static void map_vel_cy_to_a(orc_ctx* c, const double* vcy, double* va, int nzl) {
  DECL_DIMS(c);
  const int32_t* ice = FI(c, MASK_ICE_A);
#define CYI(k, j, i) (((size_t)(i) * (ny - 1) + (j)) * nzl + (k))
#define AI(k, j, i) (((size_t)(i) * ny + (j)) * nzl + (k))
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nzl; ++k) {
        double r;
        if (j == 0) r = (ice[IA(j, i)] == 1) ? vcy[CYI(k, j, i)] : 0.0;
        else if (j == ny - 1) r = (ice[IA(j, i)] == 1) ? vcy[CYI(k, j - 1, i)] : 0.0;
        else {
          int m0 = ice[IA(j - 1, i)], m1 = ice[IA(j, i)], m2 = ice[IA(j + 1, i)];
          if (m0 == 1 && m1 == 1 && m2 == 1) r = 0.5 * (vcy[CYI(k, j - 1, i)] + vcy[CYI(k, j, i)]);
          else if (m0 == 0 && m1 == 1 && m2 == 1) r = vcy[CYI(k, j, i)];
          else if (m0 == 1 && m1 == 1 && m2 == 0) r = vcy[CYI(k, j - 1, i)];
          else r = 0.0;
        }
        va[AI(k, j, i)] = r;
      }
#undef CYI
#undef AI
}

/* calc_3D_vertical_velocities :534-661 (u_3D_a/v_3D_a read before they are refreshed) */
static void calc_3D_vertical_velocities(orc_ctx* c) {
  DECL_DIMS(c);
  const double dx = c->dx;
  const double* zeta = c->g.zeta;
  const size_t na = (size_t)nx * ny;
  double *lsx = (double*)malloc(na * sizeof(double)), *lsy = (double*)malloc(na * sizeof(double));
  double *lix = (double*)malloc(na * sizeof(double)), *liy = (double*)malloc(na * sizeof(double));
  const double *Hs = FD(c, HS_A), *Hi = FD(c, HI_A);
  ddx_a_to_a(nx, ny, dx, Hs, lsx);
  ddy_a_to_a(nx, ny, dx, Hs, lsy);
  ddx_a_to_a(nx, ny, dx, Hi, lix);
  ddy_a_to_a(nx, ny, dx, Hi, liy);
  const double *u3 = FD(c, U_3D_CX), *v3 = FD(c, V_3D_CY), *u3a = FD(c, U_3D_A), *v3a = FD(c, V_3D_A);
  const double *dHsdx = FD(c, DHS_DX_A), *dHsdy = FD(c, DHS_DY_A), *dHidx = FD(c, DHI_DX_A), *dHidy = FD(c, DHI_DY_A);
  const double* dHbdt = FD(c, DHB_DT_A);
  const int32_t* sheet = FI(c, MASK_SHEET_A);
  double* w = FD(c, W_3D_A);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      size_t q = IA(j, i);
      double dHbase_dx = lsx[q] - lix[q], dHbase_dy = lsy[q] - liy[q];
      double ub, vb;
      if (i == 0) ub = u3[ICX3(nz - 1, j, 0)];
      else if (i == nx - 1) ub = u3[ICX3(nz - 1, j, nx - 2)];
      else ub = 0.5 * (u3[ICX3(nz - 1, j, i - 1)] + u3[ICX3(nz - 1, j, i)]);
      if (j == 0) vb = v3[ICY3(nz - 1, 0, i)];
      else if (j == ny - 1) vb = v3[ICY3(nz - 1, ny - 2, i)];
      else vb = 0.5 * (v3[ICY3(nz - 1, j - 1, i)] + v3[ICY3(nz - 1, j, i)]);
      if (sheet[q] == 1) w[IA3(nz - 1, j, i)] = (ub * dHbase_dx) + (vb * dHbase_dy) + dHbdt[q];
      else w[IA3(nz - 1, j, i)] = (ub * dHbase_dx) + (vb * dHbase_dy);
      for (int k = nz - 2; k >= 0; --k) {
        double du_k, du_kp1, dv_k, dv_kp1;
        if (i == 0) { du_k = (u3[ICX3(k, j, 1)] - u3[ICX3(k, j, 0)]) / dx; du_kp1 = (u3[ICX3(k + 1, j, 1)] - u3[ICX3(k + 1, j, 0)]) / dx; }
        else if (i == nx - 1) { du_k = (u3[ICX3(k, j, nx - 2)] - u3[ICX3(k, j, nx - 3)]) / dx; du_kp1 = (u3[ICX3(k + 1, j, nx - 2)] - u3[ICX3(k + 1, j, nx - 3)]) / dx; }
        else { du_k = (u3[ICX3(k, j, i)] - u3[ICX3(k, j, i - 1)]) / dx; du_kp1 = (u3[ICX3(k + 1, j, i)] - u3[ICX3(k + 1, j, i - 1)]) / dx; }
        if (j == 0) { dv_k = (v3[ICY3(k, 1, i)] - v3[ICY3(k, 0, i)]) / dx; dv_kp1 = (v3[ICY3(k + 1, 1, i)] - v3[ICY3(k + 1, 0, i)]) / dx; }
        else if (j == ny - 1) { dv_k = (v3[ICY3(k, ny - 2, i)] - v3[ICY3(k, ny - 3, i)]) / dx; dv_kp1 = (v3[ICY3(k + 1, ny - 2, i)] - v3[ICY3(k + 1, ny - 3, i)]) / dx; }
        else { dv_k = (v3[ICY3(k, j, i)] - v3[ICY3(k, j - 1, i)]) / dx; dv_kp1 = (v3[ICY3(k + 1, j, i)] - v3[ICY3(k + 1, j - 1, i)]) / dx; }
        double w1 = (du_k + du_kp1) / 2.0, w2 = (dv_k + dv_kp1) / 2.0;
        double dz = zeta[k + 1] - zeta[k], zm = 0.5 * (zeta[k + 1] + zeta[k]);
        double w3 = ((dHsdx[q] - zm * dHidx[q]) / fmax(0.1, Hi[q])) * ((u3a[IA3(k + 1, j, i)] - u3a[IA3(k, j, i)]) / dz);
        double w4 = ((dHsdy[q] - zm * dHidy[q]) / fmax(0.1, Hi[q])) * ((v3a[IA3(k + 1, j, i)] - v3a[IA3(k, j, i)]) / dz);
        w[IA3(k, j, i)] = w[IA3(k + 1, j, i)] - Hi[q] * (w1 + w2 + w3 + w4) * dz;
      }
    }
  double *ws = FD(c, W_SURF_A), *wb = FD(c, W_BASE_A);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) { ws[IA(j, i)] = w[IA3(0, j, i)]; wb[IA(j, i)] = w[IA3(nz - 1, j, i)]; }
  free(lsx); free(lsy); free(lix); free(liy);
}

/* calc_secondary_velocities :377-533 */
static void calc_secondary_velocities(orc_ctx* c) {
  DECL_DIMS(c);
  const double* zeta = c->g.zeta;
  const int dyn = c->c.choice_ice_dynamics;
  double *u3 = FD(c, U_3D_CX), *v3 = FD(c, V_3D_CY);
  double *ub = FD(c, U_BASE_CX), *vb = FD(c, V_BASE_CY), *us = FD(c, U_SURF_CX), *vs = FD(c, V_SURF_CY);
  double *uv = FD(c, U_VAV_CX), *vv = FD(c, V_VAV_CY);
  const double *uS = FD(c, U_SSA_CX), *vS = FD(c, V_SSA_CY), *u3s = FD(c, U_3D_SIA_CX), *v3s = FD(c, V_3D_SIA_CY);
  const size_t ncx = (size_t)ny * (nx - 1), ncy = (size_t)(ny - 1) * nx;
  if (dyn == DIVA_DYN_SIA) {
    memcpy(u3, u3s, sizeof(double) * ncx * nz);
    memcpy(v3, v3s, sizeof(double) * ncy * nz);
    memset(ub, 0, sizeof(double) * ncx);
    memset(vb, 0, sizeof(double) * ncy);
    calc_3D_vertical_velocities(c);
    for (size_t q = 0; q < ncx; ++q) us[q] = u3[q * nz];
    for (size_t q = 0; q < ncy; ++q) vs[q] = v3[q * nz];
    for (size_t q = 0; q < ncx; ++q) uv[q] = vavg(zeta, nz, &u3[q * nz]);
    for (size_t q = 0; q < ncy; ++q) vv[q] = vavg(zeta, nz, &v3[q * nz]);
  } else if (dyn == DIVA_DYN_SSA) {
    memcpy(ub, uS, sizeof(double) * ncx);
    memcpy(vb, vS, sizeof(double) * ncy);
    for (size_t q = 0; q < ncx; ++q) { uv[q] = uS[q]; us[q] = uS[q]; for (int k = 0; k < nz; ++k) u3[q * nz + k] = uS[q]; }
    for (size_t q = 0; q < ncy; ++q) { vv[q] = vS[q]; vs[q] = vS[q]; for (int k = 0; k < nz; ++k) v3[q * nz + k] = vS[q]; }
  } else if (dyn == DIVA_DYN_SIA_SSA) {
    for (size_t q = 0; q < ncx; ++q) for (int k = 0; k < nz; ++k) u3[q * nz + k] = u3s[q * nz + k] + uS[q];
    for (size_t q = 0; q < ncy; ++q) for (int k = 0; k < nz; ++k) v3[q * nz + k] = v3s[q * nz + k] + vS[q];
    memcpy(ub, uS, sizeof(double) * ncx);
    memcpy(vb, vS, sizeof(double) * ncy);
    calc_3D_vertical_velocities(c);
    for (size_t q = 0; q < ncx; ++q) us[q] = u3[q * nz];
    for (size_t q = 0; q < ncy; ++q) vs[q] = v3[q * nz];
    for (size_t q = 0; q < ncx; ++q) uv[q] = vavg(zeta, nz, &u3[q * nz]);
    for (size_t q = 0; q < ncy; ++q) vv[q] = vavg(zeta, nz, &v3[q * nz]);
  } else {
    calc_3D_vertical_velocities(c);
    for (size_t q = 0; q < ncx; ++q) us[q] = u3[q * nz];
    for (size_t q = 0; q < ncy; ++q) vs[q] = v3[q * nz];
  }
  map_vel_cx_to_a(c, u3, FD(c, U_3D_A), nz);
  map_vel_cy_to_a(c, v3, FD(c, V_3D_A), nz);
  map_vel_cx_to_a(c, uv, FD(c, U_VAV_A), 1);
  map_vel_cy_to_a(c, vv, FD(c, V_VAV_A), 1);
  map_vel_cx_to_a(c, us, FD(c, U_SURF_A), 1);
  map_vel_cy_to_a(c, vs, FD(c, V_SURF_A), 1);
  map_vel_cx_to_a(c, ub, FD(c, U_BASE_A), 1);
  map_vel_cy_to_a(c, vb, FD(c, V_BASE_A), 1);
  const double *uva = FD(c, U_VAV_A), *vva = FD(c, V_VAV_A), *usa = FD(c, U_SURF_A), *vsa = FD(c, V_SURF_A);
  const double *uba = FD(c, U_BASE_A), *vba = FD(c, V_BASE_A);
  double *av = FD(c, UABS_VAV_A), *as = FD(c, UABS_SURF_A), *ab = FD(c, UABS_BASE_A), *Rs = FD(c, R_SHEAR);
  const int32_t* ice = FI(c, MASK_ICE_A);
  for (size_t q = 0; q < (size_t)nx * ny; ++q) {
    av[q] = sqrt(uva[q] * uva[q] + vva[q] * vva[q]);
    as[q] = sqrt(usa[q] * usa[q] + vsa[q] * vsa[q]);
    ab[q] = sqrt(uba[q] * uba[q] + vba[q] * vba[q]);
  }
  for (size_t q = 0; q < (size_t)nx * ny; ++q) {
    if (dyn == DIVA_DYN_SIA) Rs[q] = 1.0;
    else if (dyn == DIVA_DYN_SSA) Rs[q] = 0.0;
    else Rs[q] = (ice[q] == 1) ? fmax(0.0, fmin(1.0, (1.0 - ab[q] / as[q]))) : 0.0;
  }
}

/* ------------------------------------------------------------------------ */
/* SIA, ice_velocity_module.f90:36-114                                       */

int orc_calc_sia_3d_velocities(orc_ctx* c) {
  DECL_DIMS(c);
  const double* zeta = c->g.zeta;
  const double n = c->c.n_flow;
  double zn[64], f[64], D[64];
  for (int k = 0; k < nz; ++k) zn[k] = pow(zeta[k], n);
  const int32_t* sheet = FI(c, MASK_SHEET_A);
  const double *Hcx = FD(c, HI_CX), *Hcy = FD(c, HI_CY), *sxcx = FD(c, DHS_DX_CX), *sycx = FD(c, DHS_DY_CX);
  const double *sxcy = FD(c, DHS_DX_CY), *sycy = FD(c, DHS_DY_CY), *Acx = FD(c, A_FLOW_3D_CX), *Acy = FD(c, A_FLOW_3D_CY);
  double *u3 = FD(c, U_3D_SIA_CX), *v3 = FD(c, V_3D_SIA_CY);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (i < nx - 1) {
        if (sheet[IA(j, i)] == 0 && sheet[IA(j, i + 1)] == 0) {
          for (int k = 0; k < nz; ++k) u3[ICX3(k, j, i)] = 0.0;
        } else {
          size_t q = ICX(j, i);
          double D0 = pow(ICE_DENSITY * GRAV * Hcx[q], n) * pow((sxcx[q] * sxcx[q] + sycx[q] * sycx[q]), (n - 1.0) / 2.0);
          for (int k = 0; k < nz; ++k) f[k] = Acx[ICX3(k, j, i)] * zn[k];
          vint_bottom_to_zeta(zeta, nz, f, D);
          for (int k = 0; k < nz; ++k) {
            double Dd = 2.0 * Hcx[q] * D[k];
            u3[ICX3(k, j, i)] = fmax(D0 * Dd, -1E5) * sxcx[q];
          }
        }
      }
      if (j < ny - 1) {
        if (sheet[IA(j, i)] == 0 && sheet[IA(j + 1, i)] == 0) {
          for (int k = 0; k < nz; ++k) v3[ICY3(k, j, i)] = 0.0;
        } else {
          size_t q = ICY(j, i);
          double D0 = pow(ICE_DENSITY * GRAV * Hcy[q], n) * pow((sxcy[q] * sxcy[q] + sycy[q] * sycy[q]), (n - 1.0) / 2.0);
          for (int k = 0; k < nz; ++k) f[k] = Acy[ICY3(k, j, i)] * zn[k];
          vint_bottom_to_zeta(zeta, nz, f, D);
          for (int k = 0; k < nz; ++k) {
            double Dd = 2.0 * Hcy[q] * D[k];
            v3[ICY3(k, j, i)] = fmax(D0 * Dd, -1E5) * sycy[q];
          }
        }
      }
    }
  return DIVA_OK;
}

int orc_solve_sia(orc_ctx* c, diva_report_t* rep) {
  if (rep) memset(rep, 0, sizeof(*rep));
  if (!(c->c.choice_ice_dynamics == DIVA_DYN_SIA || c->c.choice_ice_dynamics == DIVA_DYN_SIA_SSA))
    return fail(c, DIVA_BAD_INPUT, "solve_SIA should only be called when choice_ice_dynamics is SIA or SIA/SSA");
  orc_calc_sia_3d_velocities(c);
  calc_secondary_velocities(c);
  if (rep) rep->relres = -1.0;
  return DIVA_OK;
}

/* ------------------------------------------------------------------------ */
/* the viscosity (Picard) iterations                                         */

static int any_sheet(orc_ctx* c) {
  DECL_DIMS(c);
  const int32_t* s = FI(c, MASK_SHEET_A);
  long sum = 0;
  for (size_t q = 0; q < (size_t)nx * ny; ++q) sum += s[q];
  return sum != 0;
}

static void calc_driving_stress(orc_ctx* c) {
  DECL_DIMS(c);
  const double *Hcx = FD(c, HI_CX), *Hcy = FD(c, HI_CY), *sx = FD(c, DHS_DX_CX), *sy = FD(c, DHS_DY_CY);
  double *tx = FD(c, TAUDX_CX), *ty = FD(c, TAUDY_CY);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (i < nx - 1) tx[ICX(j, i)] = -ICE_DENSITY * GRAV * Hcx[ICX(j, i)] * sx[ICX(j, i)];
      if (j < ny - 1) ty[ICY(j, i)] = -ICE_DENSITY * GRAV * Hcy[ICY(j, i)] * sy[ICY(j, i)];
    }
}

static int check_nan(orc_ctx* c, const double* a, size_t n) {
  for (size_t q = 0; q < n; ++q) if (!isfinite(a[q])) return 1;
  (void)c;
  return 0;
}

static void fill_err(orc_ctx* c) {
  DECL_DIMS(c);
  double *ex = FD(c, DIVA_ERR_CX), *ey = FD(c, DIVA_ERR_CY);
  for (size_t q = 0; q < (size_t)ny * (nx - 1); ++q) ex[q] = 1E5;
  for (size_t q = 0; q < (size_t)(ny - 1) * nx; ++q) ey[q] = 1E5;
}

/* ------------------------------------------------------------------------ */
/* Anderson mixing of the viscosity iteration (picard_anderson_m > 0).  No counterpart in
 * the reference, whose update is relax_DIVA_visc_iterations (:1499-1529): the oracle's own
 * restatement of the GPU library's mixing step, to check it.  The map is one unrelaxed
 * Picard step g(u) (the velocity-limited linear solution), f = g(u) - u, dF_i / dG_i the
 * differences of consecutive residuals / map values; the next iterate is
 * g - sum gamma_i dG_i with gamma minimising |f - sum gamma_i dF_i|_2 over the n <= m most
 * recent columns (normal equations scaled to unit diagonal, + 1e-10; on a Cholesky pivot
 * below 1e-12, or when the coefficients' magnitudes sum to more than 20, the oldest column
 * is dropped).  A nonlinear residual 10 x the previous step's drops the older columns. */
#define AA_MAX 5
#define AA_GAMMA_MAX 20.0   /* largest sum of |gamma_i| a mixing step accepts, else drop columns */

static void aa_reset(orc_ctx* c) {
  const size_t n = (size_t)c->ny * (c->nx - 1) + (size_t)(c->ny - 1) * c->nx;
  for (int k = 0; k < AA_MAX; ++k) {
    if (!c->aa_dF[k]) c->aa_dF[k] = (double*)malloc(sizeof(double) * n);
    if (!c->aa_dG[k]) c->aa_dG[k] = (double*)malloc(sizeof(double) * n);
    memset(c->aa_dF[k], 0, sizeof(double) * n);
    memset(c->aa_dG[k], 0, sizeof(double) * n);
  }
  if (!c->aa_f) c->aa_f = (double*)malloc(sizeof(double) * n);
  if (!c->aa_g) c->aa_g = (double*)malloc(sizeof(double) * n);
  c->aa_have = 0; c->aa_n = 0; c->aa_head = 0; c->aa_restarts = 0; c->aa_rprev = 0.0;
  c->aa_off = 0; c->aa_since = 0; c->aa_best = 0.0;
  memset(c->aa_G, 0, sizeof(c->aa_G));
}

/* gamma from dots[0..m) = dF_i . dF_new and dots[AA_MAX..AA_MAX+m) = dF_i . f */
static void aa_coefficients(orc_ctx* c, int m, const double* dots, double relres) {
  double* G = c->aa_G;
  for (int k = 0; k < AA_MAX; ++k) c->aa_gamma[k] = 0.0;
  const double rprev = c->aa_rprev;
  c->aa_rprev = relres;
  /* mixing that has not lowered rel-res by 10 % in 20 steps is given up: relaxation */
  if (c->aa_off) return;
  if (c->aa_best == 0.0 || relres < 0.9 * c->aa_best) { c->aa_best = relres; c->aa_since = 0; }
  else if (++c->aa_since >= 20) { c->aa_off = 1; return; }
  if (!c->aa_have) { c->aa_have = 1; c->aa_n = 0; c->aa_head = 0; return; }
  const int s = c->aa_head;
  int n = c->aa_n;
  if (rprev > 0.0 && relres > 10.0 * rprev) { n = 0; c->aa_restarts++; }
  for (int i = 0; i < m; ++i) {
    G[s * AA_MAX + i] = dots[i];
    G[i * AA_MAX + s] = dots[i];
    c->aa_rhs[i] = dots[AA_MAX + i];
  }
  n = n + 1 < m ? n + 1 : m;
  c->aa_head = (s + 1) % m;
  int idx[AA_MAX];
  for (int k = 0; k < n; ++k) idx[k] = (s - k + m) % m;
  for (int nn = n; nn > 0; --nn) {
    double A[AA_MAX][AA_MAX], b[AA_MAX], dk[AA_MAX], y[AA_MAX];
    int ok = 1;
    for (int k = 0; k < nn && ok; ++k) {
      dk[k] = sqrt(G[idx[k] * AA_MAX + idx[k]]);
      ok = dk[k] > 0.0 && dk[k] < 1e300;
    }
    if (!ok) continue;
    for (int k = 0; k < nn; ++k) {
      for (int l = 0; l < nn; ++l) A[k][l] = G[idx[k] * AA_MAX + idx[l]] / (dk[k] * dk[l]);
      A[k][k] += 1e-10;
      b[k] = c->aa_rhs[idx[k]] / dk[k];
    }
    for (int k = 0; k < nn && ok; ++k) {
      double p = A[k][k];
      for (int l = 0; l < k; ++l) p -= A[k][l] * A[k][l];
      if (!(p > 1e-12)) { ok = 0; break; }
      const double r = sqrt(p);
      A[k][k] = r;
      for (int i = k + 1; i < nn; ++i) {
        double t = A[i][k];
        for (int l = 0; l < k; ++l) t -= A[i][l] * A[k][l];
        A[i][k] = t / r;
      }
    }
    if (!ok) continue;
    for (int k = 0; k < nn; ++k) {
      double t = b[k];
      for (int l = 0; l < k; ++l) t -= A[k][l] * y[l];
      y[k] = t / A[k][k];
    }
    for (int k = nn - 1; k >= 0; --k) {
      double t = y[k];
      for (int l = k + 1; l < nn; ++l) t -= A[l][k] * y[l];
      y[k] = t / A[k][k];
    }
    double gsum = 0.0;
    for (int k = 0; k < nn; ++k) {
      y[k] = y[k] / dk[k];
      ok = ok && isfinite(y[k]);
      gsum += fabs(y[k]);
    }
    if (!ok || !(gsum <= AA_GAMMA_MAX)) continue;
    for (int k = 0; k < nn; ++k) c->aa_gamma[idx[k]] = y[k];
    c->aa_n = nn;
    return;
  }
  c->aa_n = 0;
}

/* on entry u, v hold the map value g and U_CX_PREV / V_CY_PREV the iterate; on exit u, v
 * hold the mixed iterate */
static void anderson_mix(orc_ctx* c, double* u, double* v, double relres) {
  DECL_DIMS(c);
  const int m = c->c.picard_anderson_m;
  const double *up = FD(c, U_CX_PREV), *vp = FD(c, V_CY_PREV);
  const size_t ncx = (size_t)ny * (nx - 1);
  const int s = c->aa_head, have = c->aa_have;
  double dots[2 * AA_MAX] = {0};
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      for (int comp = 0; comp < 2; ++comp) {
        size_t q;
        double g, x;
        if (comp == 0) { if (i >= nx - 1) continue; q = ICX(j, i); g = u[q]; x = up[q]; }
        else { if (j >= ny - 1) continue; q = ncx + ICY(j, i); g = v[ICY(j, i)]; x = vp[ICY(j, i)]; }
        const double f = g - x;
        if (have) {
          const double df = f - c->aa_f[q];
          c->aa_dF[s][q] = df;
          c->aa_dG[s][q] = g - c->aa_g[q];
          for (int k = 0; k < m; ++k) {
            const double col = (k == s) ? df : c->aa_dF[k][q];
            dots[k] += col * df;
            dots[AA_MAX + k] += col * f;
          }
        }
        c->aa_f[q] = f;
        c->aa_g[q] = g;
      }
    }
  aa_coefficients(c, m, dots, relres);
  if (c->aa_off) {   /* mixing given up: the relaxation of the map value */
    const double rel = c->c.DIVA_visc_it_relax;
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j) {
        if (i < nx - 1) u[ICX(j, i)] = rel * c->aa_g[ICX(j, i)] + (1.0 - rel) * up[ICX(j, i)];
        if (j < ny - 1) v[ICY(j, i)] = rel * c->aa_g[ncx + ICY(j, i)] + (1.0 - rel) * vp[ICY(j, i)];
      }
    return;
  }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (i < nx - 1) {
        const size_t q = ICX(j, i);
        double w = c->aa_g[q];
        for (int k = 0; k < m; ++k) w -= c->aa_gamma[k] * c->aa_dG[k][q];
        u[q] = w;
      }
      if (j < ny - 1) {
        const size_t q = ncx + ICY(j, i);
        double w = c->aa_g[q];
        for (int k = 0; k < m; ++k) w -= c->aa_gamma[k] * c->aa_dG[k][q];
        v[ICY(j, i)] = w;
      }
    }
}

/* shared Picard loop of solve_SSA (:180-240) and solve_DIVA (:307-363) */
static int picard(orc_ctx* c, int diva, double* u, double* v, diva_report_t* rep) {
  DECL_DIMS(c);
  const diva_config_t* C = &c->c;
  const size_t ncx = (size_t)ny * (nx - 1), ncy = (size_t)(ny - 1) * nx;
  int it = 0, status = DIVA_OK;
  double resid = 0.0, relres = -1.0;
  long lin0 = c->lin_iters_total;
  const int relmode = (C->picard_stop == DIVA_STOP_RELRES);
  int exited_by_relres = 0;
  double eta = C->lin_adaptive_eta, relres_prev = 0.0;
  const int aa = relmode && C->picard_anderson_m > 0;
  int stalled = 0;   /* a rel-res loop stopped on picard_stall_its (the GPU library's rule) */
  double stall_best = 0.0;
  int stall_since = 0;
  if (aa) aa_reset(c);
  for (;;) {
    ++it;
    if (diva) calc_vertical_shear_strain_rates(c);
    calc_effective_viscosity(c, u, v);
    calc_sliding_term_beta(c, u, v);
    if (diva) {
      calc_F_integral(c);
      calc_beta_eff(c);
    } else {
      /* solve_SSA :192-206 */
      memcpy(FD(c, BETA_EFF_A), FD(c, BETA_A), sizeof(double) * (size_t)nx * ny);
      map_a_to_cx(nx, ny, FD(c, BETA_EFF_A), FD(c, BETA_EFF_CX));
      map_a_to_cy(nx, ny, FD(c, BETA_EFF_A), FD(c, BETA_EFF_CY));
      double *bcx = FD(c, BETA_EFF_CX), *bcy = FD(c, BETA_EFF_CY);
      const double *fcx = FD(c, F_GRND_CX), *fcy = FD(c, F_GRND_CY);
      for (size_t q = 0; q < ncx; ++q) bcx[q] = bcx[q] * (fcx[q] * fcx[q]);
      for (size_t q = 0; q < ncy; ++q) bcy[q] = bcy[q] * (fcy[q] * fcy[q]);
    }
    if (relmode) {
      set_sico_masks(c);
      assemble(c, u, v);
      relres = relres_current(c, u, v);
      /* adaptive tolerance factor: halved (floor 0.05) when, within 100 x the stop
       * tolerance, the residual did not fall */
      if (relres_prev > 0.0 && relres >= relres_prev && relres < 100.0 * C->picard_relres_tol)
        eta = fmax(0.05, 0.5 * eta);
      relres_prev = relres;
      if (relres <= C->picard_relres_tol) { exited_by_relres = 1; }
      else if (C->picard_stall_its > 0) {
        /* stagnation: rel-res not below 0.9 x its lowest for picard_stall_its iterations */
        if (stall_best == 0.0 || relres < 0.9 * stall_best) { stall_best = relres; stall_since = 0; }
        else if (++stall_since >= C->picard_stall_its) { exited_by_relres = 1; stalled = 1; }
      }
    }
    if (exited_by_relres) {
      if (diva) { calc_basal_stress(c); calc_basal_velocities(c); }
      break;
    }
    memcpy(FD(c, U_CX_PREV), u, sizeof(double) * ncx);
    memcpy(FD(c, V_CY_PREV), v, sizeof(double) * ncy);
    /* same adaptive linear tolerance rule as the GPU library (iterative solvers only) */
    const int adaptive = relmode && C->lin_adaptive &&
                         (c->lin_solver == ORC_LIN_GMRES_ILU || c->lin_solver == ORC_LIN_GMRES_WARM);
    if (adaptive) c->petsc_rtol = fmax(C->lin_rtol, eta * fmin(1.0, relres));
    c->true_residual = adaptive;
    int st = solve_stag_linearised(c, u, v);
    c->true_residual = 0;
    if (st != DIVA_OK) status = st;
    apply_velocity_limits(c, u, v);
    if (aa) anderson_mix(c, u, v, relres);
    else relax_visc_iterations(c, u, v, C->DIVA_visc_it_relax);
    resid = calc_visc_iter_UV_resid(c, u, v);
    int converged = 0;
    if (!relmode && resid < C->DIVA_visc_it_norm_dUV_tol) converged = 1;
    else if (it >= C->DIVA_visc_it_nit) converged = 1;

    if (!converged) estimate_visc_iter_UV_errors(c, u, v);
    if (diva) { calc_basal_stress(c); calc_basal_velocities(c); }
    if (check_nan(c, u, ncx) || check_nan(c, v, ncy)) { status = DIVA_NAN_DETECTED; break; }
    if (converged) {
      if (it >= C->DIVA_visc_it_nit && (relmode || resid >= C->DIVA_visc_it_norm_dUV_tol) && status == DIVA_OK)
        status = DIVA_MAX_PICARD;
      break;
    }
  }
  if (stalled && status == DIVA_OK) status = DIVA_MAX_PICARD;
  if (rep) {
    rep->picard_iterations = it;
    rep->linear_iterations = (int32_t)(c->lin_iters_total - lin0);
    rep->resid_UV = resid;
    rep->relres = relres;
    rep->status = status;
    rep->reserved[2] = stalled;
  }
  return status;
}

int orc_solve_diva(orc_ctx* c, diva_report_t* rep) {
  DECL_DIMS(c);
  if (rep) { memset(rep, 0, sizeof(*rep)); rep->relres = -1.0; }
  if (c->c.choice_ice_dynamics != DIVA_DYN_DIVA)
    return fail(c, DIVA_BAD_INPUT, "solve_DIVA should only be called when choice_ice_dynamics is DIVA");
  if (!any_sheet(c)) {
    memset(FD(c, U_VAV_CX), 0, sizeof(double) * (size_t)ny * (nx - 1));
    memset(FD(c, V_VAV_CY), 0, sizeof(double) * (size_t)(ny - 1) * nx);
    return DIVA_OK;
  }
  calc_driving_stress(c);
  calc_basal_conditions(c);
  determine_grounded_fractions(c);
  fill_err(c);
  int st = picard(c, 1, FD(c, U_VAV_CX), FD(c, V_VAV_CY), rep);
  if (st == DIVA_NAN_DETECTED) return fail(c, st, "NaN in the DIVA velocities");
  calc_3D_horizontal_velocities_DIVA(c);
  calc_secondary_velocities(c);
  return st;
}

int orc_solve_ssa(orc_ctx* c, diva_report_t* rep) {
  DECL_DIMS(c);
  if (rep) { memset(rep, 0, sizeof(*rep)); rep->relres = -1.0; }
  if (!(c->c.choice_ice_dynamics == DIVA_DYN_SSA || c->c.choice_ice_dynamics == DIVA_DYN_SIA_SSA))
    return fail(c, DIVA_BAD_INPUT, "solve_SSA should only be called when choice_ice_dynamics is SSA or SIA/SSA");
  if (!any_sheet(c) || c->c.choice_sliding_law == DIVA_SLIDING_NONE) {
    memset(FD(c, U_SSA_CX), 0, sizeof(double) * (size_t)ny * (nx - 1));
    memset(FD(c, V_SSA_CY), 0, sizeof(double) * (size_t)(ny - 1) * nx);
    return DIVA_OK;
  }
  calc_driving_stress(c);
  calc_basal_conditions(c);
  determine_grounded_fractions(c);
  fill_err(c);
  int st = picard(c, 0, FD(c, U_SSA_CX), FD(c, V_SSA_CY), rep);
  if (st == DIVA_NAN_DETECTED) return fail(c, st, "NaN in the SSA velocities");
  calc_secondary_velocities(c);
  return st;
}

int orc_nonlinear_residual(orc_ctx* c, double* relres) {
  /* coefficients of the next DIVA viscosity iteration at the current state */
  DECL_DIMS(c);
  double *u = FD(c, U_VAV_CX), *v = FD(c, V_VAV_CY);
  calc_driving_stress(c);
  calc_basal_conditions(c);
  determine_grounded_fractions(c);
  calc_vertical_shear_strain_rates(c);
  calc_effective_viscosity(c, u, v);
  calc_sliding_term_beta(c, u, v);
  calc_F_integral(c);
  calc_beta_eff(c);
  set_sico_masks(c);
  assemble(c, u, v);
  *relres = relres_current(c, u, v);
  (void)nx; (void)ny;
  return DIVA_OK;
}

/* The column-local stages of one DIVA viscosity iteration (A3-A7,
 * ice_velocity_module.f90:664-1086) and the basal stress and velocities
 * (:1087-1199), `sweeps` times with u_vav held fixed and no linear solve: the
 * iteration state that belongs to the given velocities.  Test infrastructure: the
 * restatement the device's diva_complete_state is checked against. */
int orc_diva_coefficients(orc_ctx* c);
int orc_complete_state(orc_ctx* c, int32_t sweeps) {
  if (sweeps < 0 || sweeps > 10000) return DIVA_BAD_INPUT;
  calc_driving_stress(c);
  calc_basal_conditions(c);
  determine_grounded_fractions(c);
  for (int s = 0; s < sweeps; ++s) {
    orc_diva_coefficients(c);
    calc_basal_stress(c);
    calc_basal_velocities(c);
  }
  return DIVA_OK;
}

/* ------------------------------------------------------------------------ */
/* context, I/O and configuration                                            */

void orc_config_defaults(diva_config_t* c) {
  memset(c, 0, sizeof(*c));
  c->choice_ice_dynamics = DIVA_DYN_DIVA;
  c->n_flow = 3.0; c->m_enh_sheet = 1.0; c->m_enh_shelf = 1.0;
  c->choice_ice_margin = DIVA_MARGIN_INFINITE_SLAB;
  c->include_SSADIVA_crossterms = 1; c->do_GL_subgrid_friction = 1;
  c->DIVA_visc_it_norm_dUV_tol = 1E-2; c->DIVA_visc_it_nit = 50; c->DIVA_visc_it_relax = 0.4;
  c->DIVA_epsilon_sq_0 = 1E-15; c->DIVA_visc_eff_min = 1E3; c->DIVA_beta_max = 1E20; c->DIVA_vel_max = 5000.0;
  c->choice_sliding_law = DIVA_SLIDING_COULOMB_REGULARISED;
  c->slid_delta_v = 1.0E-3; c->slid_Weertman_m = 3.0; c->slid_Coulomb_reg_q_plastic = 0.3;
  c->slid_Coulomb_reg_u_threshold = 100.0; c->slid_ZI_ut = 200.0; c->slid_ZI_p = 5.0;
  c->include_basal_freezing = 1; c->deltaT_basal_freezing = 2.0;
  c->choice_basal_hydrology = DIVA_HYDRO_MARTIN2011; c->Martin2011_hydro_Hb_min = 0.0; c->Martin2011_hydro_Hb_max = 1000.0;
  c->choice_ice_rheology = DIVA_RHEO_HUYBRECHTS1992; c->uniform_flow_factor = 1E-16;
  c->do_ocean_floodfill = 1;
  c->lin_rtol = 1E-8; c->lin_maxit = 2000;
  c->picard_stop = DIVA_STOP_RESID_UV; c->picard_relres_tol = 1E-6; c->lin_adaptive = 0; c->lin_adaptive_eta = 0.5;
  c->dt_thermo = 10.0;                                   /* configuration_module.f90:56, 427-430, 647 */
  c->choice_ice_heat_capacity = DIVA_HEATCAP_POUNDER1965; c->uniform_ice_heat_capacity = 2009.0;
  c->choice_ice_thermal_conductivity = DIVA_CONDUCT_RITZ1987; c->uniform_ice_thermal_conductivity = 6.626958E7;
  c->T_ocean_mean_PD_ANT = -1.7;
  c->choice_ice_integration_method = DIVA_INTEGRATION_EXPLICIT; c->dHi_rtol = 1E-10; c->dHi_maxit = 1000;
  c->choice_calving_law = DIVA_CALVING_THRESHOLD_THICKNESS; c->calving_threshold_thickness = 200.0;
  c->continental_shelf_min_height = -2000.0;
  c->precision = DIVA_PREC_FP64;
}

int orc_field_info(int32_t id, diva_field_info_t* out) {
  if (id < 0 || id >= DIVA_NUM_FIELDS || !out) return DIVA_BAD_INPUT;
  *out = g_info[id];
  return DIVA_OK;
}

int orc_create(orc_ctx** out, const diva_grid_t* g, const diva_config_t* cfg) {
  if (!out || !g || !cfg) return DIVA_BAD_INPUT;
  *out = NULL;
  if (g->nx < 5 || g->ny < 5 || g->nz < 2 || g->nz > 64 || !(g->dx > 0.0)) return DIVA_BAD_INPUT;
  orc_ctx* c = (orc_ctx*)calloc(1, sizeof(orc_ctx));
  c->g = *g; c->c = *cfg;
  c->nx = g->nx; c->ny = g->ny; c->nz = g->nz; c->dx = g->dx;
  for (int f = 0; f < DIVA_NUM_FIELDS; ++f) {
    int64_t ne = numel_kind(c->nx, c->ny, c->nz, g_info[f].grid);
    size_t es = g_info[f].dtype == DIVA_DTYPE_D ? sizeof(double) : sizeof(int32_t);
    c->F[f] = calloc((size_t)ne, es);
  }
  /* initialise_SSADIVA_solution_matrix :2814-2860 */
  const int nx = c->nx, ny = c->ny;
  c->neq = (nx - 1) * ny + nx * (ny - 1);
  c->ij2n_u = (int*)malloc(sizeof(int) * (size_t)ny * (nx - 1));
  c->ij2n_v = (int*)malloc(sizeof(int) * (size_t)(ny - 1) * nx);
  c->n2ij = (int*)malloc(sizeof(int) * 4 * (size_t)c->neq);
  for (int q = 0; q < 4 * c->neq; ++q) c->n2ij[q] = -1;
  int n = 0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      if (i < nx - 1) { c->ij2n_u[ICX(j, i)] = n; c->n2ij[4 * n] = i; c->n2ij[4 * n + 1] = j; ++n; }
      if (j < ny - 1) { c->ij2n_v[ICY(j, i)] = n; c->n2ij[4 * n + 2] = i; c->n2ij[4 * n + 3] = j; ++n; }
    }
  c->m.m = c->neq;
  c->m.nnz_max = 9 * c->neq;
  c->m.ptr = (int*)calloc((size_t)c->neq + 1, sizeof(int));
  c->m.idx = (int*)calloc((size_t)c->m.nnz_max, sizeof(int));
  c->m.val = (double*)calloc((size_t)c->m.nnz_max, sizeof(double));
  c->m.b = (double*)calloc((size_t)c->neq, sizeof(double));
  c->m.x = (double*)calloc((size_t)c->neq, sizeof(double));
  c->lin_solver = ORC_LIN_DIRECT;
  c->SOR_nit = 10000; c->SOR_tol = 2.5; c->SOR_omega = 1.3;
  c->petsc_rtol = 0.01; c->petsc_abstol = 2.5;
  *out = c;
  return DIVA_OK;
}

int orc_destroy(orc_ctx* c) {
  if (!c) return DIVA_OK;
  for (int f = 0; f < DIVA_NUM_FIELDS; ++f) { free(c->F[f]); free(c->S[f]); }
  free(c->ij2n_u); free(c->ij2n_v); free(c->n2ij);
  free(c->m.ptr); free(c->m.idx); free(c->m.val); free(c->m.b); free(c->m.x);
  for (int k = 0; k < AA_MAX; ++k) { free(c->aa_dF[k]); free(c->aa_dG[k]); }
  free(c->aa_f); free(c->aa_g);
  pool_destroy(c->pool);
  free(c);
  return DIVA_OK;
}

int orc_set_config(orc_ctx* c, const diva_config_t* cfg) { c->c = *cfg; return DIVA_OK; }

/* kind: 0 direct (banded LU), 1 SOR, 2 GMRES(30)+ILU(0) from zero (PETSc default), 3 the same from the current iterate */
int orc_set_linear_solver(orc_ctx* c, int kind, double rtol, double abstol, int sor_nit, double sor_tol, double sor_omega) {
  c->lin_solver = kind;
  c->petsc_rtol = rtol; c->petsc_abstol = abstol;
  c->SOR_nit = sor_nit; c->SOR_tol = sor_tol; c->SOR_omega = sor_omega;
  return DIVA_OK;
}

static size_t field_bytes(orc_ctx* c, int f) {
  return (size_t)numel_kind(c->nx, c->ny, c->nz, g_info[f].grid) *
         (g_info[f].dtype == DIVA_DTYPE_D ? sizeof(double) : sizeof(int32_t));
}
int orc_upload_field(orc_ctx* c, int32_t id, const void* host) {
  if (id < 0 || id >= DIVA_NUM_FIELDS || !host) return DIVA_BAD_INPUT;
  memcpy(c->F[id], host, field_bytes(c, id));
  return DIVA_OK;
}
int orc_download_field(orc_ctx* c, int32_t id, void* host) {
  if (id < 0 || id >= DIVA_NUM_FIELDS || !host) return DIVA_BAD_INPUT;
  memcpy(host, c->F[id], field_bytes(c, id));
  return DIVA_OK;
}
int orc_upload(orc_ctx* c, const diva_fields_t* f) {
  for (int q = 0; q < DIVA_NUM_FIELDS; ++q) if (f->ptr[q]) orc_upload_field(c, q, f->ptr[q]);
  return DIVA_OK;
}
int orc_download(orc_ctx* c, const diva_fields_t* f) {
  for (int q = 0; q < DIVA_NUM_FIELDS; ++q) if (f->ptr[q]) orc_download_field(c, q, f->ptr[q]);
  return DIVA_OK;
}

/* Assembled matrix of the last linear solve (0-based CSR) for operator tests. */
int orc_matrix(orc_ctx* c, int* m, int* nnz, const int** ptr, const int** idx, const double** val, const double** b, const double** x) {
  *m = c->m.m; *nnz = c->m.nnz; *ptr = c->m.ptr; *idx = c->m.idx; *val = c->m.val; *b = c->m.b; *x = c->m.x;
  return DIVA_OK;
}
/* Assemble the DIVA matrix at the current (u_vav_cx, v_vav_cy) with the current coefficient fields. */
int orc_assemble_current(orc_ctx* c) {
  set_sico_masks(c);
  assemble(c, FD(c, U_VAV_CX), FD(c, V_VAV_CY));
  return DIVA_OK;
}
/* Run the stages of solve_DIVA before the viscosity loop (tau_d, basal conditions, f_grnd). */
int orc_prepare_diva(orc_ctx* c) {
  calc_driving_stress(c);
  calc_basal_conditions(c);
  determine_grounded_fractions(c);
  return DIVA_OK;
}
/* One set of DIVA coefficient stages (A3-A7) at the current state. */
/* ------------------------------------------------------------------------ */
/* Ice-thickness update and the predictor/corrector step (the consumers of   */
/* u_vav inside a time step)                                                 */

/* Hi_from_Hb_and_Hs, utilities_module.f90:160-183 */
static double hi_from_hb_and_hs(double Hb, double Hs, double SL) {
  const double Hs_float = Hb + (SL - Hb) * SW_DENSITY / ICE_DENSITY;
  if (Hs > Hs_float) return Hs - Hb;
  return (Hs - SL) / (1.0 - ICE_DENSITY / SW_DENSITY);
}

/* determine_floating_margin_fraction, general_ice_model_data_module.f90:784-865
 * (rows 2..ny-1 only; the first and last rows keep their values) */
static void floating_margin_fraction(orc_ctx* c) {
  DECL_DIMS(c);
  const double* Hi = FD(c, HI_A);
  const int32_t *ice = FI(c, MASK_ICE_A), *cf = FI(c, MASK_CF_A), *shelf = FI(c, MASK_SHELF_A);
  double *fmf = FD(c, FLOAT_MARGIN_FRAC_A), *Heff = FD(c, HI_EFF_CF_A);
  for (int i = 0; i < nx; ++i)
    for (int j = 1; j < ny - 1; ++j) {
      const size_t q = IA(j, i);
      fmf[q] = ice[q] == 1 ? 1.0 : 0.0;
      Heff[q] = ice[q] == 1 ? Hi[q] : 0.0;
      if (!(cf[q] == 1 && shelf[q] == 1)) continue;
      int inner_neighbours = 0;
      double Hmax = 0.0;
      for (int ii = (i > 0 ? i - 1 : 0); ii <= (i < nx - 1 ? i + 1 : nx - 1); ++ii)
        for (int jj = j - 1; jj <= j + 1; ++jj) {
          const size_t p = IA(jj, ii);
          if (ice[p] == 1 && cf[p] == 0) { inner_neighbours = 1; Hmax = fmax(Hmax, Hi[p]); }
        }
      if (!inner_neighbours || Hmax < Hi[q]) { fmf[q] = 1.0; Heff[q] = Hi[q]; continue; }
      fmf[q] = Hi[q] / Hmax;
      Heff[q] = Hmax;
    }
}

/* apply_ice_thickness_BC, ice_thickness_module.f90:728-931: west, east, south, north */
static void apply_ice_thickness_bc(orc_ctx* c, double dt) {
  DECL_DIMS(c);
  const double *Hi = FD(c, HI_A), *Hb = FD(c, HB_A), *SL = FD(c, SL_A);
  double *Hn = FD(c, HI_TPLUSDT_A), *dH = FD(c, DHI_DT_A);
  const int diva = c->c.choice_ice_dynamics == DIVA_DYN_DIVA;
  const int bc[4] = {c->c.ice_thickness_west_BC, c->c.ice_thickness_east_BC, c->c.ice_thickness_south_BC,
                     c->c.ice_thickness_north_BC};
  for (int side = 0; side < 4; ++side) {
    const int xside = side < 2;
    const int n = xside ? ny : nx;                             /* points along the side */
    const int edge = side == 0 ? 0 : side == 1 ? nx - 1 : side == 2 ? 0 : ny - 1;
    const int inner = side == 0 ? 1 : side == 1 ? nx - 2 : side == 2 ? 1 : ny - 2;
    const int opposite = side == 0 ? nx - 2 : side == 1 ? 1 : side == 2 ? ny - 2 : 1;
    for (int k = 0; k < n; ++k) {
      const size_t q = xside ? IA(k, edge) : IA(edge, k);
      const size_t qi = xside ? IA(k, inner) : IA(inner, k);
      const size_t qo = xside ? IA(k, opposite) : IA(opposite, k);
      switch (bc[side]) {
        case DIVA_HBC_ZERO:
          Hn[q] = 0.0; dH[q] = -Hi[q] / dt;
          if (diva) { Hn[qi] = 0.0; dH[qi] = -Hi[qi] / dt; }
          break;
        case DIVA_HBC_INFINITE: {
          const double Hs_nb = surface_elevation(Hn[qi], Hb[qi], SL[qi]);
          Hn[q] = hi_from_hb_and_hs(Hb[q], Hs_nb, SL[q]);
          dH[q] = (Hn[q] - Hi[q]) / dt;
          break;
        }
        case DIVA_HBC_PERIODIC: Hn[q] = Hi[qo]; dH[q] = (Hn[q] - Hi[q]) / dt; break;
        case DIVA_HBC_FIXED: Hn[q] = Hi[q]; dH[q] = 0.0; break;
        default: break;                                        /* 'none' */
      }
    }
  }
}

/* The rows of calc_dHi_dt_semiimplicit (ice_thickness_module.f90:302-727) for cell (j,i):
 * *ident = 1 for a mass-balance-only or explicit row (x = b), else the over-implicit row
 * diag x + cw x_W + ce x_E + cs x_S + cn x_N = b; *x0 the first guess. */
static void semiimplicit_row(orc_ctx* c, double dt, int i, int j, int* ident, double* diag, double* cw,
                             double* ce, double* cs, double* cn, double* b, double* x0) {
  DECL_DIMS(c);
  const double fs = 2.5, dx = c->dx;
  const double *Hi = FD(c, HI_A), *u = FD(c, U_VAV_CX), *v = FD(c, V_VAV_CY);
  const double *smb = FD(c, SMB_A), *bmb = FD(c, BMB_A), *fmf = FD(c, FLOAT_MARGIN_FRAC_A);
  const int32_t *ice = FI(c, MASK_ICE_A), *shelf = FI(c, MASK_SHELF_A), *ocean = FI(c, MASK_OCEAN_A);
  const int32_t* cf = FI(c, MASK_CF_A);
  const int im1 = i > 0 ? i - 1 : 0, ip1 = i < nx - 1 ? i + 1 : nx - 1;
  const int jm1 = j > 0 ? j - 1 : 0, jp1 = j < ny - 1 ? j + 1 : ny - 1;
  const size_t q = IA(j, i), qw = IA(j, im1), qe = IA(j, ip1), qs = IA(jm1, i), qn = IA(jp1, i);
  int scheme;   /* 0 MB-only, 1 explicit, 2 semi-implicit (:327-347) */
  if (ice[q] == 0 && ice[qw] == 0 && ice[qe] == 0 && ice[qs] == 0 && ice[qn] == 0) scheme = 0;
  else if (shelf[q] == 1 && ((ocean[qw] == 1 && ice[qw] == 0) || (ocean[qe] == 1 && ice[qe] == 0) ||
                             (ocean[qs] == 1 && ice[qs] == 0) || (ocean[qn] == 1 && ice[qn] == 0))) scheme = 1;
  else if (ocean[q] == 1 && ice[q] == 0 && (shelf[qw] == 1 || shelf[qe] == 1 || shelf[qs] == 1 || shelf[qn] == 1))
    scheme = 1;
  else scheme = 2;
  double mb;
  if (cf[q] == 1 && shelf[q] == 1) mb = (smb[q] + bmb[q]) * fmf[q];
  else if (ocean[q] == 1 && shelf[q] == 0) mb = 0.0;
  else mb = smb[q] + bmb[q];
  /* a face between a shelf cell and open ocean carries nothing until the shelf cell is
   * full (float_margin_frac_a < 1), :501-531 and :573-620 */
  int cut_w = 0, cut_e = 0, cut_s = 0, cut_n = 0;
  if (i > 0) {
    if (shelf[q] == 1 && ocean[qw] == 1 && ice[qw] == 0) cut_w = fmf[q] < 1.0;
    else if (shelf[qw] == 1 && ocean[q] == 1 && ice[q] == 0) cut_w = fmf[qw] < 1.0;
  }
  if (i < nx - 1) {
    if (shelf[q] == 1 && ocean[qe] == 1 && ice[qe] == 0) cut_e = fmf[q] < 1.0;
    else if (shelf[qe] == 1 && ocean[q] == 1 && ice[q] == 0) cut_e = fmf[qe] < 1.0;
  }
  if (j > 0) {
    if (shelf[q] == 1 && ocean[qs] == 1 && ice[qs] == 0) cut_s = fmf[q] < 1.0;
    else if (shelf[qs] == 1 && ocean[q] == 1 && ice[q] == 0) cut_s = fmf[qs] < 1.0;
  }
  if (j < ny - 1) {
    if (shelf[q] == 1 && ocean[qn] == 1 && ice[qn] == 0) cut_n = fmf[q] < 1.0;
    else if (shelf[qn] == 1 && ocean[q] == 1 && ice[q] == 0) cut_n = fmf[qn] < 1.0;
  }
  *diag = 1.0; *cw = *ce = *cs = *cn = 0.0;
  if (scheme == 0) {
    *ident = 1;
    *b = fmax(0.0, Hi[q] + (mb * dt));
    *x0 = *b;
    return;
  }
  if (scheme == 1) {   /* :441-548 */
    double Qw = 0.0, Qe = 0.0, Qs = 0.0, Qn = 0.0;
    if (i > 0) { const double uu = u[ICX(j, i - 1)]; Qw = uu * (uu > 0.0 ? Hi[qw] : Hi[q]) / dx; }
    if (i < nx - 1) { const double uu = u[ICX(j, i)]; Qe = -uu * (uu > 0.0 ? Hi[q] : Hi[qe]) / dx; }
    if (j > 0) { const double vv = v[ICY(j - 1, i)]; Qs = vv * (vv > 0.0 ? Hi[qs] : Hi[q]) / dx; }
    if (j < ny - 1) { const double vv = v[ICY(j, i)]; Qn = -vv * (vv > 0.0 ? Hi[q] : Hi[qn]) / dx; }
    if (cut_w) Qw = 0.0;
    if (cut_e) Qe = 0.0;
    if (cut_s) Qs = 0.0;
    if (cut_n) Qn = 0.0;
    *ident = 1;
    *b = fmax(0.0, Hi[q] + dt * (mb + Qw + Qe + Qs + Qn));
    *x0 = *b;
    return;
  }
  /* :549-727 */
  const double uw = (i > 0 && !cut_w) ? u[ICX(j, i - 1)] : 0.0, ue = (i < nx - 1 && !cut_e) ? u[ICX(j, i)] : 0.0;
  const double vs = (j > 0 && !cut_s) ? v[ICY(j - 1, i)] : 0.0, vn = (j < ny - 1 && !cut_n) ? v[ICY(j, i)] : 0.0;
  double d = 1.0 / dt;
  if (i > 0) d = d - (fs / dx) * fmin(uw, 0.0);
  if (i < nx - 1) d = d + (fs / dx) * fmax(ue, 0.0);
  if (j > 0) d = d - (fs / dx) * fmin(vs, 0.0);
  if (j < ny - 1) d = d + (fs / dx) * fmax(vn, 0.0);
  *diag = d;
  if (i > 0) *cw = (-fs / dx) * fmax(uw, 0.0);
  if (i < nx - 1) *ce = (fs / dx) * fmin(ue, 0.0);
  if (j > 0) *cs = (-fs / dx) * fmax(vs, 0.0);
  if (j < ny - 1) *cn = (fs / dx) * fmin(vn, 0.0);
  double r = mb + Hi[q] / dt;
  if (i > 0) r = r + Hi[q] * (1.0 - fs) / dx * fmin(uw, 0.0) + Hi[qw] * (1.0 - fs) / dx * fmax(uw, 0.0);
  if (i < nx - 1) r = r - Hi[q] * (1.0 - fs) / dx * fmax(ue, 0.0) - Hi[qe] * (1.0 - fs) / dx * fmin(ue, 0.0);
  if (j > 0) r = r + Hi[q] * (1.0 - fs) / dx * fmin(vs, 0.0) + Hi[qs] * (1.0 - fs) / dx * fmax(vs, 0.0);
  if (j < ny - 1) r = r - Hi[q] * (1.0 - fs) / dx * fmax(vn, 0.0) - Hi[qn] * (1.0 - fs) / dx * fmin(vn, 0.0);
  *ident = 0;
  *b = r;
  *x0 = Hi[q];
}

/* calc_dHi_dt_semiimplicit, ice_thickness_module.f90:302-440: the rows above, solved
 * exactly (banded elimination in the cell order i outer, j inner; the matrix is
 * column diagonally dominant, so no pivoting is needed) */
static int calc_dHi_dt_semiimplicit(orc_ctx* c, double dt) {
  DECL_DIMS(c);
  const int n = nx * ny, bw = ny;
  const double* Hi = FD(c, HI_A);
  double *dH = FD(c, DHI_DT_A), *Hn = FD(c, HI_TPLUSDT_A);
  const int W = 2 * bw + 1;
  double* band = (double*)calloc((size_t)n * W, sizeof(double));
  double* x = (double*)malloc(sizeof(double) * n);
  if (!band || !x) { free(band); free(x); return DIVA_BAD_INPUT; }
#define BAND(r, col) band[(size_t)(r) * W + ((col) - (r) + bw)]
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const int r = i * ny + j;
      int ident;
      double d, cw, ce, cs, cn, b, x0;
      semiimplicit_row(c, dt, i, j, &ident, &d, &cw, &ce, &cs, &cn, &b, &x0);
      BAND(r, r) = ident ? 1.0 : d;
      if (!ident) {
        if (i > 0) BAND(r, r - ny) += cw;
        if (i < nx - 1) BAND(r, r + ny) += ce;
        if (j > 0) BAND(r, r - 1) += cs;
        if (j < ny - 1) BAND(r, r + 1) += cn;
      }
      x[r] = b;
    }
  for (int col = 0; col < n; ++col) {
    const double p = BAND(col, col);
    if (p == 0.0) { free(band); free(x); return DIVA_LINEAR_NOT_CONVERGED; }
    const int last = col + bw < n - 1 ? col + bw : n - 1;
    for (int r = col + 1; r <= last; ++r) {
      const double f = BAND(r, col) / p;
      if (f == 0.0) continue;
      for (int cc = col; cc <= last; ++cc) BAND(r, cc) -= f * BAND(col, cc);
      x[r] -= f * x[col];
    }
  }
  for (int r = n - 1; r >= 0; --r) {
    double s = x[r];
    const int last = r + bw < n - 1 ? r + bw : n - 1;
    for (int cc = r + 1; cc <= last; ++cc) s -= BAND(r, cc) * x[cc];
    x[r] = s / BAND(r, r);
  }
#undef BAND
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const size_t q = IA(j, i);
      Hn[q] = fmax(0.0, x[i * ny + j]);
      dH[q] = (Hn[q] - Hi[q]) / dt;
    }
  free(band); free(x);
  return DIVA_OK;
}

/* calc_dHi_dt_explicit, ice_thickness_module.f90:65-300 */
static void calc_dHi_dt_explicit(orc_ctx* c, double dt) {
  DECL_DIMS(c);
  const double dx = c->dx;
  const double *u = FD(c, U_VAV_CX), *v = FD(c, V_VAV_CY), *Hi = FD(c, HI_A);
  const double *smb = FD(c, SMB_A), *bmb = FD(c, BMB_A), *fmf = FD(c, FLOAT_MARGIN_FRAC_A);
  const int32_t *cf = FI(c, MASK_CF_A), *shelf = FI(c, MASK_SHELF_A), *ocean = FI(c, MASK_OCEAN_A);
  double *Qx = FD(c, QX_CX), *Qy = FD(c, QY_CY), *dH = FD(c, DHI_DT_A), *Hn = FD(c, HI_TPLUSDT_A);
  /* upwind fluxes, :91-120 */
  for (int i = 0; i < nx - 1; ++i)
    for (int j = 0; j < ny; ++j) {
      const double uu = u[ICX(j, i)];
      Qx[ICX(j, i)] = uu * (uu > 0.0 ? Hi[IA(j, i)] : Hi[IA(j, i + 1)]) * dx * dt;
    }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny - 1; ++j) {
      const double vv = v[ICY(j, i)];
      Qy[ICY(j, i)] = vv * (vv > 0.0 ? Hi[IA(j, i)] : Hi[IA(j + 1, i)]) * dx * dt;
    }
  /* mass balance and outflux limitation, :175-262 (in place, in the reference's order) */
  double* mb = (double*)malloc(sizeof(double) * (size_t)nx * ny);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const size_t q = IA(j, i);
      if (cf[q] == 1 && shelf[q] == 1) mb[q] = (smb[q] + bmb[q]) * dx * dx * dt * fmf[q];
      else if (ocean[q] == 1 && shelf[q] == 0) mb[q] = 0.0;
      else mb[q] = (smb[q] + bmb[q]) * dx * dx * dt;
      const double avail = Hi[q] * dx * dx;
      double out = 0.0;
      if (i > 0 && !(Qx[ICX(j, i - 1)] > 0.0)) out -= Qx[ICX(j, i - 1)];
      if (i < nx - 1 && !(Qx[ICX(j, i)] < 0.0)) out += Qx[ICX(j, i)];
      if (j > 0 && !(Qy[ICY(j - 1, i)] > 0.0)) out -= Qy[ICY(j - 1, i)];
      if (j < ny - 1 && !(Qy[ICY(j, i)] < 0.0)) out += Qy[ICY(j, i)];
      double r = 1.0;
      if (-mb[q] >= avail) { mb[q] = -avail; r = 0.0; }
      if (out > avail + mb[q]) r = (avail + mb[q]) / out;
      if (r < 1.0) {
        if (i > 0 && Qx[ICX(j, i - 1)] < 0.0) Qx[ICX(j, i - 1)] *= r;
        if (i < nx - 1 && Qx[ICX(j, i)] > 0.0) Qx[ICX(j, i)] *= r;
        if (j > 0 && Qy[ICY(j - 1, i)] < 0.0) Qy[ICY(j - 1, i)] *= r;
        if (j < ny - 1 && Qy[ICY(j, i)] > 0.0) Qy[ICY(j, i)] *= r;
      }
    }
  /* rate of change and thickness at t + dt, :266-290 */
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const size_t q = IA(j, i);
      double d = mb[q] / (dx * dx * dt);
      if (i > 0) d = d + Qx[ICX(j, i - 1)] / (dx * dx * dt);
      if (i < nx - 1) d = d - Qx[ICX(j, i)] / (dx * dx * dt);
      if (j > 0) d = d + Qy[ICY(j - 1, i)] / (dx * dx * dt);
      if (j < ny - 1) d = d - Qy[ICY(j, i)] / (dx * dx * dt);
      d = fmax(d, -Hi[q] / dt);
      dH[q] = d;
      Hn[q] = Hi[q] + d * dt;
    }
  free(mb);
}

/* calc_dHi_dt, ice_thickness_module.f90:26-63: the integration method, then the boundary conditions */
static int calc_dHi_dt(orc_ctx* c, double dt) {
  DECL_DIMS(c);
  int st = DIVA_OK;
  if (c->c.choice_ice_integration_method == DIVA_INTEGRATION_SEMIIMPLICIT) st = calc_dHi_dt_semiimplicit(c, dt);
  else if (c->c.choice_ice_integration_method == DIVA_INTEGRATION_NONE)
    memset(FD(c, DHI_DT_A), 0, sizeof(double) * (size_t)nx * ny);
  else calc_dHi_dt_explicit(c, dt);
  if (st) return st;
  apply_ice_thickness_bc(c, dt);
  return DIVA_OK;
}

int orc_determine_floating_margin_fraction(orc_ctx* c) { floating_margin_fraction(c); return DIVA_OK; }

int orc_calc_dHi_dt(orc_ctx* c, double dt) {
  if (!(dt > 0.0)) return DIVA_BAD_INPUT;
  int st = calc_dHi_dt(c, dt);
  if (st) return st;
  DECL_DIMS(c);
  if (check_nan(c, FD(c, DHI_DT_A), (size_t)nx * ny)) return DIVA_NAN_DETECTED;
  return DIVA_OK;
}

/* calc_critical_timestep_adv, ice_dynamics_module.f90:726-762 */
int orc_calc_critical_timestep_adv(orc_ctx* c, double dt_max, double* dt_crit_adv) {
  DECL_DIMS(c);
  const double *u = FD(c, U_VAV_CX), *v = FD(c, V_VAV_CY);
  double dtc = 2.0 * dt_max;
  for (int i = 1; i < nx - 1; ++i)
    for (int j = 1; j < ny - 1; ++j) dtc = fmin(dtc, c->dx / (fabs(u[ICX(j, i)]) + fabs(v[ICY(j, i)])));
  *dt_crit_adv = fmin(dt_max, dtc * 0.9);
  return DIVA_OK;
}

/* calc_critical_timestep_SIA, ice_dynamics_module.f90:651-725 */
int orc_calc_critical_timestep_sia(orc_ctx* c, double dt_max, double* dt_crit_sia) {
  DECL_DIMS(c);
  const int32_t* sheet = FI(c, MASK_SHEET_A);
  const double *us = FD(c, U_3D_SIA_CX), *vs = FD(c, V_3D_SIA_CY), *Hcx = FD(c, HI_CX), *Hcy = FD(c, HI_CY);
  const double *sx = FD(c, DHS_DX_CX), *sy = FD(c, DHS_DY_CY), *u3 = FD(c, U_3D_CX), *v3 = FD(c, V_3D_CY);
  double dtc = dt_max;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      double D = 1E-9;
      if (i < nx - 1 && sheet[IA(j, i)] == 1 && sheet[IA(j, i + 1)] == 1)
        D = fmax(D, fabs(vavg(c->g.zeta, nz, &us[ICX3(0, j, i)]) * Hcx[ICX(j, i)] / sx[ICX(j, i)]));
      if (j < ny - 1 && sheet[IA(j, i)] == 1 && sheet[IA(j + 1, i)] == 1)
        D = fmax(D, fabs(vavg(c->g.zeta, nz, &vs[ICY3(0, j, i)]) * Hcy[ICY(j, i)] / sy[ICY(j, i)]));
      dtc = fmin(dtc, c->dx * c->dx / (6.0 * D));
      for (int k = 0; k < nz; ++k) {
        const double ua = i == 0 ? fabs(u3[ICX3(k, j, 0)]) : i == nx - 1 ? fabs(u3[ICX3(k, j, nx - 2)])
                                 : fmax(fabs(u3[ICX3(k, j, i - 1)]), fabs(u3[ICX3(k, j, i)]));
        const double va = j == 0 ? fabs(v3[ICY3(k, 0, i)]) : j == ny - 1 ? fabs(v3[ICY3(k, ny - 2, i)])
                                 : fmax(fabs(v3[ICY3(k, j - 1, i)]), fabs(v3[ICY3(k, j, i)]));
        dtc = fmin(dtc, c->dx / (ua + va));
      }
    }
  *dt_crit_sia = dtc * 0.9;
  return DIVA_OK;
}

/* the predictor of run_ice_dynamics_pc, ice_dynamics_module.f90:360-377 */
int orc_pc_predictor(orc_ctx* c, double dt, double zeta) {
  DECL_DIMS(c);
  const size_t n = (size_t)nx * ny;
  if (!(dt > 0.0)) return DIVA_BAD_INPUT;
  memcpy(FD(c, DHIDT_HNM1_UNM1), FD(c, DHIDT_HN_UN), sizeof(double) * n);
  int st0 = calc_dHi_dt(c, dt);
  if (st0) return st0;
  memcpy(FD(c, DHIDT_HN_UN), FD(c, DHI_DT_A), sizeof(double) * n);
  double *Hi = FD(c, HI_A), *pred = FD(c, HI_PRED), *old = FD(c, HI_OLD);
  const double *hn = FD(c, DHIDT_HN_UN), *hm = FD(c, DHIDT_HNM1_UNM1);
  for (size_t q = 0; q < n; ++q)
    pred[q] = fmax(0.0, Hi[q] + dt * ((1.0 + zeta / 2.0) * hn[q] - (zeta / 2.0) * hm[q]));
  memcpy(old, Hi, sizeof(double) * n);
  memcpy(Hi, pred, sizeof(double) * n);
  return orc_update_general_ice_model_data(c);
}

/* the corrector, :404-421, and calc_pc_truncation_error, :763-816 */
int orc_pc_corrector(orc_ctx* c, double dt, double zeta, double eta_min, double* eta) {
  DECL_DIMS(c);
  const size_t n = (size_t)nx * ny;
  if (!(dt > 0.0)) return DIVA_BAD_INPUT;
  int st0 = calc_dHi_dt(c, dt);
  if (st0) return st0;
  memcpy(FD(c, DHIDT_HSTARNP1_UNP1), FD(c, DHI_DT_A), sizeof(double) * n);
  double *Hi = FD(c, HI_A), *old = FD(c, HI_OLD), *corr = FD(c, HI_CORR), *dH = FD(c, DHI_DT_A);
  memcpy(Hi, old, sizeof(double) * n);
  int st = orc_update_general_ice_model_data(c);
  if (st) return st;
  const double *hn = FD(c, DHIDT_HN_UN), *hs = FD(c, DHIDT_HSTARNP1_UNP1), *pred = FD(c, HI_PRED);
  for (size_t q = 0; q < n; ++q) {
    corr[q] = fmax(0.0, old[q] + 0.5 * dt * (hn[q] + hs[q]));
    dH[q] = (corr[q] - Hi[q]) / dt;
  }
  double* tau = FD(c, PC_TAU);
  const int32_t *sheet = FI(c, MASK_SHEET_A), *gl = FI(c, MASK_GL_A);
  double e = eta_min;
  for (int i = 1; i < nx - 1; ++i)
    for (int j = 1; j < ny - 1; ++j) {
      const size_t q = IA(j, i);
      tau[q] = fabs(zeta * (corr[q] - pred[q]) / ((3.0 * zeta + 3.0) * dt));
      int near_gl = 0;
      for (int ii = i - 1; ii <= i + 1; ++ii)
        for (int jj = j - 1; jj <= j + 1; ++jj) near_gl |= gl[IA(jj, ii)] != 0;
      if (sheet[q] == 1 && !near_gl) e = fmax(e, tau[q]);
    }
  *eta = e;
  return DIVA_OK;
}

/* remove_unconnected_shelves, ice_thickness_module.f90:932-1044: a depth-first search
 * from the interior shelf cells next to sheet ice through 4-connected shelf cells; the
 * shelf cells it never reaches lose their ice */
static void remove_unconnected_shelves(orc_ctx* c) {
  DECL_DIMS(c);
  const int32_t *shelf = FI(c, MASK_SHELF_A), *sheet = FI(c, MASK_SHEET_A);
  double* Hi = FD(c, HI_A);
  unsigned char* map = (unsigned char*)calloc((size_t)nx * ny, 1);
  int* stack = (int*)malloc(sizeof(int) * 2 * (size_t)nx * ny);
  size_t top = 0;
  for (int i = 1; i < nx - 1; ++i)
    for (int j = 1; j < ny - 1; ++j)
      if (shelf[IA(j, i)] == 1 && (sheet[IA(j, i + 1)] == 1 || sheet[IA(j, i - 1)] == 1 || sheet[IA(j + 1, i)] == 1 ||
                                   sheet[IA(j - 1, i)] == 1)) {
        stack[2 * top] = i; stack[2 * top + 1] = j; ++top;
        map[IA(j, i)] = 1;
      }
  while (top > 0) {
    --top;
    const int i = stack[2 * top], j = stack[2 * top + 1];
    if (shelf[IA(j, i)] != 1) continue;
    map[IA(j, i)] = 2;
    const int ni[4] = {i - 1, i + 1, i, i}, nj[4] = {j, j, j - 1, j + 1};
    for (int k = 0; k < 4; ++k) {
      if (ni[k] < 0 || ni[k] >= nx || nj[k] < 0 || nj[k] >= ny || map[IA(nj[k], ni[k])] != 0) continue;
      map[IA(nj[k], ni[k])] = 1;
      stack[2 * top] = ni[k]; stack[2 * top + 1] = nj[k]; ++top;
    }
  }
  for (size_t q = 0; q < (size_t)nx * ny; ++q)
    if (shelf[q] == 1 && map[q] == 0) Hi[q] = 0.0;
  free(map); free(stack);
}

/* Hi_tplusdt_a (:429-431) and update_ice_thickness (:435-648) on its default path */
int orc_pc_finish(orc_ctx* c, double dt) {
  DECL_DIMS(c);
  const size_t n = (size_t)nx * ny;
  double *Hi = FD(c, HI_A), *Hn = FD(c, HI_TPLUSDT_A);
  const double* dH = FD(c, DHI_DT_A);
  for (size_t q = 0; q < n; ++q) Hn[q] = fmax(0.0, Hi[q] + dt * dH[q]);
  memcpy(FI(c, MASK_ICE_A_PREV), FI(c, MASK_ICE_A), sizeof(int32_t) * n);   /* :446 */
  /* fixed shelf / sheet / grounding-line geometry, :449-540 */
  const int32_t *shelf = FI(c, MASK_SHELF_A), *sheet = FI(c, MASK_SHEET_A);
  const int fix[3] = {c->c.fixed_shelf_geometry, c->c.fixed_sheet_geometry, c->c.fixed_grounding_line};
  for (int f = 0; f < 3; ++f) {
    if (!fix[f]) continue;
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j) {
        const size_t q = IA(j, i);
        int nb_shelf = 0, nb_sheet = 0;
        for (int ii = (i > 0 ? i - 1 : 0); ii <= (i < nx - 1 ? i + 1 : nx - 1); ++ii)
          for (int jj = (j > 0 ? j - 1 : 0); jj <= (j < ny - 1 ? j + 1 : ny - 1); ++jj) {
            nb_shelf |= shelf[IA(jj, ii)] == 1;
            nb_sheet |= sheet[IA(jj, ii)] == 1;
          }
        int keep;
        if (f == 0) keep = shelf[q] == 1 || (sheet[q] == 1 && nb_shelf);
        else if (f == 1) keep = sheet[q] == 1 || (shelf[q] == 1 && nb_sheet);
        else keep = (sheet[q] == 1 && nb_shelf) || (shelf[q] == 1 && nb_sheet);
        if (keep) Hn[q] = Hi[q];
      }
  }
  for (size_t q = 0; q < n; ++q) Hi[q] = fmax(0.0, Hn[q]);
  int st = orc_update_general_ice_model_data(c);                            /* the masks of :556-590 */
  if (st) return st;
  floating_margin_fraction(c);
  if (c->c.choice_calving_law == DIVA_CALVING_THRESHOLD_THICKNESS) {
    /* threshold_thickness_calving (calving_module.f90:62-91), twice so that the calving
     * front may retreat by more than one cell (ice_dynamics_module.f90:562-583) */
    for (int pass = 0; pass < 2; ++pass) {
      const int32_t* cf = FI(c, MASK_CF_A);
      const double* He = FD(c, HI_EFF_CF_A);
      for (size_t q = 0; q < n; ++q)
        if (cf[q] == 1 && He[q] < c->c.calving_threshold_thickness) Hi[q] = 0.0;
      if ((st = orc_update_general_ice_model_data(c))) return st;
      if (pass == 0) floating_margin_fraction(c);
    }
  }
  remove_unconnected_shelves(c);
  const int32_t* noice = FI(c, MASK_NOICE_A);
  for (size_t q = 0; q < n; ++q)
    if (noice[q] == 1) Hi[q] = 0.0;                                          /* :586-592 */
  if (c->c.do_remove_shelves) {                                              /* :600-608 */
    const double *Hb = FD(c, HB_A), *SL = FD(c, SL_A);
    for (size_t q = 0; q < n; ++q)
      if (is_floating(Hi[q], Hb[q], SL[q])) Hi[q] = 0.0;
  }
  if (c->c.remove_shelves_larger_than_PD) {                                  /* :613-622 */
    const double *Hp = FD(c, HI_PD_A), *Bp = FD(c, HB_PD_A);
    for (size_t q = 0; q < n; ++q)
      if (Hp[q] == 0.0 && Bp[q] < 0.0) Hi[q] = 0.0;
  }
  if (c->c.continental_shelf_calving) {                                      /* :625-635 */
    const double *Hg = FD(c, HI_GIAEQ_A), *Bg = FD(c, HB_GIAEQ_A);
    for (size_t q = 0; q < n; ++q)
      if (Hg[q] == 0.0 && Bg[q] < c->c.continental_shelf_min_height) Hi[q] = 0.0;
  }
  return orc_update_general_ice_model_data(c);
}

/* apply_prescribed_retreat_mask, calving_module.f90:96-169 (frames read by the caller) */
int orc_apply_prescribed_retreat_mask(orc_ctx* c, double time, double t0, double t1) {
  DECL_DIMS(c);
  if (!(t1 > t0)) return DIVA_BAD_INPUT;
  const double wt0 = fmax(0.0, fmin(1.0, (t1 - time) / (t1 - t0))), wt1 = 1.0 - wt0;
  const double *m0 = FD(c, RETREAT_MASK0_A), *m1 = FD(c, RETREAT_MASK1_A), *Href = FD(c, RETREAT_MASK_HI_REF_A);
  double *m = FD(c, RETREAT_MASK_A), *Hi = FD(c, HI_A);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) m[IA(j, i)] = (wt0 * m0[IA(j, i)]) + (wt1 * m1[IA(j, i)]);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const size_t q = IA(j, i);
      if (m[q] < 0.999) Hi[q] = fmin(Hi[q], Href[q] * m[q]);
      if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && m[q] >= 0.999) {
        int any = 0;
        for (int di = -1; di <= 1; ++di)
          for (int dj = -1; dj <= 1; ++dj)
            if ((di || dj) && m[IA(j + dj, i + di)] < 0.999) any = 1;
        if (any) Hi[q] = fmin(Hi[q], Href[q] * m[q]);
      }
    }
  return orc_update_general_ice_model_data(c);
}

/* ------------------------------------------------------------------------ */
/* Thermodynamics: run_thermo_model with the 3D heat equation                */

#define SEC_PER_YEAR 31556943.36                 /* parameters_module.f90:12 */

/* Gaussian elimination with partial pivoting for a tridiagonal system (the algorithm of
 * LAPACK dgtsv, which tridiagonal_solve, utilities_module.f90:791-834, calls): dl, d, du
 * are overwritten, b holds the solution.  Returns 0, or k+1 for a zero pivot in row k. */
int orc_tridiagonal_solve(int n, double* dl, double* d, double* du, double* b) {
  for (int i = 0; i < n - 1; ++i) {
    if (fabs(d[i]) >= fabs(dl[i])) {
      if (d[i] == 0.0) return i + 1;
      const double fact = dl[i] / d[i];
      d[i + 1] = d[i + 1] - fact * du[i];
      b[i + 1] = b[i + 1] - fact * b[i];
      if (i < n - 2) dl[i] = 0.0;
    } else {
      const double fact = d[i] / dl[i];
      d[i] = dl[i];
      const double t = d[i + 1];
      d[i + 1] = du[i] - fact * t;
      if (i < n - 2) {
        dl[i] = du[i + 1];
        du[i + 1] = -fact * dl[i];
      }
      du[i] = t;
      const double tb = b[i];
      b[i] = b[i + 1];
      b[i + 1] = tb - fact * b[i + 1];
    }
  }
  if (d[n - 1] == 0.0) return n;
  b[n - 1] = b[n - 1] / d[n - 1];
  if (n > 1) b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / d[n - 2];
  for (int i = n - 3; i >= 0; --i) b[i] = (b[i] - du[i] * b[i + 1] - dl[i] * b[i + 2]) / d[i];
  return 0;
}

/* zeta coefficients of initialise_zeta_discretisation, derivatives_and_grids_module.f90:1930-2000 */
struct zeta_coef { double a[64], b[64], c[64], aa[64], bb[64], cc[64]; };
static void zeta_coefficients(const double* z, int nz, struct zeta_coef* q) {
  for (int k = 1; k < nz - 1; ++k) {
    const double ak = z[k] - z[k - 1], bk = z[k + 1] - z[k];
    q->a[k] = -bk / (ak * (ak + bk));
    q->b[k] = (bk - ak) / (ak * bk);
    q->c[k] = ak / (bk * (ak + bk));
    q->aa[k] = 2.0 / (ak * (ak + bk));
    q->bb[k] = -2.0 / (ak * bk);
    q->cc[k] = 2.0 / (bk * (ak + bk));
  }
}

/* replace_Ti_with_robin_solution, thermodynamics_module.f90:384-481 (ocean model 'none';
 * the shelf profile adds T0_C to T0_C + T_ocean_mean_PD_ANT, as written) */
static void robin_column(orc_ctx* c, double* Tn, int i, int j) {
  DECL_DIMS(c);
  const double* z = c->g.zeta;
  const size_t q = IA(j, i);
  const double Hi = FD(c, HI_A)[q], ghf = FD(c, GHF_A)[q], smb = FD(c, SMB_A)[q];
  const double* Tp = FD(c, TI_PMP_A);
  const double K = 9.828 * SEC_PER_YEAR * exp(-0.0057 * T0_C);
  const double kappa = K / (ICE_DENSITY * 2127.5);
  const double grad = -ghf / K;
  const double Ts = fmin(T0_C, FD(c, T_SURF_ANNUAL_A)[q]);
  if (FI(c, MASK_SHEET_A)[q] == 1) {
    if (smb > 0.0) {
      const double L = sqrt(2.0 * kappa * Hi / smb);
      for (int k = 0; k < nz; ++k) {
        const double erf1 = erf((1.0 - z[k]) * Hi / L), erf2 = erf(Hi / L);
        Tn[IA3(k, j, i)] = Ts + sqrt(PI_C) / 2.0 * L * grad * (erf1 - erf2);
      }
    } else {
      for (int k = 0; k < nz; ++k) Tn[IA3(k, j, i)] = Ts + ((T0_C - CC_C * Hi) - Ts) * z[k];
    }
  } else if (FI(c, MASK_SHELF_A)[q] == 1) {
    /* the Robin profile adds T0 to its ocean temperature, which with ocean model 'none' is
     * already T0 + T_ocean_mean_PD_ANT (:455-465, as written) */
    const double To = c->c.ocean_temperature_input ? FD(c, T_OCEAN_BASE_A)[q] : T0_C + c->c.T_ocean_mean_PD_ANT;
    for (int k = 0; k < nz; ++k) Tn[IA3(k, j, i)] = Ts + z[k] * (T0_C + To - Ts);
  } else {
    for (int k = 0; k < nz; ++k) Tn[IA3(k, j, i)] = Ts;
  }
  for (int k = 0; k < nz; ++k) Tn[IA3(k, j, i)] = fmin(Tn[IA3(k, j, i)], Tp[IA3(k, j, i)]);
}

/* solve_3D_heat_equation, thermodynamics_module.f90:124-381; returns the number of
 * unstable columns (-1 if they exceed 1 % of the grid) */
static int solve_3d_heat_equation(orc_ctx* c) {
  DECL_DIMS(c);
  const double dx = c->dx, dt = c->c.dt_thermo;
  const double* z = c->g.zeta;
  const double *Hi = FD(c, HI_A), *Hs = FD(c, HS_A);
  const int32_t *ice = FI(c, MASK_ICE_A), *shelf = FI(c, MASK_SHELF_A), *sheet = FI(c, MASK_SHEET_A);
  double *Ti = FD(c, TI_A), *dHs_dt = FD(c, DHS_DT_A);
  const double *dHi_dt = FD(c, DHI_DT_A), *dHb_dt = FD(c, DHB_DT_A);
  double *zdt = FD(c, DZETA_DT_A), *zdx = FD(c, DZETA_DX_A), *zdy = FD(c, DZETA_DY_A), *zdz = FD(c, DZETA_DZ_A);
  const double *dHs_dx = FD(c, DHS_DX_A), *dHs_dy = FD(c, DHS_DY_A), *dHi_dx = FD(c, DHI_DX_A), *dHi_dy = FD(c, DHI_DY_A);
  const double *Ts = FD(c, T_SURF_ANNUAL_A), *ghf = FD(c, GHF_A), *fh = FD(c, FRICTIONAL_HEATING_A);
  const double *Cp = FD(c, CPI_A), *Ki = FD(c, KI_A), *Tp = FD(c, TI_PMP_A);
  const double *u3 = FD(c, U_3D_A), *v3 = FD(c, V_3D_A), *w3 = FD(c, W_3D_A);
  const double *ucx = FD(c, U_3D_CX), *vcy = FD(c, V_3D_CY);
  (void)Hs;
  for (size_t q = 0; q < (size_t)nx * ny; ++q)
    dHs_dt[q] = shelf[q] == 0 ? dHi_dt[q] + dHb_dt[q] : dHi_dt[q] * (1.0 - ICE_DENSITY / SW_DENSITY);
  /* calculate_zeta_derivatives, derivatives_and_grids_module.f90:1892-1929 */
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const size_t q = IA(j, i);
      const double inv = 1.0 / Hi[q];
      zdz[q] = -inv;
      for (int k = 0; k < nz; ++k) {
        zdt[IA3(k, j, i)] = inv * (dHs_dt[q] - z[k] * dHi_dt[q]);
        zdx[IA3(k, j, i)] = inv * (dHs_dx[q] - z[k] * dHi_dx[q]);
        zdy[IA3(k, j, i)] = inv * (dHs_dy[q] - z[k] * dHi_dy[q]);
      }
    }
  for (size_t q = 0; q < (size_t)nx * ny; ++q) Ti[q * nz] = fmin(T0_C, Ts[q]);   /* layer 1 */
  const double* To_in = FD(c, T_OCEAN_BASE_A);   /* ocean_temperature_input: T0 added as at :209 */
  struct zeta_coef zc;
  zeta_coefficients(z, nz, &zc);
  double* Tn = (double*)calloc((size_t)nx * ny * nz, sizeof(double));
  unsigned char* unstable = (unsigned char*)calloc((size_t)nx * ny, 1);
  int n_unstable = 0;
  double dl[64], d[64], du[64], b[64];
  for (int i = 1; i < nx - 1; ++i)
    for (int j = 1; j < ny - 1; ++j) {
      const size_t q = IA(j, i);
      if (ice[q] == 0) {
        for (int k = 0; k < nz; ++k) Tn[IA3(k, j, i)] = Ti[IA3(0, j, i)];
        continue;
      }
      if (Hi[q] < 1.0) {
        for (int k = 0; k < nz; ++k) Tn[IA3(k, j, i)] = fmin(T0_C, Ts[q]);
        continue;
      }
      for (int k = 1; k < nz - 1; ++k) {
        const size_t p = IA3(k, j, i);
        double heat = 0.0;
        if (sheet[q] == 1)
          heat = ((-GRAV * z[k]) / Cp[p]) *
                 ((zc.a[k] * u3[IA3(k - 1, j, i)] + zc.b[k] * u3[p] + zc.c[k] * u3[IA3(k + 1, j, i)]) * dHs_dx[q] +
                  (zc.a[k] * v3[IA3(k - 1, j, i)] + zc.b[k] * v3[p] + zc.c[k] * v3[IA3(k + 1, j, i)]) * dHs_dy[q]);
        double udx, vdy;
        if (u3[p] > 0.0) udx = ucx[ICX3(k, j, i - 1)] * (Ti[p] - Ti[IA3(k, j, i - 1)]) / dx;
        else udx = ucx[ICX3(k, j, i)] * (Ti[IA3(k, j, i + 1)] - Ti[p]) / dx;
        if (v3[p] > 0.0) vdy = vcy[ICY3(k, j - 1, i)] * (Ti[p] - Ti[IA3(k, j - 1, i)]) / dx;
        else vdy = vcy[ICY3(k, j, i)] * (Ti[IA3(k, j + 1, i)] - Ti[p]) / dx;
        const double f1 = (Ki[p] * (zdz[q] * zdz[q])) / (ICE_DENSITY * Cp[p]);
        const double f2 = zdt[p] + zdx[p] * u3[p] + zdy[p] * v3[p] + zdz[q] * w3[p];
        const double f3 = heat + (udx + vdy) - Ti[p] / dt;
        dl[k - 1] = f1 * zc.aa[k] - f2 * zc.a[k];
        d[k] = f1 * zc.bb[k] - f2 * zc.b[k] - 1.0 / dt;
        du[k] = f1 * zc.cc[k] - f2 * zc.c[k];
        b[k] = f3;
      }
      d[0] = 1.0; du[0] = 0.0; b[0] = fmin(T0_C, Ts[q]);
      const size_t pb = IA3(nz - 1, j, i);
      if (shelf[q] == 1) {
        const double T_ocean = c->c.ocean_temperature_input ? To_in[q] + T0_C : T0_C + c->c.T_ocean_mean_PD_ANT;
        dl[nz - 2] = 0.0; d[nz - 1] = 1.0; b[nz - 1] = fmin(T0_C, fmin(Tp[pb], T_ocean));
      } else if (Ti[pb] >= Tp[pb]) {
        dl[nz - 2] = 0.0; d[nz - 1] = 1.0; b[nz - 1] = Tp[pb];
      } else {
        dl[nz - 2] = 1.0; d[nz - 1] = -1.0;
        b[nz - 1] = (z[nz - 1] - z[nz - 2]) * (ghf[q] + fh[q]) / (zdz[q] * Ki[pb]);
      }
      const int info = orc_tridiagonal_solve(nz, dl, d, du, b);
      for (int k = 0; k < nz; ++k) Tn[IA3(k, j, i)] = info ? NAN : b[k];
      for (int k = 0; k < nz - 1; ++k) Tn[IA3(k, j, i)] = fmin(Tn[IA3(k, j, i)], Tp[IA3(k, j, i)]);
      if (Tn[pb] >= Tp[pb])
        Tn[pb] = fmin(Tp[pb], Ti[IA3(nz - 2, j, i)] -
                                  (z[nz - 1] - z[nz - 2]) * (ghf[q] + fh[q]) / (zdz[q] * Ki[pb]));
      int bad = 0;
      double mn = INFINITY;
      for (int k = 0; k < nz; ++k) {
        const double t = Tn[IA3(k, j, i)];
        if (t != t) bad = 1;
        mn = fmin(mn, t);
      }
      if (mn < 150.0 || bad) { unstable[q] = 1; ++n_unstable; }
    }
  /* Neumann_BC_a_3D, derivatives_and_grids_module.f90:2034-2061: rows, then columns */
  for (int i = 0; i < nx; ++i)
    for (int k = 0; k < nz; ++k) {
      Tn[IA3(k, 0, i)] = Tn[IA3(k, 1, i)];
      Tn[IA3(k, ny - 1, i)] = Tn[IA3(k, ny - 2, i)];
    }
  for (int j = 0; j < ny; ++j)
    for (int k = 0; k < nz; ++k) {
      Tn[IA3(k, j, 0)] = Tn[IA3(k, j, 1)];
      Tn[IA3(k, j, nx - 1)] = Tn[IA3(k, j, nx - 2)];
    }
  const int limit = (int)ceil((double)(nx * ny) / 100.0);
  if (n_unstable >= limit) {
    free(Tn); free(unstable);
    return -1;
  }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      if (unstable[IA(j, i)]) robin_column(c, Tn, i, j);
  memcpy(Ti, Tn, sizeof(double) * (size_t)nx * ny * nz);
  free(Tn); free(unstable);
  return n_unstable;
}

/* run_thermo_model, thermodynamics_module.f90:29-121 */
int orc_run_thermo_model(orc_ctx* c, int32_t do_solve, int32_t* n_unstable) {
  DECL_DIMS(c);
  const int32_t *ice = FI(c, MASK_ICE_A), *prev = FI(c, MASK_ICE_A_PREV);
  const double *u = FD(c, U_VAV_CX), *v = FD(c, V_VAV_CY), *Ts = FD(c, T_SURF_ANNUAL_A);
  double* Ti = FD(c, TI_A);
  *n_unstable = 0;
  /* newly ice-covered columns take the temperature of an upwind ice neighbour (:46-72) */
  for (int i = 1; i < nx - 1; ++i)
    for (int j = 1; j < ny - 1; ++j) {
      if (!(ice[IA(j, i)] == 1 && prev[IA(j, i)] == 0)) continue;
      int si = -1, sj = -1;
      if (u[ICX(j, i - 1)] > 0.0 && prev[IA(j, i - 1)] == 1) { si = i - 1; sj = j; }
      else if (u[ICX(j, i)] < 0.0 && prev[IA(j, i + 1)] == 1) { si = i + 1; sj = j; }
      else if (v[ICY(j - 1, i)] > 0.0 && prev[IA(j - 1, i)] == 1) { si = i; sj = j - 1; }
      else if (v[ICY(j, i)] < 0.0 && prev[IA(j + 1, i)] == 1) { si = i; sj = j + 1; }
      for (int k = 0; k < nz; ++k)
        Ti[IA3(k, j, i)] = si >= 0 ? Ti[IA3(k, sj, si)] : fmin(Ts[IA(j, i)], T0_C);
    }
  /* calc_bottom_frictional_heating (:484-522) */
  double* fh = FD(c, FRICTIONAL_HEATING_A);
  const int no_fric = c->c.choice_ice_dynamics == DIVA_DYN_SIA || c->c.choice_sliding_law == DIVA_SLIDING_NONE;
  if (no_fric) {
    for (size_t q = 0; q < (size_t)nx * ny; ++q) fh[q] = 0.0;
  } else {
    const double *beta = FD(c, BETA_A), *ub = FD(c, U_BASE_A), *vb = FD(c, V_BASE_A);
    const int32_t* sheet = FI(c, MASK_SHEET_A);
    for (int i = 1; i < nx - 1; ++i)
      for (int j = 1; j < ny - 1; ++j) {
        const size_t q = IA(j, i);
        fh[q] = sheet[q] == 1 ? beta[q] * (ub[q] * ub[q] + vb[q] * vb[q]) : 0.0;
      }
  }
  /* calc_heat_capacity, calc_thermal_conductivity (:523-608) */
  double *Cp = FD(c, CPI_A), *Ki = FD(c, KI_A);
  const size_t n3 = (size_t)nx * ny * nz;
  for (size_t p = 0; p < n3; ++p) {
    Cp[p] = c->c.choice_ice_heat_capacity == DIVA_HEATCAP_UNIFORM ? c->c.uniform_ice_heat_capacity
                                                                   : 2115.3 + 7.79293 * (Ti[p] - T0_C);
    Ki[p] = c->c.choice_ice_thermal_conductivity == DIVA_CONDUCT_UNIFORM ? c->c.uniform_ice_thermal_conductivity
                                                                          : 3.101E+08 * exp(-0.0057 * Ti[p]);
  }
  orc_calc_pressure_melting_point(c);
  if (do_solve) {
    if (!(c->c.dt_thermo > 0.0)) return DIVA_BAD_INPUT;
    const int nu = solve_3d_heat_equation(c);
    if (nu < 0) {
      snprintf(c->err, sizeof(c->err), "heat equation solver unstable for more than 1%% of grid cells");
      return DIVA_NAN_DETECTED;
    }
    *n_unstable = nu;
  }
  return orc_calc_ice_rheology(c);
}

int orc_diva_coefficients(orc_ctx* c) {
  double *u = FD(c, U_VAV_CX), *v = FD(c, V_VAV_CY);
  calc_vertical_shear_strain_rates(c);
  calc_effective_viscosity(c, u, v);
  calc_sliding_term_beta(c, u, v);
  calc_F_integral(c);
  calc_beta_eff(c);
  return DIVA_OK;
}
int orc_secondary_velocities(orc_ctx* c) { calc_secondary_velocities(c); return DIVA_OK; }
int orc_3d_horizontal_velocities_diva(orc_ctx* c) { calc_3D_horizontal_velocities_DIVA(c); return DIVA_OK; }
long orc_linear_iterations(orc_ctx* c) { return c->lin_iters_total; }

int orc_state_save(orc_ctx* c) {
  for (int f = 0; f < DIVA_NUM_FIELDS; ++f) {
    size_t nb = field_bytes(c, f);
    if (!c->S[f]) c->S[f] = malloc(nb);
    memcpy(c->S[f], c->F[f], nb);
  }
  return DIVA_OK;
}
int orc_state_restore(orc_ctx* c) {
  for (int f = 0; f < DIVA_NUM_FIELDS; ++f) if (c->S[f]) memcpy(c->F[f], c->S[f], field_bytes(c, f));
  return DIVA_OK;
}

const char* orc_last_error(const orc_ctx* c) { return c ? c->err : ""; }

/* Schoof (2006) SSA ice-stream solution, utilities_module.f90:836-878 */
void orc_schoof2006(double tantheta, double h0, double A_flow, double y, double n_flow, double m, double L,
                    double* U, double* tauc) {
  double B = pow(A_flow, -1.0 / n_flow);
  double f = ICE_DENSITY * GRAV * h0 * tantheta;
  double W = L * pow(m + 1.0, 1.0 / m);
  *tauc = f * pow(fabs(y / L), m);
  double ua = -2.0 * pow(f, 3) * pow(L, 4) / (pow(B, 3) * pow(h0, 3));
  double ub = (1.0 / 4.0) * (pow(y / L, 4.0) - pow(m + 1.0, 4.0 / m));
  double uc = (-3.0 / ((m + 1.0) * (m + 4.0))) * (pow(fabs(y / L), m + 4.0) - pow(m + 1.0, 1.0 + (4.0 / m)));
  double ud = (3.0 / (pow(m + 1.0, 2) * (2.0 * m + 4.0))) * (pow(fabs(y / L), 2 * m + 4.0) - pow(m + 1.0, 2.0 + (4.0 / m)));
  double ue = (-1.0 / (pow(m + 1.0, 3) * (3.0 * m + 4.0))) * (pow(fabs(y / L), 3 * m + 4.0) - pow(m + 1.0, 3.0 + (4.0 / m)));
  *U = ua * (ub + uc + ud + ue);
  if (fabs(y) > W) *U = 0.0;
}

/* column quadratures for known-answer tests */
double orc_vertical_integrate(const double* zeta, int nz, const double* f) { return vint(zeta, nz, f); }
double orc_vertical_average(const double* zeta, int nz, const double* f) { return vavg(zeta, nz, f); }
void orc_vertical_integration_from_bottom_to_zeta(const double* zeta, int nz, const double* f, double* out) {
  vint_bottom_to_zeta(zeta, nz, f, out);
}

/* Threads of this context's GMRES (timed CPU baseline only; 1 keeps the sequential
 * algorithm the parity tests use, more splits ILU(0) into block-Jacobi over row blocks). */
int orc_set_threads(orc_ctx* c, int32_t threads) {
  if (!c || threads < 1 || threads > ORC_MAX_THREADS) return DIVA_BAD_INPUT;
  pool_destroy(c->pool);
  c->pool = threads > 1 ? pool_create(threads) : NULL;
  c->threads = threads;
  return DIVA_OK;
}

int orc_num_threads(void) { return ORC_MAX_THREADS; }
