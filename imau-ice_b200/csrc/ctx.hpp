// ctx.hpp -- device-resident state of one grid and the launchers shared by
// the translation units of libdiva_b200.so.
#pragma once
#include <cuda_runtime.h>
#include <cmath>
#include <string>
#include "common.cuh"

namespace diva {

constexpr int kMaxLevels = 12;
constexpr int kCoarseDirectMax = 64;
// Adaptive linear tolerance (lin_adaptive): rtol = max(lin_rtol, eta * min(1, rel-res)),
// eta starting at lin_adaptive_eta and halved, down to kEtaFloor, whenever a viscosity
// iteration within kEtaWindow x the stop tolerance fails to lower the nonlinear residual:
// near the target a loose solve can stall a relaxed Picard iteration at the noise its own
// linear error injects, while early iterations are often non-monotone and left alone.
constexpr double kEtaFloor = 0.05, kEtaWindow = 100.0;
__host__ __device__ inline double eta_after(double eta, double relres, double prev, double tol) {
  const bool stalled = prev > 0.0 && relres >= prev && relres < kEtaWindow * tol;
  return stalled ? (0.5 * eta > kEtaFloor ? 0.5 * eta : kEtaFloor) : eta;
}    // unknowns of a coarsest level solved directly

// One multigrid level of the staggered DIVA operator.  Coefficients are the
// rediscretised Na (a-grid), Nb (b-grid) and the reaction terms Bx = beta_eff_cx*dx^2
// (cx) and By (cy) of the level's grid; idu/idv are the inverse effective
// diagonals used by the Gauss-Seidel smoother.
struct Level {
  Dims d;
  double *Na, *Nb, *Bx, *By, *idu, *idv;
  double *xu, *xv, *bu, *bv, *ru, *rv;
  double *tu, *tv;   // x after pre-smoothing (tiled levels): read over halos by the post-smoothing kernel
};

// Boundary condition codes of the velocity unknowns (diva_bc_t), per side.
struct BCs {
  int uW, uE, uS, uN, vW, vE, vS, vN;
};

// Float planes of each tiled level for the mixed-precision preconditioner.
enum { F32_NA = 0, F32_NB, F32_BX, F32_BY, F32_IDU, F32_IDV };

// Krylov vectors on the fine level, each a (u,v) pair of planes.
enum { KV_X = 0, KV_R, KV_RHAT, KV_P, KV_PHAT, KV_V, KV_S, KV_SHAT, KV_T, KV_B, KV_COUNT };

// Device scalars of the linear solver and of the Picard bookkeeping.
enum {
  SC_RHO = 0, SC_ALPHA, SC_OMEGA, SC_BETA, SC_RNORM2, SC_BNORM2, SC_SNORM2, SC_TMP0, SC_TMP1, SC_TMP2,
  SC_RES1, SC_RES2, SC_NCNT, SC_RR, SC_BB, SC_NANFLAG, SC_FLAG,
  // device-side control of a graph-launched viscosity iteration
  SC_TARGET2, SC_LIN_IT, SC_LIN_FULL, SC_LIN_FAILED, SC_PIC_IT, SC_EXIT_RELRES, SC_CONVERGED, SC_RESID,
  SC_RELRES, SC_NAN, SC_SOLVED, SC_HALFDONE,
  SC_ETA, SC_RELRES_PREV,   // adaptive linear tolerance factor and the previous nonlinear residual
  SC_SUM_LIN, SC_SUM_FULL, SC_N_SOLVED,   // totals of a graph-launched viscosity loop
  // Anderson mixing of the viscosity iteration (picard_anderson_m > 0): history columns held,
  // the ring slot the next one goes to, whether the previous map value is stored, the
  // nonlinear residual the last mixing step saw, the Gram matrix of the residual
  // differences, its right-hand side and the mixing coefficients
  SC_AA_N, SC_AA_HEAD, SC_AA_HAVE, SC_AA_RPREV, SC_AA_RESTARTS,
  SC_STALLED, SC_STALL_BEST, SC_STALL_SINCE,   // stagnation stop: flag, lowest rel-res, iterations since
  SC_AA_OFF, SC_AA_BEST, SC_AA_SINCE,   // mixing given up; best rel-res so far; steps since it improved
  SC_AA_G, SC_AA_RHS = SC_AA_G + 25, SC_AA_GAMMA = SC_AA_RHS + 5,
  SC_COUNT = SC_AA_GAMMA + 5
};
constexpr int kAAMax = 5;             // largest Anderson depth
constexpr int kAAPartials = 2 * kAAMax;   // block partials of one mixing step
constexpr double kAAGammaMax = 20.0;      // largest sum of |gamma_i| a mixing step accepts
constexpr int kAAPatience = 20;           // steps without a 10 % better rel-res before mixing is given up

// One Anderson mixing step's coefficients from the inner products of the newest residual
// difference dF_s with every history column (dots[0..m)) and of the residual f with them
// (dots[kAAMax..kAAMax+m)), on the device scalars SC_AA_*.  The first call of a solve only
// records that a map value exists (gamma = 0: the plain step g).  A nonlinear residual
// more than 10 x the one the previous step saw drops the older columns.  gamma solves the
// normal equations of the least-squares problem over the n most recent columns, scaled to
// unit diagonal and regularised by 1e-10; when the Cholesky factorisation meets a pivot
// below 1e-12, or the coefficients sum to more than kAAGammaMax in magnitude (an
// extrapolation far outside the history), the oldest column is dropped and the solve
// repeated (down to none: the plain step).
__host__ __device__ inline void aa_coefficients(double* sc, int m, const double* dots) {
  double* G = sc + SC_AA_G;
  double* rhs = sc + SC_AA_RHS;
  double* gam = sc + SC_AA_GAMMA;
  const double relres = sc[SC_RELRES], rprev = sc[SC_AA_RPREV];
  for (int k = 0; k < kAAMax; ++k) gam[k] = 0.0;
  sc[SC_AA_RPREV] = relres;
  // Mixing that has not lowered rel-res by 10 % in kAAPatience steps is given up for the
  // rest of the solve and the reference's relaxation takes over (launch_picard_update reads
  // SC_AA_OFF): where the velocity limit is active the limited map is not smooth, the mixed
  // iteration wanders, while the relaxed one settles on the limited fixed point.
  if (sc[SC_AA_OFF] != 0.0) return;
  if (sc[SC_AA_BEST] == 0.0 || relres < 0.9 * sc[SC_AA_BEST]) {
    sc[SC_AA_BEST] = relres;
    sc[SC_AA_SINCE] = 0.0;
  } else if ((sc[SC_AA_SINCE] += 1.0) >= (double)kAAPatience) {
    sc[SC_AA_OFF] = 1.0;
    return;
  }
  if (sc[SC_AA_HAVE] == 0.0) {
    sc[SC_AA_HAVE] = 1.0;
    sc[SC_AA_N] = 0.0;
    sc[SC_AA_HEAD] = 0.0;
    return;
  }
  const int s = (int)sc[SC_AA_HEAD];
  int n = (int)sc[SC_AA_N];
  if (rprev > 0.0 && relres > 10.0 * rprev) {
    n = 0;
    sc[SC_AA_RESTARTS] += 1.0;
  }
  for (int i = 0; i < m; ++i) {
    G[s * kAAMax + i] = dots[i];
    G[i * kAAMax + s] = dots[i];
    rhs[i] = dots[kAAMax + i];
  }
  n = n + 1 < m ? n + 1 : m;
  sc[SC_AA_HEAD] = (double)((s + 1) % m);
  int idx[kAAMax];
  for (int k = 0; k < n; ++k) idx[k] = (s - k + m) % m;   // newest first
  for (int nn = n; nn > 0; --nn) {
    double A[kAAMax][kAAMax], b[kAAMax], dk[kAAMax];
    bool ok = true;
    for (int k = 0; k < nn && ok; ++k) {
      dk[k] = sqrt(G[idx[k] * kAAMax + idx[k]]);
      ok = dk[k] > 0.0 && dk[k] < 1e300;
    }
    if (!ok) continue;
    for (int k = 0; k < nn; ++k) {
      for (int l = 0; l < nn; ++l) A[k][l] = G[idx[k] * kAAMax + idx[l]] / (dk[k] * dk[l]);
      A[k][k] += 1e-10;
      b[k] = rhs[idx[k]] / dk[k];
    }
    // Cholesky A = L L^T in the lower triangle
    for (int k = 0; k < nn && ok; ++k) {
      double p = A[k][k];
      for (int l = 0; l < k; ++l) p -= A[k][l] * A[k][l];
      if (!(p > 1e-12)) { ok = false; break; }
      const double r = sqrt(p);
      A[k][k] = r;
      for (int i = k + 1; i < nn; ++i) {
        double t = A[i][k];
        for (int l = 0; l < k; ++l) t -= A[i][l] * A[k][l];
        A[i][k] = t / r;
      }
    }
    if (!ok) continue;
    double y[kAAMax];
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
      ok = ok && (y[k] == y[k]) && fabs(y[k]) < 1e300;
      gsum += fabs(y[k]);
    }
    if (!ok || !(gsum <= kAAGammaMax)) continue;
    for (int k = 0; k < nn; ++k) gam[idx[k]] = y[k];
    sc[SC_AA_N] = (double)nn;
    return;
  }
  sc[SC_AA_N] = 0.0;
}

// The graph-launched viscosity loop: one instantiated graph per starting buffer of
// the viscosity double buffer; the launch and pass counts of each captured region of
// one iteration turn the loop's totals into launches and passes.
struct PicardGraphs {
  bool valid = false;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  void* visc_buf[2] = {nullptr, nullptr};   // buffer holding the current viscosity when exec[p] starts
  long long n_pre = 0, n_head = 0, n_first = 0, n_second = 0, n_tail = 0, n_post = 0;
  double p_pre = 0, p_head = 0, p_first = 0, p_second = 0, p_tail = 0;
};

struct Ctx {
  diva_grid_t g;
  diva_config_t c;
  Dims d;
  Zeta zt;
  BCs bc;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  void* f[DIVA_NUM_FIELDS] = {};      // device pointer of each field
  void* saved[DIVA_NUM_FIELDS] = {};  // state snapshot (diva_state_save)
  bool have_saved = false;
  // work buffers
  double* visc_prev = nullptr;        // second buffer of visc_eff_3D_a (Picard double buffering)
  double* afac = nullptr;             // 0.5 * A^(-1/n), per solve
  double* quad[4] = {};               // grounded fractions of the four quadrants (NW, NE, SW, SE)
  double* err_cand[2] = {};           // DIVA_err candidates (cx, cy)
  double* staging = nullptr;          // upload/download staging (largest field)
  double* col_eps = nullptr;          // column coefficients: mean-flow strain rate per column
  int* col_flags = nullptr;           // column coefficients: shear faces with ice
  double* taub_seen[2] = {};          // basal stress (cx, cy) the last K1 of the viscosity loop read
  float* f32[kMaxLevels][6] = {};     // float copies of each tiled level (F32_*, precision 'mixed')
  int8_t* rtu = nullptr;              // finest-level row types ('BC' ice margins)
  int8_t* rtv = nullptr;
  int* ff_ocean = nullptr;            // flood-fill state
  int* ff_flag = nullptr;
  double* scal = nullptr;             // device scalars (SC_*)
  double* h_scal = nullptr;           // pinned host mirror
  double* partials = nullptr;         // block partial sums
  int max_blocks = 0;
  double* kv[KV_COUNT][2] = {};       // Krylov vectors (u,v)
  // Anderson mixing history (u,v plane pairs): ring of residual differences dF and map
  // differences dG, and the previous residual f = g - u and map value g
  double* aa_dF[kAAMax][2] = {};
  double* aa_dG[kAAMax][2] = {};
  double* aa_f[2] = {};
  double* aa_g[2] = {};
  Level lv[kMaxLevels];
  int nlev = 0;
  // inverse of the coarsest level's reduced matrix (when it has few enough unknowns)
  bool coarse_direct = false;
  int coarse_n = 0;
  double* coarse_A = nullptr;         // probed matrix, row-major n x n
  double* coarse_inv = nullptr;       // its inverse
  int* coarse_singular = nullptr;     // set by the inversion: relax instead
  // row tables of the one-block sub-cycle levels (grid and boundary conditions only)
  uint16_t* sub_tab = nullptr;
  size_t sub_tab_off[kMaxLevels] = {};
  int sub_cls[kMaxLevels][5] = {};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  PicardGraphs graphs[2];               // [0] solve_SSA, [1] solve_DIVA
  bool graphs_disabled = false;         // set if graph construction failed: host-driven loop
  bool tiled = false;                   // large levels smoothed by the tiled kernels
  bool tiles_disabled = false;          // per-colour kernels on every level
  int tile_override[kMaxLevels] = {};   // tile edge of a tiled level: 0 by its size, else 16 or 32
  // counters of the last solve
  long lin_iters = 0, mg_cycles = 0;
  long long launches = 0;            // kernels launched since create
  double fine_passes = 0.0;
  std::string err;

  template <class T> T* F(int id) const { return static_cast<T*>(f[id]); }
  double* D(int id) const { return static_cast<double*>(f[id]); }
  int* I(int id) const { return static_cast<int*>(f[id]); }
};

// status helpers
int set_error(Ctx* c, int code, const std::string& msg);
int check_cuda(Ctx* c, cudaError_t e, const char* what);
#define DIVA_CUDA(ctx, call)                                       \
  do {                                                             \
    cudaError_t e__ = (call);                                      \
    if (e__ != cudaSuccess) return check_cuda((ctx), e__, #call);  \
  } while (0)
#define DIVA_LAUNCHED(ctx, what)                                   \
  do {                                                             \
    cudaError_t e__ = cudaGetLastError();                          \
    if (e__ != cudaSuccess) return check_cuda((ctx), e__, (what)); \
  } while (0)

// geometry.cu
int launch_update_general_ice_model_data(Ctx* c);
int launch_pressure_melting_point(Ctx* c);
int launch_ice_rheology(Ctx* c);
int launch_basal_conditions(Ctx* c);
int launch_grounded_fractions(Ctx* c);
int launch_driving_stress(Ctx* c);
int launch_sico_masks(Ctx* c);

// picard.cu
int launch_prepare_afac(Ctx* c);
// K1: the coefficients of one viscosity iteration from (u, v), the previous viscosity and
// the basal stress.  K1_WRITE_SHEAR also writes du_dz_3D_cx / dv_dz_3D_cy; K1_LOOP (the
// viscosity loop) keeps what it needs to write them after the loop instead
// (launch_visc_b_output); K1_COLUMNS_ONLY launches the column kernel alone (timing).
enum { K1_WRITE_SHEAR = 0, K1_LOOP = 1, K1_COLUMNS_ONLY = 2 };
int launch_diva_coefficients(Ctx* c, const double* u, const double* v, bool diva, int what = K1_WRITE_SHEAR);
int launch_picard_update(Ctx* c, double* u, double* v, const double* xu, const double* xv, bool diva);
// Anderson mixing step before launch_picard_update (picard_anderson_m > 0): the map value
// g = velocity-limited linear solution, its residual f = g - u, the new history columns
// and the mixing coefficients (device scalars); launch_picard_update then forms the
// mixed iterate g - sum gamma_i dG_i in place of the relaxation.
int launch_anderson_prepare(Ctx* c, const double* u, const double* v, const double* xu, const double* xv);
int anderson_reset(Ctx* c);   // empty history at the start of a solve (zeroed columns)
int launch_commit_err(Ctx* c);
int launch_basal_stress_velocities(Ctx* c);
int launch_visc_b_output(Ctx* c);   // after the viscosity loop: visc_eff_3D_b and the shear strain rates
int launch_3d_horizontal_velocities(Ctx* c);
int launch_secondary_velocities(Ctx* c);
int launch_sia(Ctx* c);
int launch_ssa_beta_eff(Ctx* c);
int launch_zero_velocities(Ctx* c, double* u, double* v);
int launch_ctl_end(Ctx* c, bool relmode);
int launch_err_commit_pred(Ctx* c);
int launch_basal_pred(Ctx* c);
int launch_any_sheet(Ctx* c, int* result);

// solver.cu
int solver_init(Ctx* c);
size_t solver_table_entries(const Ctx* c);   // uint16 entries of the sub-cycle row tables      // per-context solver choices (after the configuration is known)
// Coefficients of all levels from N_a, N_b, beta_eff, taud.  The inverse of the coarsest
// level's matrix (the coarse step of the V-cycle preconditioner) is formed when inv_when is
// 0; with 1 only in the viscosity iterations coarse_inverse_due() picks (the device
// iteration counter of the graph-launched loop), with 2 not at all (an older inverse stays).
// The operator itself, and so the converged answer, is always current.
int solver_setup(Ctx* c, int inv_when = 0);
// Viscosity iterations that refresh the coarse inverse: the first three, then every fourth.
// Its one-block Gauss-Jordan elimination costs as much as a fifth of an iteration's V-cycle,
// while the coarsest grid's coefficients change slowly once the iteration has settled.
__host__ __device__ inline bool coarse_inverse_due(int it) { return it <= 3 || (it - 1) % 4 == 0; }
// The stagnation stop of a rel-res loop (picard_stall_its): track the lowest rel-res and the
// iterations since it last fell by 10 %; true once that count reaches stall_its.
__host__ __device__ inline bool stall_after(double relres, double* best, double* since, int stall_its) {
  if (stall_its <= 0) return false;
  if (*best == 0.0 || relres < 0.9 * *best) {
    *best = relres;
    *since = 0.0;
    return false;
  }
  *since += 1.0;
  return *since >= (double)stall_its;
}
int solver_solve(Ctx* c, const double* u0, const double* v0, double rtol, int maxit, int* iters, double* relres0);
int solver_relres(Ctx* c, const double* u, const double* v, double* relres);
int solver_fill_boundary(Ctx* c, double* u, double* v);
int solver_row_types(Ctx* c);   // finest-level row types of choice_ice_margin 'BC' (after the SICO masks)
int solver_smooth_fine(Ctx* c, int sweeps);
int solver_smooth_fine_values(const Ctx* c);
int solver_matvec_fine(Ctx* c, int reps);
int solver_vcycle_fine(Ctx* c, int reps);
int solver_subcycle(Ctx* c, int reps);
double solver_vcycle_bytes(const Ctx* c);
int solver_build_picard_graphs(Ctx* c, bool diva);
// the viscosity loops of n contexts (solve_DIVA) side by side in one instantiated graph
int solver_build_batch_graph(Ctx* const* cs, int n, cudaGraphExec_t* exec, void** bufs);
void solver_destroy_graphs(Ctx* c);
// tile edge (16 or 32) of each level's smoothing kernels, 0 for levels not smoothed by
// the tiled kernels; returns the number of levels
int solver_tile_edges(const Ctx* c, int32_t* edges, int n);

}  // namespace diva

// the opaque handle of the C ABI
struct diva_ctx {
  diva::Ctx c;
};
