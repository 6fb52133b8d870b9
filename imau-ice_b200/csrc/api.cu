// api.cu -- the C ABI of libdiva_b200.so (include/diva.h): context, device
// memory, Fortran-order upload/download, and the host-side sequencing of
// solve_SIA / solve_SSA / solve_DIVA (ice_velocity_module.f90:36-374).
//
// All device memory of a context is one cudaMalloc'd arena carved at create
// time; no call after diva_create allocates.  Every kernel runs on the
// context's stream.  The viscosity loop is one CUDA graph launch per solve
// (device-side loop; the host waits once, at its end); the host-driven fallback
// synchronises once per viscosity iteration and once per Krylov half-step.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <string>
#include "ctx.hpp"

using namespace diva;

namespace diva {

int set_error(Ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}
int check_cuda(Ctx* c, cudaError_t e, const char* what) {
  return set_error(c, DIVA_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace diva

namespace {

const diva_field_info_t g_info[DIVA_NUM_FIELDS] = {
#define X(ID, name, grid, type) {#name, DIVA_GRID_##grid, DIVA_DTYPE_##type},
    DIVA_FIELD_LIST(X)
#undef X
};

bool is3d(int kind) { return kind >= DIVA_GRID_A3; }
int base_kind(int kind) { return is3d(kind) ? kind - DIVA_GRID_A3 : kind; }

int64_t host_numel(int nx, int ny, int nz, int kind) {
  const int64_t n2[4] = {(int64_t)ny * nx, (int64_t)ny * (nx - 1), (int64_t)(ny - 1) * nx, (int64_t)(ny - 1) * (nx - 1)};
  return (is3d(kind) ? nz : 1) * n2[base_kind(kind)];
}

// Fortran-order host array <-> padded, layer-major device layout
template <typename T>
__global__ void k_unpack(Dims d, int kind, const T* __restrict__ src, T* __restrict__ dst) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  const int bk = kind >= DIVA_GRID_A3 ? kind - DIVA_GRID_A3 : kind;
  const int hny = (bk == DIVA_GRID_CY || bk == DIVA_GRID_B) ? d.ny - 1 : d.ny;
  const int hnx = (bk == DIVA_GRID_CX || bk == DIVA_GRID_B) ? d.nx - 1 : d.nx;
  if (j >= hny || i >= hnx) return;
  const long long col = (long long)i * hny + j;
  if (kind >= DIVA_GRID_A3) {
    for (int k = 0; k < d.nz; ++k) dst[(long long)k * d.plane + d.at(j, i)] = src[col * d.nz + k];
  } else {
    dst[d.at(j, i)] = src[col];
  }
}
template <typename T>
__global__ void k_pack(Dims d, int kind, const T* __restrict__ src, T* __restrict__ dst) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  const int bk = kind >= DIVA_GRID_A3 ? kind - DIVA_GRID_A3 : kind;
  const int hny = (bk == DIVA_GRID_CY || bk == DIVA_GRID_B) ? d.ny - 1 : d.ny;
  const int hnx = (bk == DIVA_GRID_CX || bk == DIVA_GRID_B) ? d.nx - 1 : d.nx;
  if (j >= hny || i >= hnx) return;
  const long long col = (long long)i * hny + j;
  if (kind >= DIVA_GRID_A3) {
    for (int k = 0; k < d.nz; ++k) dst[col * d.nz + k] = src[(long long)k * d.plane + d.at(j, i)];
  } else {
    dst[col] = src[d.at(j, i)];
  }
}

__global__ void k_fill(double* p, long long n, double v) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) p[t] = v;
}

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

struct Carver {
  char* base;
  size_t off = 0;
  bool dry;
  void* take(size_t bytes) {
    void* p = dry ? nullptr : base + off;
    off += align256(bytes);
    return p;
  }
};

void config_defaults(diva_config_t* c) {
  // configuration_module.f90:271-367, 424-426, 702
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
  c->lin_rtol = 1E-8; c->lin_maxit = 500;
  c->picard_stop = DIVA_STOP_RESID_UV; c->picard_relres_tol = 1E-6; c->lin_adaptive = 0; c->lin_adaptive_eta = 0.5;
  c->dt_thermo = 10.0;                                   // configuration_module.f90:56, 427-430, 647
  c->choice_ice_heat_capacity = DIVA_HEATCAP_POUNDER1965; c->uniform_ice_heat_capacity = 2009.0;
  c->choice_ice_thermal_conductivity = DIVA_CONDUCT_RITZ1987; c->uniform_ice_thermal_conductivity = 6.626958E7;
  c->T_ocean_mean_PD_ANT = -1.7;
  c->choice_ice_integration_method = DIVA_INTEGRATION_EXPLICIT; c->dHi_rtol = 1E-10; c->dHi_maxit = 1000;
  c->choice_calving_law = DIVA_CALVING_THRESHOLD_THICKNESS; c->calving_threshold_thickness = 200.0;
  c->continental_shelf_min_height = -2000.0;
  c->precision = DIVA_PREC_FP64;
}

int validate_config(Ctx* c, const diva_config_t* cfg) {
  if (cfg->choice_ice_dynamics < 0 || cfg->choice_ice_dynamics > 3) return set_error(c, DIVA_BAD_INPUT, "choice_ice_dynamics");
  if (cfg->choice_ice_margin < 0 || cfg->choice_ice_margin > 1) return set_error(c, DIVA_BAD_INPUT, "choice_ice_margin");
  if (cfg->choice_sliding_law < 0 || cfg->choice_sliding_law > 6) return set_error(c, DIVA_BAD_INPUT, "choice_sliding_law");
  if (cfg->DIVA_visc_it_nit < 1) return set_error(c, DIVA_BAD_INPUT, "DIVA_visc_it_nit must be >= 1");
  if (!(cfg->n_flow > 0.0)) return set_error(c, DIVA_BAD_INPUT, "n_flow must be > 0");
  if (cfg->lin_maxit < 1) return set_error(c, DIVA_BAD_INPUT, "lin_maxit must be >= 1");
  if (cfg->precision != DIVA_PREC_FP64 && cfg->precision != DIVA_PREC_MIXED)
    return set_error(c, DIVA_BAD_INPUT, "precision must be DIVA_PREC_FP64 or DIVA_PREC_MIXED");
  if (cfg->lin_adaptive && !(cfg->lin_adaptive_eta > 0.0 && cfg->lin_adaptive_eta < 1.0))
    return set_error(c, DIVA_BAD_INPUT, "lin_adaptive_eta must lie in (0, 1)");
  if (cfg->picard_anderson_m < 0 || cfg->picard_anderson_m > kAAMax)
    return set_error(c, DIVA_BAD_INPUT, "picard_anderson_m must lie in 0..5");
  if (cfg->picard_anderson_m > 0 && cfg->picard_stop != DIVA_STOP_RELRES)
    return set_error(c, DIVA_BAD_INPUT, "picard_anderson_m > 0 needs picard_stop = DIVA_STOP_RELRES");
  if (cfg->picard_stall_its < 0) return set_error(c, DIVA_BAD_INPUT, "picard_stall_its must be >= 0");
  const int bcs[8] = {cfg->BC_u_west, cfg->BC_u_east, cfg->BC_u_south, cfg->BC_u_north,
                      cfg->BC_v_west, cfg->BC_v_east, cfg->BC_v_south, cfg->BC_v_north};
  for (int b : bcs)
    if (b < 0 || b > 2) return set_error(c, DIVA_BAD_INPUT, "boundary condition code");
  return DIVA_OK;
}

void apply_config(Ctx* c, const diva_config_t* cfg) {
  c->c = *cfg;
  c->bc = BCs{cfg->BC_u_west, cfg->BC_u_east, cfg->BC_u_south, cfg->BC_u_north,
              cfg->BC_v_west, cfg->BC_v_east, cfg->BC_v_south, cfg->BC_v_north};
  for (int k = 0; k < c->zt.nz; ++k) c->zt.zn[k] = pow(c->zt.z[k], cfg->n_flow);
}

// multigrid hierarchy: halve every direction with at least 9 points
void plan_levels(Ctx* c) {
  int nx = c->d.nx, ny = c->d.ny;
  double dx = c->d.dx;
  c->nlev = 0;
  for (;;) {
    Dims L;
    L.nx = nx; L.ny = ny; L.nz = c->d.nz;
    L.ld = c->nlev == 0 ? c->d.ld : ((ny + 15) / 16) * 16;
    L.plane = (long long)L.nx * L.ld;
    L.dx = dx;
    c->lv[c->nlev].d = L;
    c->nlev++;
    if (c->nlev == kMaxLevels) break;
    const bool cx = nx >= 9, cy = ny >= 9;
    if (!cx && !cy) break;
    if (cx) { nx = (nx + 2) / 2; dx *= 2.0; }
    if (cy) ny = (ny + 2) / 2;
  }
}

size_t carve(Ctx* c, Carver& cv) {
  const Dims& d = c->d;
  for (int f = 0; f < DIVA_NUM_FIELDS; ++f) {
    const size_t es = g_info[f].dtype == DIVA_DTYPE_D ? sizeof(double) : sizeof(int);
    c->f[f] = cv.take((is3d(g_info[f].grid) ? d.nz : 1) * d.plane * es);
  }
  c->visc_prev = (double*)cv.take(sizeof(double) * d.nz * d.plane);
  c->afac = (double*)cv.take(sizeof(double) * d.nz * d.plane);
  for (int q = 0; q < 4; ++q) c->quad[q] = (double*)cv.take(sizeof(double) * d.plane);
  for (int q = 0; q < 2; ++q) c->err_cand[q] = (double*)cv.take(sizeof(double) * d.plane);
  c->staging = (double*)cv.take(sizeof(double) * d.nz * d.plane);
  c->col_eps = (double*)cv.take(sizeof(double) * d.plane);
  c->col_flags = (int*)cv.take(sizeof(int) * d.plane);
  for (int q = 0; q < 2; ++q) c->taub_seen[q] = (double*)cv.take(sizeof(double) * d.plane);
  for (int l = 0; l < c->nlev; ++l)
    for (int k = 0; k < 6; ++k) c->f32[l][k] = (float*)cv.take(sizeof(float) * c->lv[l].d.plane);
  c->rtu = (int8_t*)cv.take(d.plane);
  c->rtv = (int8_t*)cv.take(d.plane);
  c->ff_ocean = (int*)cv.take(sizeof(int) * 2 * d.plane);
  c->ff_flag = (int*)cv.take(sizeof(int) * 4);
  c->scal = (double*)cv.take(sizeof(double) * SC_COUNT);
  c->coarse_A = (double*)cv.take(sizeof(double) * kCoarseDirectMax * kCoarseDirectMax);
  c->coarse_inv = (double*)cv.take(sizeof(double) * kCoarseDirectMax * kCoarseDirectMax);
  c->coarse_singular = (int*)cv.take(sizeof(int) * 4);
  c->sub_tab = (uint16_t*)cv.take(sizeof(uint16_t) * (solver_table_entries(c) + 8));
  const dim3 g = grid2d(d.ny, d.nx);
  c->max_blocks = g.x * g.y;
  c->partials = (double*)cv.take(sizeof(double) * (kAAPartials > 4 ? kAAPartials : 4) * c->max_blocks);
  for (int k = 0; k < KV_COUNT; ++k)
    for (int q = 0; q < 2; ++q) c->kv[k][q] = (double*)cv.take(sizeof(double) * d.plane);
  for (int q = 0; q < 2; ++q) {
    for (int k = 0; k < kAAMax; ++k) {
      c->aa_dF[k][q] = (double*)cv.take(sizeof(double) * d.plane);
      c->aa_dG[k][q] = (double*)cv.take(sizeof(double) * d.plane);
    }
    c->aa_f[q] = (double*)cv.take(sizeof(double) * d.plane);
    c->aa_g[q] = (double*)cv.take(sizeof(double) * d.plane);
  }
  for (int l = 0; l < c->nlev; ++l) {
    Level& L = c->lv[l];
    const size_t pb = sizeof(double) * L.d.plane;
    L.Na = (double*)cv.take(pb); L.Nb = (double*)cv.take(pb); L.Bx = (double*)cv.take(pb); L.By = (double*)cv.take(pb);
    L.idu = (double*)cv.take(pb); L.idv = (double*)cv.take(pb);
    L.xu = (double*)cv.take(pb); L.xv = (double*)cv.take(pb); L.bu = (double*)cv.take(pb); L.bv = (double*)cv.take(pb);
    L.ru = (double*)cv.take(pb); L.rv = (double*)cv.take(pb);
    L.tu = (double*)cv.take(pb); L.tv = (double*)cv.take(pb);
  }
  return cv.off;
}

size_t field_dev_bytes(const Ctx* c, int f) {
  const size_t es = g_info[f].dtype == DIVA_DTYPE_D ? sizeof(double) : sizeof(int);
  return (is3d(g_info[f].grid) ? c->d.nz : 1) * c->d.plane * es;
}

int begin(Ctx* c) {
  c->lin_iters = 0;
  c->mg_cycles = 0;
  c->fine_passes = 0.0;
  c->err.clear();
  DIVA_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  return DIVA_OK;
}
int finish(Ctx* c, diva_report_t* rep) {
  DIVA_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  DIVA_CUDA(c, cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  DIVA_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  if (rep) {
    rep->elapsed_ms = ms;
    rep->linear_iterations = (int32_t)c->lin_iters;
    rep->mg_cycles = (int32_t)c->mg_cycles;
    rep->fine_passes = c->fine_passes;
  }
  return DIVA_OK;
}

int fill_const(Ctx* c, double* p, double v) {
  const long long n = c->d.plane;
  k_fill<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(p, n, v); c->launches++;
  DIVA_LAUNCHED(c, "k_fill");
  return DIVA_OK;
}

// The viscosity iteration as one graph launch per iteration (see solver.cu):
// the Krylov loop and the skip of a converged iteration run on the device;
// the host reads one status block per iteration and mirrors the viscosity
// buffer swap the graph performed.  In steps, so that a batch of contexts can
// keep one iteration of each in flight on its own stream (diva_solve_diva_batch).
struct GraphLoop {
  bool diva = true;
  int it = 0;
  double resid = 0.0, relres = -1.0;
  bool by_relres = false, done = false;
};

int graph_loop_begin(Ctx* c, GraphLoop& L) {
  double init[SC_COUNT - SC_TARGET2] = {};
  init[SC_RELRES - SC_TARGET2] = -1.0;
  init[SC_ETA - SC_TARGET2] = c->c.lin_adaptive_eta;
  DIVA_CUDA(c, cudaMemcpyAsync(c->scal + SC_TARGET2, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
  L.it = 0; L.resid = 0.0; L.relres = -1.0; L.by_relres = false; L.done = false;
  return anderson_reset(c);
}

// enqueue the whole viscosity loop (one graph launch) and the copy of its status block
int graph_loop_launch(Ctx* c, GraphLoop& L) {
  PicardGraphs& G = c->graphs[L.diva ? 1 : 0];
  int parity;
  if (c->f[DIVA_F_VISC_EFF_3D_A] == G.visc_buf[0]) parity = 0;
  else if (c->f[DIVA_F_VISC_EFF_3D_A] == G.visc_buf[1]) parity = 1;
  else return set_error(c, DIVA_CUDA_ERROR, "viscosity buffers out of step with the captured graphs");
  DIVA_CUDA(c, cudaGraphLaunch(G.exec[parity], c->stream));
  DIVA_CUDA(c, cudaMemcpyAsync(c->h_scal + SC_TARGET2, c->scal + SC_TARGET2,
                               sizeof(double) * (SC_COUNT - SC_TARGET2), cudaMemcpyDeviceToHost, c->stream));
  return DIVA_OK;
}

// wait for the loop and account for it: every iteration swapped the viscosity buffers
int graph_loop_collect(Ctx* c, GraphLoop& L) {
  PicardGraphs& G = c->graphs[L.diva ? 1 : 0];
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  const double* h = c->h_scal;
  L.it = (int)h[SC_PIC_IT];
  if (L.it & 1) std::swap(c->f[DIVA_F_VISC_EFF_3D_A], *reinterpret_cast<void**>(&c->visc_prev));
  const long lin = (long)h[SC_SUM_LIN], full = (long)h[SC_SUM_FULL], solved = (long)h[SC_N_SOLVED];
  c->lin_iters += lin;
  c->mg_cycles += lin + full;
  c->launches += (long long)L.it * (G.n_pre + G.n_post) + solved * (G.n_head + G.n_tail) + lin * G.n_first +
                 full * G.n_second;
  c->fine_passes += L.it * G.p_pre + solved * (G.p_head + G.p_tail) + lin * G.p_first + full * G.p_second;
  L.relres = h[SC_RELRES];
  L.done = true;
  if (h[SC_NAN] != 0.0) return set_error(c, DIVA_NAN_DETECTED, "NaN in the viscosity iteration");
  if (h[SC_EXIT_RELRES] != 0.0) {
    L.by_relres = true;
    return DIVA_OK;
  }
  L.resid = h[SC_RESID];
  if (h[SC_CONVERGED] == 0.0) return set_error(c, DIVA_TIMEOUT, "viscosity iteration did not stop");
  return DIVA_OK;
}

int graph_loop_end(Ctx* c, const GraphLoop& L, diva_report_t* rep) {
  const diva_config_t& C = c->c;
  const bool relmode = C.picard_stop == DIVA_STOP_RELRES;
  int status = DIVA_OK;
  const bool stalled = c->h_scal[SC_STALLED] != 0.0;
  if (!L.by_relres && L.it >= C.DIVA_visc_it_nit && (relmode || L.resid >= C.DIVA_visc_it_norm_dUV_tol))
    status = DIVA_MAX_PICARD;
  if (stalled) status = DIVA_MAX_PICARD;   // stopped on picard_stall_its short of the tolerance
  if (rep) {
    rep->picard_iterations = L.it;
    rep->resid_UV = L.resid;
    rep->relres = L.relres;
    rep->status = status;
    rep->reserved[0] = (int32_t)c->h_scal[SC_LIN_FAILED];
    rep->reserved[1] = 1;   // graph-launched
    rep->reserved[2] = stalled ? 1 : 0;
  }
  return status;
}

int picard_graph(Ctx* c, bool diva, diva_report_t* rep) {
  GraphLoop L;
  L.diva = diva;
  int st = graph_loop_begin(c, L);
  if (!st) st = graph_loop_launch(c, L);
  if (!st) st = graph_loop_collect(c, L);
  if (st) return st;
  return graph_loop_end(c, L, rep);
}

// the viscosity iteration shared by solve_SSA (:180-240) and solve_DIVA (:307-363)
int picard(Ctx* c, bool diva, double* u, double* v, diva_report_t* rep) {
  if (!c->graphs_disabled) {
    if (solver_build_picard_graphs(c, diva) == DIVA_OK) return picard_graph(c, diva, rep);
    c->graphs_disabled = true;   // conditional graph nodes unavailable: host-driven loop below
  }
  const diva_config_t& C = c->c;
  const bool relmode = C.picard_stop == DIVA_STOP_RELRES;
  int it = 0, st = DIVA_OK, lin_fail = 0;
  bool stalled_exit = false;
  double stall_best = 0.0, stall_since = 0.0;
  double resid = 0.0, relres = -1.0, eta = C.lin_adaptive_eta, relres_prev = 0.0;
  if (C.picard_anderson_m > 0) {
    double init[SC_COUNT - SC_AA_N] = {};
    DIVA_CUDA(c, cudaMemcpyAsync(c->scal + SC_AA_N, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
    if ((st = anderson_reset(c))) return st;
  }
  for (;;) {
    ++it;
    if ((st = launch_diva_coefficients(c, u, v, diva, K1_LOOP))) return st;
    if ((st = solver_setup(c, coarse_inverse_due(it) ? 0 : 2))) return st;
    if (relmode) {
      if ((st = solver_relres(c, u, v, &relres))) return st;
      eta = eta_after(eta, relres, relres_prev, C.picard_relres_tol);   // as the graph's k_ctl_relres does
      relres_prev = relres;
      if (!std::isfinite(relres)) return set_error(c, DIVA_NAN_DETECTED, "NaN in the nonlinear residual");
      const bool stop_stall = relres > C.picard_relres_tol &&
                              stall_after(relres, &stall_best, &stall_since, C.picard_stall_its);
      if (relres <= C.picard_relres_tol || stop_stall) {
        stalled_exit = stop_stall;
        if (diva && (st = launch_basal_stress_velocities(c))) return st;
        break;
      }
    }
    double rtol = C.lin_rtol;
    if (relmode && C.lin_adaptive) rtol = std::max(C.lin_rtol, eta * std::min(1.0, relres));
    int iters = 0;
    st = solver_solve(c, u, v, rtol, C.lin_maxit, &iters, nullptr);
    if (st == DIVA_LINEAR_NOT_CONVERGED) {
      ++lin_fail;   // the reference does not check PETSc/SOR convergence either; keep iterating
    } else if (st) {
      return st;
    }
    if (C.picard_anderson_m > 0) {
      // the mixing step reads this iteration's nonlinear residual from the device scalars
      DIVA_CUDA(c, cudaMemcpyAsync(c->scal + SC_RELRES, &relres, sizeof(double), cudaMemcpyHostToDevice, c->stream));
      if ((st = launch_anderson_prepare(c, u, v, c->kv[KV_X][0], c->kv[KV_X][1]))) return st;
    }
    if ((st = launch_picard_update(c, u, v, c->kv[KV_X][0], c->kv[KV_X][1], diva))) return st;
    DIVA_CUDA(c, cudaMemcpyAsync(c->h_scal + SC_RES1, c->scal + SC_RES1, 3 * sizeof(double), cudaMemcpyDeviceToHost,
                                 c->stream));
    DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
    const double r1 = c->h_scal[SC_RES1], r2 = c->h_scal[SC_RES2], cnt = c->h_scal[SC_RES1 + 2];
    if (!std::isfinite(r1) || !std::isfinite(r2)) return set_error(c, DIVA_NAN_DETECTED, "NaN in the velocities");
    resid = (cnt > 0.0) ? 2.0 * sqrt(r1) / std::max(sqrt(r2), 1E-8) : 0.0;
    bool converged = false;
    if (!relmode && resid < C.DIVA_visc_it_norm_dUV_tol) converged = true;
    else if (it >= C.DIVA_visc_it_nit) converged = true;
    if (!converged) launch_commit_err(c);
    if (converged) break;
  }
  int status = DIVA_OK;
  if ((it >= C.DIVA_visc_it_nit || stalled_exit) &&
      ((relmode && !(relres >= 0.0 && relres <= C.picard_relres_tol)) ||
       (!relmode && resid >= C.DIVA_visc_it_norm_dUV_tol)))
    status = DIVA_MAX_PICARD;
  if (stalled_exit) status = DIVA_MAX_PICARD;
  if (rep) {
    rep->picard_iterations = it;
    rep->resid_UV = resid;
    rep->relres = relres;
    rep->status = status;
    rep->reserved[0] = lin_fail;
    rep->reserved[1] = 0;   // host-driven
    rep->reserved[2] = stalled_exit ? 1 : 0;
  }
  return status;
}

int prepare_velocity_solve(Ctx* c) {
  int st;
  if ((st = launch_driving_stress(c))) return st;
  if ((st = launch_basal_conditions(c))) return st;
  if ((st = launch_grounded_fractions(c))) return st;
  if ((st = fill_const(c, c->D(DIVA_F_DIVA_ERR_CX), 1E5))) return st;
  if ((st = fill_const(c, c->D(DIVA_F_DIVA_ERR_CY), 1E5))) return st;
  if ((st = launch_prepare_afac(c))) return st;
  // set_sico_masks (:1678) depends only on TAF and Hi, which do not change
  // during the viscosity iteration: once per solve gives the same masks
  if ((st = launch_sico_masks(c))) return st;
  if ((st = solver_row_types(c))) return st;
  return DIVA_OK;
}

}  // namespace

extern "C" {

void diva_config_defaults(diva_config_t* cfg) {
  if (cfg) config_defaults(cfg);
}

void diva_grid_init(diva_grid_t* g, int32_t nx, int32_t ny, double dx, double xmin, double ymin) {
  if (!g) return;
  memset(g, 0, sizeof(*g));
  g->nx = nx; g->ny = ny; g->nz = 15; g->dx = dx; g->xmin = xmin; g->ymin = ymin;
  const double z[15] = {0.00, 0.10, 0.20, 0.30, 0.40, 0.50, 0.60, 0.70, 0.80, 0.90, 0.925, 0.95, 0.975, 0.99, 1.00};
  for (int k = 0; k < 15; ++k) g->zeta[k] = z[k];
}

int diva_field_info(int32_t id, diva_field_info_t* out) {
  if (id < 0 || id >= DIVA_NUM_FIELDS || !out) return DIVA_BAD_INPUT;
  *out = g_info[id];
  return DIVA_OK;
}

int64_t diva_field_numel(const diva_grid_t* g, int32_t id) {
  if (!g || id < 0 || id >= DIVA_NUM_FIELDS) return -1;
  return host_numel(g->nx, g->ny, g->nz, g_info[id].grid);
}

int diva_create(diva_ctx_t** out, const diva_grid_t* g, const diva_config_t* cfg) {
  if (!out || !g || !cfg) return DIVA_BAD_INPUT;
  *out = nullptr;
  if (g->nx < 5 || g->ny < 5 || g->nz < 2 || g->nz > kMaxNz || !(g->dx > 0.0)) return DIVA_BAD_INPUT;
  for (int k = 1; k < g->nz; ++k)
    if (!(g->zeta[k] > g->zeta[k - 1])) return DIVA_BAD_INPUT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return DIVA_CUDA_ERROR;
  diva_ctx* h = new diva_ctx();
  Ctx* c = &h->c;
  int st = validate_config(c, cfg);
  if (st) { delete h; return st; }
  c->g = *g;
  c->d.nx = g->nx; c->d.ny = g->ny; c->d.nz = g->nz;
  c->d.ld = ((g->ny + 15) / 16) * 16;
  c->d.plane = (long long)c->d.nx * c->d.ld;
  c->d.dx = g->dx;
  c->zt.nz = g->nz;
  for (int k = 0; k < g->nz; ++k) {
    c->zt.z[k] = g->zeta[k];
    c->zt.z2[k] = pow(g->zeta[k], 2.0);
  }
  apply_config(c, cfg);
  plan_levels(c);
  // DIVA_NO_GRAPHS=1 launches the same kernels one by one instead of from
  // CUDA graphs (kernel-level profilers list them individually that way)
  if (const char* e = getenv("DIVA_NO_GRAPHS")) c->graphs_disabled = (e[0] == '1');
  // DIVA_NO_TILES=1 smooths every level with the per-colour kernels (same results)
  if (const char* e = getenv("DIVA_NO_TILES")) c->tiles_disabled = (e[0] == '1');
  Carver dry{nullptr, 0, true};
  const size_t bytes = carve(c, dry);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete h; return DIVA_CUDA_ERROR; }
  c->own_stream = true;
  if (cudaMalloc(&c->arena, bytes) != cudaSuccess) {
    cudaStreamDestroy(c->stream);
    delete h;
    return DIVA_CUDA_ERROR;
  }
  c->arena_bytes = bytes;
  Carver real{c->arena, 0, false};
  carve(c, real);
  if (cudaMallocHost(&c->h_scal, sizeof(double) * SC_COUNT) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaMemsetAsync(c->arena, 0, bytes, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess || solver_init(c) != DIVA_OK) {
    diva_destroy(h);
    return DIVA_CUDA_ERROR;
  }
  *out = h;
  return DIVA_OK;
}

int diva_destroy(diva_ctx_t* h) {
  if (!h) return DIVA_OK;
  Ctx* c = &h->c;
  if (c->stream) cudaStreamSynchronize(c->stream);
  solver_destroy_graphs(c);
  for (int f = 0; f < DIVA_NUM_FIELDS; ++f)
    if (c->saved[f]) cudaFree(c->saved[f]);
  if (c->arena) cudaFree(c->arena);
  if (c->h_scal) cudaFreeHost(c->h_scal);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete h;
  return DIVA_OK;
}

int diva_set_config(diva_ctx_t* h, const diva_config_t* cfg) {
  if (!h || !cfg) return DIVA_BAD_INPUT;
  int st = validate_config(&h->c, cfg);
  if (st) return st;
  apply_config(&h->c, cfg);
  solver_destroy_graphs(&h->c);   // captured kernel arguments carry the configuration
  return solver_init(&h->c);
}

int diva_set_stream(diva_ctx_t* h, void* stream) {
  if (!h) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  if (stream) {
    if (c->own_stream) cudaStreamDestroy(c->stream);
    c->stream = static_cast<cudaStream_t>(stream);
    c->own_stream = false;
  }
  return DIVA_OK;
}

int diva_upload_field(diva_ctx_t* h, int32_t id, const void* host) {
  if (!h || !host || id < 0 || id >= DIVA_NUM_FIELDS) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  const int kind = g_info[id].grid;
  const size_t es = g_info[id].dtype == DIVA_DTYPE_D ? sizeof(double) : sizeof(int);
  const size_t n = (size_t)host_numel(c->d.nx, c->d.ny, c->d.nz, kind);
  DIVA_CUDA(c, cudaMemcpyAsync(c->staging, host, n * es, cudaMemcpyHostToDevice, c->stream));
  if (g_info[id].dtype == DIVA_DTYPE_D) {
    k_unpack<double><<<grid2d(c->d.ny, c->d.nx), block2d(), 0, c->stream>>>(c->d, kind, c->staging, c->D(id)); c->launches++;
  } else {
    k_unpack<int><<<grid2d(c->d.ny, c->d.nx), block2d(), 0, c->stream>>>(c->d, kind, (const int*)c->staging, c->I(id)); c->launches++;
  }
  DIVA_LAUNCHED(c, "k_unpack");
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int diva_download_field(diva_ctx_t* h, int32_t id, void* host) {
  if (!h || !host || id < 0 || id >= DIVA_NUM_FIELDS) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  const int kind = g_info[id].grid;
  const size_t es = g_info[id].dtype == DIVA_DTYPE_D ? sizeof(double) : sizeof(int);
  const size_t n = (size_t)host_numel(c->d.nx, c->d.ny, c->d.nz, kind);
  if (g_info[id].dtype == DIVA_DTYPE_D) {
    k_pack<double><<<grid2d(c->d.ny, c->d.nx), block2d(), 0, c->stream>>>(c->d, kind, c->D(id), c->staging); c->launches++;
  } else {
    k_pack<int><<<grid2d(c->d.ny, c->d.nx), block2d(), 0, c->stream>>>(c->d, kind, c->I(id), (int*)c->staging); c->launches++;
  }
  DIVA_LAUNCHED(c, "k_pack");
  DIVA_CUDA(c, cudaMemcpyAsync(host, c->staging, n * es, cudaMemcpyDeviceToHost, c->stream));
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int diva_upload(diva_ctx_t* h, const diva_fields_t* f) {
  if (!h || !f) return DIVA_BAD_INPUT;
  for (int q = 0; q < DIVA_NUM_FIELDS; ++q)
    if (f->ptr[q]) {
      int st = diva_upload_field(h, q, f->ptr[q]);
      if (st) return st;
    }
  return DIVA_OK;
}

int diva_download(diva_ctx_t* h, const diva_fields_t* f) {
  if (!h || !f) return DIVA_BAD_INPUT;
  for (int q = 0; q < DIVA_NUM_FIELDS; ++q)
    if (f->ptr[q]) {
      int st = diva_download_field(h, q, f->ptr[q]);
      if (st) return st;
    }
  return DIVA_OK;
}

int diva_update_general_ice_model_data(diva_ctx_t* h) {
  if (!h) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  int st = launch_update_general_ice_model_data(c);
  if (st) return st;
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int diva_calc_pressure_melting_point(diva_ctx_t* h) {
  if (!h) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  int st = launch_pressure_melting_point(c);
  if (st) return st;
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int diva_calc_ice_rheology(diva_ctx_t* h) {
  if (!h) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  int st = launch_ice_rheology(c);
  if (st) return st;
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int diva_calc_sia_3d_velocities(diva_ctx_t* h) {
  if (!h) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  int st = launch_sia(c);
  if (st) return st;
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int diva_solve_sia(diva_ctx_t* h, diva_report_t* rep) {
  if (!h) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  if (rep) { memset(rep, 0, sizeof(*rep)); rep->relres = -1.0; }
  if (!(c->c.choice_ice_dynamics == DIVA_DYN_SIA || c->c.choice_ice_dynamics == DIVA_DYN_SIA_SSA))
    return set_error(c, DIVA_BAD_INPUT, "solve_SIA should only be called when choice_ice_dynamics is SIA or SIA/SSA");
  int st;
  if ((st = begin(c))) return st;
  if ((st = launch_sia(c))) return st;
  if ((st = launch_secondary_velocities(c))) return st;
  return finish(c, rep);
}

int diva_solve_diva(diva_ctx_t* h, diva_report_t* rep) {
  if (!h) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  if (rep) { memset(rep, 0, sizeof(*rep)); rep->relres = -1.0; }
  if (c->c.choice_ice_dynamics != DIVA_DYN_DIVA)
    return set_error(c, DIVA_BAD_INPUT, "solve_DIVA should only be called when choice_ice_dynamics is DIVA");
  int st;
  if ((st = begin(c))) return st;
  int any = 0;
  if ((st = launch_any_sheet(c, &any))) return st;
  if (!any) {
    if ((st = launch_zero_velocities(c, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY)))) return st;
    return finish(c, rep);
  }
  if ((st = prepare_velocity_solve(c))) return st;
  const int pst = picard(c, true, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY), rep);
  if (pst != DIVA_OK && pst != DIVA_MAX_PICARD) return pst;
  if ((st = launch_visc_b_output(c))) return st;
  if ((st = launch_3d_horizontal_velocities(c))) return st;
  if ((st = launch_secondary_velocities(c))) return st;
  if ((st = finish(c, rep))) return st;
  return pst;
}

// solve_DIVA for several contexts at once.  Each context runs its graph-launched
// viscosity loop on its own stream, all launched before any is waited for, so the
// iterations of different members overlap on the GPU.  A context that cannot use the
// graph-launched loop (graph construction unavailable) is solved on its own after
// the others.  reports[k] receives the report of ctxs[k]; the return value is
// DIVA_OK if every member returned OK, else the first other status.
int diva_solve_diva_batch(diva_ctx_t** hs, int32_t n, diva_report_t* reports) {
  if (!hs || n < 1 || !reports) return DIVA_BAD_INPUT;
  for (int k = 0; k < n; ++k) {
    if (!hs[k]) return DIVA_BAD_INPUT;
    for (int m = 0; m < k; ++m)
      if (hs[m] == hs[k]) return set_error(&hs[0]->c, DIVA_BAD_INPUT, "a context appears twice in the batch");
  }
  std::vector<int> status(n, DIVA_OK);
  std::vector<GraphLoop> loops(n);
  std::vector<char> active(n, 0), sequential(n, 0);
  // set-up of every member up to its first iteration
  for (int k = 0; k < n; ++k) {
    Ctx* c = &hs[k]->c;
    diva_report_t* rep = &reports[k];
    memset(rep, 0, sizeof(*rep));
    rep->relres = -1.0;
    int st = DIVA_OK;
    if (c->c.choice_ice_dynamics != DIVA_DYN_DIVA) {
      st = set_error(c, DIVA_BAD_INPUT, "solve_DIVA should only be called when choice_ice_dynamics is DIVA");
    } else if (!(st = begin(c))) {
      int any = 0;
      if (!(st = launch_any_sheet(c, &any))) {
        if (!any) {
          if (!(st = launch_zero_velocities(c, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY)))) st = finish(c, rep);
        } else if (!(st = prepare_velocity_solve(c))) {
          if (!c->graphs_disabled && solver_build_picard_graphs(c, true) == DIVA_OK) {
            loops[k].diva = true;
            if (!(st = graph_loop_begin(c, loops[k]))) active[k] = 1;
          } else {
            c->graphs_disabled = true;
            sequential[k] = 1;
          }
        }
      }
    }
    status[k] = st;
    if (st) rep->status = st;
  }
  // launch every active member's loop, then collect them in turn (one pass)
  for (;;) {
    bool any = false;
    for (int k = 0; k < n; ++k)
      if (active[k]) {
        int st = graph_loop_launch(&hs[k]->c, loops[k]);
        if (st) { status[k] = st; active[k] = 0; reports[k].status = st; }
        else any = true;
      }
    if (!any) break;
    for (int k = 0; k < n; ++k)
      if (active[k]) {
        int st = graph_loop_collect(&hs[k]->c, loops[k]);
        if (st) { status[k] = st; active[k] = 0; reports[k].status = st; }
        else if (loops[k].done) {
          active[k] = 0;
          status[k] = graph_loop_end(&hs[k]->c, loops[k], &reports[k]);
          Ctx* c = &hs[k]->c;
          int s2;
          if ((s2 = launch_visc_b_output(c)) || (s2 = launch_3d_horizontal_velocities(c)) ||
              (s2 = launch_secondary_velocities(c)) || (s2 = finish(c, &reports[k]))) {
            status[k] = s2;
          }
          reports[k].status = status[k];
        }
      }
  }
  // members without graph-launched iterations
  for (int k = 0; k < n; ++k)
    if (sequential[k]) {
      Ctx* c = &hs[k]->c;
      const int pst = picard(c, true, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY), &reports[k]);
      int st = pst;
      if (pst == DIVA_OK || pst == DIVA_MAX_PICARD) {
        int s2;
        if ((s2 = launch_visc_b_output(c)) || (s2 = launch_3d_horizontal_velocities(c)) ||
            (s2 = launch_secondary_velocities(c)) || (s2 = finish(c, &reports[k])))
          st = s2;
      }
      status[k] = st;
      reports[k].status = st;
    }
  for (int k = 0; k < n; ++k)
    if (status[k] != DIVA_OK) return status[k];
  return DIVA_OK;
}

// ---- persistent batches: every member's viscosity loop in one graph launch ----------
}  // extern "C"

struct diva_batch {
  std::vector<diva_ctx_t*> members;
  std::vector<void*> bufs;            // the viscosity buffer each member's captured loop starts from
  std::vector<diva_config_t> cfgs;    // the configurations the loops were captured with
  cudaGraphExec_t exec = nullptr;
  cudaStream_t stream = nullptr;      // the batch graph's launch stream
  cudaEvent_t done = nullptr;
  std::vector<cudaEvent_t> ready;     // one per member: its prelude has been enqueued
};

namespace {
void batch_free(diva_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (cudaEvent_t e : b->ready)
    if (e) cudaEventDestroy(e);
  if (b->done) cudaEventDestroy(b->done);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}
}  // namespace

extern "C" {

int diva_batch_create(diva_ctx_t** hs, int32_t n, diva_batch_t** out) {
  if (!hs || n < 1 || !out) return DIVA_BAD_INPUT;
  *out = nullptr;
  for (int k = 0; k < n; ++k) {
    if (!hs[k]) return DIVA_BAD_INPUT;
    for (int m = 0; m < k; ++m)
      if (hs[m] == hs[k]) return set_error(&hs[0]->c, DIVA_BAD_INPUT, "a context appears twice in the batch");
    if (hs[k]->c.c.choice_ice_dynamics != DIVA_DYN_DIVA)
      return set_error(&hs[k]->c, DIVA_BAD_INPUT, "batch members must have choice_ice_dynamics DIVA");
  }
  std::vector<Ctx*> cs(n);
  for (int k = 0; k < n; ++k) {
    cs[k] = &hs[k]->c;
    if (cs[k]->graphs_disabled) return set_error(cs[k], DIVA_UNSUPPORTED, "member without graph-launched loops");
    if (int st = solver_build_picard_graphs(cs[k], true)) return st;
  }
  diva_batch* b = new diva_batch;
  b->members.assign(hs, hs + n);
  b->bufs.resize(n);
  b->ready.resize(n, nullptr);
  for (int k = 0; k < n; ++k) b->cfgs.push_back(cs[k]->c);
  bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) == cudaSuccess;
  for (int k = 0; k < n && ok; ++k) ok = cudaEventCreateWithFlags(&b->ready[k], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    batch_free(b);
    return set_error(cs[0], DIVA_CUDA_ERROR, "batch stream or events");
  }
  if (int st = solver_build_batch_graph(cs.data(), n, &b->exec, b->bufs.data())) {
    batch_free(b);
    return st;
  }
  *out = b;
  return DIVA_OK;
}

int diva_batch_destroy(diva_batch_t* b) {
  batch_free(b);
  return DIVA_OK;
}

int diva_batch_solve_diva(diva_batch_t* b, diva_report_t* reports) {
  if (!b || !reports) return DIVA_BAD_INPUT;
  const int n = (int)b->members.size();
  std::vector<GraphLoop> loops(n);
  std::vector<int> status(n, DIVA_OK), any(n, 1);
  // preludes on the members' streams (each as solve_DIVA's before its loop)
  for (int k = 0; k < n; ++k) {
    Ctx* c = &b->members[k]->c;
    diva_report_t* rep = &reports[k];
    memset(rep, 0, sizeof(*rep));
    rep->relres = -1.0;
    if (memcmp(&c->c, &b->cfgs[k], sizeof(diva_config_t)) != 0 || !c->graphs[1].valid)
      return set_error(c, DIVA_BAD_INPUT, "batch member reconfigured since diva_batch_create");
    int st;
    if ((st = begin(c)) || (st = launch_any_sheet(c, &any[k]))) return st;
    if (any[k] && (st = prepare_velocity_solve(c))) return st;
    loops[k].diva = true;
    if ((st = graph_loop_begin(c, loops[k]))) return st;
    // the captured loop reads the viscosity from the buffer it was captured with
    if (c->f[DIVA_F_VISC_EFF_3D_A] != b->bufs[k]) {
      DIVA_CUDA(c, cudaMemcpyAsync(b->bufs[k], c->f[DIVA_F_VISC_EFF_3D_A], sizeof(double) * c->d.nz * c->d.plane,
                                   cudaMemcpyDeviceToDevice, c->stream));
      c->visc_prev = static_cast<double*>(c->f[DIVA_F_VISC_EFF_3D_A]);
      c->f[DIVA_F_VISC_EFF_3D_A] = b->bufs[k];
    }
    DIVA_CUDA(c, cudaEventRecord(b->ready[k], c->stream));
    DIVA_CUDA(c, cudaStreamWaitEvent(b->stream, b->ready[k], 0));
  }
  // one launch runs every member's viscosity loop
  Ctx* c0 = &b->members[0]->c;
  DIVA_CUDA(c0, cudaGraphLaunch(b->exec, b->stream));
  DIVA_CUDA(c0, cudaEventRecord(b->done, b->stream));
  for (int k = 0; k < n; ++k) {
    Ctx* c = &b->members[k]->c;
    DIVA_CUDA(c, cudaStreamWaitEvent(c->stream, b->done, 0));
    DIVA_CUDA(c, cudaMemcpyAsync(c->h_scal + SC_TARGET2, c->scal + SC_TARGET2,
                                 sizeof(double) * (SC_COUNT - SC_TARGET2), cudaMemcpyDeviceToHost, c->stream));
  }
  // accounting and the solves' tails on the members' streams
  int first_bad = DIVA_OK;
  for (int k = 0; k < n; ++k) {
    Ctx* c = &b->members[k]->c;
    int st = graph_loop_collect(c, loops[k]);   // also mirrors the loop's viscosity buffer swaps
    if (!any[k]) {
      // no sheet ice: solve_DIVA sets the velocities to zero and solves nothing (:276-285);
      // the member's captured loop ran all the same, and its outcome is dropped
      st = launch_zero_velocities(c, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY));
      c->err.clear();
      if (!st) st = finish(c, &reports[k]);
      reports[k].picard_iterations = 0;
    } else {
      if (!st) st = graph_loop_end(c, loops[k], &reports[k]);
      if (st == DIVA_OK || st == DIVA_MAX_PICARD) {
        int s2 = launch_visc_b_output(c);
        if (!s2) s2 = launch_3d_horizontal_velocities(c);
        if (!s2) s2 = launch_secondary_velocities(c);
        if (!s2) s2 = finish(c, &reports[k]);
        if (s2) st = s2;
      }
    }
    status[k] = st;
    reports[k].status = st;
    if (st != DIVA_OK && first_bad == DIVA_OK) first_bad = st;
  }
  return first_bad;
}

int diva_solve_ssa(diva_ctx_t* h, diva_report_t* rep) {
  if (!h) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  if (rep) { memset(rep, 0, sizeof(*rep)); rep->relres = -1.0; }
  if (!(c->c.choice_ice_dynamics == DIVA_DYN_SSA || c->c.choice_ice_dynamics == DIVA_DYN_SIA_SSA))
    return set_error(c, DIVA_BAD_INPUT, "solve_SSA should only be called when choice_ice_dynamics is SSA or SIA/SSA");
  int st;
  if ((st = begin(c))) return st;
  int any = 0;
  if ((st = launch_any_sheet(c, &any))) return st;
  if (!any || c->c.choice_sliding_law == DIVA_SLIDING_NONE) {
    if ((st = launch_zero_velocities(c, c->D(DIVA_F_U_SSA_CX), c->D(DIVA_F_V_SSA_CY)))) return st;
    return finish(c, rep);
  }
  if ((st = prepare_velocity_solve(c))) return st;
  const int pst = picard(c, false, c->D(DIVA_F_U_SSA_CX), c->D(DIVA_F_V_SSA_CY), rep);
  if (pst != DIVA_OK && pst != DIVA_MAX_PICARD) return pst;
  if ((st = launch_visc_b_output(c))) return st;
  if ((st = launch_secondary_velocities(c))) return st;
  if ((st = finish(c, rep))) return st;
  return pst;
}

int diva_nonlinear_residual(diva_ctx_t* h, double* relres) {
  if (!h || !relres) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  int st;
  if ((st = launch_driving_stress(c))) return st;
  if ((st = launch_basal_conditions(c))) return st;
  if ((st = launch_grounded_fractions(c))) return st;
  if ((st = launch_prepare_afac(c))) return st;
  if ((st = launch_diva_coefficients(c, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY), true))) return st;
  if ((st = launch_sico_masks(c))) return st;
  if ((st = solver_row_types(c))) return st;
  if ((st = solver_setup(c))) return st;
  return solver_relres(c, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY), relres);
}

int diva_complete_state(diva_ctx_t* h, int32_t sweeps) {
  if (!h || sweeps < 0 || sweeps > 10000) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  int st;
  if ((st = launch_driving_stress(c))) return st;
  if ((st = launch_basal_conditions(c))) return st;
  if ((st = launch_grounded_fractions(c))) return st;
  if ((st = launch_prepare_afac(c))) return st;
  for (int s = 0; s < sweeps; ++s) {
    if ((st = launch_diva_coefficients(c, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY), true))) return st;
    if ((st = launch_basal_stress_velocities(c))) return st;
  }
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int diva_state_save(diva_ctx_t* h) {
  if (!h) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  for (int f = 0; f < DIVA_NUM_FIELDS; ++f) {
    const size_t nb = field_dev_bytes(c, f);
    if (!c->saved[f]) DIVA_CUDA(c, cudaMalloc(&c->saved[f], nb));
    DIVA_CUDA(c, cudaMemcpyAsync(c->saved[f], c->f[f], nb, cudaMemcpyDeviceToDevice, c->stream));
  }
  c->have_saved = true;
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int diva_state_restore(diva_ctx_t* h) {
  if (!h) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  if (!c->have_saved) return set_error(c, DIVA_BAD_INPUT, "no saved state");
  for (int f = 0; f < DIVA_NUM_FIELDS; ++f)
    DIVA_CUDA(c, cudaMemcpyAsync(c->f[f], c->saved[f], field_dev_bytes(c, f), cudaMemcpyDeviceToDevice, c->stream));
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int diva_get_tile_edges(diva_ctx_t* h, int32_t* edges, int32_t n, int32_t* nlev) {
  if (!h || !edges || !nlev || n < 0) return DIVA_BAD_INPUT;
  *nlev = solver_tile_edges(&h->c, edges, n < kMaxLevels ? n : kMaxLevels);
  for (int l = kMaxLevels; l < n; ++l) edges[l] = 0;
  return DIVA_OK;
}

int diva_set_tile_edges(diva_ctx_t* h, const int32_t* edges, int32_t n) {
  if (!h || (n > 0 && !edges) || n < 0 || n > kMaxLevels) return DIVA_BAD_INPUT;
  for (int l = 0; l < n; ++l)
    if (edges[l] != 0 && edges[l] != 16 && edges[l] != 32) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  for (int l = 0; l < kMaxLevels; ++l) c->tile_override[l] = l < n ? edges[l] : 0;
  solver_destroy_graphs(c);   // captured launches carry the tile shapes
  return DIVA_OK;
}

int diva_profile_kernel(diva_ctx_t* h, int32_t which, int32_t reps, double* ms, double* bytes) {
  if (!h || !ms || !bytes || reps < 1 || which < 0 || which > 5) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  const double nc = (double)c->d.nx * c->d.ny, w = sizeof(double), nz = c->d.nz;
  int st = DIVA_OK;
  DIVA_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  for (int r = 0; r < reps && !st; ++r) {
    switch (which) {
      case 0: st = launch_diva_coefficients(c, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY), true, K1_LOOP); break;
      case 1: st = solver_smooth_fine(c, 1); break;
      case 2: st = solver_matvec_fine(c, 1); break;
      case 3: st = solver_vcycle_fine(c, 1); break;
      case 4: st = solver_subcycle(c, 1); break;
      case 5: st = launch_diva_coefficients(c, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY), true, K1_COLUMNS_ONLY); break;
    }
  }
  if (st) return st;
  DIVA_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  DIVA_CUDA(c, cudaEventSynchronize(c->ev1));
  float t = 0.f;
  DIVA_CUDA(c, cudaEventElapsedTime(&t, c->ev0, c->ev1));
  *ms = t / reps;
  // algorithmic bytes per launch (compulsory traffic per column, FP64):
  //  0: read A-factor and the previous viscosity, write the new one (3 nz) + 15 2D fields
  //  1: fine-level smoothing of one V-cycle: the tiled pre- and post-smoothing kernels (24 values,
  //     solver_smooth_fine_values), or one per-colour sweep on untiled grids (10)
  //  2: operator application: u, v, N_a, N_b, beta_x, beta_y read, A u, A v written (8)
  //  3: one V-cycle: per level 4 sweeps, a residual and the transfers, weighted by its points
  //  4: the one-block coarse levels of a V-cycle (latency-bound; bytes as for 3 over those levels)
  const double per_col[3] = {(3 * nz + 15) * w, solver_smooth_fine_values(c) * w, 8 * w};
  //  5: the column launches of 0 without the b-grid faces: A-factor and previous viscosity
  //     read, viscosity written (3 nz), with the 2D fields they read and write (12)
  *bytes = which < 3 ? per_col[which] * nc
                     : (which == 3 ? solver_vcycle_bytes(c) : (which == 5 ? (3 * nz + 12) * w * nc : 0.0));
  return DIVA_OK;
}

int64_t diva_kernel_launches(const diva_ctx_t* h) { return h ? (int64_t)h->c.launches : -1; }

const char* diva_last_error(const diva_ctx_t* h) { return h ? h->c.err.c_str() : ""; }

const char* diva_status_string(int32_t s) {
  switch (s) {
    case DIVA_OK: return "OK";
    case DIVA_MAX_PICARD: return "MAX_PICARD";
    case DIVA_LINEAR_NOT_CONVERGED: return "LINEAR_NOT_CONVERGED";
    case DIVA_NAN_DETECTED: return "NAN_DETECTED";
    case DIVA_BAD_INPUT: return "BAD_INPUT";
    case DIVA_CUDA_ERROR: return "CUDA_ERROR";
    case DIVA_TIMEOUT: return "TIMEOUT";
    case DIVA_UNSUPPORTED: return "UNSUPPORTED";
  }
  return "UNKNOWN";
}

}  // extern "C"
