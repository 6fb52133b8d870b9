/*
 * diva.h -- C ABI of the B200 ice-velocity library (libdiva_b200.so).
 *
 * Drop-in replacement for the velocity hot path of IMAU-ICE:
 *   SUBROUTINE solve_SIA ( grid, ice)   src/ice_velocity_module.f90:36-114
 *   SUBROUTINE solve_SSA ( grid, ice)   src/ice_velocity_module.f90:115-248
 *   SUBROUTINE solve_DIVA( grid, ice)   src/ice_velocity_module.f90:249-374
 * plus the routines that prepare their inputs on the same device-resident
 * state:
 *   update_general_ice_model_data       src/general_ice_model_data_module.f90:30-86
 *   calc_pressure_melting_point         src/thermodynamics_module.f90:609-640
 *   calc_ice_rheology                   src/thermodynamics_module.f90:641-753
 *
 * The Fortran reference passes TYPE(type_grid) and TYPE(type_ice_model) and
 * reads its settings from the global C%.  Here the grid and the settings are
 * given once to diva_create(), the ice fields are copied in and out through
 * diva_upload()/diva_download() (host arrays in Fortran order, shapes as in
 * diva_fields.h), and everything in between stays resident in GPU memory.
 *
 * All entry points return a diva_status_t; 0 is success.  No entry point
 * terminates the process (the reference calls crash() -> MPI_ABORT).
 */
#ifndef DIVA_H
#define DIVA_H

#include <stddef.h>
#include <stdint.h>
#include "diva_fields.h"

#ifdef __cplusplus
extern "C" {
#endif

#define DIVA_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
typedef enum {
  DIVA_OK = 0,
  DIVA_MAX_PICARD = 1,          /* viscosity iteration hit its cap (non-fatal, as in the reference) */
  DIVA_LINEAR_NOT_CONVERGED = 2,/* linear solve missed its tolerance within its iteration cap */
  DIVA_NAN_DETECTED = 3,        /* NaN/Inf in the solution (check_for_NaN_dp_* analogue) */
  DIVA_BAD_INPUT = 4,           /* invalid argument, size, option or calling mode */
  DIVA_CUDA_ERROR = 5,          /* a CUDA runtime call failed */
  DIVA_TIMEOUT = 6,             /* a bounded device-side loop ran out of iterations */
  DIVA_UNSUPPORTED = 7          /* option not implemented by this backend */
} diva_status_t;

/* ---- field identifiers (diva_fields.h) --------------------------------- */
typedef enum {
#define DIVA_X_ENUM(ID, name, grid, type) DIVA_F_##ID,
  DIVA_FIELD_LIST(DIVA_X_ENUM)
#undef DIVA_X_ENUM
  DIVA_NUM_FIELDS
} diva_field_id_t;

typedef enum { DIVA_GRID_A = 0, DIVA_GRID_CX, DIVA_GRID_CY, DIVA_GRID_B,
               DIVA_GRID_A3, DIVA_GRID_CX3, DIVA_GRID_CY3, DIVA_GRID_B3 } diva_grid_kind_t;
typedef enum { DIVA_DTYPE_D = 0, DIVA_DTYPE_I = 1 } diva_dtype_t;

typedef struct {
  const char* name;   /* reference component name, e.g. "u_vav_cx" */
  int grid;           /* diva_grid_kind_t */
  int dtype;          /* diva_dtype_t */
} diva_field_info_t;

/* ---- option enums (string options of the reference's C%) ---------------- */
typedef enum { DIVA_DYN_SIA = 0, DIVA_DYN_SSA = 1, DIVA_DYN_SIA_SSA = 2, DIVA_DYN_DIVA = 3 } diva_dynamics_t;
typedef enum { DIVA_MARGIN_INFINITE_SLAB = 0, DIVA_MARGIN_BC = 1 } diva_margin_t;
typedef enum { DIVA_BC_INFINITE = 0, DIVA_BC_ZERO = 1, DIVA_BC_PERIODIC = 2 } diva_bc_t;
typedef enum { DIVA_SLIDING_NONE = 0, DIVA_SLIDING_WEERTMAN = 1, DIVA_SLIDING_COULOMB = 2,
               DIVA_SLIDING_COULOMB_REGULARISED = 3, DIVA_SLIDING_TSAI2015 = 4,
               DIVA_SLIDING_SCHOOF2005 = 5, DIVA_SLIDING_ZOET_IVERSON = 6 } diva_sliding_t;
typedef enum { DIVA_HYDRO_DRY = 0, DIVA_HYDRO_SATURATED = 1, DIVA_HYDRO_MARTIN2011 = 2 } diva_hydro_t;
typedef enum { DIVA_RHEO_UNIFORM = 0, DIVA_RHEO_HUYBRECHTS1992 = 1 } diva_rheology_t;
/* Picard stop test: the reference's step norm resid_UV (ice_velocity_module.f90:1530-1601),
 * or the FP64 nonlinear residual ||b(u) - A(u) u|| / ||b(u)||. */
typedef enum { DIVA_STOP_RESID_UV = 0, DIVA_STOP_RELRES = 1 } diva_stop_t;
/* Arithmetic of the linear solves: plain FP64, or MIXED: the finest multigrid level's
 * smoother (tile kernels) runs in FP32 on FP32 copies of the coefficients, inside the
 * FP64 BiCGStab whose residuals, and the nonlinear residual and Picard norms, stay FP64.
 * MIXED needs the tiled smoother (no periodic side) and a grid of at least 9 points in one
 * direction; otherwise the solve returns DIVA_UNSUPPORTED. */
typedef enum { DIVA_PREC_FP64 = 0, DIVA_PREC_MIXED = 1 } diva_precision_t;
typedef enum { DIVA_INTEGRATION_EXPLICIT = 0, DIVA_INTEGRATION_SEMIIMPLICIT = 1,
               DIVA_INTEGRATION_NONE = 2 } diva_integration_t;
typedef enum { DIVA_HEATCAP_UNIFORM = 0, DIVA_HEATCAP_POUNDER1965 = 1 } diva_heatcap_t;
/* Calving law of update_ice_thickness (calving_module.f90:30-91). */
typedef enum { DIVA_CALVING_NONE = 0, DIVA_CALVING_THRESHOLD_THICKNESS = 1 } diva_calving_t;
typedef enum { DIVA_CONDUCT_UNIFORM = 0, DIVA_CONDUCT_RITZ1987 = 1 } diva_conductivity_t;
/* Ice thickness at the domain boundary (apply_ice_thickness_BC, ice_thickness_module.f90:728-931). */
typedef enum { DIVA_HBC_ZERO = 0, DIVA_HBC_INFINITE = 1, DIVA_HBC_PERIODIC = 2, DIVA_HBC_FIXED = 3,
               DIVA_HBC_NONE = 4 } diva_hbc_t;

/* ---- grid (TYPE(type_grid), data_types_module.f90:13-29) --------------- */
typedef struct {
  int32_t nx, ny, nz;     /* a-grid size; number of scaled-zeta layers */
  double dx;              /* square cells, dx = dy [m] */
  double xmin, ymin;      /* x(1), y(1) [m] (informational) */
  double zeta[64];        /* C%zeta(1:nz), 0 at the surface, 1 at the base */
} diva_grid_t;

/* ---- configuration (the C% fields the path reads) ----------------------- */
typedef struct {
  int32_t choice_ice_dynamics;          /* diva_dynamics_t        configuration_module.f90:271 */
  double  n_flow;                       /* Glen exponent                                   :272 */
  double  m_enh_sheet, m_enh_shelf;     /* enhancement factors                         :273-274 */
  int32_t choice_ice_margin;            /* diva_margin_t                                   :275 */
  int32_t include_SSADIVA_crossterms;   /*                                                 :276 */
  int32_t do_GL_subgrid_friction;       /*                                                 :277 */
  double  DIVA_visc_it_norm_dUV_tol;    /*                                                 :282 */
  int32_t DIVA_visc_it_nit;             /*                                                 :283 */
  double  DIVA_visc_it_relax;           /*                                                 :284 */
  double  DIVA_epsilon_sq_0;            /*                                                 :285 */
  double  DIVA_visc_eff_min;            /*                                                 :286 */
  double  DIVA_beta_max;                /*                                                 :287 */
  double  DIVA_vel_max;                 /*                                                 :288 */
  int32_t BC_u_west, BC_u_east, BC_u_south, BC_u_north;   /* diva_bc_t               :289-292 */
  int32_t BC_v_west, BC_v_east, BC_v_south, BC_v_north;   /* diva_bc_t               :293-296 */
  int32_t choice_sliding_law;           /* diva_sliding_t                                  :349 */
  double  slid_delta_v;                 /*                                                 :351 */
  double  slid_Weertman_m;              /*                                                 :352 */
  double  slid_Coulomb_reg_q_plastic;   /*                                                 :353 */
  double  slid_Coulomb_reg_u_threshold; /*                                                 :354 */
  double  slid_ZI_ut, slid_ZI_p;        /*                                             :355-356 */
  int32_t include_basal_freezing;       /*                                                 :357 */
  double  deltaT_basal_freezing;        /*                                                 :358 */
  int32_t choice_basal_hydrology;       /* diva_hydro_t                                    :361 */
  double  Martin2011_hydro_Hb_min, Martin2011_hydro_Hb_max;  /*                       :362-363 */
  int32_t choice_ice_rheology;          /* diva_rheology_t                                 :424 */
  double  uniform_flow_factor;          /*                                                 :425 */
  int32_t do_ocean_floodfill;           /*                                                 :702 */
  /* Coulomb law with tauc_a given as input (choice_param_basal_roughness 'SSA_icestream',
   * basal_conditions_and_sliding_module.f90:1021-1023) instead of tan(phi_fric) * Neff */
  int32_t prescribed_tauc;
  /* linear solve: replaces DIVA_PETSc_rtol/abstol (:301-302) and DIVA_SOR_* (:298-300) */
  double  lin_rtol;                     /* relative residual target of every linear solve */
  int32_t lin_maxit;                    /* Krylov iteration cap per linear solve */
  /* Picard stop rule */
  int32_t picard_stop;                  /* diva_stop_t */
  double  picard_relres_tol;            /* used when picard_stop == DIVA_STOP_RELRES */
  int32_t lin_adaptive;                 /* RELRES mode: linear rtol tied to the current nonlinear residual */
  double  lin_adaptive_eta;             /* that rtol: max(lin_rtol, eta * min(1, rel-res)); default 0.5 */
  int32_t precision;                    /* diva_precision_t */
  /* ice thickness boundary conditions, diva_hbc_t (configuration_module.f90:325-328, default zero) */
  int32_t ice_thickness_west_BC, ice_thickness_east_BC, ice_thickness_south_BC, ice_thickness_north_BC;
  /* thermodynamics (configuration_module.f90:56, 424-430, 647); the ocean model is 'none':
   * the shelf base sits at T0 + T_ocean_mean_PD_ANT */
  double  dt_thermo;                           /* :56, default 10 yr */
  int32_t choice_ice_heat_capacity;            /* diva_heatcap_t, default Pounder1965 */
  double  uniform_ice_heat_capacity;           /* :428, 2009 */
  int32_t choice_ice_thermal_conductivity;     /* diva_conductivity_t, default Ritz1987 */
  double  uniform_ice_thermal_conductivity;    /* :430, 6.626958E7 */
  double  T_ocean_mean_PD_ANT;                 /* :647, -1.7 */
  /* ice-thickness integration (configuration_module.f90:308-314): diva_integration_t, and
   * for 'semi-implicit' the relative residual and iteration cap of its linear solve
   * (replacing dHi_SOR_* / dHi_PETSc_*) */
  int32_t choice_ice_integration_method;
  double  dHi_rtol;
  int32_t dHi_maxit;
  /* update_ice_thickness options (configuration_module.f90:335-337, 414), default off */
  int32_t fixed_shelf_geometry, fixed_sheet_geometry, fixed_grounding_line, do_remove_shelves;
  /* 1: the heat equation takes the ocean temperature at the shelf base (deg C, what
   * interpolate_ocean_depth gives an ocean model) from T_ocean_base_a; 0: ocean model
   * 'none', T_ocean_mean_PD_ANT everywhere */
  int32_t ocean_temperature_input;
  /* calving law (configuration_module.f90:412-413): diva_calving_t, default
   * 'threshold_thickness' with 200 m, as in the reference */
  int32_t choice_calving_law;
  double  calving_threshold_thickness;
  /* remove floating ice where the present-day geometry (Hi_PD_a, Hb_PD_a) has open
   * ocean; remove ice where the GIA-equilibrium geometry (Hi_GIAeq_a, Hb_GIAeq_a) has
   * no ice on a bed deeper than continental_shelf_min_height (configuration_module.f90:
   * 415-417; default off, -2000 m) */
  int32_t remove_shelves_larger_than_PD, continental_shelf_calving;
  double  continental_shelf_min_height;
  /* Nonlinear iteration (no reference counterpart): 0 = the reference's relaxed Picard
   * update u <- relax x + (1 - relax) u_prev (ice_velocity_module.f90:1499-1529); m in 1..5 =
   * Anderson mixing of depth m on the unrelaxed Picard map g(u) (the velocity-limited
   * linear solution): u <- g - sum_i gamma_i (g_i+1 - g_i), with gamma minimising
   * || f - sum_i gamma_i (f_i+1 - f_i) ||_2 over the last m residuals f = g(u) - u
   * (velocities on the cx and cy points); safeguards: columns are dropped while the
 * coefficients' magnitudes sum to more than 20, all but the newest when the nonlinear
 * residual grows tenfold, and mixing that has not lowered the nonlinear residual by 10 %
 * in 20 steps hands over to the relaxation for the rest of the solve (where the
 * velocity limit is active the mixed iteration wanders, the relaxed one settles).
 * Needs picard_stop = DIVA_STOP_RELRES: the
   * stop test is the nonlinear residual, so the converged state solves the same equations
   * as with the relaxed update; only the path there, and its length, change. */
  int32_t picard_anderson_m;
  /* Stop a rel-res iteration that has stopped making progress (no reference counterpart):
   * with picard_stop = DIVA_STOP_RELRES and picard_stall_its = K > 0, the loop ends with
   * DIVA_MAX_PICARD once the nonlinear residual has not fallen below 0.9 x its lowest value
   * so far for K viscosity iterations in a row.  This is the case where the velocity limit
   * DIVA_vel_max (apply_velocity_limits, ice_velocity_module.f90:1432-1498) is active: the
   * limited iteration settles on, or cycles around, states that do not solve the unlimited
   * equations.  0 (the default) keeps iterating to DIVA_visc_it_nit. */
  int32_t picard_stall_its;
  int32_t reserved[7];
} diva_config_t;

/* ---- per-solve report --------------------------------------------------- */
typedef struct {
  int32_t status;                 /* diva_status_t of the solve */
  int32_t picard_iterations;      /* viscosity iterations taken */
  int32_t linear_iterations;      /* Krylov iterations summed over the solve */
  int32_t mg_cycles;              /* multigrid V-cycles summed over the solve */
  double  resid_UV;               /* last step norm (ice_velocity_module.f90:1530-1601) */
  double  relres;                 /* last FP64 nonlinear relative residual (-1 if not evaluated) */
  double  fine_passes;            /* fine-grid-equivalent stencil passes (for byte counting) */
  double  elapsed_ms;             /* device time of the call (CUDA events); 0 for the CPU oracle */
  int32_t reserved[8];
} diva_report_t;

/* Host pointers for upload/download, indexed by diva_field_id_t; NULL = skip. */
typedef struct { void* ptr[DIVA_NUM_FIELDS]; } diva_fields_t;

typedef struct diva_ctx diva_ctx_t;

/* Defaults of configuration_module.f90:271-367, 424-426, 702 (with the velocity
 * options of the reference's default run: DIVA, infinite slab, cross terms). */
void diva_config_defaults(diva_config_t* cfg);
/* C%zeta default (configuration_module.f90:168-170) and nz = 15. */
void diva_grid_init(diva_grid_t* grid, int32_t nx, int32_t ny, double dx, double xmin, double ymin);

int  diva_field_info(int32_t id, diva_field_info_t* out);
/* Number of elements of a field on this grid (e.g. nz*ny*(nx-1) for CX3). */
int64_t diva_field_numel(const diva_grid_t* grid, int32_t id);

/* Allocate all device state for one grid; replaces allocate_ice_model
 * (ice_dynamics_module.f90:1034-1251) and initialise_SSADIVA_solution_matrix
 * (ice_velocity_module.f90:2814-2860).  All fields start at zero. */
int  diva_create(diva_ctx_t** ctx, const diva_grid_t* grid, const diva_config_t* cfg);
int  diva_destroy(diva_ctx_t* ctx);
int  diva_set_config(diva_ctx_t* ctx, const diva_config_t* cfg);
/* Bind a CUDA stream (cudaStream_t as void*; NULL = the library's own stream). */
int  diva_set_stream(diva_ctx_t* ctx, void* stream);

int  diva_upload(diva_ctx_t* ctx, const diva_fields_t* host);
int  diva_download(diva_ctx_t* ctx, const diva_fields_t* host);
int  diva_upload_field(diva_ctx_t* ctx, int32_t id, const void* host);
int  diva_download_field(diva_ctx_t* ctx, int32_t id, void* host);

/* update_general_ice_model_data (general_ice_model_data_module.f90:30-86). */
int  diva_update_general_ice_model_data(diva_ctx_t* ctx);
/* calc_pressure_melting_point (thermodynamics_module.f90:609-640). */
int  diva_calc_pressure_melting_point(diva_ctx_t* ctx);
/* calc_ice_rheology (thermodynamics_module.f90:641-753). */
int  diva_calc_ice_rheology(diva_ctx_t* ctx);

/* solve_SIA (ice_velocity_module.f90:36-114); needs choice_ice_dynamics SIA or SIA/SSA. */
int  diva_solve_sia(diva_ctx_t* ctx, diva_report_t* rep);
/* solve_SSA (ice_velocity_module.f90:115-248); needs SSA or SIA/SSA. */
int  diva_solve_ssa(diva_ctx_t* ctx, diva_report_t* rep);
/* solve_DIVA (ice_velocity_module.f90:249-374); needs DIVA. */
int  diva_solve_diva(diva_ctx_t* ctx, diva_report_t* rep);
/* solve_DIVA for n contexts at once (an ensemble; no single routine of the reference:
 * its members would be separate solve_DIVA calls).  Each context runs its
 * graph-launched viscosity loop on its own stream, all members in flight at once,
 * so the iterations of different members overlap on the GPU.  reports[k] is the report
 * of ctxs[k] (its status included); returns DIVA_OK if every member is OK, else the
 * first other status.  Contexts must be distinct. */
int  diva_solve_diva_batch(diva_ctx_t** ctxs, int32_t n, diva_report_t* reports);
/* A persistent batch: the viscosity loops of n contexts (an ensemble's members) captured
 * side by side in ONE CUDA graph, instantiated once by diva_batch_create and replayed by
 * every diva_batch_solve_diva, which is solve_DIVA for all members with a single graph
 * launch for all their viscosity iterations (each member's loop still ends on its own test;
 * the launch ends when the last member's has).  The members' preludes and tails (driving
 * stress, basal conditions, grounded fractions before; 3D and secondary velocities after)
 * run on the members' own streams around it.  reports[k] is member k's report; returns
 * DIVA_OK if every member is OK, else the first other status.  The members must stay
 * alive and unconfigured for the batch's lifetime (a diva_set_config on a member makes
 * the next solve return DIVA_BAD_INPUT); a member with no sheet ice gets zero velocities,
 * as from solve_DIVA, after its captured loop has run regardless.  No single routine of
 * the reference: its members would be separate solve_DIVA calls. */
typedef struct diva_batch diva_batch_t;
int  diva_batch_create(diva_ctx_t** ctxs, int32_t n, diva_batch_t** batch);
int  diva_batch_solve_diva(diva_batch_t* batch, diva_report_t* reports);
int  diva_batch_destroy(diva_batch_t* batch);
/* The SIA 3D velocity loop of solve_SIA (ice_velocity_module.f90:60-105) alone,
 * in any dynamics mode (used for "DIVA plus SIA" diagnostics). */
int  diva_calc_sia_3d_velocities(diva_ctx_t* ctx);

/* ---- ice-thickness update and the predictor/corrector step ------------------
 * The consumers of u_vav_cx / v_vav_cy inside a time step (run_ice_dynamics_pc,
 * ice_dynamics_module.f90:243-432), on the device; the time-step control itself
 * (dt_crit, pc_zeta, pc_eta, the event clock) is host logic around these calls. */
/* determine_floating_margin_fraction (general_ice_model_data_module.f90:784-865):
 * float_margin_frac_a and Hi_eff_cf_a of rows 2..ny-1 from Hi_a and the masks. */
int  diva_determine_floating_margin_fraction(diva_ctx_t* ctx);
/* calc_dHi_dt (ice_thickness_module.f90:26-63) with choice_ice_integration_method
 * 'explicit' (:65-300: upwind fluxes Qx_cx/Qy_cy of u_vav, mass balance SMB_a + BMB_a with
 * the floating fraction at calving fronts and none on open ocean, outfluxes rescaled so
 * no cell goes negative, dHi_dt_a and Hi_tplusdt_a = Hi_a + dt dHi_dt_a), 'semi-implicit'
 * (:302-727: per cell a mass-balance-only, explicit or over-implicit upwind row, fs = 2.5,
 * solved to dHi_rtol by BiCGStab with a Jacobi preconditioner) or 'none' (dHi_dt_a = 0),
 * then apply_ice_thickness_BC (:728-931; west, east, south, north in that order). */
int  diva_calc_dHi_dt(diva_ctx_t* ctx, double dt);
/* calc_critical_timestep_adv (ice_dynamics_module.f90:726-762):
 * min(dt_max, 0.9 min over interior a-points of dx / (|u_vav_cx| + |v_vav_cy|)). */
int  diva_calc_critical_timestep_adv(diva_ctx_t* ctx, double dt_max, double* dt_crit_adv);
/* calc_critical_timestep_SIA (ice_dynamics_module.f90:651-725), for the direct time
 * stepping of SIA and SIA/SSA dynamics: 0.9 x min(dt_max, dx^2 / (6 D_SIA) over sheet
 * faces with D_SIA = max(1e-9, |vertical average of u_3D_SIA x Hi / dHs_dx| on the
 * face), dx / (|u_3D| + |v_3D|) of every layer and cell) -- reads u_3D_SIA_cx,
 * v_3D_SIA_cy (solve_SIA) and u_3D_cx, v_3D_cy. */
int  diva_calc_critical_timestep_sia(diva_ctx_t* ctx, double dt_max, double* dt_crit_sia);
/* The predictor of run_ice_dynamics_pc (:360-377): dHidt_Hnm1_unm1 = dHidt_Hn_un;
 * calc_dHi_dt(dt); dHidt_Hn_un = dHi_dt_a; Hi_pred = max(0, Hi + dt ((1 + zeta/2)
 * dHidt_Hn_un - zeta/2 dHidt_Hnm1_unm1)); Hi_old = Hi; Hi = Hi_pred;
 * update_general_ice_model_data.  The velocity solve follows (the caller's). */
int  diva_pc_predictor(diva_ctx_t* ctx, double dt, double zeta);
/* The corrector (:408-421) and calc_pc_truncation_error (:763-816): calc_dHi_dt(dt);
 * dHidt_Hstarnp1_unp1 = dHi_dt_a; Hi = Hi_old; update_general_ice_model_data;
 * Hi_corr = max(0, Hi_old + dt/2 (dHidt_Hn_un + dHidt_Hstarnp1_unp1));
 * dHi_dt_a = (Hi_corr - Hi) / dt; pc_tau and *eta = max(eta_min, pc_tau over interior
 * sheet cells with no grounding line in their 3 x 3 neighbourhood). */
int  diva_pc_corrector(diva_ctx_t* ctx, double dt, double zeta, double eta_min, double* eta);
/* Hi_tplusdt_a = max(0, Hi_a + dt dHi_dt_a) (:429-431), then update_ice_thickness
 * (:435-648): mask_ice_a_prev = mask_ice_a; [fixed_shelf_geometry, fixed_sheet_geometry,
 * fixed_grounding_line keep Hi_tplusdt_a = Hi_a on shelf / sheet / grounding-line
 * cells]; Hi_a = max(0, Hi_tplusdt_a); masks; determine_floating_margin_fraction;
 * [choice_calving_law 'threshold_thickness' (the default): twice, Hi_a = 0 on
 * calving-front cells with Hi_eff_cf_a < calving_threshold_thickness, then masks (and
 * the floating margin fraction after the first pass) (:562-583, calving_module.f90:
 * 62-91)]; remove_unconnected_shelves (ice_thickness_module.f90:
 * 932-1044: shelf cells not 4-connected through shelf to a shelf cell next to sheet ice
 * lose their ice); Hi_a = 0 where mask_noice_a (region%mask_noice); [do_remove_shelves:
 * Hi_a = 0 on floating cells]; [remove_shelves_larger_than_PD: Hi_a = 0 where Hi_PD_a = 0
 * and Hb_PD_a < 0]; [continental_shelf_calving: Hi_a = 0 where Hi_GIAeq_a = 0 and
 * Hb_GIAeq_a < continental_shelf_min_height] (:600-635); and
 * update_general_ice_model_data. */
int  diva_pc_finish(diva_ctx_t* ctx, double dt);

/* apply_prescribed_retreat_mask (calving_module.f90:96-169), the last removal step of
 * update_ice_thickness when do_apply_prescribed_retreat_mask is set; call it after
 * diva_pc_finish.  The caller reads the mask's time frames (NetCDF in the reference)
 * and uploads them as ice_fraction_retreat_mask0_a / _mask1_a with the reference
 * thickness retreat_mask_Hi_ref_a; t0 < t1 are the frames' times.  On the device:
 * ice_fraction_retreat_mask_a = wt0 mask0 + (1 - wt0) mask1 with wt0 = clamp((t1 -
 * time) / (t1 - t0), 0, 1); Hi_a = min(Hi_a, Hi_ref * mask) where the mask is below
 * 0.999, and also at interior cells whose mask is not but a neighbour's is (3 x 3);
 * then update_general_ice_model_data. */
int  diva_apply_prescribed_retreat_mask(diva_ctx_t* ctx, double time, double t0, double t1);

/* run_thermo_model with choice_thermo_model '3D_heat_equation' (thermodynamics_module.f90:
 * 29-121): temperature of newly ice-covered columns from their upwind neighbour,
 * frictional heating, heat capacity, conductivity, pressure melting point, then (when
 * do_solve_heat_equation) solve_3D_heat_equation (:124-381: one implicit column solve
 * per interior column over C%dt_thermo, unstable columns replaced by the Robin
 * solution, :384-481), then calc_ice_rheology.  *n_unstable receives the number of
 * unstable columns; more than 1 % of the grid returns DIVA_NAN_DETECTED (the reference
 * crashes).  The column systems are solved by Gaussian elimination with partial
 * pivoting in the order of LAPACK's dgtsv, which the reference calls. */
int  diva_run_thermo_model(diva_ctx_t* ctx, int32_t do_solve_heat_equation, int32_t* n_unstable);

/* FP64 nonlinear residual of the current (u_vav_cx, v_vav_cy): evaluates the
 * coefficients of the next viscosity iteration (A3-A7) and returns
 * ||b - A u||_2 / ||b||_2 over the interior rows.  Leaves the state unchanged
 * except for the coefficient fields. */
int  diva_nonlinear_residual(diva_ctx_t* ctx, double* relres);

/* Complete the state the DIVA viscosity iteration carries from given velocities:
 * `sweeps` passes of the column-local stages of one viscosity iteration -- vertical
 * shear strain rates, effective viscosity, beta, F2, beta_eff (A3-A7,
 * ice_velocity_module.f90:664-1086) -- and the basal stress and velocities
 * (:1087-1199), with u_vav_cx / v_vav_cy held fixed and no linear solve.  The
 * first of those stages reads the previous viscosity and basal stress
 * (calc_vertical_shear_strain_rates, :664-721), so a context given only velocities
 * (a restart without viscosity, an observation, a predicted guess) starts
 * diva_solve_diva as far from its fixed point as a cold start; completing the state
 * first lets it start from the velocities' own.  No reference counterpart.
 * 0 <= sweeps <= 10000. */
int  diva_complete_state(diva_ctx_t* ctx, int32_t sweeps);

/* Tile shapes of the multigrid smoother.  The levels above the one-block sub-cycle
 * are smoothed by tiled kernels of edge 16 or 32; by default a level takes 32 while
 * its 32 x 32 tiles still fill the GPU, and tiles 1.5x as wide along i (32 x 48,
 * 16 x 24) where the square ones give just over one block per SM and the wide ones
 * fit in one.  diva_get_tile_edges writes each level's edge along j (0 for levels not
 * smoothed by tiles) into edges[0..n) and the level count into *nlev;
 * diva_set_tile_edges fixes the edge of levels 0..n-1 (16 or 32: square tiles; 0 for
 * the default) until the next call, e.g. from an autotuner that times candidates
 * with diva_profile_kernel.  The solution does not depend on the shape, only the
 * time per V-cycle. */
int  diva_get_tile_edges(diva_ctx_t* ctx, int32_t* edges, int32_t n, int32_t* nlev);
int  diva_set_tile_edges(diva_ctx_t* ctx, const int32_t* edges, int32_t n);

/* Snapshot / restore of the Picard state that persists across calls
 * (velocities, visc_eff_3D_a, taub, u_3D_a, v_3D_a, u_3D_cx, v_3D_cy ...):
 * a device-side checkpoint, replacing a cold restart from u = 0. */
int  diva_state_save(diva_ctx_t* ctx);
int  diva_state_restore(diva_ctx_t* ctx);

/* Time one hot kernel of the current state in isolation: `which` selects
 *   0  the column coefficients of one viscosity iteration: column prep, layer viscosity and
 *      column integrals (viscosity, F2, beta, beta_eff) + the b-grid face kernel
 *   1  one full Gauss-Seidel sweep (4 colours) of the fine-level operator
 *   2  one fine-level operator application (matrix-free A x with dot products)
 *   3  one multigrid V-cycle (the preconditioner of one Krylov half-step)
 *   4  the one-block coarse-level part of a V-cycle alone
 *   5  the column launches of 0 without the b-grid face kernel
 * `reps` launches are bracketed by CUDA events on the context's stream;
 * returns the mean device time per launch and the algorithmic bytes one launch
 * must move.  Needs a context that has completed a solve; kind 0 leaves the
 * coefficient fields of the next viscosity iteration behind (5 too), kinds 1-4 touch
 * only solver scratch vectors. */
int  diva_profile_kernel(diva_ctx_t* ctx, int32_t which, int32_t reps, double* ms_per_launch,
                         double* bytes_per_launch);

/* Allocation-free step norm of one viscosity iteration.
 * No counterpart in the reference: it exists for callers that cannot let a
 * library allocate GPU memory -- a host model that budgets all device memory
 * through its own pool, or code that must not trigger cudaMalloc while other
 * work shares the device.  It computes resid_UV exactly as the reference's
 * calc_visc_iter_UV_resid does (2 ||u - u_prev|| / max(||u + u_prev||, 1e-8)
 * over cx and cy points with |u| above 1e-6 m/yr, 0 if there are none) from
 * device arrays the caller owns, and writes it to resid_uv (one double in
 * device memory).  Layout: u arrays (j,i) at i*ld_cx + j for i < nx-1,
 * j < ny (ld_cx >= ny); v arrays (j,i) at i*ld_cy + j for j < ny-1 (ld_cy >=
 * ny-1); Fortran arrays u_vav_cx(ny,nx-1) and v_vav_cy(ny-1,nx) copied to the
 * device as they are fit with ld_cx = ny, ld_cy = ny-1.  Runs on `stream`
 * (cudaStream_t; NULL = legacy default stream) and does not synchronise.
 * It allocates nothing: its scratch is a static 384 KiB device array that
 * every GPU loading the library holds until exit, enough for grids of at most
 * 16384 thread blocks of 32 x 8 columns, i.e. ceil(ny/32) * ceil(nx/8) <=
 * 16384 (2048 x 2048 fits); larger grids return DIVA_BAD_INPUT.  The first
 * call on a device (more exactly: in each CUDA context, so again after a
 * cudaDeviceReset) looks up the scratch array's device address with that
 * device current and caches it, so make that first call before any stream
 * capture.  All calls share the scratch array: calls that overlap on the GPU
 * race, so serialise them. */
int  diva_visc_iter_uv_resid_noalloc(int32_t nx, int32_t ny, const double* u_cx, const double* u_cx_prev,
                                     int32_t ld_cx, const double* v_cy, const double* v_cy_prev, int32_t ld_cy,
                                     double* resid_uv, void* stream);

/* Number of kernels this context has launched since diva_create. */
int64_t diva_kernel_launches(const diva_ctx_t* ctx);

const char* diva_last_error(const diva_ctx_t* ctx);
const char* diva_status_string(int32_t status);

#ifdef __cplusplus
}
#endif
#endif /* DIVA_H */
