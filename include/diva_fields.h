/*
 * diva_fields.h -- the ice-model field table of the velocity hot path.
 *
 * Every entry mirrors a component of IMAU-ICE's TYPE(type_ice_model)
 * (src/data_types_module.f90:56-325) that the velocity solvers in
 * src/ice_velocity_module.f90, or the routines that prepare their inputs
 * (src/general_ice_model_data_module.f90:30-988,
 *  src/thermodynamics_module.f90:609-753,
 *  src/basal_conditions_and_sliding_module.f90:31-240),
 * read or write.  Shapes follow src/ice_dynamics_module.f90:1034-1251.
 *
 * X(ID, name, grid, type)
 *   grid: A  (ny,nx)       CX (ny,nx-1)      CY (ny-1,nx)      B (ny-1,nx-1)
 *         A3 (nz,ny,nx)    CX3 (nz,ny,nx-1)  CY3 (nz,ny-1,nx)  B3 (nz,ny-1,nx-1)
 *   type: D = REAL(dp) (double), I = default INTEGER (int32)
 * Host arrays passed through the C ABI are in Fortran (column-major) order
 * with exactly these shapes, i.e. the memory of the reference's own arrays.
 */
#ifndef DIVA_FIELDS_H
#define DIVA_FIELDS_H

#define DIVA_FIELD_LIST(X)                                   \
  /* geometry and forcing (inputs) */                        \
  X(HI_A,                 Hi_a,                 A,   D)      \
  X(HB_A,                 Hb_a,                 A,   D)      \
  X(SL_A,                 SL_a,                 A,   D)      \
  X(DHB_DT_A,             dHb_dt_a,             A,   D)      \
  X(TI_A,                 Ti_a,                 A3,  D)      \
  X(BETA_SQ_A,            beta_sq_a,            A,   D)      \
  X(PHI_FRIC_A,           phi_fric_a,           A,   D)      \
  X(ALPHA_SQ_A,           alpha_sq_a,           A,   D)      \
  X(TAUC_A,               tauc_a,               A,   D)      \
  /* update_general_ice_model_data */                        \
  X(HS_A,                 Hs_a,                 A,   D)      \
  X(TAF_A,                TAF_a,                A,   D)      \
  X(MASK_LAND_A,          mask_land_a,          A,   I)      \
  X(MASK_OCEAN_A,         mask_ocean_a,         A,   I)      \
  X(MASK_ICE_A,           mask_ice_a,           A,   I)      \
  X(MASK_SHEET_A,         mask_sheet_a,         A,   I)      \
  X(MASK_SHELF_A,         mask_shelf_a,         A,   I)      \
  X(MASK_COAST_A,         mask_coast_a,         A,   I)      \
  X(MASK_MARGIN_A,        mask_margin_a,        A,   I)      \
  X(MASK_GL_A,            mask_gl_a,            A,   I)      \
  X(MASK_CF_A,            mask_cf_a,            A,   I)      \
  X(MASK_A,               mask_a,               A,   I)      \
  X(HI_CX,                Hi_cx,                CX,  D)      \
  X(HI_CY,                Hi_cy,                CY,  D)      \
  X(HI_B,                 Hi_b,                 B,   D)      \
  X(DHI_DX_A,             dHi_dx_a,             A,   D)      \
  X(DHI_DY_A,             dHi_dy_a,             A,   D)      \
  X(DHS_DX_A,             dHs_dx_a,             A,   D)      \
  X(DHS_DY_A,             dHs_dy_a,             A,   D)      \
  X(DHS_DX_CX,            dHs_dx_cx,            CX,  D)      \
  X(DHS_DY_CX,            dHs_dy_cx,            CX,  D)      \
  X(DHS_DX_CY,            dHs_dx_cy,            CY,  D)      \
  X(DHS_DY_CY,            dHs_dy_cy,            CY,  D)      \
  /* rheology */                                             \
  X(A_FLOW_3D_A,          A_flow_3D_a,          A3,  D)      \
  X(A_FLOW_3D_CX,         A_flow_3D_cx,         CX3, D)      \
  X(A_FLOW_3D_CY,         A_flow_3D_cy,         CY3, D)      \
  X(A_FLOW_VAV_A,         A_flow_vav_a,         A,   D)      \
  X(A_FLOW_VAV_CX,        A_flow_vav_cx,        CX,  D)      \
  X(A_FLOW_VAV_CY,        A_flow_vav_cy,        CY,  D)      \
  X(TI_PMP_A,             Ti_pmp_a,             A3,  D)      \
  /* basal conditions */                                     \
  X(PORE_WATER_PRESSURE_A, pore_water_pressure_a, A, D)      \
  X(OVERBURDEN_PRESSURE_A, overburden_pressure_a, A, D)      \
  X(NEFF_A,               Neff_a,               A,   D)      \
  /* velocity solver: driving stress, grounded fractions */  \
  X(TAUDX_CX,             taudx_cx,             CX,  D)      \
  X(TAUDY_CY,             taudy_cy,             CY,  D)      \
  X(F_GRND_A,             f_grnd_a,             A,   D)      \
  X(F_GRND_CX,            f_grnd_cx,            CX,  D)      \
  X(F_GRND_CY,            f_grnd_cy,            CY,  D)      \
  X(F_GRND_B,             f_grnd_b,             B,   D)      \
  /* velocity solver: viscosity, friction, F-integrals */    \
  X(DU_DZ_3D_CX,          du_dz_3D_cx,          CX3, D)      \
  X(DV_DZ_3D_CY,          dv_dz_3D_cy,          CY3, D)      \
  X(VISC_EFF_3D_A,        visc_eff_3D_a,        A3,  D)      \
  X(VISC_EFF_3D_B,        visc_eff_3D_b,        B3,  D)      \
  X(VISC_EFF_INT_A,       visc_eff_int_a,       A,   D)      \
  X(VISC_EFF_INT_B,       visc_eff_int_b,       B,   D)      \
  X(N_A,                  N_a,                  A,   D)      \
  X(N_B,                  N_b,                  B,   D)      \
  X(N_CX,                 N_cx,                 CX,  D)      \
  X(N_CY,                 N_cy,                 CY,  D)      \
  X(BETA_A,               beta_a,               A,   D)      \
  X(F2_A,                 F2_a,                 A,   D)      \
  X(BETA_EFF_A,           beta_eff_a,           A,   D)      \
  X(BETA_EFF_CX,          beta_eff_cx,          CX,  D)      \
  X(BETA_EFF_CY,          beta_eff_cy,          CY,  D)      \
  X(F1_3D_A,              F1_3D_a,              A3,  D)      \
  /* velocity solver: velocities and Picard state */         \
  X(U_VAV_CX,             u_vav_cx,             CX,  D)      \
  X(V_VAV_CY,             v_vav_cy,             CY,  D)      \
  X(U_SSA_CX,             u_SSA_cx,             CX,  D)      \
  X(V_SSA_CY,             v_SSA_cy,             CY,  D)      \
  X(U_CX_PREV,            u_cx_prev,            CX,  D)      \
  X(V_CY_PREV,            v_cy_prev,            CY,  D)      \
  X(DIVA_ERR_CX,          DIVA_err_cx,          CX,  D)      \
  X(DIVA_ERR_CY,          DIVA_err_cy,          CY,  D)      \
  X(TAUB_CX,              taub_cx,              CX,  D)      \
  X(TAUB_CY,              taub_cy,              CY,  D)      \
  X(U_BASE_CX,            u_base_cx,            CX,  D)      \
  X(V_BASE_CY,            v_base_cy,            CY,  D)      \
  X(U_SURF_CX,            u_surf_cx,            CX,  D)      \
  X(V_SURF_CY,            v_surf_cy,            CY,  D)      \
  X(U_3D_CX,              u_3D_cx,              CX3, D)      \
  X(V_3D_CY,              v_3D_cy,              CY3, D)      \
  X(U_3D_SIA_CX,          u_3D_SIA_cx,          CX3, D)      \
  X(V_3D_SIA_CY,          v_3D_SIA_cy,          CY3, D)      \
  X(W_3D_A,               w_3D_a,               A3,  D)      \
  X(U_3D_A,               u_3D_a,               A3,  D)      \
  X(V_3D_A,               v_3D_a,               A3,  D)      \
  X(U_VAV_A,              u_vav_a,              A,   D)      \
  X(V_VAV_A,              v_vav_a,              A,   D)      \
  X(U_SURF_A,             u_surf_a,             A,   D)      \
  X(V_SURF_A,             v_surf_a,             A,   D)      \
  X(U_BASE_A,             u_base_a,             A,   D)      \
  X(V_BASE_A,             v_base_a,             A,   D)      \
  X(UABS_VAV_A,           uabs_vav_a,           A,   D)      \
  X(UABS_SURF_A,          uabs_surf_a,          A,   D)      \
  X(UABS_BASE_A,          uabs_base_a,          A,   D)      \
  X(W_SURF_A,             w_surf_a,             A,   D)      \
  X(W_BASE_A,             w_base_a,             A,   D)      \
  X(R_SHEAR,              R_shear,              A,   D)      \
  /* SICOPOLIS-style solver masks (set_sico_masks) */        \
  X(DIVA_MASK_COMBI,      DIVA_mask_combi,      A,   I)      \
  X(DIVA_ISFRONT_INNER,   DIVA_isfront_inner,   A,   I)      \
  X(DIVA_ISFRONT_OUTER,   DIVA_isfront_outer,   A,   I)      \
  /* ice-thickness update and predictor/corrector step   */ \
  /* (ice_thickness_module.f90:26-300, 728-931;          */ \
  /*  ice_dynamics_module.f90:243-432, 726-816;          */ \
  /*  general_ice_model_data_module.f90:784-865);        */ \
  /* SMB_a is SMB%SMB_year and BMB_a is BMB%BMB          */ \
  /* (data_types_module.f90:732, 742), m/yr of ice       */ \
  X(SMB_A,                SMB_a,                A,   D)      \
  X(BMB_A,                BMB_a,                A,   D)      \
  X(FLOAT_MARGIN_FRAC_A,  float_margin_frac_a,  A,   D)      \
  X(HI_EFF_CF_A,          Hi_eff_cf_a,          A,   D)      \
  X(QX_CX,                Qx_cx,                CX,  D)      \
  X(QY_CY,                Qy_cy,                CY,  D)      \
  X(DHI_DT_A,             dHi_dt_a,             A,   D)      \
  X(HI_TPLUSDT_A,         Hi_tplusdt_a,         A,   D)      \
  X(HI_PRED,              Hi_pred,              A,   D)      \
  X(HI_CORR,              Hi_corr,              A,   D)      \
  X(HI_OLD,               Hi_old,               A,   D)      \
  X(DHIDT_HN_UN,          dHidt_Hn_un,          A,   D)      \
  X(DHIDT_HNM1_UNM1,      dHidt_Hnm1_unm1,      A,   D)      \
  X(DHIDT_HSTARNP1_UNP1,  dHidt_Hstarnp1_unp1,  A,   D)      \
  X(PC_TAU,               pc_tau,               A,   D)      \
  X(MASK_ICE_A_PREV,      mask_ice_a_prev,      A,   I)      \
  X(MASK_NOICE_A,         mask_noice_a,         A,   I)      \
  /* reference geometries read by update_ice_thickness's  */ \
  /* remove_shelves_larger_than_PD / continental_shelf_   */ \
  /* calving (refgeo_PD, refgeo_GIAeq: Hi and Hb)          */ \
  X(HI_PD_A,              Hi_PD_a,              A,   D)      \
  X(HB_PD_A,              Hb_PD_a,              A,   D)      \
  X(HI_GIAEQ_A,           Hi_GIAeq_a,           A,   D)      \
  X(HB_GIAEQ_A,           Hb_GIAeq_a,           A,   D)      \
  /* prescribed retreat mask (calving_module.f90:96-169): */ \
  /* the two time frames, the reference thickness, and   */ \
  /* the mask interpolated to the model time (output)    */ \
  X(RETREAT_MASK0_A,      ice_fraction_retreat_mask0_a, A, D)  \
  X(RETREAT_MASK1_A,      ice_fraction_retreat_mask1_a, A, D)  \
  X(RETREAT_MASK_HI_REF_A, retreat_mask_Hi_ref_a,       A, D)  \
  X(RETREAT_MASK_A,       ice_fraction_retreat_mask_a,  A, D)  \
  /* thermodynamics (thermodynamics_module.f90:29-608,   */ \
  /*  derivatives_and_grids_module.f90:1892-2061);       */ \
  /* T_surf_annual_a is SUM(climate%T2m)/12 and GHF_a    */ \
  /* ice%GHF_a (J m-2 yr-1)                              */ \
  X(T_SURF_ANNUAL_A,      T_surf_annual_a,      A,   D)      \
  X(GHF_A,                GHF_a,                A,   D)      \
  X(T_OCEAN_BASE_A,       T_ocean_base_a,       A,   D)      \
  X(FRICTIONAL_HEATING_A, frictional_heating_a, A,   D)      \
  X(CPI_A,                Cpi_a,                A3,  D)      \
  X(KI_A,                 Ki_a,                 A3,  D)      \
  X(DHS_DT_A,             dHs_dt_a,             A,   D)      \
  X(DZETA_DT_A,           dzeta_dt_a,           A3,  D)      \
  X(DZETA_DX_A,           dzeta_dx_a,           A3,  D)      \
  X(DZETA_DY_A,           dzeta_dy_a,           A3,  D)      \
  X(DZETA_DZ_A,           dzeta_dz_a,           A,   D)

#endif /* DIVA_FIELDS_H */
