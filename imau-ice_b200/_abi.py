"""ctypes mirror of include/diva.h.

The structs below have the same member order and types as the C definitions,
so ctypes lays them out identically.  They are shared by the CUDA library
(``libdiva_b200.so``, symbols ``diva_*``) and by the CPU oracle used in tests
(``liboracle.so``, symbols ``orc_*``), which implement the same entry points.
"""
import ctypes as C

MAX_NZ = 64

# status codes (diva_status_t)
OK, MAX_PICARD, LINEAR_NOT_CONVERGED, NAN_DETECTED, BAD_INPUT, CUDA_ERROR, TIMEOUT, UNSUPPORTED = range(8)
STATUS_NAMES = {0: "OK", 1: "MAX_PICARD", 2: "LINEAR_NOT_CONVERGED", 3: "NAN_DETECTED",
                4: "BAD_INPUT", 5: "CUDA_ERROR", 6: "TIMEOUT", 7: "UNSUPPORTED"}

# option enums (string options of the reference's C%)
DYN = {"SIA": 0, "SSA": 1, "SIA/SSA": 2, "DIVA": 3}
MARGIN = {"infinite_slab": 0, "BC": 1}
BC = {"infinite": 0, "zero": 1, "periodic": 2}
SLIDING = {"no_sliding": 0, "Weertman": 1, "Coulomb": 2, "Coulomb_regularised": 3,
           "Tsai2015": 4, "Schoof2005": 5, "Zoet-Iverson": 6}
HYDRO = {"dry": 0, "saturated": 1, "Martin2011": 2}
RHEO = {"uniform": 0, "Huybrechts1992": 1}
STOP = {"resid_UV": 0, "relres": 1}
PREC = {"fp64": 0, "mixed": 1}
HBC = {"zero": 0, "infinite": 1, "periodic": 2, "fixed": 3, "none": 4}
HEATCAP = {"uniform": 0, "Pounder1965": 1}
CONDUCT = {"uniform": 0, "Ritz1987": 1}
INTEGRATION = {"explicit": 0, "semi-implicit": 1, "none": 2}
CALVING = {"none": 0, "threshold_thickness": 1}

GRID_KINDS = ["A", "CX", "CY", "B", "A3", "CX3", "CY3", "B3"]


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("dx", C.c_double), ("xmin", C.c_double), ("ymin", C.c_double),
                ("zeta", C.c_double * MAX_NZ)]


class Config(C.Structure):
    _fields_ = [
        ("choice_ice_dynamics", C.c_int32),
        ("n_flow", C.c_double),
        ("m_enh_sheet", C.c_double), ("m_enh_shelf", C.c_double),
        ("choice_ice_margin", C.c_int32),
        ("include_SSADIVA_crossterms", C.c_int32),
        ("do_GL_subgrid_friction", C.c_int32),
        ("DIVA_visc_it_norm_dUV_tol", C.c_double),
        ("DIVA_visc_it_nit", C.c_int32),
        ("DIVA_visc_it_relax", C.c_double),
        ("DIVA_epsilon_sq_0", C.c_double),
        ("DIVA_visc_eff_min", C.c_double),
        ("DIVA_beta_max", C.c_double),
        ("DIVA_vel_max", C.c_double),
        ("BC_u_west", C.c_int32), ("BC_u_east", C.c_int32), ("BC_u_south", C.c_int32), ("BC_u_north", C.c_int32),
        ("BC_v_west", C.c_int32), ("BC_v_east", C.c_int32), ("BC_v_south", C.c_int32), ("BC_v_north", C.c_int32),
        ("choice_sliding_law", C.c_int32),
        ("slid_delta_v", C.c_double),
        ("slid_Weertman_m", C.c_double),
        ("slid_Coulomb_reg_q_plastic", C.c_double),
        ("slid_Coulomb_reg_u_threshold", C.c_double),
        ("slid_ZI_ut", C.c_double), ("slid_ZI_p", C.c_double),
        ("include_basal_freezing", C.c_int32),
        ("deltaT_basal_freezing", C.c_double),
        ("choice_basal_hydrology", C.c_int32),
        ("Martin2011_hydro_Hb_min", C.c_double), ("Martin2011_hydro_Hb_max", C.c_double),
        ("choice_ice_rheology", C.c_int32),
        ("uniform_flow_factor", C.c_double),
        ("do_ocean_floodfill", C.c_int32),
        ("prescribed_tauc", C.c_int32),
        ("lin_rtol", C.c_double),
        ("lin_maxit", C.c_int32),
        ("picard_stop", C.c_int32),
        ("picard_relres_tol", C.c_double),
        ("lin_adaptive", C.c_int32),
        ("lin_adaptive_eta", C.c_double),
        ("precision", C.c_int32),
        ("ice_thickness_west_BC", C.c_int32), ("ice_thickness_east_BC", C.c_int32),
        ("ice_thickness_south_BC", C.c_int32), ("ice_thickness_north_BC", C.c_int32),
        ("dt_thermo", C.c_double),
        ("choice_ice_heat_capacity", C.c_int32),
        ("uniform_ice_heat_capacity", C.c_double),
        ("choice_ice_thermal_conductivity", C.c_int32),
        ("uniform_ice_thermal_conductivity", C.c_double),
        ("T_ocean_mean_PD_ANT", C.c_double),
        ("choice_ice_integration_method", C.c_int32),
        ("dHi_rtol", C.c_double),
        ("dHi_maxit", C.c_int32),
        ("fixed_shelf_geometry", C.c_int32), ("fixed_sheet_geometry", C.c_int32),
        ("fixed_grounding_line", C.c_int32), ("do_remove_shelves", C.c_int32),
        ("ocean_temperature_input", C.c_int32),
        ("choice_calving_law", C.c_int32),
        ("calving_threshold_thickness", C.c_double),
        ("remove_shelves_larger_than_PD", C.c_int32), ("continental_shelf_calving", C.c_int32),
        ("continental_shelf_min_height", C.c_double),
        ("picard_anderson_m", C.c_int32),
        ("picard_stall_its", C.c_int32),
        ("reserved", C.c_int32 * 7),
    ]


class Report(C.Structure):
    _fields_ = [("status", C.c_int32), ("picard_iterations", C.c_int32),
                ("linear_iterations", C.c_int32), ("mg_cycles", C.c_int32),
                ("resid_UV", C.c_double), ("relres", C.c_double),
                ("fine_passes", C.c_double), ("elapsed_ms", C.c_double),
                ("reserved", C.c_int32 * 8)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}
        d["linear_not_converged"] = self.reserved[0]   # linear solves that missed their tolerance
        d["graph_launched"] = self.reserved[1]         # 1 if the iterations ran as CUDA graphs
        d["stalled"] = self.reserved[2]                # 1 if a rel-res loop stopped on picard_stall_its
        return d


class FieldInfo(C.Structure):
    _fields_ = [("name", C.c_char_p), ("grid", C.c_int32), ("dtype", C.c_int32)]


# Options given as strings (as in the reference's config files) map to enums.
ENUM_OPTIONS = {
    "choice_ice_dynamics": DYN, "choice_ice_margin": MARGIN,
    "BC_u_west": BC, "BC_u_east": BC, "BC_u_south": BC, "BC_u_north": BC,
    "BC_v_west": BC, "BC_v_east": BC, "BC_v_south": BC, "BC_v_north": BC,
    "choice_sliding_law": SLIDING, "choice_basal_hydrology": HYDRO,
    "choice_ice_rheology": RHEO, "picard_stop": STOP, "precision": PREC,
    "ice_thickness_west_BC": HBC, "ice_thickness_east_BC": HBC, "ice_thickness_south_BC": HBC,
    "ice_thickness_north_BC": HBC,
    "choice_ice_heat_capacity": HEATCAP, "choice_ice_thermal_conductivity": CONDUCT,
    "choice_ice_integration_method": INTEGRATION,
    "choice_calving_law": CALVING,
}


def bind(lib, prefix):
    """Declare argument and return types of the shared entry points of ``lib``."""
    vp, i32, dp = C.c_void_p, C.c_int32, C.POINTER(C.c_double)
    sig = {
        "config_defaults": (None, [C.POINTER(Config)]),
        "field_info": (C.c_int, [i32, C.POINTER(FieldInfo)]),
        "create": (C.c_int, [C.POINTER(vp), C.POINTER(Grid), C.POINTER(Config)]),
        "destroy": (C.c_int, [vp]),
        "set_config": (C.c_int, [vp, C.POINTER(Config)]),
        "upload_field": (C.c_int, [vp, i32, vp]),
        "download_field": (C.c_int, [vp, i32, vp]),
        "update_general_ice_model_data": (C.c_int, [vp]),
        "calc_pressure_melting_point": (C.c_int, [vp]),
        "calc_ice_rheology": (C.c_int, [vp]),
        "solve_sia": (C.c_int, [vp, C.POINTER(Report)]),
        "solve_ssa": (C.c_int, [vp, C.POINTER(Report)]),
        "solve_diva": (C.c_int, [vp, C.POINTER(Report)]),
        "calc_sia_3d_velocities": (C.c_int, [vp]),
        "nonlinear_residual": (C.c_int, [vp, dp]),
        "complete_state": (C.c_int, [vp, i32]),
        "state_save": (C.c_int, [vp]),
        "state_restore": (C.c_int, [vp]),
        "determine_floating_margin_fraction": (C.c_int, [vp]),
        "calc_dHi_dt": (C.c_int, [vp, C.c_double]),
        "calc_critical_timestep_adv": (C.c_int, [vp, C.c_double, dp]),
        "calc_critical_timestep_sia": (C.c_int, [vp, C.c_double, dp]),
        "pc_predictor": (C.c_int, [vp, C.c_double, C.c_double]),
        "pc_corrector": (C.c_int, [vp, C.c_double, C.c_double, C.c_double, dp]),
        "pc_finish": (C.c_int, [vp, C.c_double]),
        "apply_prescribed_retreat_mask": (C.c_int, [vp, C.c_double, C.c_double, C.c_double]),
        "run_thermo_model": (C.c_int, [vp, i32, C.POINTER(C.c_int32)]),
        "last_error": (C.c_char_p, [vp]),
    }
    fns = {}
    for name, (res, args) in sig.items():
        f = getattr(lib, prefix + name)
        f.restype = res
        f.argtypes = args
        fns[name] = f
    return fns
