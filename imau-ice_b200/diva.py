"""Host-side mirror of IMAU-ICE's velocity interface.

The reference exposes ``solve_SIA(grid, ice)``, ``solve_SSA(grid, ice)`` and
``solve_DIVA(grid, ice)`` (src/ice_velocity_module.f90:36, :115, :249), which
read TYPE(type_grid), update TYPE(type_ice_model) in place and take their
settings from the global ``C%``.  This module keeps that shape:

* ``Grid`` describes the square grid (nx, ny, dx, zeta);
* an ice model is a ``dict`` of NumPy arrays named after the reference's
  components (``ice["Hi_a"]``, ``ice["u_vav_cx"]``, ...), Fortran-ordered with
  the reference's shapes, e.g. ``(ny, nx-1)`` for a cx-grid field and
  ``(nz, ny, nx)`` for a 3D a-grid field, so ``ice["Hi_a"][j, i]`` is
  ``ice%Hi_a(j+1, i+1)``;
* ``solve_DIVA(grid, ice, config)`` etc. copy the inputs to the GPU, run the
  solve there and write the outputs back into ``ice``.

For repeated solves on one grid, ``Context`` keeps the whole state resident on
the GPU between calls (upload once, solve many times, download on request),
which is how a Fortran shim over the C ABI drives the library.

The product backend is ``libdiva_b200.so`` (CUDA, sm_100a).  There is no CPU
fallback: if the library or a GPU is missing, creating a context raises.
"""
import ctypes as C
import os
import numpy as np

from . import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libdiva_b200.so")

ZETA_DEFAULT = [0.00, 0.10, 0.20, 0.30, 0.40, 0.50, 0.60, 0.70, 0.80, 0.90,
                0.925, 0.95, 0.975, 0.99, 1.00]   # configuration_module.f90:168-170


class DivaError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class Backend:
    """A loaded implementation of the diva.h entry points (``prefix`` + name)."""

    def __init__(self, path, prefix, name):
        if not os.path.exists(path):
            raise DivaError(_abi.BAD_INPUT, f"library not built: {path}")
        self.lib = C.CDLL(path)
        self.fns = _abi.bind(self.lib, prefix)
        self.prefix = prefix
        self.name = name
        self.path = path
        self._fields = None

    def fields(self):
        if self._fields is None:
            out, info, i = [], _abi.FieldInfo(), 0
            while self.fns["field_info"](i, C.byref(info)) == 0:
                out.append((info.name.decode(), _abi.GRID_KINDS[info.grid], "f8" if info.dtype == 0 else "i4"))
                i += 1
            self._fields = out
        return self._fields

    def default_config(self):
        cfg = _abi.Config()
        self.fns["config_defaults"](C.byref(cfg))
        return cfg


_CUDA = None


def cuda_backend():
    """The product backend; loads ``lib/libdiva_b200.so`` once."""
    global _CUDA
    if _CUDA is None:
        _CUDA = Backend(LIB_PATH, "diva_", "cuda")
    return _CUDA


class Grid:
    """TYPE(type_grid) (data_types_module.f90:13-29): a regular square grid."""

    def __init__(self, nx, ny, dx, zeta=None, xmin=0.0, ymin=0.0):
        self.nx, self.ny, self.dx = int(nx), int(ny), float(dx)
        self.zeta = np.asarray(ZETA_DEFAULT if zeta is None else zeta, dtype=np.float64)
        self.nz = len(self.zeta)
        self.xmin, self.ymin = float(xmin), float(ymin)
        if self.nz > _abi.MAX_NZ or self.nz < 2:
            raise DivaError(_abi.BAD_INPUT, f"nz={self.nz} outside 2..{_abi.MAX_NZ}")

    @property
    def x(self):
        return self.xmin + self.dx * np.arange(self.nx)

    @property
    def y(self):
        return self.ymin + self.dx * np.arange(self.ny)

    def to_c(self):
        g = _abi.Grid()
        g.nx, g.ny, g.nz, g.dx, g.xmin, g.ymin = self.nx, self.ny, self.nz, self.dx, self.xmin, self.ymin
        for k, z in enumerate(self.zeta):
            g.zeta[k] = z
        return g

    def shape(self, kind):
        nx, ny, nz = self.nx, self.ny, self.nz
        return {"A": (ny, nx), "CX": (ny, nx - 1), "CY": (ny - 1, nx), "B": (ny - 1, nx - 1),
                "A3": (nz, ny, nx), "CX3": (nz, ny, nx - 1), "CY3": (nz, ny - 1, nx),
                "B3": (nz, ny - 1, nx - 1)}[kind]


def make_config(backend, overrides=None):
    """Reference defaults with ``overrides`` (strings for the string options)."""
    cfg = backend.default_config()
    for k, v in (overrides or {}).items():
        if k in _abi.ENUM_OPTIONS and isinstance(v, str):
            v = _abi.ENUM_OPTIONS[k][v]
        if not hasattr(cfg, k):
            raise DivaError(_abi.BAD_INPUT, f"unknown config option {k}")
        setattr(cfg, k, v)
    return cfg


class Context:
    """Device-resident state of one grid (allocate_ice_model + solution matrix)."""

    def __init__(self, grid, config=None, backend=None):
        self.backend = backend or cuda_backend()
        self.grid = grid
        self.fields = {name: (kind, dt) for name, kind, dt in self.backend.fields()}
        self.ids = {name: i for i, (name, _, _) in enumerate(self.backend.fields())}
        self.cfg = config if isinstance(config, _abi.Config) else make_config(self.backend, config)
        self._g = grid.to_c()
        h = C.c_void_p()
        st = self.backend.fns["create"](C.byref(h), C.byref(self._g), C.byref(self.cfg))
        if st != 0:
            raise DivaError(st, f"{self.backend.prefix}create failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.backend.fns["destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st not in (0, _abi.MAX_PICARD):
            err = self.backend.fns["last_error"](self.h)
            raise DivaError(st, f"{what}: {err.decode() if err else ''}")
        return st

    def set_config(self, overrides):
        self.cfg = make_config(self.backend, overrides) if not isinstance(overrides, _abi.Config) else overrides
        self._check(self.backend.fns["set_config"](self.h, C.byref(self.cfg)), "set_config")

    # ---- field I/O ---------------------------------------------------------
    def empty(self, name):
        kind, dt = self.fields[name]
        return np.zeros(self.grid.shape(kind), dtype=dt, order="F")

    def upload(self, ice):
        for name, arr in ice.items():
            if name not in self.fields:
                continue
            kind, dt = self.fields[name]
            a = np.asfortranarray(arr, dtype=dt)
            if a.shape != self.grid.shape(kind):
                raise DivaError(_abi.BAD_INPUT, f"{name}: shape {a.shape} != {self.grid.shape(kind)}")
            self._check(self.backend.fns["upload_field"](self.h, self.ids[name], a.ctypes.data), f"upload {name}")

    def download(self, names=None, out=None):
        """Fields as Fortran-ordered host arrays.  ``out`` may hold preallocated arrays
        (e.g. views of pinned memory) to fill instead of allocating new ones."""
        res = {}
        for name in (names or self.fields.keys()):
            a = None if out is None else out.get(name)
            if a is None:
                a = self.empty(name)
            else:
                kind, dt = self.fields[name]
                if a.dtype != dt or a.shape != self.grid.shape(kind) or not a.flags.f_contiguous:
                    raise DivaError(_abi.BAD_INPUT, f"{name}: output array must be Fortran-ordered {dt} "
                                                   f"{self.grid.shape(kind)}")
            self._check(self.backend.fns["download_field"](self.h, self.ids[name], a.ctypes.data), f"download {name}")
            res[name] = a
        return res

    # ---- restart files ----------------------------------------------------------
    def save_restart(self, path, names=None):
        """Write the grid, the configuration and the fields (all by default) to an .npz
        file: a restart of the whole device state, velocities and viscosity included
        (the reference's restart file, netcdf_module.f90:31-127, holds the geometry and
        temperature but not the velocity-solver state)."""
        import json
        arrays = self.download(names)
        cfg = {name: getattr(self.cfg, name) for name, _ in _abi.Config._fields_ if name != "reserved"}
        meta = {"_grid": np.array([self.grid.nx, self.grid.ny], dtype=np.int64),
                "_grid_f": np.array([self.grid.dx, self.grid.xmin, self.grid.ymin]),
                "_zeta": self.grid.zeta,
                "_config_json": np.array(json.dumps(cfg))}
        np.savez(path, **arrays, **meta)

    @classmethod
    def load_restart(cls, path, backend=None):
        """A new context with the grid, configuration and fields of a restart file."""
        z = np.load(path)
        nx, ny = (int(v) for v in z["_grid"])
        dx, xmin, ymin = (float(v) for v in z["_grid_f"])
        grid = Grid(nx, ny, dx, zeta=z["_zeta"], xmin=xmin, ymin=ymin)
        be = backend or cuda_backend()
        if "_config_json" in z.files:
            # by field name onto the library's defaults: files stay readable when
            # configuration fields are added
            import json
            cfg = be.default_config()
            for name, value in json.loads(str(z["_config_json"])).items():
                if hasattr(cfg, name):
                    setattr(cfg, name, value)
        else:
            raw = z["_config"].tobytes()
            if len(raw) != C.sizeof(_abi.Config):
                raise DivaError(_abi.BAD_INPUT, "restart file written with another configuration layout")
            cfg = _abi.Config.from_buffer_copy(raw)
        ctx = cls(grid, cfg, be)
        ctx.upload({k: np.asfortranarray(z[k]) for k in z.files if not k.startswith("_")})
        return ctx

    # ---- the reference's routines ---------------------------------------------
    def update_general_ice_model_data(self):
        self._check(self.backend.fns["update_general_ice_model_data"](self.h), "update_general_ice_model_data")

    def calc_pressure_melting_point(self):
        self._check(self.backend.fns["calc_pressure_melting_point"](self.h), "calc_pressure_melting_point")

    def calc_ice_rheology(self):
        self._check(self.backend.fns["calc_ice_rheology"](self.h), "calc_ice_rheology")

    def _solve(self, fn, what):
        rep = _abi.Report()
        self._check(self.backend.fns[fn](self.h, C.byref(rep)), what)
        return rep.as_dict()

    def solve_SIA(self):
        return self._solve("solve_sia", "solve_SIA")

    def solve_SSA(self):
        return self._solve("solve_ssa", "solve_SSA")

    def solve_DIVA(self):
        return self._solve("solve_diva", "solve_DIVA")

    def calc_sia_3d_velocities(self):
        self._check(self.backend.fns["calc_sia_3d_velocities"](self.h), "calc_sia_3d_velocities")

    def complete_state(self, sweeps=30):
        """diva_complete_state: the viscosity iteration's carried state (viscosity,
        beta_eff, basal stress) for the current u_vav_cx / v_vav_cy, by ``sweeps``
        column-local passes without a linear solve."""
        self._check(self.backend.fns["complete_state"](self.h, int(sweeps)), "complete_state")

    def nonlinear_residual(self):
        r = C.c_double()
        self._check(self.backend.fns["nonlinear_residual"](self.h, C.byref(r)), "nonlinear_residual")
        return r.value

    # ---- the ice-thickness update and the predictor/corrector stages ---------------
    def determine_floating_margin_fraction(self):
        """general_ice_model_data_module.f90:784-865."""
        self._check(self.backend.fns["determine_floating_margin_fraction"](self.h),
                    "determine_floating_margin_fraction")

    def calc_dHi_dt(self, dt):
        """ice_thickness_module.f90:26-300 ('explicit') with apply_ice_thickness_BC."""
        self._check(self.backend.fns["calc_dHi_dt"](self.h, float(dt)), "calc_dHi_dt")

    def calc_critical_timestep_SIA(self, dt_max):
        """calc_critical_timestep_SIA (ice_dynamics_module.f90:651-725)."""
        r = C.c_double()
        self._check(self.backend.fns["calc_critical_timestep_sia"](self.h, float(dt_max), C.byref(r)),
                    "calc_critical_timestep_sia")
        return r.value

    def calc_critical_timestep_adv(self, dt_max):
        """ice_dynamics_module.f90:726-762; returns dt_crit_adv."""
        r = C.c_double()
        self._check(self.backend.fns["calc_critical_timestep_adv"](self.h, float(dt_max), C.byref(r)),
                    "calc_critical_timestep_adv")
        return r.value

    def pc_predictor(self, dt, zeta):
        """The predictor stage of run_ice_dynamics_pc (ice_dynamics_module.f90:360-377)."""
        self._check(self.backend.fns["pc_predictor"](self.h, float(dt), float(zeta)), "pc_predictor")

    def pc_corrector(self, dt, zeta, eta_min):
        """The corrector stage and calc_pc_truncation_error (:404-421, :763-816); returns pc_eta."""
        r = C.c_double()
        self._check(self.backend.fns["pc_corrector"](self.h, float(dt), float(zeta), float(eta_min), C.byref(r)),
                    "pc_corrector")
        return r.value

    def pc_finish(self, dt):
        """Hi_tplusdt_a and the thickness update of the step (:429-431, :435-648 in part)."""
        self._check(self.backend.fns["pc_finish"](self.h, float(dt)), "pc_finish")

    def apply_prescribed_retreat_mask(self, time, t0, t1):
        """apply_prescribed_retreat_mask (calving_module.f90:96-169) at model ``time``
        between the uploaded frames at t0 and t1; call after pc_finish."""
        self._check(self.backend.fns["apply_prescribed_retreat_mask"](self.h, float(time), float(t0), float(t1)),
                    "apply_prescribed_retreat_mask")

    def run_thermo_model(self, do_solve_heat_equation=True):
        """run_thermo_model with the 3D heat equation (thermodynamics_module.f90:29-121);
        returns the number of unstable columns replaced by the Robin solution."""
        n = C.c_int32()
        self._check(self.backend.fns["run_thermo_model"](self.h, int(bool(do_solve_heat_equation)), C.byref(n)),
                    "run_thermo_model")
        return n.value

    def state_save(self):
        self._check(self.backend.fns["state_save"](self.h), "state_save")

    def state_restore(self):
        self._check(self.backend.fns["state_restore"](self.h), "state_restore")

    # ---- CUDA-library extras ---------------------------------------------------
    def set_stream(self, stream_handle):
        """Run all of this context's work on a caller's CUDA stream (cudaStream_t as int)."""
        f = self.backend.lib.diva_set_stream
        f.argtypes = [C.c_void_p, C.c_void_p]
        self._check(f(self.h, C.c_void_p(stream_handle)), "set_stream")

    def kernel_launches(self):
        """Kernels this context has launched since creation (diva_kernel_launches)."""
        f = self.backend.lib.diva_kernel_launches
        f.argtypes = [C.c_void_p]
        f.restype = C.c_int64
        return int(f(self.h))

    def get_tile_edges(self):
        """(edge of each multigrid level's tiled smoother, 0 where untiled; level count)."""
        f = self.backend.lib.diva_get_tile_edges
        f.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32)]
        e, n = (C.c_int32 * 12)(), C.c_int32()
        self._check(f(self.h, e, 12, C.byref(n)), "get_tile_edges")
        return [int(e[k]) for k in range(n.value)]

    def set_tile_edges(self, edges):
        """Fix the tile edge (16, 32, or 0 for the default) of levels 0..len(edges)-1."""
        f = self.backend.lib.diva_set_tile_edges
        f.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.c_int32]
        e = (C.c_int32 * max(1, len(edges)))(*[int(v) for v in edges])
        self._check(f(self.h, e, len(edges)), "set_tile_edges")

    def profile_kernel(self, which, reps=20):
        """(ms per launch, algorithmic bytes per launch) of one hot kernel (diva_profile_kernel)."""
        f = self.backend.lib.diva_profile_kernel
        f.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        ms, nb = C.c_double(), C.c_double()
        self._check(f(self.h, which, reps, C.byref(ms), C.byref(nb)), "profile_kernel")
        return ms.value, nb.value


# Fields each routine writes (downloaded back into the caller's dict).
OUT_UPDATE = ["Hs_a", "TAF_a", "mask_land_a", "mask_ocean_a", "mask_ice_a", "mask_sheet_a", "mask_shelf_a",
              "mask_coast_a", "mask_margin_a", "mask_gl_a", "mask_cf_a", "mask_a", "Hi_cx", "Hi_cy", "Hi_b",
              "dHi_dx_a", "dHi_dy_a", "dHs_dx_a", "dHs_dy_a", "dHs_dx_cx", "dHs_dy_cx", "dHs_dx_cy", "dHs_dy_cy",
              "A_flow_3D_cx", "A_flow_3D_cy", "A_flow_vav_cx", "A_flow_vav_cy"]
OUT_RHEOLOGY = ["A_flow_3D_a", "A_flow_vav_a", "A_flow_3D_cx", "A_flow_3D_cy", "A_flow_vav_cx", "A_flow_vav_cy"]
OUT_SECONDARY = ["u_3D_cx", "v_3D_cy", "w_3D_a", "u_3D_a", "v_3D_a", "u_vav_cx", "v_vav_cy",
                 "u_surf_cx", "v_surf_cy", "u_base_cx", "v_base_cy", "u_vav_a", "v_vav_a", "u_surf_a", "v_surf_a",
                 "u_base_a", "v_base_a", "uabs_vav_a", "uabs_surf_a", "uabs_base_a", "w_surf_a", "w_base_a", "R_shear"]
OUT_PICARD = ["taudx_cx", "taudy_cy", "f_grnd_a", "f_grnd_cx", "f_grnd_cy", "f_grnd_b", "Neff_a",
              "pore_water_pressure_a", "overburden_pressure_a", "tauc_a",
              "visc_eff_3D_a", "visc_eff_int_a", "visc_eff_3D_b", "visc_eff_int_b", "N_a", "N_b", "N_cx", "N_cy",
              "beta_a", "beta_eff_a", "beta_eff_cx", "beta_eff_cy", "u_cx_prev", "v_cy_prev",
              "DIVA_err_cx", "DIVA_err_cy", "DIVA_mask_combi", "DIVA_isfront_inner", "DIVA_isfront_outer"]
OUT_DIVA = OUT_PICARD + ["du_dz_3D_cx", "dv_dz_3D_cy", "F2_a", "F1_3D_a", "taub_cx", "taub_cy"] + OUT_SECONDARY
OUT_SSA = OUT_PICARD + ["u_SSA_cx", "v_SSA_cy"] + OUT_SECONDARY
OUT_SIA = ["u_3D_SIA_cx", "v_3D_SIA_cy"] + OUT_SECONDARY


def _run(grid, ice, config, backend, fn, outputs):
    ctx = Context(grid, config, backend)
    try:
        ctx.upload(ice)
        rep = getattr(ctx, fn)()
        ice.update(ctx.download(outputs) if outputs is not None else ctx.download())
        return rep
    finally:
        ctx.close()


def update_general_ice_model_data(grid, ice, config=None, backend=None):
    """general_ice_model_data_module.f90:30-86 on the GPU; updates ``ice`` in place."""
    return _run(grid, ice, config, backend, "update_general_ice_model_data", OUT_UPDATE)


def calc_ice_rheology(grid, ice, config=None, backend=None):
    """thermodynamics_module.f90:641-753 on the GPU; updates ``ice`` in place."""
    return _run(grid, ice, config, backend, "calc_ice_rheology", OUT_RHEOLOGY)


def solve_SIA(grid, ice, config=None, backend=None):
    """ice_velocity_module.f90:36-114 on the GPU; updates ``ice`` in place."""
    return _run(grid, ice, config, backend, "solve_SIA", OUT_SIA)


def solve_SSA(grid, ice, config=None, backend=None):
    """ice_velocity_module.f90:115-248 on the GPU; updates ``ice`` in place."""
    return _run(grid, ice, config, backend, "solve_SSA", OUT_SSA)


class Batch:
    """A persistent batch (diva_batch_create): the viscosity loops of ``contexts`` captured
    into one CUDA graph once; every ``solve_DIVA()`` is solve_DIVA for all members with a
    single graph launch for their iterations.  The contexts must stay open and keep their
    configuration while the batch lives."""

    def __init__(self, contexts):
        if not contexts:
            raise DivaError(_abi.BAD_INPUT, "a batch needs at least one context")
        self.contexts = list(contexts)
        be = self.contexts[0].backend
        if be.name != "cuda" or any(c.backend is not be for c in self.contexts):
            raise DivaError(_abi.UNSUPPORTED, "batches run on the CUDA library, all members on it")
        lib = be.lib
        self._create = lib.diva_batch_create
        self._create.restype = C.c_int
        self._create.argtypes = [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)]
        self._solve = lib.diva_batch_solve_diva
        self._solve.restype = C.c_int
        self._solve.argtypes = [C.c_void_p, C.POINTER(_abi.Report)]
        self._destroy = lib.diva_batch_destroy
        self._destroy.restype = C.c_int
        self._destroy.argtypes = [C.c_void_p]
        self.h = C.c_void_p()
        n = len(self.contexts)
        hs = (C.c_void_p * n)(*[c.h for c in self.contexts])
        st = self._create(hs, n, C.byref(self.h))
        if st != 0:
            err = be.fns["last_error"](self.contexts[0].h)
            raise DivaError(st, f"diva_batch_create: {err.decode() if err else ''}")

    def solve_DIVA(self, raise_on_error=True):
        n = len(self.contexts)
        reps = (_abi.Report * n)()
        st = self._solve(self.h, reps)
        out = [r.as_dict() for r in reps]
        if raise_on_error:
            for k, (c, r) in enumerate(zip(self.contexts, out)):
                if r["status"] not in (0, _abi.MAX_PICARD):
                    err = c.backend.fns["last_error"](c.h)
                    raise DivaError(r["status"], f"batch member {k}: {err.decode() if err else ''}")
            if st not in (0, _abi.MAX_PICARD) and all(r["status"] in (0, _abi.MAX_PICARD) for r in out):
                err = self.contexts[0].backend.fns["last_error"](self.contexts[0].h)
                raise DivaError(st, f"diva_batch_solve_diva: {err.decode() if err else ''}")
        return out

    def close(self):
        if self.h:
            self._destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_DIVA_batch(contexts, raise_on_error=True):
    """solve_DIVA for several contexts at once (diva_solve_diva_batch): each on its own
    stream, every member's graph-launched viscosity loop in flight at once, so small
    members share the GPU.  Returns the reports in order; raises DivaError naming the
    first member whose status is neither OK nor MAX_PICARD, unless raise_on_error is
    False (then each report's status says how its member ended)."""
    if not contexts:
        return []
    be = contexts[0].backend
    if any(c.backend is not be for c in contexts):
        raise DivaError(_abi.BAD_INPUT, "all contexts of a batch must use the same backend")
    f = getattr(be.lib, be.prefix + "solve_diva_batch", None)
    if f is None:
        raise DivaError(_abi.UNSUPPORTED, f"{be.name} backend has no batched solve")
    f.restype = C.c_int
    f.argtypes = [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(_abi.Report)]
    n = len(contexts)
    hs = (C.c_void_p * n)(*[c.h for c in contexts])
    reps = (_abi.Report * n)()
    st = f(hs, n, reps)
    out = [r.as_dict() for r in reps]
    if st not in (0, _abi.MAX_PICARD) and all(r["status"] in (0, _abi.MAX_PICARD) for r in out):
        err = be.fns["last_error"](contexts[0].h)   # rejected before any member ran
        raise DivaError(st, f"solve_DIVA_batch: {err.decode() if err else ''}")
    for k, (c, r) in enumerate(zip(contexts, out)):
        if raise_on_error and r["status"] not in (0, _abi.MAX_PICARD):
            err = be.fns["last_error"](c.h)
            raise DivaError(r["status"], f"solve_DIVA_batch member {k}: {err.decode() if err else ''}")
    return out


def solve_DIVA(grid, ice, config=None, backend=None):
    """ice_velocity_module.f90:249-374 on the GPU; updates ``ice`` in place."""
    return _run(grid, ice, config, backend, "solve_DIVA", OUT_DIVA)
