"""Seeded synthetic inputs for the velocity benchmarks.

No public dataset is involved: the benchmark configurations are synthetic.
Grid sizes follow the reference's own rule nx = 1 + 2*floor((xmax-xmid)/dx)
(IMAU_ICE_main_model.f90:699-706).  The marine channel borrows only the
shape of the MISMIP+ set-up (a trough deepening downstream, side walls, a
floating shelf past a grounding line); the ice cap is a dome on Gaussian
random topography with ragged margins.  Every field is a deterministic
function of (seed, dx).

Arrays are Fortran-ordered with the reference's shapes: (ny, nx) for
a-grid fields and (nz, ny, nx) for 3D fields.
"""
import numpy as np

RHO_I, RHO_SW = 910.0, 1028.0


def _axis(half_width, dx):
    n = 1 + 2 * int(np.floor(half_width / dx + 1e-9))
    return -dx * (n // 2) + dx * np.arange(n)


def _grf(rng, ny, nx, dx, corr_len):
    """Zero-mean, unit-variance Gaussian random field with a Gaussian spectrum."""
    w = rng.standard_normal((ny, nx))
    ky = np.fft.fftfreq(ny, d=dx)[:, None]
    kx = np.fft.fftfreq(nx, d=dx)[None, :]
    filt = np.exp(-0.5 * (2 * np.pi * corr_len) ** 2 * (kx ** 2 + ky ** 2))
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
    f -= f.mean()
    s = f.std()
    return f / s if s > 0 else f


def _smooth3(a):
    """One pass of a 1-2-1 binomial filter in each direction (edges replicated)."""
    p = np.pad(a, 1, mode="edge")
    a = 0.25 * p[:-2, 1:-1] + 0.5 * p[1:-1, 1:-1] + 0.25 * p[2:, 1:-1]
    p = np.pad(a, 1, mode="edge")
    return 0.25 * p[1:-1, :-2] + 0.5 * p[1:-1, 1:-1] + 0.25 * p[1:-1, 2:]


def _lognormal_friction(rng, ny, nx, median=1e4, sigma=0.5):
    g = _smooth3(rng.standard_normal((ny, nx)))
    g = (g - g.mean()) / g.std()
    return np.exp(np.log(median) + sigma * g)


def _temperature(rng, zeta, ny, nx, t_top, t_bot, dx, corr):
    """Englacial temperature rising from t_top at the surface towards t_bot at the base."""
    pert = _grf(rng, ny, nx, dx, corr)
    T = t_top + (t_bot - t_top - 3.0) * zeta[:, None, None] ** 1.5 + 1.5 * pert[None, :, :]
    return np.clip(T, t_top, t_bot)


def _fortran(d):
    return {k: np.asfortranarray(v) for k, v in d.items()}


ZETA = np.array([0.00, 0.10, 0.20, 0.30, 0.40, 0.50, 0.60, 0.70, 0.80, 0.90,
                 0.925, 0.95, 0.975, 0.99, 1.00])


def marine_channel(seed=1, dx=5e3, zeta=ZETA, calving_front=False):
    """Config 1: 640 x 80 km channel (129 x 17 at 5 km), grounding line near x = 450 km.

    Bed: a trough from +100 m to -700 m along flow with a seeded low-order
    perturbation and ~500 m tanh side walls.  Thickness: 2000 m at the divide,
    thinning to flotation at x_gl = 450 km, then a thinning floating shelf.
    Temperature 243-273 K; Weertman friction coefficient lognormal
    (median 1e4, sigma 0.5).

    ``calving_front=True`` cuts the shelf for the 'BC' ice-margin rows: open
    ocean in the last column, every third interior row one column shorter (a
    ragged front, so v rows meet it too), one open-ocean cell inside the shelf
    (fronts facing both ways) and one ice-free land cell inside the shelf
    (shelf-next-to-land rows).  No velocity point lies between two ocean cells
    away from the domain boundary on purpose: with 'BC' the reference gives
    ice-free cells zero viscosity and zero friction, so such rows keep only
    b-grid shear terms (or none) and the matrix becomes singular.
    """
    rng = np.random.default_rng(seed)
    x, y = _axis(320e3, dx), _axis(40e3, dx)
    nx, ny = len(x), len(y)
    X, Y = np.meshgrid(x, y)                      # (ny, nx)
    xr = X - x[0]
    L = x[-1] - x[0]
    amps = rng.uniform(-30.0, 30.0, 3)
    phases = rng.uniform(0, 2 * np.pi, 3)
    pert = sum(a * np.sin(2 * np.pi * (k + 1) * xr / L + p) for k, (a, p) in enumerate(zip(amps, phases)))
    b_center = 100.0 - 800.0 * xr / L + pert
    walls = 500.0 * 0.5 * (1.0 + np.tanh((np.abs(Y) - 28e3) / 5e3))
    Hb = b_center + walls
    x_gl = 450e3
    b_gl = 100.0 - 800.0 * x_gl / L + sum(a * np.sin(2 * np.pi * (k + 1) * x_gl / L + p)
                                          for k, (a, p) in enumerate(zip(amps, phases)))
    Hf_gl = max(0.0, -b_gl) * RHO_SW / RHO_I
    # centre-line thickness, then a surface that is flat across the channel:
    # ice thins against the side walls instead of following them
    s = np.clip(xr / x_gl, 0.0, None)
    H_grounded = Hf_gl + (2000.0 - Hf_gl) * np.sqrt(np.clip(1.0 - s, 0.0, None))
    H_shelf = 0.9 * Hf_gl * np.exp(-(xr - x_gl) / 200e3)
    Hs_center = np.where(xr < x_gl, b_center + H_grounded, H_shelf * (1.0 - RHO_I / RHO_SW))
    H_center = np.where(xr < x_gl, H_grounded, H_shelf)
    H = np.minimum(H_center, np.maximum(0.0, Hs_center - Hb))
    H = H * (1.0 + 0.02 * _grf(rng, ny, nx, dx, 30e3))
    H = np.maximum(H, 0.0)
    if calving_front:
        H[:, nx - 1] = 0.0
        H[2:ny - 2:3, nx - 2] = 0.0
        H[ny // 2 - 2, nx - 20] = 0.0
        jl, il = ny // 2 + 1, nx - 12
        H[jl, il] = 0.0
        Hb[jl, il] = 50.0
    T = _temperature(rng, zeta, ny, nx, 243.0, 273.0, dx, 60e3)
    fields = {
        "Hi_a": H, "Hb_a": Hb, "SL_a": np.zeros((ny, nx)), "dHb_dt_a": np.zeros((ny, nx)),
        "Ti_a": T, "beta_sq_a": _lognormal_friction(rng, ny, nx),
    }
    config = {
        "choice_ice_dynamics": "DIVA", "choice_ice_margin": "infinite_slab",
        "include_SSADIVA_crossterms": 1, "do_GL_subgrid_friction": 1, "include_basal_freezing": 0,
        "choice_sliding_law": "Weertman", "slid_Weertman_m": 3.0,
        "choice_ice_rheology": "Huybrechts1992",
        "BC_u_west": "zero", "BC_u_east": "infinite", "BC_u_south": "infinite", "BC_u_north": "infinite",
        "BC_v_west": "zero", "BC_v_east": "infinite", "BC_v_south": "zero", "BC_v_north": "zero",
        "DIVA_visc_it_norm_dUV_tol": 1e-3, "DIVA_visc_it_nit": 200, "DIVA_visc_it_relax": 0.4,
        "lin_rtol": 1e-8,
    }
    grid = dict(nx=nx, ny=ny, dx=dx, zeta=zeta, xmin=x[0], ymin=y[0])
    return grid, config, _fortran(fields)


def _dome(seed, dx, zeta, half_x, half_y, rx, ry, bed_corr, margin_corr, t_corr, s_max, h_max):
    """A dome on Gaussian random topography (bed rescaled to [-500, 2500] m) whose margin
    radius is perturbed by a second random field; thickness = surface - bed, clipped to
    [0, h_max], so margins are ragged where the bed rises through the dome."""
    rng = np.random.default_rng(seed)
    x, y = _axis(half_x, dx), _axis(half_y, dx)
    nx, ny = len(x), len(y)
    X, Y = np.meshgrid(x, y)
    g = _grf(rng, ny, nx, dx, bed_corr)
    Hb = -500.0 + 3000.0 * (g - g.min()) / (g.max() - g.min())
    r = np.sqrt((X / rx) ** 2 + (Y / ry) ** 2)
    rm = 1.0 + 0.05 * np.clip(_grf(rng, ny, nx, dx, margin_corr), -2.0, 2.0)
    Hs = s_max * np.clip(1.0 - (r / rm) ** 2, 0.0, None)
    H = np.clip(Hs - Hb, 0.0, h_max)
    H = np.where(Hs > 0.0, H, 0.0)
    T = _temperature(rng, zeta, ny, nx, 240.0, 273.0, dx, t_corr)
    fields = {
        "Hi_a": H, "Hb_a": Hb, "SL_a": np.zeros((ny, nx)), "dHb_dt_a": np.zeros((ny, nx)),
        "Ti_a": T, "beta_sq_a": _lognormal_friction(rng, ny, nx),
    }
    config = {
        "choice_ice_dynamics": "DIVA", "choice_ice_margin": "infinite_slab",
        "include_SSADIVA_crossterms": 1, "do_GL_subgrid_friction": 1, "include_basal_freezing": 0,
        "choice_sliding_law": "Weertman", "slid_Weertman_m": 3.0,
        "choice_ice_rheology": "Huybrechts1992",
        "DIVA_visc_it_norm_dUV_tol": 1e-3, "DIVA_visc_it_nit": 200, "DIVA_visc_it_relax": 0.4,
        "lin_rtol": 1e-8,
    }
    grid = dict(nx=nx, ny=ny, dx=dx, zeta=zeta, xmin=x[0], ymin=y[0])
    return grid, config, _fortran(fields)


def ice_cap(seed=2, dx=5e3, zeta=ZETA):
    """Config 2: 1600 x 2800 km ice cap (321 x 561 at 5 km).

    Bed correlation length ~150 km, dome 3400 m high, thickness at most 3200 m;
    temperature 240-273 K; Weertman friction coefficient lognormal.
    """
    return _dome(seed, dx, zeta, 800e3, 1400e3, 760e3, 1340e3, 150e3, 40e3, 200e3, 3400.0, 3200.0)


def ice_sheet(seed=5, dx=4e3, zeta=ZETA):
    """Config 5's large member: a 6000 x 6000 km continental ice sheet (1501 x 1501 at
    4 km), the same construction as the ice cap at continental scale (bed correlation
    length ~300 km, dome 4200 m high, thickness at most 4000 m)."""
    return _dome(seed, dx, zeta, 3000e3, 3000e3, 2850e3, 2850e3, 300e3, 80e3, 400e3, 4200.0, 4000.0)


def ensemble(n=64, seed=0, sizes=("channel", "icecap", "sheet")):
    """Config 5: n members with sizes drawn (seeded) from the marine channel (129 x 17),
    the ice cap (321 x 561) and the continental sheet (1501 x 1501); per member the
    friction coefficient is scaled by a log-uniform factor in [0.3, 3] and the flow
    factor (through the enhancement factor) by one in [0.5, 2].  Returns a list of
    (name, grid, config, fields)."""
    rng = np.random.default_rng(seed)
    gens = {"channel": marine_channel, "icecap": ice_cap, "sheet": ice_sheet}
    out = []
    for k in range(n):
        kind = sizes[int(rng.integers(len(sizes)))]
        fb = float(np.exp(rng.uniform(np.log(0.3), np.log(3.0))))
        fa = float(np.exp(rng.uniform(np.log(0.5), np.log(2.0))))
        g, cfg, f = gens[kind](seed=1000 + k)
        f = dict(f)
        if "beta_sq_a" in f:
            f["beta_sq_a"] = np.asfortranarray(f["beta_sq_a"] * fb)
        cfg = dict(cfg, m_enh_sheet=fa, m_enh_shelf=fa)
        out.append((f"{kind}-{k}", g, cfg, f))
    return out


def schoof_icestream(dx=10e3, half_width=400e3, zeta=ZETA, A=1e-17, L=100e3, m=0.5,
                     tantheta=3e-4, H0=2000.0):
    """The SSA_icestream benchmark (Schoof 2006): an infinite slab on a slope
    (reference_fields_module.f90:573-603) with the till yield stress of
    utilities_module.f90:836-878 (calc_bed_roughness_SSA_icestream,
    basal_conditions_and_sliding_module.f90:814-843); nx = 7 as in
    IMAU_ICE_main_model.f90:703."""
    x = dx * (np.arange(7) - 3)
    y = _axis(half_width, dx)
    nx, ny = len(x), len(y)
    X, Y = np.meshgrid(x, y)
    f = RHO_I * 9.81 * H0 * tantheta
    tauc = f * np.abs(Y / L) ** m
    fields = {
        "Hi_a": np.full((ny, nx), H0), "Hb_a": -tantheta * X, "SL_a": np.full((ny, nx), -1e4),
        "dHb_dt_a": np.zeros((ny, nx)), "Ti_a": np.full((len(zeta), ny, nx), 260.0),
        "tauc_a": tauc,
    }
    config = {
        "choice_ice_dynamics": "SSA", "choice_ice_margin": "infinite_slab",
        "choice_sliding_law": "Coulomb", "prescribed_tauc": 1, "include_basal_freezing": 0,
        "choice_ice_rheology": "uniform", "uniform_flow_factor": A,
        "DIVA_visc_it_norm_dUV_tol": 1e-6, "DIVA_visc_it_nit": 500, "DIVA_visc_it_relax": 0.4,
        "lin_rtol": 1e-10,
    }
    grid = dict(nx=nx, ny=ny, dx=dx, zeta=zeta, xmin=x[0], ymin=y[0])
    return grid, config, _fortran(fields)


CONFIGS = {1: marine_channel, 2: ice_cap, 5: ice_sheet}
