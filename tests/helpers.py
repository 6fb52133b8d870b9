"""Shared drivers for the parity tests: one call sequence, two backends."""
import numpy as np

from imau_ice_b200 import diva, synth

INT_FIELDS = {"mask_land_a", "mask_ocean_a", "mask_ice_a", "mask_sheet_a", "mask_shelf_a", "mask_coast_a",
              "mask_margin_a", "mask_gl_a", "mask_cf_a", "mask_a", "DIVA_mask_combi", "DIVA_isfront_inner",
              "DIVA_isfront_outer"}


def make_case(cfg_id, dx=None, seed=None, overrides=None, **gen_kw):
    gen = synth.CONFIGS[cfg_id]
    kw = dict(gen_kw)
    if dx is not None:
        kw["dx"] = dx
    if seed is not None:
        kw["seed"] = seed
    g, cfg, fields = gen(**kw)
    cfg = dict(cfg)
    cfg.update(overrides or {})
    return diva.Grid(**g), cfg, fields


def prepare(ctx, fields):
    """The input preparation the reference does before solve_DIVA: geometry, masks, rheology."""
    ctx.upload(fields)
    ctx.update_general_ice_model_data()
    ctx.calc_pressure_melting_point()
    ctx.calc_ice_rheology()
    ctx.update_general_ice_model_data()


def run(backend, grid, cfg, fields, solve="solve_DIVA", oracle_solver=None, post=None):
    ctx = diva.Context(grid, cfg, backend)
    if oracle_solver is not None:
        import oracle_backend
        oracle_backend.set_linear_solver(ctx, *oracle_solver)
    prepare(ctx, fields)
    rep = getattr(ctx, solve)() if solve else None
    if post:
        post(ctx)
    out = ctx.download()
    ctx.close()
    return rep, out


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def compare(gpu, ref, names, rtol):
    """Return {name: rel-L2} for float fields and mismatch counts for int fields."""
    res = {}
    for n in names:
        if n in INT_FIELDS:
            res[n] = int(np.count_nonzero(gpu[n] != ref[n]))
        else:
            res[n] = rel_l2(gpu[n], ref[n])
    return res
