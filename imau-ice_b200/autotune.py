"""Tile-shape autotuner of the multigrid smoother.

The levels above the one-block sub-cycle are smoothed by tiled kernels whose tile
edge is 16 or 32; the default picks 32 while the level's 32 x 32 tiles still fill
the GPU.  Whether that is the faster choice depends on the level's size, the
operator and the precision, so ``tune_tile_edges`` measures it: for every
assignment of {16, 32} to the tiled levels it times one V-cycle on the context's
current operator (``diva_profile_kernel`` kind 3, CUDA events on the context's
stream), keeps the fastest, and sets it with ``diva_set_tile_edges``.  The solution
is the same bit for bit whatever the edges (the tiled smoother reproduces the
per-colour sweeps), so tuning changes time only.  Results are cached per grid
shape and configuration in a JSON file when ``cache`` is given, so an ensemble
tunes each member size once.
"""
import itertools
import json
import os


def cache_key(ctx):
    g, c = ctx.grid, ctx.cfg
    return f"{g.nx}x{g.ny}x{g.nz}:prec{int(c.precision)}:margin{int(c.choice_ice_margin)}"


def candidates(edges):
    """Every assignment of 16 / 32 to the tiled levels (edge != 0) of ``edges``."""
    tiled = [l for l, e in enumerate(edges) if e]
    for combo in itertools.product((16, 32), repeat=len(tiled)):
        out = [0] * len(edges)
        for l, v in zip(tiled, combo):
            out[l] = v
        yield out


def tune_tile_edges(ctx, reps=20, trials=3, cache=None):
    """Pick and set the fastest tile edges for ``ctx``; returns (edges, {edges: ms}).
    Contexts of other backends than the CUDA library have no tiles: ([], {})."""
    if getattr(getattr(ctx, "backend", None), "name", "cuda") != "cuda":
        return [], {}
    key = cache_key(ctx)
    if cache and os.path.exists(cache):
        with open(cache) as f:
            known = json.load(f)
        if key in known:
            ctx.set_tile_edges(known[key])
            return known[key], {}
    ctx.nonlinear_residual()          # coefficients and operator at the current state
    ctx.set_tile_edges([])
    default = ctx.get_tile_edges()
    timings = {}
    for e in candidates(default):
        ctx.set_tile_edges(e)
        timings[tuple(e)] = min(ctx.profile_kernel(3, reps)[0] for _ in range(trials))
    best = list(min(timings, key=timings.get)) if timings else default
    ctx.set_tile_edges(best)
    if cache:
        known = {}
        if os.path.exists(cache):
            with open(cache) as f:
                known = json.load(f)
        known[key] = best
        with open(cache, "w") as f:
            json.dump(known, f, indent=1, sort_keys=True)
    return best, timings
