"""Tile shapes of the multigrid smoother on the GPU: any per-level choice of 16 / 32
gives the bit-identical solve, and the autotuner sets a valid choice."""
import numpy as np
import pytest
import torch

from imau_ice_b200 import autotune, diva
import helpers

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU (B200)")]


def solve(edges=None, tune=False):
    g, cfg, f = helpers.make_case(2, dx=5e3, overrides={"picard_stop": "relres", "picard_relres_tol": 1e-6,
                                                        "DIVA_visc_it_nit": 300, "lin_adaptive": 1})
    ctx = diva.Context(g, cfg)
    helpers.prepare(ctx, f)
    ctx.nonlinear_residual()        # what the tuner does first: every run starts from the same state
    if edges is not None:
        ctx.set_tile_edges(edges)
    chosen = autotune.tune_tile_edges(ctx, reps=5, trials=1)[0] if tune else ctx.get_tile_edges()
    r = ctx.solve_DIVA()
    o = ctx.download(["u_vav_cx", "v_vav_cy", "visc_eff_3D_a"])
    ctx.close()
    return r, o, chosen


def test_tile_edges_change_time_not_the_solution():
    r0, o0, e0 = solve()
    assert e0[0] == 32 and all(e in (0, 16, 32) for e in e0)      # 321 x 561: 32 x 32 tiles on level 0
    r1, o1, e1 = solve([16] * len(e0))
    assert e1[0] == 16
    r2, o2, e2 = solve(tune=True)
    assert all((a == 0) == (b == 0) for a, b in zip(e0, e2))
    for r, o in ((r1, o1), (r2, o2)):
        assert r["picard_iterations"] == r0["picard_iterations"] and r["mg_cycles"] == r0["mg_cycles"]
        for k in o0:
            assert np.array_equal(o[k], o0[k]), k
