"""Behaviour of the C ABI on the GPU: determinism, checkpoint/restore, the
reference-shaped Python API, error codes, and failure handling without any
device fault (bad inputs are injected on the host)."""
import numpy as np
import pytest

from imau_ice_b200 import _abi, diva
import helpers

pytestmark = pytest.mark.gpu


def small():
    return helpers.make_case(2, dx=40e3, overrides={"lin_rtol": 1e-10})


def test_bitwise_deterministic(cuda):
    g, cfg, f = small()
    r1, o1 = helpers.run(cuda, g, cfg, f)
    r2, o2 = helpers.run(cuda, g, cfg, f)
    assert r1["picard_iterations"] == r2["picard_iterations"]
    for k in ("u_vav_cx", "v_vav_cy", "visc_eff_3D_a", "w_3D_a"):
        assert np.array_equal(o1[k], o2[k]), k


def test_state_save_restore_reproduces_a_solve(cuda):
    g, cfg, f = small()
    ctx = diva.Context(g, cfg, cuda)
    helpers.prepare(ctx, f)
    ctx.state_save()
    r1 = ctx.solve_DIVA()
    a = ctx.download(["u_vav_cx", "v_vav_cy", "u_3D_a"])
    ctx.state_restore()
    r2 = ctx.solve_DIVA()
    b = ctx.download(["u_vav_cx", "v_vav_cy", "u_3D_a"])
    ctx.close()
    assert r1["picard_iterations"] == r2["picard_iterations"]
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_warm_start_converges_faster(cuda):
    g, cfg, f = helpers.make_case(2, dx=40e3, overrides={"picard_stop": "relres", "picard_relres_tol": 1e-6,
                                                         "DIVA_visc_it_nit": 300, "lin_adaptive": 1})
    ctx = diva.Context(g, cfg, cuda)
    helpers.prepare(ctx, f)
    cold = ctx.solve_DIVA()
    warm = ctx.solve_DIVA()          # second call starts from the converged state
    ctx.close()
    assert cold["relres"] <= 1e-6 and warm["relres"] <= 1e-6
    assert warm["picard_iterations"] < cold["picard_iterations"]


def test_reference_shaped_functions(cuda):
    g, cfg, f = small()
    ice = dict(f)
    diva.update_general_ice_model_data(g, ice, cfg, cuda)
    diva.calc_ice_rheology(g, ice, cfg, cuda)
    diva.update_general_ice_model_data(g, ice, cfg, cuda)
    assert "mask_sheet_a" in ice and ice["mask_sheet_a"].sum() > 0 and ice["A_flow_3D_a"].min() > 0
    rep = diva.solve_DIVA(g, ice, cfg, cuda)
    assert rep["picard_iterations"] >= 1
    assert ice["u_vav_cx"].shape == (g.ny, g.nx - 1) and ice["u_3D_cx"].shape == (g.nz, g.ny, g.nx - 1)
    assert np.isfinite(ice["u_vav_cx"]).all()


def test_wrong_dynamics_mode_is_rejected(cuda):
    g, cfg, f = small()
    ctx = diva.Context(g, cfg, cuda)
    with pytest.raises(diva.DivaError) as e:
        ctx.solve_SIA()
    assert e.value.status == _abi.BAD_INPUT
    ctx.close()


def test_bc_margins_need_a_coarser_level(cuda):
    """The 'BC' front rows live on the finest multigrid level; a grid below 9 points in
    both directions has no coarser level and is refused instead of solved without them."""
    n = 8
    g = diva.Grid(n, n, 5e3)
    f = {"Hi_a": np.full((n, n), 300.0), "Hb_a": np.full((n, n), -600.0), "SL_a": np.zeros((n, n)),
         "Ti_a": np.full((g.nz, n, n), 260.0), "beta_sq_a": np.full((n, n), 1e4)}
    f["Hb_a"][:, :3] = 100.0        # grounded ice upstream (a solve without sheet ice returns early)
    f["Hi_a"][:, -2:] = 0.0
    ctx = diva.Context(g, {"choice_ice_margin": "BC"}, cuda)
    helpers.prepare(ctx, {k: np.asfortranarray(v) for k, v in f.items()})
    with pytest.raises(diva.DivaError) as e:
        ctx.solve_DIVA()
    assert e.value.status == _abi.UNSUPPORTED
    ctx.close()


@pytest.mark.parametrize("dx", [5e3, 2.5e3])
def test_bc_margins_same_result_on_every_launch_path(cuda, monkeypatch, dx):
    """The cut shelf with 'BC' margins through the graph-launched viscosity loop, the
    host-driven loop (DIVA_NO_GRAPHS=1) and the per-colour smoothing kernels
    (DIVA_NO_TILES=1): the same iterations, bit for bit."""
    g, cfg, f = helpers.make_case(1, dx=dx, overrides={"choice_ice_margin": "BC", "lin_rtol": 1e-10},
                                  calving_front=True)
    r1, o1 = helpers.run(cuda, g, cfg, f)
    monkeypatch.setenv("DIVA_NO_GRAPHS", "1")
    r2, o2 = helpers.run(cuda, g, cfg, f)
    monkeypatch.setenv("DIVA_NO_TILES", "1")
    r3, o3 = helpers.run(cuda, g, cfg, f)
    assert r1["graph_launched"] == 1 and r2["graph_launched"] == 0
    assert r1["picard_iterations"] == r2["picard_iterations"] == r3["picard_iterations"]
    for k in ("u_vav_cx", "v_vav_cy", "u_3D_cx"):
        assert np.array_equal(o1[k], o2[k]) and np.array_equal(o1[k], o3[k]), k
    assert np.abs(o1["u_vav_cx"]).max() > 100.0


def test_bc_margins_singular_geometry_is_reported(cuda):
    """'BC' with a wide open-ocean strip: rows between ocean cells are empty in the
    reference's matrix (zero viscosity and friction there), so the system is singular;
    the solve ends with an error status instead of returning velocities."""
    g, cfg, f = helpers.make_case(1, overrides={"choice_ice_margin": "BC", "DIVA_visc_it_nit": 20})
    H = np.array(f["Hi_a"])
    H[:, -12:] = 0.0
    f = dict(f, Hi_a=np.asfortranarray(H))
    ctx = diva.Context(g, cfg, cuda)
    helpers.prepare(ctx, f)
    with pytest.raises(diva.DivaError) as e:
        ctx.solve_DIVA()
    assert e.value.status in (_abi.NAN_DETECTED, _abi.LINEAR_NOT_CONVERGED)
    ctx.close()


def test_bad_grid_rejected(cuda):
    with pytest.raises(diva.DivaError) as e:
        diva.Context(diva.Grid(3, 3, 1e3), {}, cuda)
    assert e.value.status == _abi.BAD_INPUT


def test_nan_input_is_reported_not_faulted(cuda):
    """A corrupt input (NaN thickness) ends the solve with NAN_DETECTED; the context stays usable."""
    g, cfg, f = small()
    bad = dict(f)
    H = np.array(f["Hi_a"])
    H[g.ny // 2, g.nx // 2] = np.nan
    bad["Hi_a"] = np.asfortranarray(H)
    ctx = diva.Context(g, cfg, cuda)
    helpers.prepare(ctx, bad)
    with pytest.raises(diva.DivaError) as e:
        ctx.solve_DIVA()
    assert e.value.status == _abi.NAN_DETECTED
    zeros = {k: ctx.empty(k) for k in ("u_vav_cx", "v_vav_cy", "visc_eff_3D_a", "taub_cx", "taub_cy",
                                       "u_3D_a", "v_3D_a")}
    ctx.upload(zeros)                        # recover on the same context from a cold state
    helpers.prepare(ctx, f)
    rep = ctx.solve_DIVA()
    ctx.close()
    assert rep["status"] in (_abi.OK, _abi.MAX_PICARD)


def test_linear_iteration_cap_is_bounded(cuda):
    g, cfg, f = helpers.make_case(2, dx=40e3, overrides={"lin_maxit": 1, "lin_rtol": 1e-14, "DIVA_visc_it_nit": 5})
    ctx = diva.Context(g, cfg, cuda)
    helpers.prepare(ctx, f)
    rep = ctx.solve_DIVA()
    ctx.close()
    assert rep["picard_iterations"] == 5 and rep["linear_iterations"] == 5


@pytest.mark.parametrize("anderson_m", [0, 3])
def test_graph_launched_iterations_match_direct_launches(cuda, monkeypatch, anderson_m):
    """Each viscosity iteration runs as one CUDA graph (device-side Krylov loop);
    launching the same kernels one by one gives bit-identical results, with the
    reference's relaxation and with Anderson mixing."""
    g, cfg, f = helpers.make_case(2, dx=40e3, overrides={"picard_stop": "relres", "picard_relres_tol": 1e-6,
                                                         "DIVA_visc_it_nit": 300, "lin_adaptive": 1,
                                                         "picard_anderson_m": anderson_m})
    rg, og = helpers.run(cuda, g, cfg, f)
    monkeypatch.setenv("DIVA_NO_GRAPHS", "1")
    rd, od = helpers.run(cuda, g, cfg, f)
    assert rg["graph_launched"] == 1 and rd["graph_launched"] == 0
    assert rg["picard_iterations"] == rd["picard_iterations"]
    assert rg["linear_iterations"] == rd["linear_iterations"] and rg["mg_cycles"] == rd["mg_cycles"]
    for k in ("u_vav_cx", "v_vav_cy", "visc_eff_3D_a", "DIVA_err_cx", "taub_cx", "u_3D_cx"):
        assert np.array_equal(og[k], od[k]), k


@pytest.mark.parametrize("dx", [5e3, 10e3])
def test_tiled_smoothing_matches_per_colour_kernels(cuda, monkeypatch, dx):
    """The large levels are smoothed by tile kernels that recompute a halo; the
    per-colour kernels (DIVA_NO_TILES=1) give bit-identical results.  5 km uses
    the 32 x 32 tiles on the finest level, 10 km the 16 x 16 tiles."""
    g, cfg, f = helpers.make_case(2, dx=dx, overrides={"picard_stop": "relres", "picard_relres_tol": 1e-6,
                                                       "DIVA_visc_it_nit": 300, "lin_adaptive": 1})
    rt, ot = helpers.run(cuda, g, cfg, f)
    monkeypatch.setenv("DIVA_NO_TILES", "1")
    rp, op = helpers.run(cuda, g, cfg, f)
    assert rt["status"] == rp["status"] and rt["status"] in (0, 1), (rt, rp)   # OK or the iteration cap
    assert rt["picard_iterations"] == rp["picard_iterations"]
    assert rt["linear_iterations"] == rp["linear_iterations"] and rt["mg_cycles"] == rp["mg_cycles"]
    for k in ("u_vav_cx", "v_vav_cy", "visc_eff_3D_a", "u_3D_cx"):
        assert np.array_equal(ot[k], op[k]), k


def test_batch_solve_matches_individual_solves(cuda):
    """diva_solve_diva_batch keeps one iteration of every member in flight on its own
    stream; each member's result is bit-identical to solving it alone."""
    ov = {"picard_stop": "relres", "picard_relres_tol": 1e-6, "DIVA_visc_it_nit": 300, "lin_adaptive": 1}
    cases = [helpers.make_case(1, overrides=ov), helpers.make_case(2, dx=40e3, overrides=ov),
             helpers.make_case(2, dx=10e3, overrides=dict(ov, DIVA_visc_it_nit=40))]
    names = ("u_vav_cx", "v_vav_cy", "visc_eff_3D_a", "u_3D_cx", "w_3D_a")
    alone = [helpers.run(cuda, g, cfg, f, post=None) for g, cfg, f in cases]
    ctxs = []
    for g, cfg, f in cases:
        ctx = diva.Context(g, cfg, cuda)
        helpers.prepare(ctx, f)
        ctxs.append(ctx)
    reps = diva.solve_DIVA_batch(ctxs)
    outs = [ctx.download(list(names)) for ctx in ctxs]
    for ctx in ctxs:
        ctx.close()
    for (ra, oa), rb, ob in zip(alone, reps, outs):
        assert ra["status"] == rb["status"] and ra["picard_iterations"] == rb["picard_iterations"]
        assert ra["mg_cycles"] == rb["mg_cycles"]
        for k in names:
            assert np.array_equal(oa[k], ob[k]), k
    assert reps[2]["status"] == _abi.MAX_PICARD   # the capped member ends like the lone solve


def test_persistent_batch_graph_matches_individual_solves(cuda):
    """diva_batch_create captures every member's viscosity loop into one CUDA graph;
    diva_batch_solve_diva replays it as one launch.  Each member's result is bit-identical
    to solving it alone, on the first replay and on a second one from the same cold
    states (the members' viscosity buffers then start in another order, which the batch
    restores before its launch), and a member reconfigured after capture is refused."""
    ov = {"picard_stop": "relres", "picard_relres_tol": 1e-6, "DIVA_visc_it_nit": 300, "lin_adaptive": 1}
    cases = [helpers.make_case(1, overrides=ov), helpers.make_case(2, dx=40e3, overrides=ov),
             helpers.make_case(2, dx=20e3, overrides=dict(ov, picard_anderson_m=3, lin_adaptive_eta=0.1,
                                                          picard_stall_its=30)),
             helpers.make_case(2, dx=10e3, overrides=dict(ov, DIVA_visc_it_nit=40, precision="mixed"))]
    names = ("u_vav_cx", "v_vav_cy", "visc_eff_3D_a", "u_3D_cx", "w_3D_a")
    alone = [helpers.run(cuda, g, cfg, f) for g, cfg, f in cases]
    ctxs = []
    for g, cfg, f in cases:
        ctx = diva.Context(g, cfg, cuda)
        helpers.prepare(ctx, f)
        ctx.state_save()
        ctxs.append(ctx)
    batch = diva.Batch(ctxs)
    for replay in range(2):
        for ctx in ctxs:
            ctx.state_restore()
        reps = batch.solve_DIVA()
        outs = [ctx.download(list(names)) for ctx in ctxs]
        for (ra, oa), rb, ob in zip(alone, reps, outs):
            assert ra["status"] == rb["status"] and ra["picard_iterations"] == rb["picard_iterations"], replay
            assert ra["mg_cycles"] == rb["mg_cycles"] and ra["stalled"] == rb["stalled"], replay
            for k in names:
                assert np.array_equal(oa[k], ob[k]), (replay, k)
    assert reps[2]["stalled"] == 1 and reps[3]["status"] == _abi.MAX_PICARD
    ctxs[1].set_config(dict(cases[1][1], lin_adaptive_eta=0.3))
    with pytest.raises(diva.DivaError) as e:
        batch.solve_DIVA()
    assert e.value.status == _abi.BAD_INPUT
    batch.close()
    for ctx in ctxs:
        ctx.close()


def test_batch_solve_rejects_repeated_context(cuda):
    g, cfg, f = helpers.make_case(2, dx=40e3)
    ctx = diva.Context(g, cfg, cuda)
    helpers.prepare(ctx, f)
    with pytest.raises(diva.DivaError):
        diva.solve_DIVA_batch([ctx, ctx])
    ctx.close()


def test_ensemble_members_equal_lone_solves(cuda):
    """An ensemble solved through the partition/batch driver on one rank gives each
    member exactly its lone solve (same iterations, bit-identical velocities)."""
    import dist_worker
    from imau_ice_b200 import ensemble
    members = dist_worker.small_channel_members(3)
    g, cfg, f = helpers.make_case(2, dx=40e3, overrides={"lin_rtol": 1e-10})
    members.append(("icecap-3", g, cfg, f))
    res, parts = ensemble.solve_ensemble(members, cuda)
    assert parts == [[0, 1, 2, 3]] and sorted(res) == [0, 1, 2, 3]
    for k, (name, grid, c, fields) in enumerate(members):
        r, o = helpers.run(cuda, grid, c, fields)
        assert res[k]["report"]["picard_iterations"] == r["picard_iterations"], name
        assert np.array_equal(res[k]["u_vav_cx"], o["u_vav_cx"]), name
        assert np.array_equal(res[k]["v_vav_cy"], o["v_vav_cy"]), name


def test_mixed_precision_is_validated(cuda):
    g, cfg, f = small()
    with pytest.raises(diva.DivaError) as e:
        diva.Context(g, dict(cfg, precision=2), cuda)
    assert e.value.status == _abi.BAD_INPUT
    ctx = diva.Context(g, dict(cfg, precision="mixed", BC_u_west="periodic", BC_u_east="periodic"), cuda)
    helpers.prepare(ctx, f)
    with pytest.raises(diva.DivaError) as e:
        ctx.solve_DIVA()
    assert e.value.status == _abi.UNSUPPORTED
    ctx.close()


@pytest.mark.parametrize("case", ["channel_5km", "icecap_5km"])
def test_mixed_precision_matches_fp64(cuda, case):
    """precision 'mixed' (FP32 finest-level smoother inside FP64 BiCGStab) reaches the same
    nonlinear tolerance as the FP64 solver; the velocities agree to the tolerance's size."""
    cfg_id = 1 if case.startswith("channel") else 2
    ov = {"picard_stop": "relres", "picard_relres_tol": 1e-6, "DIVA_visc_it_nit": 500, "lin_adaptive": 1,
          "lin_rtol": 1e-10}
    g, cfg, f = helpers.make_case(cfg_id, overrides=ov)
    r64, o64 = helpers.run(cuda, g, cfg, f)
    r32, o32 = helpers.run(cuda, g, dict(cfg, precision="mixed"), f)
    assert r64["status"] == 0, r64
    assert r32["status"] == 0, r32
    assert r32["relres"] <= 1e-6
    a = np.concatenate([o64["u_vav_cx"].ravel(), o64["v_vav_cy"].ravel()])
    b = np.concatenate([o32["u_vav_cx"].ravel(), o32["v_vav_cy"].ravel()])
    assert helpers.rel_l2(b, a) <= 1e-5
    assert abs(r32["picard_iterations"] - r64["picard_iterations"]) <= 0.1 * r64["picard_iterations"] + 2


def test_restart_file_continues_bit_for_bit(cuda, tmp_path):
    """save_restart / load_restart of a GPU context: the reloaded context's next solve is
    the original context's, bit for bit."""
    g, cfg, f = small()
    ctx = diva.Context(g, cfg, cuda)
    helpers.prepare(ctx, f)
    ctx.solve_DIVA()
    path = tmp_path / "restart.npz"
    ctx.save_restart(path)
    ctx2 = diva.Context.load_restart(path, cuda)
    r1, r2 = ctx.solve_DIVA(), ctx2.solve_DIVA()
    assert r1["picard_iterations"] == r2["picard_iterations"]
    a, b = ctx.download(["u_vav_cx", "v_vav_cy", "visc_eff_3D_a", "u_3D_cx"]), ctx2.download(
        ["u_vav_cx", "v_vav_cy", "visc_eff_3D_a", "u_3D_cx"])
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    ctx.close()
    ctx2.close()


def test_complete_state_matches_the_oracle_and_warm_starts(cuda, oracle):
    """diva_complete_state from the oracle's converged velocities: the completed
    viscosity, beta_eff and basal stress agree with the oracle's, and solve_DIVA
    started from them stops within a few iterations (a cold start needs > 20)."""
    import oracle_backend as ob
    from imau_ice_b200 import synth
    g, cfg, f = synth.ice_cap(seed=310, dx=20e3)
    f = dict(f)
    f["beta_sq_a"] = np.asfortranarray(f["beta_sq_a"] * 4.0)
    cfg = dict(cfg, picard_stop="relres", picard_relres_tol=1e-6, DIVA_visc_it_nit=500, lin_adaptive=1,
               lin_rtol=1e-10)
    grid = diva.Grid(**g)
    ctx = diva.Context(grid, cfg, oracle)
    ob.set_linear_solver(ctx, ob.LIN_GMRES_WARM, rtol=1e-10, abstol=0.0)
    helpers.prepare(ctx, f)
    cold = ctx.solve_DIVA()["picard_iterations"]
    uv = ctx.download(["u_vav_cx", "v_vav_cy"])
    ctx.close()
    names = ["visc_eff_3D_a", "beta_eff_cx", "beta_eff_cy", "taub_cx", "taub_cy", "u_base_cx", "v_base_cy"]
    out = []
    for be in (cuda, oracle):
        ctx = diva.Context(grid, cfg, be)
        helpers.prepare(ctx, f)
        ctx.upload(uv)
        ctx.complete_state(30)
        out.append(ctx.download(names))
        if be is cuda:
            rep = ctx.solve_DIVA()
        ctx.close()
    for k in names:
        assert helpers.rel_l2(out[0][k], out[1][k]) <= 1e-9, k
    assert cold > 20 and rep["status"] == 0 and rep["picard_iterations"] <= 3, (cold, rep)


def test_anderson_mixing_is_validated(cuda):
    g, cfg, f = small()
    for bad in ({"picard_anderson_m": 6, "picard_stop": "relres"}, {"picard_anderson_m": -1},
                {"picard_anderson_m": 2, "picard_stop": "resid_UV"}):
        with pytest.raises(diva.DivaError) as e:
            diva.Context(g, dict(cfg, **bad), cuda)
        assert e.value.status == _abi.BAD_INPUT, bad


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_anderson_mixing_reaches_the_same_equations_in_fewer_iterations(cuda, oracle, precision):
    """The 321 x 561 ice cap to rel-res 1e-6 with the bench's adaptive linear tolerance:
    Anderson mixing of depth 3 (linear tolerance factor 0.1) needs far fewer viscosity
    iterations than the reference's relaxation (factor 0.5), and the state it stops at
    satisfies the reference equations as the oracle evaluates them."""
    ov = {"picard_stop": "relres", "picard_relres_tol": 1e-6, "DIVA_visc_it_nit": 500, "lin_adaptive": 1,
          "lin_rtol": 1e-10}
    g, cfg, f = helpers.make_case(2, overrides=ov)
    r0, o0 = helpers.run(cuda, g, cfg, f)
    r1, o1 = helpers.run(cuda, g, dict(cfg, picard_anderson_m=3, lin_adaptive_eta=0.1, precision=precision), f)
    assert r0["status"] == 0 and r1["status"] == 0, (r0, r1)
    assert r1["relres"] <= 1e-6
    assert r1["picard_iterations"] <= 0.5 * r0["picard_iterations"], (r0, r1)
    octx = diva.Context(g, cfg, oracle)
    helpers.prepare(octx, f)
    oracle.lib.orc_prepare_diva(octx.h)
    octx.upload({k: o1[k] for k in ("u_vav_cx", "v_vav_cy", "visc_eff_3D_a", "taub_cx", "taub_cy")})
    r = octx.nonlinear_residual()
    octx.close()
    assert r <= 2e-6, r

