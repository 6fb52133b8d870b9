"""The device thickness update and predictor/corrector stages against the oracle,
through the C ABI: bit-exact for the same inputs (both sides follow the reference's
IEEE operation order, the CUDA file without FMA contraction), and close after a few
time steps whose velocities each side solves itself."""
import numpy as np
import pytest

from imau_ice_b200 import diva, dynamics, synth
import helpers
import oracle_backend as ob

pytestmark = pytest.mark.gpu

THICK = ["Qx_cx", "Qy_cy", "dHi_dt_a", "Hi_tplusdt_a", "float_margin_frac_a", "Hi_eff_cf_a"]


def random_case(backend, seed, bc, dyn="DIVA", nx=37, ny=29, dx=10e3):
    rng = np.random.default_rng(seed)
    g = diva.Grid(nx, ny, dx)
    Hb = rng.uniform(-600.0, 400.0, (ny, nx))
    H = np.where(rng.random((ny, nx)) < 0.8, rng.uniform(50.0, 1500.0, (ny, nx)), 0.0)
    f = {"Hi_a": H, "Hb_a": Hb, "SL_a": np.zeros((ny, nx)), "Ti_a": np.full((g.nz, ny, nx), 260.0),
         "SMB_a": rng.uniform(-2.0, 1.0, (ny, nx)), "BMB_a": rng.uniform(-3.0, 0.5, (ny, nx)),
         "u_vav_cx": rng.uniform(-400.0, 400.0, (ny, nx - 1)), "v_vav_cy": rng.uniform(-400.0, 400.0, (ny - 1, nx))}
    cfg = {"choice_ice_dynamics": dyn, "ice_thickness_west_BC": bc[0], "ice_thickness_east_BC": bc[1],
           "ice_thickness_south_BC": bc[2], "ice_thickness_north_BC": bc[3]}
    ctx = diva.Context(g, cfg, backend)
    ctx.upload({k: np.asfortranarray(v) for k, v in f.items()})
    ctx.update_general_ice_model_data()
    ctx.determine_floating_margin_fraction()
    return ctx


BCS = [("zero", "zero", "zero", "zero"), ("infinite", "periodic", "fixed", "none"),
       ("periodic", "infinite", "infinite", "zero")]


@pytest.mark.parametrize("bc", BCS)
def test_calc_dHi_dt_bit_exact(cuda, oracle, bc):
    out = []
    for be in (cuda, oracle):
        ctx = random_case(be, 3, bc)
        ctx.calc_dHi_dt(2.5)
        out.append(ctx.download(THICK + ["mask_cf_a"]))
        ctx.close()
    for k in THICK:
        assert np.array_equal(out[0][k], out[1][k]), k


def test_critical_timestep_bit_exact(cuda, oracle):
    v = []
    for be in (cuda, oracle):
        ctx = random_case(be, 4, BCS[0])
        v.append((ctx.calc_critical_timestep_adv(10.0), ctx.calc_critical_timestep_adv(1e-3)))
        ctx.close()
    assert v[0] == v[1]


def test_predictor_corrector_stages_bit_exact(cuda, oracle):
    names = ["Hi_a", "Hi_pred", "Hi_old", "Hi_corr", "dHi_dt_a", "dHidt_Hn_un", "dHidt_Hnm1_unm1",
             "dHidt_Hstarnp1_unp1", "pc_tau", "Hi_tplusdt_a", "mask_ice_a", "mask_gl_a", "float_margin_frac_a"]
    out, eta = [], []
    for be in (cuda, oracle):
        ctx = random_case(be, 5, BCS[1])
        ctx.pc_predictor(1.5, 1.2)
        e = ctx.pc_corrector(1.5, 1.2, 1e-8)
        ctx.pc_finish(1.0)
        out.append(ctx.download(names))
        eta.append(e)
        ctx.close()
    assert eta[0] == eta[1]
    for k in names:
        assert np.array_equal(out[0][k], out[1][k]), k


def test_time_steps_against_the_oracle(cuda, oracle):
    """Four predictor/corrector steps of the marine channel at 20 km, each side solving
    its own velocities to the nonlinear rel-res 1e-8 (linear solves to 1e-12, so both
    sit on the same fixed point whatever their iteration counts): the same time steps,
    thickness and velocities to that tolerance."""
    g, cfg, f = synth.marine_channel(dx=20e3)
    f = dict(f)
    f["SMB_a"] = np.asfortranarray(np.full_like(f["Hi_a"], 0.3))
    f["BMB_a"] = np.asfortranarray(np.where(f["Hb_a"] < -400.0, -1.0, 0.0))
    cfg = dict(cfg, lin_rtol=1e-12, picard_stop="relres", picard_relres_tol=1e-8, DIVA_visc_it_nit=500,
               ice_thickness_west_BC="infinite", ice_thickness_east_BC="zero",
               ice_thickness_south_BC="infinite", ice_thickness_north_BC="infinite")
    res = []
    for be in (cuda, oracle):
        ctx = diva.Context(diva.Grid(**g), cfg, be)
        if be is oracle:
            ob.set_linear_solver(ctx, ob.LIN_GMRES_WARM, 1e-12, 0.0)
        helpers.prepare(ctx, f)
        ctx.determine_floating_margin_fraction()
        pc = dynamics.PCTimeStepper(ctx, start_time=0.0, end_time=1000.0)
        dts = [pc.step() for _ in range(4)]
        res.append((dts, pc.pc_eta, ctx.download(["Hi_a", "u_vav_cx", "v_vav_cy"]), pc.reports))
        ctx.close()
    (d0, e0, o0, _), (d1, e1, o1, _) = res
    assert all(r["status"] == 0 for r in res[0][3]) and all(r["status"] == 0 for r in res[1][3])
    np.testing.assert_allclose(d0, d1, rtol=1e-9)
    assert helpers.rel_l2(o0["Hi_a"], o1["Hi_a"]) <= 1e-5
    assert helpers.rel_l2(np.concatenate([o0["u_vav_cx"].ravel(), o0["v_vav_cy"].ravel()]),
                          np.concatenate([o1["u_vav_cx"].ravel(), o1["v_vav_cy"].ravel()])) <= 1e-5


@pytest.mark.parametrize("case", ["grounded", "shelf"])
def test_semiimplicit_matches_the_oracle(cuda, oracle, case):
    """The semi-implicit thickness solve: the oracle eliminates exactly, the GPU runs
    BiCGStab to dHi_rtol = 1e-13; all row types (mass-balance-only, explicit next to the
    calving front, over-implicit) on the shelf case."""
    import test_thickness
    out = []
    for be in (cuda, oracle):
        if case == "grounded":
            ctx, g = test_thickness.grounded_case(be, "semi-implicit")
        else:
            ctx = random_case(be, 6, ("none", "none", "none", "none"))
            ctx.set_config({"choice_ice_integration_method": "semi-implicit", "dHi_rtol": 1e-13,
                            "choice_ice_dynamics": "DIVA", "ice_thickness_west_BC": "none",
                            "ice_thickness_east_BC": "none", "ice_thickness_south_BC": "none",
                            "ice_thickness_north_BC": "none"})
        ctx.calc_dHi_dt(20.0)
        out.append(ctx.download(["Hi_tplusdt_a", "dHi_dt_a"]))
        ctx.close()
    np.testing.assert_allclose(out[0]["Hi_tplusdt_a"], out[1]["Hi_tplusdt_a"], rtol=1e-10, atol=1e-8)
    np.testing.assert_allclose(out[0]["dHi_dt_a"], out[1]["dHi_dt_a"], rtol=1e-9, atol=1e-9)


def test_unconnected_shelves_match_the_oracle(cuda, oracle):
    import test_thickness
    out = []
    for be in (cuda, oracle):
        ctx, _ = test_thickness.island_case(be)
        ctx.pc_finish(1.0)
        out.append(ctx.download(["Hi_a", "mask_ice_a", "mask_shelf_a", "mask_ice_a_prev", "float_margin_frac_a"]))
        ctx.close()
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k


@pytest.mark.parametrize("flag", ["fixed_shelf_geometry", "fixed_sheet_geometry", "fixed_grounding_line",
                                  "do_remove_shelves"])
def test_update_ice_thickness_options_bit_exact(cuda, oracle, flag):
    import test_thickness
    out = [test_thickness.options_case(be, flag)[1] for be in (cuda, oracle)]
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k


@pytest.mark.parametrize("law", ["none", "threshold_thickness"])
def test_calving_bit_exact(cuda, oracle, law):
    import test_thickness
    out = []
    for be in (cuda, oracle):
        ctx, _ = test_thickness.calving_case(be, law)
        ctx.pc_finish(1.0)
        out.append(ctx.download(["Hi_a", "mask_ice_a", "mask_cf_a", "Hi_eff_cf_a", "float_margin_frac_a"]))
        ctx.close()
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k


@pytest.mark.parametrize("flag", ["remove_shelves_larger_than_PD", "continental_shelf_calving"])
def test_reference_geometry_removal_bit_exact(cuda, oracle, flag):
    import test_thickness
    out = []
    for be in (cuda, oracle):
        ctx, _ = test_thickness.refgeo_case(be, flag)
        ctx.pc_finish(1.0)
        out.append(ctx.download(["Hi_a", "mask_ice_a", "mask_shelf_a"]))
        ctx.close()
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k


def test_prescribed_retreat_mask_bit_exact(cuda, oracle):
    import test_thickness
    out = []
    for be in (cuda, oracle):
        ctx = test_thickness.retreat_case(be)[0]
        ctx.apply_prescribed_retreat_mask(25.0, 0.0, 100.0)
        out.append(ctx.download(["Hi_a", "ice_fraction_retreat_mask_a", "mask_ice_a"]))
        ctx.close()
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k


def test_critical_timestep_sia_bit_exact(cuda, oracle):
    """From the oracle's state after solve_SIA, both sides' calc_critical_timestep_SIA
    agree exactly (same vertical averages in the same order, no FMA contraction)."""
    g, cfg, f = synth.ice_cap(dx=40e3)
    cfg = dict(cfg, choice_ice_dynamics="SIA")
    ctx = diva.Context(diva.Grid(**g), cfg, oracle)
    helpers.prepare(ctx, f)
    ctx.solve_SIA()
    state = ctx.download()
    dts = [ctx.calc_critical_timestep_SIA(10.0)]
    ctx.close()
    ctx = diva.Context(diva.Grid(**g), cfg, cuda)
    ctx.upload(state)
    dts.append(ctx.calc_critical_timestep_SIA(10.0))
    ctx.close()
    assert dts[0] == dts[1] and 0.0 < dts[0] <= 9.0
