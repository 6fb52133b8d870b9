"""The device 3D heat equation against the oracle through the C ABI, from identical
states: the column solves, the bed and shelf conditions, frictional heating, the new-ice
columns and the Robin replacement.  The arithmetic is the same sequence on both sides;
exp (conductivity, rate factor) and erf (Robin profile) are each side's library, so
temperatures agree to a few ulps rather than bit for bit."""
import numpy as np
import pytest

from imau_ice_b200 import diva, synth
import helpers
import oracle_backend as ob
import test_thermo  # noqa: E402  (the slab geometry of the CPU tests)

pytestmark = pytest.mark.gpu

EXACT = ["frictional_heating_a", "dHs_dt_a", "dzeta_dt_a", "dzeta_dx_a", "dzeta_dy_a", "dzeta_dz_a", "Cpi_a"]
CLOSE = ["Ti_a", "Ki_a", "A_flow_3D_a", "Ti_pmp_a"]


def compare(og, oo):
    for k in EXACT:
        assert np.array_equal(og[k], oo[k], equal_nan=True), k
    for k in CLOSE:
        np.testing.assert_allclose(og[k], oo[k], rtol=1e-12, atol=0, err_msg=k)


def test_heat_equation_after_a_solve_matches_the_oracle(cuda, oracle):
    g, cfg, f = synth.marine_channel(dx=20e3)
    f = dict(f)
    ny, nx = f["Hi_a"].shape
    f["T_surf_annual_a"] = np.asfortranarray(np.full((ny, nx), 243.0))
    f["GHF_a"] = np.asfortranarray(np.full((ny, nx), 1.7e6))
    f["SMB_a"] = np.asfortranarray(np.full((ny, nx), 0.3))
    f["mask_ice_a_prev"] = np.ones((ny, nx), dtype=np.int32, order="F")
    grid = diva.Grid(**g)
    cfg = dict(cfg, lin_rtol=1e-10)
    ctx = diva.Context(grid, cfg, oracle)
    ob.set_linear_solver(ctx, ob.LIN_GMRES_WARM, 1e-10, 0.0)
    helpers.prepare(ctx, f)
    ctx.solve_DIVA()
    state = ctx.download()
    n_o = ctx.run_thermo_model(True)
    oo = ctx.download()
    ctx.close()
    ctx = diva.Context(grid, cfg, cuda)
    ctx.upload(state)                                 # the oracle's post-solve state, field for field
    n_g = ctx.run_thermo_model(True)
    og = ctx.download()
    ctx.close()
    assert n_g == n_o == 0
    compare(og, oo)


@pytest.mark.parametrize("case", ["steady", "robin", "new_ice", "shelf_ocean_input"])
def test_slab_cases_match_the_oracle(cuda, oracle, case):
    g, f = test_thermo.slab()
    cfg = {"choice_ice_heat_capacity": "uniform", "choice_ice_thermal_conductivity": "uniform",
           "choice_sliding_law": "no_sliding", "dt_thermo": 1e12 if case == "steady" else 10.0}
    if case == "robin":
        f["T_surf_annual_a"][7, 8] = 100.0
        f["T_surf_annual_a"][12, 3] = 90.0
    if case == "new_ice":
        f["mask_ice_a_prev"][4, 5] = 0
        f["Ti_a"][:, 4, 4] = np.linspace(250.0, 260.0, g.nz)
        cfg.update(choice_ice_heat_capacity="Pounder1965", choice_ice_thermal_conductivity="Ritz1987")
    if case == "shelf_ocean_input":                   # a floating slab, the shelf-base temperature
        f["Hb_a"] = np.full(f["Hi_a"].shape, -3000.0)  # from T_ocean_base_a, one Robin column on it
        f["T_ocean_base_a"] = np.random.default_rng(7).uniform(-3.0, -2.0, f["Hi_a"].shape)
        f["T_surf_annual_a"][7, 8] = 100.0
        cfg.update(ocean_temperature_input=1)
    out, n = [], []
    for be in (cuda, oracle):
        ctx = diva.Context(g, cfg, be)
        ctx.upload({k: np.asfortranarray(v) for k, v in f.items()})
        ctx.update_general_ice_model_data()
        ctx.calc_pressure_melting_point()
        ctx.upload({"u_vav_cx": np.full((g.ny, g.nx - 1), 5.0)})
        n.append(ctx.run_thermo_model(True))
        out.append(ctx.download())
        ctx.close()
    assert n[0] == n[1]
    compare(out[0], out[1])


def test_coupled_time_steps_match_the_oracle(cuda, oracle):
    """Predictor/corrector steps with the thermodynamics event on both sides, each solving
    its own velocities to the nonlinear rel-res 1e-8: time steps, thickness and
    temperature agree to that tolerance."""
    from imau_ice_b200 import dynamics
    g, cfg, f = synth.marine_channel(dx=20e3)
    f = dict(f)
    ny, nx = f["Hi_a"].shape
    for k, v in (("SMB_a", 0.3), ("BMB_a", 0.0), ("T_surf_annual_a", 243.0), ("GHF_a", 1.7e6)):
        f[k] = np.asfortranarray(np.full((ny, nx), v))
    f["mask_ice_a_prev"] = np.ones((ny, nx), dtype=np.int32, order="F")
    cfg = dict(cfg, lin_rtol=1e-12, picard_stop="relres", picard_relres_tol=1e-8, DIVA_visc_it_nit=500,
               dt_thermo=0.02, ice_thickness_west_BC="infinite", ice_thickness_east_BC="zero",
               ice_thickness_south_BC="infinite", ice_thickness_north_BC="infinite")
    res = []
    for be in (cuda, oracle):
        ctx = diva.Context(diva.Grid(**g), cfg, be)
        if be is oracle:
            ob.set_linear_solver(ctx, ob.LIN_GMRES_WARM, 1e-12, 0.0)
        helpers.prepare(ctx, f)
        ctx.determine_floating_margin_fraction()
        pc = dynamics.PCTimeStepper(ctx, 0.0, 1000.0, thermo=True)
        dts = [pc.step() for _ in range(4)]
        res.append((dts, pc.thermo_solves, ctx.download(["Hi_a", "Ti_a"])))
        ctx.close()
    (d0, n0, o0), (d1, n1, o1) = res
    assert n0 == n1 >= 1
    np.testing.assert_allclose(d0, d1, rtol=1e-9)
    assert helpers.rel_l2(o0["Hi_a"], o1["Hi_a"]) <= 1e-5
    assert helpers.rel_l2(o0["Ti_a"], o1["Ti_a"]) <= 1e-9
