"""The explicit ice-thickness update and the predictor/corrector stages on the CPU
oracle: an independent NumPy restatement of calc_dHi_dt_explicit
(ice_thickness_module.f90:65-300), known answers of the boundary conditions
(:728-931) and of the advective time-step limit (ice_dynamics_module.f90:726-762),
mass conservation, and a few predictor/corrector steps (:243-432)."""
import numpy as np
import pytest

from imau_ice_b200 import diva, dynamics, synth
import helpers
import oracle_backend as ob

RHO_I, RHO_SW = 910.0, 1028.0


def small_case(seed=0, nx=11, ny=9, dx=10e3, bc="none", dyn="DIVA"):
    rng = np.random.default_rng(seed)
    g = diva.Grid(nx, ny, dx)
    Hb = rng.uniform(-600.0, 400.0, (ny, nx))
    H = np.where(rng.random((ny, nx)) < 0.8, rng.uniform(50.0, 1500.0, (ny, nx)), 0.0)
    f = {"Hi_a": H, "Hb_a": Hb, "SL_a": np.zeros((ny, nx)), "Ti_a": np.full((g.nz, ny, nx), 260.0),
         "SMB_a": rng.uniform(-2.0, 1.0, (ny, nx)), "BMB_a": rng.uniform(-3.0, 0.5, (ny, nx)),
         "u_vav_cx": rng.uniform(-400.0, 400.0, (ny, nx - 1)), "v_vav_cy": rng.uniform(-400.0, 400.0, (ny - 1, nx))}
    cfg = {"choice_ice_dynamics": dyn, "ice_thickness_west_BC": bc, "ice_thickness_east_BC": bc,
           "ice_thickness_south_BC": bc, "ice_thickness_north_BC": bc}
    ctx = diva.Context(g, cfg, ob.oracle_backend())
    ctx.upload({k: np.asfortranarray(v) for k, v in f.items()})
    ctx.update_general_ice_model_data()
    ctx.determine_floating_margin_fraction()
    return ctx, g


def numpy_dHi_dt(o, dx, dt):
    """calc_dHi_dt_explicit restated with NumPy (the outflux limitation as the reference's
    sequential in-place loop, i outer and j inner)."""
    H, u, v = o["Hi_a"], o["u_vav_cx"], o["v_vav_cy"]
    ny, nx = H.shape
    Qx = u * np.where(u > 0, H[:, :-1], H[:, 1:]) * dx * dt
    Qy = v * np.where(v > 0, H[:-1, :], H[1:, :]) * dx * dt
    msmb = o["SMB_a"] + o["BMB_a"]
    cf_shelf = (o["mask_cf_a"] == 1) & (o["mask_shelf_a"] == 1)
    open_ocean = (o["mask_ocean_a"] == 1) & (o["mask_shelf_a"] == 0)
    mb = np.where(cf_shelf, msmb * dx * dx * dt * o["float_margin_frac_a"],
                  np.where(open_ocean, 0.0, msmb * dx * dx * dt))
    for i in range(nx):
        for j in range(ny):
            avail = H[j, i] * dx * dx
            out = 0.0
            if i > 0 and not Qx[j, i - 1] > 0: out -= Qx[j, i - 1]
            if i < nx - 1 and not Qx[j, i] < 0: out += Qx[j, i]
            if j > 0 and not Qy[j - 1, i] > 0: out -= Qy[j - 1, i]
            if j < ny - 1 and not Qy[j, i] < 0: out += Qy[j, i]
            r = 1.0
            if -mb[j, i] >= avail:
                mb[j, i] = -avail
                r = 0.0
            if out > avail + mb[j, i]:
                r = (avail + mb[j, i]) / out
            if r < 1.0:
                if i > 0 and Qx[j, i - 1] < 0: Qx[j, i - 1] *= r
                if i < nx - 1 and Qx[j, i] > 0: Qx[j, i] *= r
                if j > 0 and Qy[j - 1, i] < 0: Qy[j - 1, i] *= r
                if j < ny - 1 and Qy[j, i] > 0: Qy[j, i] *= r
    den = dx * dx * dt
    d = mb / den
    d[:, 1:] = d[:, 1:] + Qx / den
    d[:, :-1] = d[:, :-1] - Qx / den
    d[1:, :] = d[1:, :] + Qy / den
    d[:-1, :] = d[:-1, :] - Qy / den
    d = np.maximum(d, -H / dt)
    return Qx, Qy, d, H + d * dt


@pytest.mark.parametrize("seed", range(3))
def test_explicit_update_matches_a_numpy_restatement(seed):
    ctx, g = small_case(seed)
    dt = 2.5
    ctx.calc_dHi_dt(dt)
    o = ctx.download()
    Qx, Qy, d, Hn = numpy_dHi_dt(o, g.dx, dt)
    # the column sums in d are accumulated in the reference's term order only up to
    # reassociation, so 1e-12; fluxes are elementwise and exact
    np.testing.assert_array_equal(o["Qx_cx"], Qx)
    np.testing.assert_array_equal(o["Qy_cy"], Qy)
    np.testing.assert_allclose(o["dHi_dt_a"], d, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(o["Hi_tplusdt_a"], Hn, rtol=1e-12, atol=1e-9)
    assert o["Hi_tplusdt_a"].min() >= -1e-9                    # outfluxes were limited


def test_explicit_update_conserves_mass():
    ctx, g = small_case(5)
    dt = 1.0
    ctx.calc_dHi_dt(dt)
    o = ctx.download()
    # fluxes only cross interior faces: the volume change is the applied mass balance,
    # wherever the -Hi/dt floor did not act
    Qx, Qy, d, Hn = numpy_dHi_dt(o, g.dx, dt)
    floor = np.isclose(o["dHi_dt_a"], -o["Hi_a"] / dt)
    vol = (o["Hi_tplusdt_a"] - o["Hi_a"]).sum() * g.dx ** 2
    div = np.zeros_like(o["Hi_a"])
    div[:, 1:] += o["Qx_cx"]; div[:, :-1] -= o["Qx_cx"]; div[1:, :] += o["Qy_cy"]; div[:-1, :] -= o["Qy_cy"]
    mb = (o["dHi_dt_a"] * dt * g.dx ** 2 - div)
    assert abs(div.sum()) <= 1e-6 * np.abs(o["Qx_cx"]).sum()
    assert np.isclose(vol, mb.sum() + div.sum(), rtol=1e-10)
    assert floor.sum() < floor.size


def test_thickness_boundary_conditions():
    ny, nx = 9, 11
    for bc, check in [
        ("zero", lambda o: np.all(o["Hi_tplusdt_a"][:, :2] == 0) and np.all(o["Hi_tplusdt_a"][:2, :] == 0)
         and np.all(o["Hi_tplusdt_a"][:, -2:] == 0) and np.all(o["Hi_tplusdt_a"][-2:, :] == 0)),
        ("fixed", lambda o: np.all(o["Hi_tplusdt_a"][:, 0] == o["Hi_a"][:, 0]) and np.all(o["dHi_dt_a"][0, :] == 0)),
        ("periodic", lambda o: np.all(o["Hi_tplusdt_a"][1:-1, 0] == o["Hi_a"][1:-1, nx - 2])
         and np.all(o["Hi_tplusdt_a"][-1, :] == o["Hi_a"][1, :])),
    ]:
        ctx, g = small_case(1, nx=nx, ny=ny, bc=bc)
        ctx.calc_dHi_dt(1.0)
        assert check(ctx.download()), bc
    # 'infinite': the edge cell takes the surface of its inner neighbour at t + dt
    ctx, g = small_case(2, nx=nx, ny=ny, bc="none")
    ctx.set_config({"choice_ice_dynamics": "DIVA", "ice_thickness_west_BC": "infinite", "ice_thickness_east_BC": "none",
                    "ice_thickness_south_BC": "none", "ice_thickness_north_BC": "none"})
    ctx.calc_dHi_dt(1.0)
    o = ctx.download()
    Hn, Hb, SL = o["Hi_tplusdt_a"], o["Hb_a"], o["SL_a"]
    Hs_in = Hn[:, 1] + np.maximum(SL[:, 1] - RHO_I / RHO_SW * Hn[:, 1], Hb[:, 1])
    Hs_float = Hb[:, 0] + (SL[:, 0] - Hb[:, 0]) * RHO_SW / RHO_I
    expect = np.where(Hs_in > Hs_float, Hs_in - Hb[:, 0], (Hs_in - SL[:, 0]) / (1.0 - RHO_I / RHO_SW))
    np.testing.assert_allclose(Hn[:, 0], expect, rtol=1e-14)
    # with SIA dynamics only the edge row/column is zeroed
    ctx, g = small_case(1, nx=nx, ny=ny, bc="zero", dyn="SIA")
    ctx.calc_dHi_dt(1.0)
    o = ctx.download()
    assert np.all(o["Hi_tplusdt_a"][:, 0] == 0) and np.any(o["Hi_tplusdt_a"][2:-2, 1] != 0)


def test_critical_timestep_known_answer():
    ctx, g = small_case(0)
    u = np.full((g.ny, g.nx - 1), 100.0)
    v = np.zeros((g.ny - 1, g.nx))
    v[3, 4] = -300.0
    ctx.upload({"u_vav_cx": u, "v_vav_cy": v})
    assert ctx.calc_critical_timestep_adv(10.0) == min(10.0, 0.9 * g.dx / 400.0)
    assert ctx.calc_critical_timestep_adv(1e-3) == 1e-3                    # capped at dt_max


def test_floating_margin_fraction_known_answer():
    ny, nx = 7, 7
    g = diva.Grid(nx, ny, 1e3)
    H = np.zeros((ny, nx))
    H[:, :3] = 400.0            # a shelf ...
    H[3, 3] = 100.0             # ... and a thin calving-front cell beyond it
    f = {"Hi_a": H, "Hb_a": np.full((ny, nx), -1000.0), "SL_a": np.zeros((ny, nx)),
         "Ti_a": np.full((g.nz, ny, nx), 260.0)}
    ctx = diva.Context(g, {}, ob.oracle_backend())
    ctx.upload({k: np.asfortranarray(v) for k, v in f.items()})
    ctx.update_general_ice_model_data()
    ctx.determine_floating_margin_fraction()
    o = ctx.download(["float_margin_frac_a", "Hi_eff_cf_a", "mask_cf_a"])
    assert o["mask_cf_a"][3, 3] == 1
    # its non-front ice neighbours are the interior shelf cells of column 1 (400 m)
    assert o["float_margin_frac_a"][3, 3] == 100.0 / 400.0 and o["Hi_eff_cf_a"][3, 3] == 400.0
    assert o["float_margin_frac_a"][3, 5] == 0.0 and o["float_margin_frac_a"][3, 1] == 1.0


def test_predictor_corrector_steps_on_the_oracle():
    g, cfg, f = synth.marine_channel(dx=20e3)
    f = dict(f)
    f["SMB_a"] = np.asfortranarray(np.full_like(f["Hi_a"], 0.3))
    f["BMB_a"] = np.asfortranarray(np.where(f["Hb_a"] < -400.0, -1.0, 0.0))
    cfg = dict(cfg, lin_rtol=1e-10, ice_thickness_west_BC="infinite", ice_thickness_east_BC="zero",
               ice_thickness_south_BC="infinite", ice_thickness_north_BC="infinite")
    ctx = diva.Context(diva.Grid(**g), cfg, ob.oracle_backend())
    ob.set_linear_solver(ctx, ob.LIN_GMRES_WARM, 1e-10, 0.0)
    helpers.prepare(ctx, f)
    ctx.determine_floating_margin_fraction()
    pc = dynamics.PCTimeStepper(ctx, start_time=0.0, end_time=1000.0)
    H0 = ctx.download(["Hi_a"])["Hi_a"].copy()
    n = pc.run(max_steps=4)
    o = ctx.download(["Hi_a", "pc_tau", "dHi_dt_a"])
    assert n == 4 and len(pc.reports) == 4
    assert pc.time > 0.0 and pc.dt_crit_ice >= pc.dt_min
    assert o["Hi_a"].min() >= 0.0 and np.isfinite(o["Hi_a"]).all()
    change = np.abs(o["Hi_a"] - H0)
    assert np.all(o["Hi_a"][:, -2:] == 0.0)                        # the 'zero' east edge (two columns, DIVA)
    assert 0.0 < change[2:-2, 2:-2].max() < 50.0                    # a few years of flow inside
    assert pc.pc_eta >= pc.pc_eta_min and np.isfinite(pc.pc_eta)


def test_restart_file_continues_the_run(tmp_path):
    """A restart written after a solve and a time step, read into a new context, continues
    exactly as the original context does."""
    g, cfg, f = synth.marine_channel(dx=20e3)
    f = dict(f)
    f["SMB_a"] = np.asfortranarray(np.full_like(f["Hi_a"], 0.3))
    cfg = dict(cfg, lin_rtol=1e-10, ice_thickness_west_BC="infinite", ice_thickness_east_BC="zero",
               ice_thickness_south_BC="infinite", ice_thickness_north_BC="infinite")
    ctx = diva.Context(diva.Grid(**g), cfg, ob.oracle_backend())
    ob.set_linear_solver(ctx, ob.LIN_GMRES_WARM, 1e-10, 0.0)
    helpers.prepare(ctx, f)
    ctx.determine_floating_margin_fraction()
    pc = dynamics.PCTimeStepper(ctx, 0.0, 1000.0)
    pc.step()
    path = tmp_path / "restart.npz"
    ctx.save_restart(path)
    ctx2 = diva.Context.load_restart(path, ob.oracle_backend())
    ob.set_linear_solver(ctx2, ob.LIN_GMRES_WARM, 1e-10, 0.0)
    r1, r2 = ctx.solve_DIVA(), ctx2.solve_DIVA()
    a, b = ctx.download(), ctx2.download()
    assert r1["picard_iterations"] == r2["picard_iterations"]
    for k in a:
        assert np.array_equal(a[k], b[k], equal_nan=True), k


def grounded_case(backend, method, seed=7, nx=13, ny=11, dx=10e3):
    rng = np.random.default_rng(seed)
    g = diva.Grid(nx, ny, dx)
    f = {"Hi_a": rng.uniform(500.0, 1500.0, (ny, nx)), "Hb_a": np.full((ny, nx), 200.0), "SL_a": np.zeros((ny, nx)),
         "Ti_a": np.full((g.nz, ny, nx), 260.0), "SMB_a": rng.uniform(-1.0, 1.0, (ny, nx)),
         "BMB_a": np.zeros((ny, nx)), "u_vav_cx": rng.uniform(-300.0, 300.0, (ny, nx - 1)),
         "v_vav_cy": rng.uniform(-300.0, 300.0, (ny - 1, nx))}
    cfg = {"choice_ice_integration_method": method, "dHi_rtol": 1e-13}
    for side in ("west", "east", "south", "north"):
        cfg[f"ice_thickness_{side}_BC"] = "none"
    ctx = diva.Context(g, cfg, backend)
    ctx.upload({k: np.asfortranarray(v) for k, v in f.items()})
    ctx.update_general_ice_model_data()
    ctx.determine_floating_margin_fraction()
    return ctx, g


def test_semiimplicit_conserves_mass_and_reduces_to_the_mass_balance():
    ctx, g = grounded_case(ob.oracle_backend(), "semi-implicit")
    dt = 20.0
    ctx.calc_dHi_dt(dt)
    o = ctx.download(["Hi_a", "Hi_tplusdt_a", "SMB_a", "dHi_dt_a"])
    # every cell is an over-implicit row and the fluxes are conservative across faces
    assert np.isclose((o["Hi_tplusdt_a"] - o["Hi_a"]).sum(), dt * o["SMB_a"].sum(), rtol=1e-10, atol=1e-6)
    np.testing.assert_allclose(o["dHi_dt_a"], (o["Hi_tplusdt_a"] - o["Hi_a"]) / dt, rtol=1e-14)
    # with the ice at rest the row is (1/dt) x = MB + H/dt
    ctx.upload({"u_vav_cx": np.zeros((g.ny, g.nx - 1)), "v_vav_cy": np.zeros((g.ny - 1, g.nx))})
    ctx.calc_dHi_dt(dt)
    o = ctx.download(["Hi_a", "Hi_tplusdt_a", "SMB_a"])
    np.testing.assert_allclose(o["Hi_tplusdt_a"], o["Hi_a"] + o["SMB_a"] * dt, rtol=1e-13)


def test_semiimplicit_approaches_the_explicit_scheme_for_small_steps():
    out = {}
    for m in ("explicit", "semi-implicit"):
        ctx, g = grounded_case(ob.oracle_backend(), m)
        ctx.calc_dHi_dt(1e-3)
        out[m] = ctx.download(["dHi_dt_a"])["dHi_dt_a"]
    np.testing.assert_allclose(out["semi-implicit"], out["explicit"], rtol=1e-3, atol=1e-3)


def test_semiimplicit_row_types_on_a_shelf():
    """Mass-balance-only cells (no ice nearby), explicit cells (shelf next to open ocean and
    open ocean next to the shelf) and over-implicit cells side by side."""
    ctx, g = small_case(4, bc="none")
    ctx.set_config({"choice_ice_integration_method": "semi-implicit", "choice_ice_dynamics": "DIVA",
                    "ice_thickness_west_BC": "none", "ice_thickness_east_BC": "none",
                    "ice_thickness_south_BC": "none", "ice_thickness_north_BC": "none"})
    ctx.calc_dHi_dt(5.0)
    o = ctx.download(["Hi_tplusdt_a", "dHi_dt_a", "mask_ice_a"])
    assert np.isfinite(o["Hi_tplusdt_a"]).all() and o["Hi_tplusdt_a"].min() >= 0.0


def island_case(backend):
    """Grounded ice in the west, a shelf attached to it, and a floating island (not
    4-connected to the attached shelf) in the east; a no-ice patch on the grounded part."""
    ny, nx = 15, 21
    g = diva.Grid(nx, ny, 10e3)
    Hb = np.full((ny, nx), -800.0)
    Hb[:, :6] = 300.0
    H = np.zeros((ny, nx))
    H[2:-2, :10] = 400.0                 # sheet (x < 6) and the shelf attached to it
    H[5:9, 13:17] = 300.0                # the floating island
    H[6:8, 10:13] = 0.0
    noice = np.zeros((ny, nx), dtype=np.int32)
    noice[3, 2] = 1
    f = {"Hi_a": H, "Hb_a": Hb, "SL_a": np.zeros((ny, nx)), "Ti_a": np.full((g.nz, ny, nx), 260.0),
         "mask_noice_a": noice}
    ctx = diva.Context(g, {}, backend)
    ctx.upload({k: np.asfortranarray(v) for k, v in f.items()})
    ctx.update_general_ice_model_data()
    ctx.determine_floating_margin_fraction()
    return ctx, H


def test_unconnected_shelves_and_the_no_ice_mask_lose_their_ice():
    ctx, H = island_case(ob.oracle_backend())
    ctx.pc_finish(1.0)                                # dHi_dt_a = 0: only the geometry clean-up acts
    o = ctx.download(["Hi_a", "mask_ice_a_prev"])
    assert np.all(o["Hi_a"][5:9, 13:17] == 0.0)     # the island is gone
    assert np.all(o["Hi_a"][2:-2, 6:10][H[2:-2, 6:10] > 0] == 400.0)   # the attached shelf stays
    assert o["Hi_a"][3, 2] == 0.0 and o["Hi_a"][4, 2] == 400.0         # the no-ice mask
    assert o["mask_ice_a_prev"][6, 14] == 1                             # the step's ice mask kept


OPTIONS = ["fixed_shelf_geometry", "fixed_sheet_geometry", "fixed_grounding_line", "do_remove_shelves"]


def options_case(backend, flag):
    """The island case with dHi_dt_a = 1 m/yr everywhere and one option of
    update_ice_thickness (ice_dynamics_module.f90:449-608) switched on; returns the
    masks and thickness before pc_finish(1.0) and the thickness after it."""
    ctx, H = island_case(backend)
    ctx.set_config({flag: 1})
    g = ctx.grid
    ctx.upload({"dHi_dt_a": np.ones((g.ny, g.nx))})
    before = ctx.download(["mask_shelf_a", "mask_sheet_a", "Hi_a"])
    ctx.pc_finish(1.0)
    after = ctx.download(["Hi_a", "mask_ice_a", "mask_shelf_a", "mask_sheet_a", "mask_gl_a",
                          "float_margin_frac_a"])
    ctx.close()
    return before, after


@pytest.mark.parametrize("flag", OPTIONS)
def test_update_ice_thickness_options(flag):
    """Fixed shelf / sheet / grounding-line geometry keep Hi_a (ice_dynamics_module.f90:
    465-530: the masked cells and their 8-neighbours across the grounding line); the
    others take dHi_dt_a; do_remove_shelves zeroes every floating cell (:600-606)."""
    from scipy.ndimage import binary_dilation
    before, o = options_case(ob.oracle_backend(), flag)
    shelf, sheet, H0 = before["mask_shelf_a"] == 1, before["mask_sheet_a"] == 1, before["Hi_a"]
    near_shelf = binary_dilation(shelf, np.ones((3, 3), bool))
    near_sheet = binary_dilation(sheet, np.ones((3, 3), bool))
    kept = {"fixed_shelf_geometry": shelf | (sheet & near_shelf),
            "fixed_sheet_geometry": sheet | (shelf & near_sheet),
            "fixed_grounding_line": (sheet & near_shelf) | (shelf & near_sheet),
            "do_remove_shelves": np.zeros_like(shelf)}[flag]
    grounded = sheet & (H0 > 0)
    grounded[3, 2] = False                                # the no-ice cell
    assert o["Hi_a"][3, 2] == 0.0
    if flag == "do_remove_shelves":
        assert np.all(o["Hi_a"][shelf] == 0.0)
        np.testing.assert_array_equal(o["Hi_a"][grounded], H0[grounded] + 1.0)
        return
    np.testing.assert_array_equal(o["Hi_a"][grounded & kept], H0[grounded & kept])
    np.testing.assert_array_equal(o["Hi_a"][grounded & ~kept], H0[grounded & ~kept] + 1.0)


def calving_case(backend, law):
    """A grounded sheet (x < 5), a 400 m shelf thinning to 180 / 150 / 120 m over its
    last three columns, open ocean beyond; dHi_dt_a = 0."""
    ny, nx = 7, 20
    g = diva.Grid(nx, ny, 10e3)
    Hb = np.full((ny, nx), -800.0)
    Hb[:, :5] = 300.0
    H = np.zeros((ny, nx))
    H[:, :14] = np.where(np.arange(14) < 5, 600.0, 400.0)
    H[:, 14], H[:, 15], H[:, 16] = 180.0, 150.0, 120.0
    f = {"Hi_a": H, "Hb_a": Hb, "SL_a": np.zeros((ny, nx)), "Ti_a": np.full((g.nz, ny, nx), 260.0)}
    ctx = diva.Context(g, {"choice_calving_law": law}, backend)
    ctx.upload({k: np.asfortranarray(v) for k, v in f.items()})
    ctx.update_general_ice_model_data()
    ctx.determine_floating_margin_fraction()
    return ctx, H


def test_threshold_thickness_calving_retreats_the_front_two_cells():
    """threshold_thickness_calving (calving_module.f90:62-91) applied twice per update
    (ice_dynamics_module.f90:562-583): the 120 m front column goes (its effective
    thickness is its 150 m neighbour's), then the 150 m column (effective 180 m); the
    180 m column waits for the next update.  The domain's edge rows are never calving
    front (the masks leave the border out), so they keep their ice.  With law 'none'
    nothing calves."""
    out = {}
    for law in ("none", "threshold_thickness"):
        ctx, H = calving_case(ob.oracle_backend(), law)
        ctx.pc_finish(1.0)
        out[law] = ctx.download(["Hi_a"])["Hi_a"]
        ctx.close()
    np.testing.assert_array_equal(out["none"], H)
    c = out["threshold_thickness"]
    assert np.all(c[1:-1, 15:] == 0.0)
    np.testing.assert_array_equal(c[1:-1, :15], H[1:-1, :15])
    np.testing.assert_array_equal(c[[0, -1]], H[[0, -1]])


def refgeo_case(backend, flag):
    ctx, H = calving_case(backend, "none")
    ny, nx = H.shape
    Hpd, Bpd = H.copy(), np.full((ny, nx), -800.0)
    Hpd[:, 10:] = 0.0                                  # the present-day front at x = 10
    Heq, Beq = H.copy(), np.full((ny, nx), -800.0)
    Heq[:, 12:] = 0.0
    Beq[:, 12:] = -2500.0                              # beyond the shelf edge from x = 12
    ctx.upload({k: np.asfortranarray(v) for k, v in
                {"Hi_PD_a": Hpd, "Hb_PD_a": Bpd, "Hi_GIAeq_a": Heq, "Hb_GIAeq_a": Beq}.items()})
    ctx.set_config({"choice_calving_law": "none", flag: 1})
    return ctx, H


@pytest.mark.parametrize("flag,edge", [("remove_shelves_larger_than_PD", 10), ("continental_shelf_calving", 12)])
def test_reference_geometry_removal(flag, edge):
    """remove_shelves_larger_than_PD / continental_shelf_calving (ice_dynamics_module.f90:
    613-635): ice goes where the reference geometry has open ocean (PD) or no ice on a bed
    below continental_shelf_min_height (GIA equilibrium)."""
    ctx, H = refgeo_case(ob.oracle_backend(), flag)
    ctx.pc_finish(1.0)
    o = ctx.download(["Hi_a"])["Hi_a"]
    ctx.close()
    assert np.all(o[:, edge:] == 0.0)
    np.testing.assert_array_equal(o[:, :edge], H[:, :edge])


def retreat_case(backend):
    ctx, H = calving_case(backend, "none")
    ny, nx = H.shape
    m0, m1 = np.ones((ny, nx)), np.ones((ny, nx))
    m1[:, 12:] = 0.0                                   # the later frame has retreated to x = 12
    m1[:, 11] = 0.5
    Href = np.full((ny, nx), 300.0)
    ctx.upload({k: np.asfortranarray(v) for k, v in {"ice_fraction_retreat_mask0_a": m0,
                                                      "ice_fraction_retreat_mask1_a": m1,
                                                      "retreat_mask_Hi_ref_a": Href}.items()})
    return ctx, H, m0, m1, Href


def test_prescribed_retreat_mask_caps_the_thickness():
    """apply_prescribed_retreat_mask (calving_module.f90:96-169) a quarter of the way from
    the frame at t0 = 0 to the one at t1 = 100: mask = 0.75 m0 + 0.25 m1; thickness
    capped at Href * mask where the mask is below 0.999 and at interior cells next to
    such a cell; elsewhere untouched."""
    ctx, H, m0, m1, Href = retreat_case(ob.oracle_backend())
    ctx.apply_prescribed_retreat_mask(25.0, 0.0, 100.0)
    o = ctx.download(["Hi_a", "ice_fraction_retreat_mask_a"])
    ctx.close()
    m = 0.75 * m0 + 0.25 * m1
    np.testing.assert_array_equal(o["ice_fraction_retreat_mask_a"], m)
    ny, nx = H.shape
    low = m < 0.999
    near = np.zeros_like(low)
    for dj in (-1, 0, 1):
        for di in (-1, 0, 1):
            near[1:-1, 1:-1] |= np.roll(np.roll(low, dj, 0), di, 1)[1:-1, 1:-1]
    capped = low | near
    want = np.where(capped, np.minimum(H, Href * m), H)
    np.testing.assert_array_equal(o["Hi_a"], want)
    assert capped[3, 10] and not capped[3, 9] and o["Hi_a"][3, 10] == 300.0


def test_bad_arguments_are_rejected_on_the_host():
    """Invalid calls return DIVA_BAD_INPUT before any work: a retreat-mask frame
    interval that is empty or reversed, a negative number of completion sweeps."""
    ctx, _ = calving_case(ob.oracle_backend(), "none")
    for t0, t1 in ((0.0, 0.0), (10.0, 5.0)):
        with pytest.raises(diva.DivaError) as e:
            ctx.apply_prescribed_retreat_mask(1.0, t0, t1)
        assert e.value.status == 4
    with pytest.raises(diva.DivaError) as e:
        ctx.complete_state(-1)
    assert e.value.status == 4
    ctx.close()


def test_critical_timestep_sia_known_answer():
    """calc_critical_timestep_SIA (ice_dynamics_module.f90:651-725) on a sheet with a
    uniform SIA velocity profile: D = |u_vav Hi / dHs_dx| on the x faces, the 3D
    advective limit from u_3D, times 0.9."""
    ny, nx = 9, 11
    g = diva.Grid(nx, ny, 10e3)
    ctx = diva.Context(g, {"choice_ice_dynamics": "SIA"}, ob.oracle_backend())
    f = {"Hi_a": np.full((ny, nx), 1000.0), "Hb_a": np.full((ny, nx), 100.0), "SL_a": np.zeros((ny, nx)),
         "Ti_a": np.full((g.nz, ny, nx), 260.0)}
    ctx.upload({k: np.asfortranarray(v) for k, v in f.items()})
    ctx.update_general_ice_model_data()
    u = np.full((g.nz, ny, nx - 1), 50.0)
    ctx.upload({"u_3D_SIA_cx": np.asfortranarray(u), "v_3D_SIA_cy": np.zeros((g.nz, ny - 1, nx)),
                "dHs_dx_cx": np.full((ny, nx - 1), -2e-3), "dHs_dy_cy": np.full((ny - 1, nx), 1.0),
                "Hi_cx": np.full((ny, nx - 1), 1000.0), "Hi_cy": np.full((ny - 1, nx), 1000.0),
                "u_3D_cx": np.full((g.nz, ny, nx - 1), 20.0), "v_3D_cy": np.full((g.nz, ny - 1, nx), 5.0)})
    dt = ctx.calc_critical_timestep_SIA(100.0)
    D = 50.0 * 1000.0 / 2e-3
    assert dt == pytest.approx(0.9 * min(100.0, 1e8 / (6.0 * D), 1e4 / 25.0), rel=1e-12)
    ctx.close()


@pytest.mark.parametrize("dyn", ["SIA", "SIA/SSA"])
def test_direct_time_stepping(dyn):
    """run_ice_dynamics_direct with SIA or hybrid SIA/SSA: each solve when its event is
    due, the step bounded by the critical time steps and the start-up cap, thickness
    changing."""
    from imau_ice_b200 import dynamics
    g, cfg, f = synth.ice_cap(dx=80e3)
    cfg = dict(cfg, choice_ice_dynamics=dyn)
    f = dict(f)
    f["SMB_a"] = np.asfortranarray(np.full(f["Hi_a"].shape, 0.3))
    ctx = diva.Context(diva.Grid(**g), cfg, ob.oracle_backend())
    helpers.prepare(ctx, f)
    H0 = ctx.download(["Hi_a"])["Hi_a"]
    st = dynamics.DirectTimeStepper(ctx, 0.0, 1000.0, dt_min=0.1, dt_max=10.0, dt_startup_phase=10.0)
    dts = [st.step() for _ in range(4)]
    H1 = ctx.download(["Hi_a"])["Hi_a"]
    ctx.close()
    assert len(st.reports) >= 2 and all(r["status"] == 0 for r in st.reports)
    assert all(0.0 < d <= 10.0 for d in dts) and st.time == pytest.approx(sum(dts))
    assert dts[0] == pytest.approx(0.1)           # the start-up cap at t = 0 is dt_min
    assert np.abs(H1 - H0).max() > 0.0
    with pytest.raises(ValueError):
        dynamics.DirectTimeStepper(diva.Context(diva.Grid(**g), dict(cfg, choice_ice_dynamics="DIVA"),
                                                ob.oracle_backend()), 0.0, 10.0)


def test_direct_time_stepping_with_the_heat_equation():
    """The thermodynamics event of the direct scheme: run_thermo_model every step, the
    heat equation when dt_thermo has elapsed, and the step cut at that event."""
    from imau_ice_b200 import dynamics
    g, cfg, f = synth.ice_cap(dx=80e3)
    cfg = dict(cfg, choice_ice_dynamics="SIA", dt_thermo=0.25)
    f = dict(f)
    ny, nx = f["Hi_a"].shape
    for k, v in (("SMB_a", 0.3), ("T_surf_annual_a", 245.0), ("GHF_a", 1.7e6)):
        f[k] = np.asfortranarray(np.full((ny, nx), v))
    f["mask_ice_a_prev"] = np.ones((ny, nx), dtype=np.int32, order="F")
    ctx = diva.Context(diva.Grid(**g), cfg, ob.oracle_backend())
    helpers.prepare(ctx, f)
    T0 = ctx.download(["Ti_a"])["Ti_a"]
    st = dynamics.DirectTimeStepper(ctx, 0.0, 1000.0, dt_min=0.1, dt_max=10.0, dt_startup_phase=10.0, thermo=True)
    times = []
    for _ in range(6):
        st.step()
        times.append(st.time)
    T1 = ctx.download(["Ti_a"])["Ti_a"]
    ctx.close()
    assert st.thermo_solves >= 1 and np.abs(T1 - T0).max() > 0.0
    assert any(abs(t - 0.25) < 1e-12 or abs(t - 0.5) < 1e-12 for t in times)   # steps end on the event
