"""The 3D heat equation on the CPU oracle (thermodynamics_module.f90:29-481): the
column solver against NumPy, the steady conductive profile, newly ice-covered columns,
and the Robin replacement of unstable columns."""
import ctypes as C

import numpy as np
import pytest

from imau_ice_b200 import diva, synth
import helpers
import oracle_backend as ob

T0 = 273.16


def dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@pytest.mark.parametrize("seed", range(4))
def test_tridiagonal_solver_matches_numpy(oracle, seed):
    rng = np.random.default_rng(seed)
    n = 15
    dl, du = rng.normal(size=n - 1), rng.normal(size=n - 1)
    d = rng.normal(size=n) * (3.0 if seed % 2 == 0 else 0.3)   # odd seeds need row interchanges
    b = rng.normal(size=n)
    A = np.diag(d) + np.diag(dl, -1) + np.diag(du, 1)
    x = b.copy()
    info = oracle.lib.orc_tridiagonal_solve(n, dptr(dl.copy()), dptr(d.copy()), dptr(du.copy()), dptr(x))
    assert info == 0
    np.testing.assert_allclose(A @ x, b, rtol=0, atol=1e-10 * np.abs(b).max())


def slab(nx=21, ny=21, H=2000.0, Ts=240.0, ghf=5e5, smb=0.2):
    g = diva.Grid(nx, ny, 10e3)
    f = {"Hi_a": np.full((ny, nx), H), "Hb_a": np.full((ny, nx), 500.0), "SL_a": np.zeros((ny, nx)),
         "Ti_a": np.full((g.nz, ny, nx), Ts), "T_surf_annual_a": np.full((ny, nx), Ts),
         "GHF_a": np.full((ny, nx), ghf), "SMB_a": np.full((ny, nx), smb),
         "mask_ice_a_prev": np.ones((ny, nx), dtype=np.int32)}
    return g, f


def thermo_ctx(g, f, **cfg):
    base = {"choice_ice_heat_capacity": "uniform", "choice_ice_thermal_conductivity": "uniform",
            "choice_sliding_law": "no_sliding"}
    base.update(cfg)
    ctx = diva.Context(g, base, ob.oracle_backend())
    ctx.upload({k: np.asfortranarray(v) for k, v in f.items()})
    ctx.update_general_ice_model_data()
    ctx.calc_pressure_melting_point()
    return ctx


def test_steady_conductive_profile():
    """No flow, no heating, a very long step: T rises linearly with depth by GHF H / K."""
    g, f = slab()
    ctx = thermo_ctx(g, f, dt_thermo=1e12)
    assert ctx.run_thermo_model(True) == 0
    T = ctx.download(["Ti_a"])["Ti_a"][:, 10, 10]
    K = 6.626958e7
    expect = 240.0 + 5e5 * 2000.0 / K * np.asarray(g.zeta)
    np.testing.assert_allclose(T, expect, rtol=0, atol=1e-6)


def test_new_ice_takes_the_upwind_column():
    g, f = slab(nx=11, ny=9)
    f["mask_ice_a_prev"][4, 5] = 0                    # (4,5) became ice this step
    f["Ti_a"][:, 4, 4] = np.linspace(250.0, 260.0, g.nz)
    ctx = thermo_ctx(g, f)
    ctx.upload({"u_vav_cx": np.full((g.ny, g.nx - 1), 5.0)})   # flow from the west
    ctx.run_thermo_model(False)
    T = ctx.download(["Ti_a"])["Ti_a"]
    np.testing.assert_array_equal(T[:, 4, 5], T[:, 4, 4])


def test_unstable_columns_take_the_robin_solution():
    g, f = slab()
    f["T_surf_annual_a"][7, 8] = 100.0                # a column far too cold for the solver's limit
    f["T_surf_annual_a"][12, 3] = 90.0
    ctx = thermo_ctx(g, f, dt_thermo=10.0)
    assert ctx.run_thermo_model(True) == 2
    o = ctx.download(["Ti_a", "Ti_pmp_a"])
    K = 9.828 * 31556943.36 * np.exp(-0.0057 * T0)
    kappa = K / (910.0 * 2127.5)
    z = np.asarray(g.zeta)
    for (j, i), Ts in (((7, 8), 100.0), ((12, 3), 90.0)):
        L = np.sqrt(2.0 * kappa * 2000.0 / 0.2)
        from math import erf
        prof = Ts + np.sqrt(np.pi) / 2.0 * L * (-5e5 / K) * (
            np.array([erf((1.0 - zk) * 2000.0 / L) for zk in z]) - erf(2000.0 / L))
        np.testing.assert_allclose(o["Ti_a"][:, j, i], np.minimum(prof, o["Ti_pmp_a"][:, j, i]), rtol=1e-14)


def test_too_many_unstable_columns_is_an_error():
    g, f = slab(nx=11, ny=9)
    f["T_surf_annual_a"][4, 5] = 100.0                # 1 of 99 cells: ceil(0.99) = 1 is already too many
    ctx = thermo_ctx(g, f)
    with pytest.raises(diva.DivaError) as e:
        ctx.run_thermo_model(True)
    assert e.value.status == 3                        # DIVA_NAN_DETECTED (the reference crashes)


def test_heat_equation_after_a_velocity_solve():
    """The channel after a DIVA solve: advection, strain and frictional heating on; the
    temperatures stay between the surface value and the pressure melting point."""
    g, cfg, f = synth.marine_channel(dx=20e3)
    f = dict(f)
    ny, nx = f["Hi_a"].shape
    f["T_surf_annual_a"] = np.asfortranarray(np.full((ny, nx), 243.0))
    f["GHF_a"] = np.asfortranarray(np.full((ny, nx), 1.7e6))
    f["SMB_a"] = np.asfortranarray(np.full((ny, nx), 0.3))
    f["mask_ice_a_prev"] = np.ones((ny, nx), dtype=np.int32, order="F")
    ctx = diva.Context(diva.Grid(**g), dict(cfg, lin_rtol=1e-10), ob.oracle_backend())
    ob.set_linear_solver(ctx, ob.LIN_GMRES_WARM, 1e-10, 0.0)
    helpers.prepare(ctx, f)
    ctx.solve_DIVA()
    T_before = ctx.download(["Ti_a"])["Ti_a"].copy()
    n = ctx.run_thermo_model(True)
    o = ctx.download(["Ti_a", "Ti_pmp_a", "frictional_heating_a", "Ki_a", "Cpi_a"])
    assert n == 0
    assert np.isfinite(o["Ti_a"]).all()
    assert (o["Ti_a"] <= o["Ti_pmp_a"] + 1e-9).all() and o["Ti_a"].min() > 200.0
    assert o["frictional_heating_a"].max() > 0.0
    # conductivity and heat capacity of the temperatures the step started from (:523-608)
    np.testing.assert_allclose(o["Ki_a"], 3.101e8 * np.exp(-0.0057 * T_before), rtol=1e-14)
    np.testing.assert_allclose(o["Cpi_a"], 2115.3 + 7.79293 * (T_before - T0), rtol=1e-14)
    assert np.abs(o["Ti_a"] - T_before).max() > 1e-3                  # the step changed the temperatures


def test_time_steps_with_thermodynamics():
    """Predictor/corrector steps with the thermodynamics event: the heat equation runs when
    its clock is due (dt_thermo), the rheology follows the new temperatures."""
    from imau_ice_b200 import dynamics
    g, cfg, f = synth.marine_channel(dx=20e3)
    f = dict(f)
    ny, nx = f["Hi_a"].shape
    for k, v in (("SMB_a", 0.3), ("BMB_a", 0.0), ("T_surf_annual_a", 243.0), ("GHF_a", 1.7e6)):
        f[k] = np.asfortranarray(np.full((ny, nx), v))
    f["mask_ice_a_prev"] = np.ones((ny, nx), dtype=np.int32, order="F")
    cfg = dict(cfg, lin_rtol=1e-10, dt_thermo=0.02, ice_thickness_west_BC="infinite", ice_thickness_east_BC="zero",
               ice_thickness_south_BC="infinite", ice_thickness_north_BC="infinite")
    ctx = diva.Context(diva.Grid(**g), cfg, ob.oracle_backend())
    ob.set_linear_solver(ctx, ob.LIN_GMRES_WARM, 1e-10, 0.0)
    helpers.prepare(ctx, f)
    ctx.determine_floating_margin_fraction()
    T0_field = ctx.download(["Ti_a", "A_flow_3D_a"])
    pc = dynamics.PCTimeStepper(ctx, 0.0, 1000.0, thermo=True)
    pc.run(max_steps=4)
    o = ctx.download(["Ti_a", "A_flow_3D_a"])
    assert pc.thermo_solves >= 1
    assert np.abs(o["Ti_a"] - T0_field["Ti_a"]).max() > 1e-3
    assert not np.array_equal(o["A_flow_3D_a"], T0_field["A_flow_3D_a"])


def test_shelf_base_takes_the_ocean_input():
    """ocean_temperature_input: the shelf-base temperature is T0 + T_ocean_base_a instead of
    T0 + T_ocean_mean_PD_ANT (thermodynamics_module.f90:189-218, :296-300). Both stay below
    the pressure melting point of the 2000 m slab (T0 - 1.74), which would otherwise take
    the base to the basal-gradient value (:323-326)."""
    g, f = slab()
    f["Hb_a"] = np.full(f["Hi_a"].shape, -3000.0)         # a floating slab
    f["T_ocean_base_a"] = np.full(f["Hi_a"].shape, -2.5)
    base = {}
    for flag in (0, 1):
        ctx = thermo_ctx(g, f, ocean_temperature_input=flag, T_ocean_mean_PD_ANT=-3.0)
        assert ctx.run_thermo_model(True) == 0
        o = ctx.download(["Ti_a", "mask_shelf_a"])
        assert o["mask_shelf_a"][10, 10] == 1
        base[flag] = o["Ti_a"][-1, 10, 10]
    assert base[0] == T0 - 3.0 and base[1] == -2.5 + T0
