"""Pins of the CPU oracle (no GPU).

The reference ships no tests and cannot be compiled here, so the oracle is
pinned by known answers derived from the reference's own code: the Schoof
(2006) SSA ice-stream solution (utilities_module.f90:836-878), exact column
quadratures, grounded fractions of hand-built quads, the flood-fill's
connectivity rule, properties of the assembled DIVA matrix and the first-call
viscosity rule; plus regression fixtures in tests/golden/.
"""
import ctypes as C
import os

import numpy as np
import pytest

from imau_ice_b200 import diva, synth
import helpers
import oracle_backend as ob

ZETA = np.array(synth.ZETA)
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def dptr(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


# ---- column quadratures (utilities_module.f90:21-124) ------------------------------
def test_vertical_quadratures(oracle):
    lib = oracle.lib
    nz = len(ZETA)
    for f, exact in [(np.ones(nz), 1.0), (ZETA.copy(), 0.5)]:
        assert lib.orc_vertical_integrate(dptr(ZETA), nz, dptr(f)) == pytest.approx(exact, rel=1e-15)
        assert lib.orc_vertical_average(dptr(ZETA), nz, dptr(f)) == pytest.approx(exact, rel=1e-15)
    f = ZETA ** 2
    trap = np.sum(0.5 * (f[1:] + f[:-1]) * np.diff(ZETA))
    assert lib.orc_vertical_integrate(dptr(ZETA), nz, dptr(f)) == pytest.approx(trap, rel=1e-15)
    out = np.zeros(nz)
    lib.orc_vertical_integration_from_bottom_to_zeta(dptr(ZETA), nz, dptr(np.ones(nz)), out.ctypes.data_as(C.POINTER(C.c_double)))
    np.testing.assert_allclose(out, -(1.0 - ZETA), rtol=0, atol=1e-15)


# ---- grounded fractions (general_ice_model_data_module.f90:521-783) ---------------
def frac(lib, nw, ne, sw, se):
    return lib.orc_calc_fraction_above_zero(nw, ne, sw, se)


def bilinear_fraction(nw, ne, sw, se, n=1000):
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x)
    f = sw * (1 - X) * (1 - Y) + se * X * (1 - Y) + nw * (1 - X) * Y + ne * X * Y
    return float((f > 0).mean())


def test_fraction_above_zero_known_answers(oracle):
    lib = oracle.lib
    assert frac(lib, 1, 2, 3, 4) == 1.0
    assert frac(lib, -1, -2, -3, -4) == 0.0
    # planar grounding line parallel to y: f = x - 0.3 -> 70 % grounded (scenario 3, parallel branch)
    assert frac(lib, -0.3, 0.7, -0.3, 0.7) == pytest.approx(0.7, abs=1e-12)
    assert frac(lib, 0.3, 0.3, -0.7, -0.7) == pytest.approx(0.3, abs=1e-12)   # f = y - 0.7


@pytest.mark.parametrize("seed", range(6))
def test_fraction_above_zero_matches_the_bilinear_area(oracle, seed):
    rng = np.random.default_rng(seed)
    lib = oracle.lib
    done = 0
    while done < 20:
        v = rng.uniform(-1, 1, 4)
        if np.min(np.abs(v)) < 0.02 or abs(v[1] + v[2] - v[0] - v[3]) < 0.02:
            continue
        phi = frac(lib, *v)
        assert phi == pytest.approx(bilinear_fraction(*v), abs=3e-3)
        assert phi + frac(lib, *(-v)) == pytest.approx(1.0, abs=1e-9)   # complementarity
        done += 1


# ---- masks and flood-fill (:87-348, :868-988) --------------------------------------
def mask_case(Hi, Hb, SL=None, floodfill=1):
    ny, nx = Hi.shape
    g = diva.Grid(nx, ny, 1e3)
    fields = {"Hi_a": Hi, "Hb_a": Hb, "SL_a": np.zeros_like(Hi) if SL is None else SL,
              "Ti_a": np.full((g.nz, ny, nx), 260.0)}
    ctx = diva.Context(g, {"do_ocean_floodfill": floodfill}, ob.oracle_backend())
    ctx.upload({k: np.asfortranarray(v) for k, v in fields.items()})
    ctx.update_general_ice_model_data()
    out = ctx.download()
    ctx.close()
    return out


def test_floodfill_lake_stays_land():
    ny, nx = 11, 13
    Hb = np.full((ny, nx), 100.0)
    Hb[:, :3] = -200.0            # ocean along the west edge
    Hb[4:7, 7:10] = -50.0          # enclosed depression: a lake, not ocean
    out = mask_case(np.zeros((ny, nx)), Hb)
    assert out["mask_ocean_a"][:, :3].all()
    assert out["mask_ocean_a"][4:7, 7:10].sum() == 0
    assert out["mask_land_a"][4:7, 7:10].all()


def test_floodfill_diagonal_connectivity():
    ny, nx = 9, 9
    Hb = np.full((ny, nx), 100.0)
    Hb[0, 0] = -100.0              # edge seed
    for k in range(1, 6):          # a diagonal channel of single cells
        Hb[k, k] = -100.0
    out = mask_case(np.zeros((ny, nx)), Hb)
    assert all(out["mask_ocean_a"][k, k] == 1 for k in range(6))


@pytest.mark.parametrize("seed", range(4))
def test_floodfill_equals_edge_connected_components(seed):
    from scipy import ndimage
    rng = np.random.default_rng(seed)
    ny, nx = 23, 31
    Hb = ndimage.uniform_filter(rng.normal(0, 300, (ny, nx)), 3) - 20
    Hi = np.where(rng.random((ny, nx)) < 0.3, rng.uniform(0, 300, (ny, nx)), 0.0)
    out = mask_case(Hi, Hb)
    floating = Hi < (0.0 - Hb) * 1028.0 / 910.0
    lab, _ = ndimage.label(floating, structure=np.ones((3, 3)))
    edge = set(np.unique(np.concatenate([lab[0], lab[-1], lab[:, 0], lab[:, -1]]))) - {0}
    expect = np.isin(lab, list(edge)) & floating
    np.testing.assert_array_equal(out["mask_ocean_a"].astype(bool), expect)
    np.testing.assert_array_equal(out["mask_ice_a"], (Hi > np.finfo(float).tiny).astype(np.int32))
    sheet = (out["mask_ice_a"] == 1) & (out["mask_land_a"] == 1)
    np.testing.assert_array_equal(out["mask_sheet_a"].astype(bool), sheet)


# ---- the DIVA matrix and the first viscosity iteration ------------------------------
def prepared(cfg_id=1, dx=None, overrides=None):
    g, cfg, f = helpers.make_case(cfg_id, dx=dx, overrides=overrides)
    ctx = diva.Context(g, cfg, ob.oracle_backend())
    helpers.prepare(ctx, f)
    return ctx, g


def test_first_cold_iteration_takes_the_minimum_viscosity():
    """visc_eff_3D_a and taub are zero before the first call (allocate_ice_model), so
    du/dz = 0/0 on the first iteration and MAX(NaN, visc_eff_min) = visc_eff_min."""
    ctx, g = prepared()
    lib = ctx.backend.lib
    lib.orc_prepare_diva(ctx.h)
    lib.orc_diva_coefficients(ctx.h)
    out = ctx.download(["visc_eff_3D_a", "du_dz_3D_cx", "mask_ice_a"])
    ice = out["mask_ice_a"] == 1
    assert np.isnan(out["du_dz_3D_cx"]).any()
    assert np.all(out["visc_eff_3D_a"][:, ice] == 1e3)


def test_assembled_matrix_structure():
    ctx, g = prepared()
    lib = ctx.backend.lib
    lib.orc_prepare_diva(ctx.h)
    ctx.upload({"u_vav_cx": np.full((g.ny, g.nx - 1), 10.0), "v_vav_cy": np.zeros((g.ny - 1, g.nx))})
    for _ in range(2):
        lib.orc_diva_coefficients(ctx.h)
    lib.orc_assemble_current(ctx.h)
    ptr, idx, val, b, x = ob.matrix(ctx)
    import scipy.sparse as sp
    n = len(b)
    assert n == (g.nx - 1) * g.ny + g.nx * (g.ny - 1)       # ice_velocity_module.f90:2831
    A = sp.csr_matrix((val, idx, ptr), shape=(n, n))
    nnz = np.diff(ptr)
    assert nnz.max() == 9 and set(np.unique(nnz)) <= {1, 2, 9}
    free = np.where(nnz == 9)[0]
    Af = A[free][:, free]
    assert abs(Af - Af.T).max() <= 1e-12 * abs(Af).max()     # free-free couplings are symmetric
    assert np.all(A.diagonal()[free] < 0)
    bnd = np.where(nnz <= 2)[0]
    assert np.all(A.diagonal()[bnd] == 1.0) and np.all(b[bnd] == 0.0)


def test_bc_margin_rows():
    """choice_ice_margin = 'BC' on the cut shelf: stress rows at every ice/ocean face
    (ice_velocity_module.f90:2192-2341, 4 entries, rhs = the depth-integrated pressure
    imbalance), identity rows where shelf meets ice-free land (:1787-1796), and a
    non-singular matrix."""
    g, cfg, f = synth.marine_channel(calving_front=True)
    grid = diva.Grid(**g)
    ctx = diva.Context(grid, dict(cfg, choice_ice_margin="BC"), ob.oracle_backend())
    helpers.prepare(ctx, f)
    lib = ctx.backend.lib
    lib.orc_prepare_diva(ctx.h)
    lib.orc_diva_coefficients(ctx.h)
    lib.orc_assemble_current(ctx.h)
    ptr, idx, val, b, x = ob.matrix(ctx)
    m = ctx.download(["Hi_a", "DIVA_mask_combi"])
    H, combi = m["Hi_a"], m["DIVA_mask_combi"]
    nx, ny = grid.nx, grid.ny
    eq = {}
    n = 0
    for i in range(nx):                                     # ice_velocity_module.f90:2840-2855
        for j in range(ny):
            if i < nx - 1:
                eq[("u", j, i)] = n; n += 1
            if j < ny - 1:
                eq[("v", j, i)] = n; n += 1
    nnz = np.diff(ptr)
    fronts = idents = 0
    for (kind, j, i), r in eq.items():
        j2, i2 = (j, i + 1) if kind == "u" else (j + 1, i)
        if (kind == "u" and i in (0, nx - 2)) or (kind == "v" and j in (0, ny - 2)) or j == 0 or j == ny - 1 \
                or i == 0 or i == nx - 1:
            continue
        if {combi[j, i], combi[j2, i2]} == {1, 3}:
            assert nnz[r] == 1 and val[ptr[r]] == 1.0 and b[r] == 0.0
            idents += 1
        elif (H[j, i] > 0) != (H[j2, i2] > 0) and 3 in (combi[j, i], combi[j2, i2]):
            Hf = max(H[j, i], H[j2, i2])
            assert nnz[r] == 4 and b[r] > 0.0 and b[r] < 0.5 * 910.0 * 9.81 * Hf ** 2
            fronts += 1
    assert idents == 4 and fronts == 19      # 5 notches x (1 u + 2 v) + 4 around the open cell
    import scipy.sparse as sp
    A = sp.csr_matrix((val, idx, ptr), shape=(len(b), len(b))).toarray()
    s = np.linalg.svd(A, compute_uv=False)
    assert s[-1] > 1e-3


# ---- the Schoof (2006) SSA ice stream: known answer of the SSA path ----------------
def test_ssa_matches_schoof2006():
    g, cfg, f = synth.schoof_icestream(dx=10e3)
    cfg = dict(cfg, DIVA_visc_it_nit=300)
    grid = diva.Grid(**g)
    orc = ob.oracle_backend()
    ctx = diva.Context(grid, cfg, orc)
    ob.set_linear_solver(ctx, ob.LIN_GMRES_WARM, rtol=1e-12, abstol=0.0)
    helpers.prepare(ctx, f)
    ctx.solve_SSA()
    o = ctx.download(["u_SSA_cx", "v_SSA_cy", "A_flow_vav_a"])
    U, tc = C.c_double(), C.c_double()
    orc.lib.orc_schoof2006(3e-4, 2000.0, o["A_flow_vav_a"][0, 0], 0.0, 3.0, 0.5, 100e3, C.byref(U), C.byref(tc))
    assert U.value == pytest.approx(1491.80, rel=1e-4)
    assert abs(1.0 - o["u_SSA_cx"].max() / U.value) < 0.05
    assert np.abs(o["v_SSA_cy"]).max() < 1e-3


# ---- regression fixtures ------------------------------------------------------------
def test_golden_channel_regression():
    path = os.path.join(GOLDEN, "channel_cfg1.npz")
    gold = np.load(path)
    g, cfg, f = helpers.make_case(1, overrides={"lin_rtol": 1e-12})
    rep, out = helpers.run(ob.oracle_backend(), g, cfg, f, oracle_solver=(ob.LIN_GMRES_WARM, 1e-12, 0.0))
    assert rep["picard_iterations"] == int(gold["picard_iterations"])
    for k in gold.files:
        if k == "picard_iterations":
            continue
        if gold[k].dtype.kind in "iu":
            np.testing.assert_array_equal(out[k], gold[k], err_msg=k)
        else:
            assert helpers.rel_l2(out[k], gold[k]) < 1e-9, k
