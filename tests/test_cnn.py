"""The warm-start network on the CPU: the flat weight layout and tap convention of
the PyTorch reference, and the finding the network's output channels rest on -- the
viscosity iteration warm-starts from its whole carried state (velocities, basal
stress, viscosity), not from the velocities alone (oracle, no GPU)."""
import numpy as np
import torch
import torch.nn.functional as F

from imau_ice_b200 import diva, learned, synth
import cnn_reference as ref
import helpers
import oracle_backend as ob


def test_weight_layout_counts_every_parameter():
    lay, total = learned.weight_layout()
    assert total == sum(9 * ci * co + co for _, ci, co in learned.LAYERS) + learned.N_OUT * (learned.HEAD_C + 1)
    offs = sorted((v[0], v[2]) for v in lay.values())
    assert offs[0][0] == 0 and all(b[0] > a[1] for a, b in zip(offs, offs[1:]))


def test_tap_convention_is_cross_correlation():
    """Flat [tap][cout][cin] with tap = 3(dy+1) + (dx+1): the output at (y, x) reads the
    input at (y+dy, x+dx)."""
    lay, total = learned.weight_layout()
    w = np.zeros(total, np.float32)
    wo, (_, co, ci), _, _ = lay["e1a"]
    dy, dx = -1, 1
    w[wo + (3 * (dy + 1) + (dx + 1)) * co * ci + 0 * ci + 0] = 1.0      # cout 0 <- cin 0 at (dy, dx)
    ww, b = ref.unflatten(w)["e1a"]
    x = torch.zeros(1, 16, 8, 8)
    x[0, 0, 4, 5] = 1.0
    y = F.conv2d(x, ww, b, padding=1)
    assert y[0, 0, 4 - dy, 5 - dx] == 1.0 and y.abs().sum() == 1.0


def test_reference_forward_shapes_and_bf16_rounding():
    rng = np.random.default_rng(0)
    _, total = learned.weight_layout()
    w = rng.normal(0, 0.1, total).astype(np.float32)
    feat = rng.normal(0, 1, (2, 12, 16, 16)).astype(np.float32)
    o32, o16 = ref.forward(feat, w), ref.forward(feat, w, bf16=True)
    assert o32.shape == (2, 12, 16, learned.N_OUT)
    assert torch.allclose(o32, o16, rtol=0.1, atol=0.05 * float(o32.abs().max()))


def test_targets_and_features_channels():
    ny, nx, nz = 5, 7, 3
    f = {"Hi_a": np.full((ny, nx), 2000.0), "Hb_a": np.full((ny, nx), -500.0), "dHs_dx_a": np.full((ny, nx), 1e-3),
         "dHs_dy_a": np.zeros((ny, nx)), "A_flow_vav_a": np.full((ny, nx), 1e-16), "beta_sq_a": np.full((ny, nx), 1e4),
         "mask_sheet_a": np.ones((ny, nx)), "mask_shelf_a": np.zeros((ny, nx)),
         "u_vav_cx": np.full((ny, nx - 1), 10.0), "v_vav_cy": np.full((ny - 1, nx), -10.0),
         "taub_cx": np.full((ny, nx - 1), 1000.0), "taub_cy": np.zeros((ny - 1, nx)),
         "visc_eff_3D_a": np.full((nz, ny, nx), 1e9)}
    c, t = ref.features(f, 8, 8), ref.targets(f, 8, 8)
    np.testing.assert_allclose(c[0, 0, :8], [2.0, -0.5, 0.1, 0.0, 1.0, 0.0, 1.0, 0.0], atol=1e-6)
    assert np.all(c[ny:] == 0) and np.all(c[:, nx:] == 0)
    m = ref.valid_mask(8, 8, ny, nx, nz)
    np.testing.assert_allclose(t[0, 0, :4 + nz], [np.arcsinh(1.0), -np.arcsinh(1.0), np.arcsinh(1.0), 0.0, 1.0, 1.0, 1.0],
                               atol=1e-6)
    assert m[:, :, 0].sum() == ny * (nx - 1) and m[:, :, 1].sum() == (ny - 1) * nx and not m[:, :, 4 + nz:].any()
    assert np.all(t[~m] == 0)


def test_the_iteration_warm_starts_from_its_whole_state():
    """Given the converged velocities but a cold viscosity and basal stress, solve_DIVA
    iterates about as long as from a cold start; given all three it stops at once
    (ice_velocity_module.f90:664-721: the vertical shear of the first iteration comes
    from the previous viscosity and basal stress)."""
    g, cfg, f = synth.ice_cap(seed=310, dx=20e3)
    f = dict(f)
    f["beta_sq_a"] = np.asfortranarray(f["beta_sq_a"] * 4.0)
    cfg = dict(cfg, picard_stop="relres", picard_relres_tol=1e-6, DIVA_visc_it_nit=500, lin_adaptive=1,
               lin_rtol=1e-10)

    def run(state=None):
        ctx = diva.Context(diva.Grid(**g), cfg, ob.oracle_backend())
        ob.set_linear_solver(ctx, ob.LIN_GMRES_WARM, rtol=1e-10, abstol=0.0)
        helpers.prepare(ctx, f)
        if state:
            ctx.upload(state)
        r = ctx.solve_DIVA()
        s = ctx.download(["u_vav_cx", "v_vav_cy", "taub_cx", "taub_cy", "visc_eff_3D_a"])
        ctx.close()
        return r["picard_iterations"], s

    cold, s = run()
    uv, _ = run({k: s[k] for k in ("u_vav_cx", "v_vav_cy")})
    full, _ = run(s)
    assert cold > 20 and uv >= 0.8 * cold and full <= 2


def test_complete_state_lets_velocities_alone_warm_start():
    """diva_complete_state on the oracle: the converged velocities plus 30 column-local
    sweeps start solve_DIVA at its fixed point."""
    g, cfg, f = synth.ice_cap(seed=310, dx=20e3)
    f = dict(f)
    f["beta_sq_a"] = np.asfortranarray(f["beta_sq_a"] * 4.0)
    cfg = dict(cfg, picard_stop="relres", picard_relres_tol=1e-6, DIVA_visc_it_nit=500, lin_adaptive=1,
               lin_rtol=1e-10)
    its, uv = [], None
    for sweeps in (None, 30):
        ctx = diva.Context(diva.Grid(**g), cfg, ob.oracle_backend())
        ob.set_linear_solver(ctx, ob.LIN_GMRES_WARM, rtol=1e-10, abstol=0.0)
        helpers.prepare(ctx, f)
        if uv is not None:
            ctx.upload(uv)
            ctx.complete_state(sweeps)
        its.append(ctx.solve_DIVA()["picard_iterations"])
        uv = ctx.download(["u_vav_cx", "v_vav_cy"])
        ctx.close()
    assert its[0] > 20 and its[1] <= 2, its


def test_the_network_needs_the_cuda_library():
    """No host implementation of the network: another backend is refused up front."""
    with np.testing.assert_raises(diva.DivaError):
        learned.WarmStartNet(diva.Grid(37, 29, 10e3), backend=ob.oracle_backend())
