"""The warm-start network's CUDA kernels (tcgen05 implicit-GEMM convolutions, head,
Adam, the context <-> tensor kernels) against the PyTorch FP32 reference
(tests/cnn_reference.py) with the device's BF16 roundings, and the end-to-end effect
on solve_DIVA."""
import numpy as np
import pytest
import torch

from imau_ice_b200 import diva, learned, synth
import cnn_reference as ref
import helpers

pytestmark = pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU (B200)")


def small_net(ny=29, nx=37, batch=2, seed=3):
    g = diva.Grid(nx, ny, 10e3)
    return g, learned.WarmStartNet(g, batch=batch, capacity=0, seed=seed)


def random_batch(net, n, seed):
    Hp, Wp = net.padded_shape
    rng = np.random.default_rng(seed)
    feat = rng.normal(0, 1, (n, Hp, Wp, learned.IN_C)).astype(np.float32)
    feat[..., 8:] = 0.0
    feat = torch.as_tensor(feat).to(torch.bfloat16).float().numpy()       # representable in BF16
    tgt = rng.normal(0, 1, (n, Hp, Wp, learned.N_OUT)).astype(np.float32)
    return feat, tgt


def dev(a, dtype):
    return torch.as_tensor(a).to(dtype).cuda().contiguous()


@pytest.mark.gpu
def test_forward_matches_the_reference():
    g, net = small_net()
    feat, _ = random_batch(net, 2, 0)
    out = torch.zeros(2, *net.padded_shape, learned.N_OUT, device="cuda")
    f = dev(feat, torch.bfloat16)
    net.forward(f.data_ptr(), out.data_ptr(), 2)
    want = ref.forward(feat, net.get_weights(), bf16=True)
    err = (out.cpu() - want).abs().max() / want.abs().max()
    assert err < 2e-2, float(err)
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("velocities_only", [False, True])
def test_gradients_match_autograd(velocities_only):
    g, net = small_net()
    feat, tgt = random_batch(net, 2, 1)
    lw = np.ones(learned.N_OUT, np.float32)
    if velocities_only:
        net.velocities_only()
        lw[2:] = 0.0
    w = torch.as_tensor(net.get_weights()).requires_grad_(True)
    mask = ref.valid_mask(*net.padded_shape, g.ny, g.nx, g.nz)
    mask = np.broadcast_to(mask, (2,) + mask.shape)
    loss_ref = ref.loss(ref.forward(feat, w, bf16=True), torch.as_tensor(tgt), mask, lw)
    loss_ref.backward()
    gref = w.grad.numpy()
    f, t = dev(feat, torch.bfloat16), dev(tgt, torch.float32)    # held: the kernels read them
    loss = net.train_step(f.data_ptr(), t.data_ptr(), 2, 0.0)
    gdev = net.grads()
    assert abs(loss - loss_ref.item()) <= 2e-2 * loss_ref.item()
    lay, _ = learned.weight_layout()
    for name, (wo, shape, bo, nb) in lay.items():
        n = int(np.prod(shape))
        for a, b, what in ((gdev[wo:wo + n], gref[wo:wo + n], "w"), (gdev[bo:bo + nb], gref[bo:bo + nb], "b")):
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            assert rel < 5e-2, (name, what, rel)
    net.close()


@pytest.mark.gpu
def test_training_lowers_the_loss_and_predict_writes_the_state():
    g, net = small_net(batch=2)
    feat, tgt = random_batch(net, 2, 2)
    f, t = dev(feat, torch.bfloat16), dev(tgt * 0.3, torch.float32)
    losses = [net.train_step(f.data_ptr(), t.data_ptr(), 2, 3e-3) for _ in range(60)]
    assert losses[-1] < 0.5 * losses[0]
    # a network whose head ignores its input writes constant fields through predict
    lay, total = learned.weight_layout()
    w = np.zeros(total, np.float32)
    hb = lay["head"][2]
    w[hb:hb + 4] = [np.arcsinh(5.0), np.arcsinh(-2.0), np.arcsinh(3.0), 0.0]
    w[hb + 4:hb + 4 + g.nz] = 1.0                                    # visc = 1e9
    net.set_weights(w)
    gg, cfg, fl = synth.marine_channel(dx=20e3)
    grid = diva.Grid(**gg)
    net2 = learned.WarmStartNet(grid, batch=1)
    net2.set_weights(w)
    ctx = diva.Context(grid, cfg)
    helpers.prepare(ctx, fl)
    net2.predict(ctx, complete_sweeps=0)
    o = ctx.download(["u_vav_cx", "v_vav_cy", "taub_cx", "taub_cy", "visc_eff_3D_a"])
    np.testing.assert_allclose(o["u_vav_cx"], 50.0, rtol=1e-6)
    np.testing.assert_allclose(o["v_vav_cy"], -20.0, rtol=1e-6)
    np.testing.assert_allclose(o["taub_cx"], 3000.0, rtol=1e-6)
    np.testing.assert_allclose(o["visc_eff_3D_a"], 1e9, rtol=1e-6)
    ctx.close()
    net.close()
    net2.close()


@pytest.mark.gpu
def test_warm_start_from_the_trained_network_cuts_iterations():
    """Ice caps at 20 km (friction x4): train on 96 solved members, then the held-out
    members converge to the same tolerance from the prediction (velocities plus 10
    state-completion sweeps) in fewer viscosity iterations than from cold, to the same
    velocities."""
    def case(seed):
        gg, cfg, fl = synth.ice_cap(seed=seed, dx=20e3)
        fl = dict(fl)
        fl["beta_sq_a"] = np.asfortranarray(fl["beta_sq_a"] * 4.0)
        cfg = dict(cfg, picard_stop="relres", picard_relres_tol=1e-6, DIVA_visc_it_nit=500, lin_adaptive=1,
                   lin_rtol=1e-10)
        return diva.Grid(**gg), cfg, fl

    grid = case(0)[0]
    net = learned.WarmStartNet(grid, batch=8, capacity=96, seed=0)
    net.velocities_only()                   # predict's default mode completes the rest
    seed = 0
    while net.num_samples < 96:
        _, cfg, fl = case(seed)
        ctx = diva.Context(grid, cfg)
        helpers.prepare(ctx, fl)
        if ctx.solve_DIVA()["status"] == 0:
            net.add_sample(ctx)
        ctx.close()
        seed += 1
    l0 = net.train(1, lr=1e-3, seed=1)
    l1 = net.train(150, lr=1e-3, seed=2)
    assert l1 < 0.2 * l0
    cold, warm = [], []
    for s in range(1000, 1004):
        _, cfg, fl = case(s)
        res = []
        for use in (False, True):
            ctx = diva.Context(grid, cfg)
            helpers.prepare(ctx, fl)
            if use:
                net.predict(ctx)
            r = ctx.solve_DIVA()
            res.append((r, ctx.download(["u_vav_cx", "v_vav_cy"])))
            ctx.close()
        (rc, oc), (rw, ow) = res
        if rc["status"] != 0:
            continue
        # the warm start is judged by the solve itself: the same stop rule, rel-res <= 1e-6
        assert rw["status"] == 0 and 0 <= rw["relres"] <= 1e-6
        cold.append(rc["picard_iterations"])
        warm.append(rw["picard_iterations"])
        # Two states that both meet rel-res 1e-6 need not be close: these 20 km caps are
        # ill-conditioned enough that the oracle itself, started from its own solution
        # perturbed by 10 %, converges 1e-4 .. 5e-2 (seed 1001) away from its cold solve.
        # Only a gross departure (another branch of the iteration) fails here.
        a = np.concatenate([oc["u_vav_cx"].ravel(), oc["v_vav_cy"].ravel()])
        b = np.concatenate([ow["u_vav_cx"].ravel(), ow["v_vav_cy"].ravel()])
        assert helpers.rel_l2(b, a) <= 0.1
    assert cold and np.mean(warm) < 0.95 * np.mean(cold), (cold, warm)
    net.close()
