"""Entry points of spawned ranks for the multi-process (gloo) tests.  A spawned
child imports this module afresh, so it loads the package itself first."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import conftest  # noqa: E402,F401  (imports imau-ice_b200 as imau_ice_b200 and puts oracle/ on the path)


def ensemble_rank(rank, world, port, q, members_fn):
    import torch.distributed as dist
    import oracle_backend
    from imau_ice_b200 import ensemble
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res, parts = ensemble.solve_ensemble(members_fn(), oracle_backend.oracle_backend(), rank, world)
        q.put((rank, {k: (v["report"]["picard_iterations"], v["u_vav_cx"], v["v_vav_cy"]) for k, v in res.items()},
               parts))
    finally:
        dist.destroy_process_group()


def small_channel_members(n=4):
    import numpy as np
    from imau_ice_b200 import diva, synth
    out = []
    for k in range(n):
        g, cfg, f = synth.marine_channel(seed=100 + k, dx=10e3)
        f = dict(f)
        f["beta_sq_a"] = np.asfortranarray(f["beta_sq_a"] * (0.5 + 0.5 * k))
        out.append((f"channel-{k}", diva.Grid(**g), dict(cfg, lin_rtol=1e-10), f))
    return out
