"""Regenerate tests/golden/channel_cfg1.npz: the oracle's solve_DIVA of the
129 x 17 marine channel (seed 1), reference stop rule, linear solves by
GMRES(30)+ILU(0) from the current iterate to 1e-12.  These are regression
fixtures of the oracle (the reference itself cannot run here); the GPU parity
tests compare against them as well.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import conftest  # noqa: E402,F401  (loads the package and the oracle path)
import helpers  # noqa: E402
import oracle_backend as ob  # noqa: E402

FIELDS = ["mask_ice_a", "mask_sheet_a", "mask_shelf_a", "mask_ocean_a", "mask_gl_a", "mask_cf_a", "mask_a",
          "DIVA_mask_combi", "u_vav_cx", "v_vav_cy", "f_grnd_cx", "f_grnd_cy", "N_a", "beta_eff_cx",
          "taub_cx", "w_surf_a", "uabs_surf_a", "Hs_a", "TAF_a"]


def main():
    g, cfg, f = helpers.make_case(1, overrides={"lin_rtol": 1e-12})
    rep, out = helpers.run(ob.oracle_backend(), g, cfg, f, oracle_solver=(ob.LIN_GMRES_WARM, 1e-12, 0.0))
    data = {k: out[k] for k in FIELDS}
    data["picard_iterations"] = np.array(rep["picard_iterations"])
    np.savez_compressed(os.path.join(HERE, "channel_cfg1.npz"), **data)
    print("picard iterations", rep["picard_iterations"])


if __name__ == "__main__":
    main()
