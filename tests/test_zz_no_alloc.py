"""The allocation-free step norm (diva_visc_iter_uv_resid_noalloc).

Callers that cannot let the library allocate device memory (a host model with
its own pool allocator, or code that must not call cudaMalloc while it shares
the device) get one entry point whose scratch is a static device array.  This
file is collected last: if it fails, a run that stops at the first failure has
already run every other test.  It checks, through the C ABI, that the entry
point reproduces the step norm the existing solve_DIVA entry point reports, on
two calls in a row, and that grids beyond its scratch are rejected.
"""
import ctypes as C

import numpy as np
import pytest

from imau_ice_b200 import _abi, diva
import helpers

pytestmark = pytest.mark.gpu


def _fn(lib):
    f = lib.diva_visc_iter_uv_resid_noalloc
    f.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                  C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _to_device(a):
    """A Fortran array as the caller's own device buffer (Fortran order, leading dimension = rows)."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda()


def test_noalloc_step_norm_matches_solve_diva(cuda):
    import torch
    g, cfg, f = helpers.make_case(2, dx=40e3, overrides={"lin_rtol": 1e-10})
    ctx = diva.Context(g, cfg, cuda)
    helpers.prepare(ctx, f)
    fn = _fn(cuda.lib)
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    for call in range(2):           # a cold solve, then a warm one: two different step norms
        rep = ctx.solve_DIVA()      # the existing entry point reports resid_UV of its last iteration
        o = ctx.download(["u_vav_cx", "u_cx_prev", "v_vav_cy", "v_cy_prev"])
        u, up, v, vp = (_to_device(o[k]) for k in ("u_vav_cx", "u_cx_prev", "v_vav_cy", "v_cy_prev"))
        for _ in range(2):          # and twice on the same inputs: the shared scratch carries nothing over
            out.fill_(-1.0)
            st = fn(g.nx, g.ny, u.data_ptr(), up.data_ptr(), g.ny, v.data_ptr(), vp.data_ptr(), g.ny - 1,
                    out.data_ptr(), None)
            torch.cuda.synchronize()
            assert st == _abi.OK
            assert out.item() == pytest.approx(rep["resid_UV"], rel=1e-12, abs=1e-300), call
    ctx.close()


def test_noalloc_rejects_grids_beyond_its_scratch(cuda):
    import torch
    fn = _fn(cuda.lib)
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    # ceil(3000/32) * ceil(3000/8) = 94 * 375 blocks > 16384: rejected before any launch
    assert fn(3000, 3000, p, p, 3000, p, p, 2999, p, None) == _abi.BAD_INPUT
    assert fn(1, 5, p, p, 5, p, p, 4, p, None) == _abi.BAD_INPUT


def test_noalloc_padded_rows_on_a_side_stream_allocates_nothing(cuda):
    """Caller arrays with padded leading dimensions (ld_cx = ny + 3, ld_cy = ny + 2) on a
    stream of the caller's own: the same norm as unpadded arrays on the default stream, and
    the device's free memory does not move over repeated calls (the entry point allocates
    nothing; the first call may load the library's device code, so it is made before)."""
    import torch
    fn = _fn(cuda.lib)
    rng = np.random.default_rng(7)
    ny, nx = 45, 37
    u, up = rng.normal(0, 100, (2, ny, nx - 1))
    v, vp = rng.normal(0, 100, (2, ny - 1, nx))
    u[3:9, 4:7] = 0.0                      # points below the velocity tolerance are left out

    def dev(a, ld):
        t = torch.zeros((a.shape[1], ld), dtype=torch.float64)
        t[:, :a.shape[0]] = torch.from_numpy(a.T.copy())
        return t.cuda()

    out0 = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    out1 = torch.full((1,), -2.0, dtype=torch.float64, device="cuda")
    plain = [dev(a, a.shape[0]) for a in (u, up, v, vp)]
    padded = [dev(u, ny + 3), dev(up, ny + 3), dev(v, ny + 2), dev(vp, ny + 2)]
    assert fn(nx, ny, plain[0].data_ptr(), plain[1].data_ptr(), ny, plain[2].data_ptr(), plain[3].data_ptr(),
              ny - 1, out0.data_ptr(), None) == _abi.OK
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        st = fn(nx, ny, padded[0].data_ptr(), padded[1].data_ptr(), ny + 3, padded[2].data_ptr(),
                padded[3].data_ptr(), ny + 2, out1.data_ptr(), C.c_void_p(side.cuda_stream))
        assert st == _abi.OK
    side.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    m = np.abs(u) > 1e-6
    mv = np.abs(v) > 1e-6
    r1 = np.sum((u - up)[m] ** 2) + np.sum((v - vp)[mv] ** 2)
    r2 = np.sum((u + up)[m] ** 2) + np.sum((v + vp)[mv] ** 2)
    want = 2.0 * np.sqrt(r1) / max(np.sqrt(r2), 1e-8)
    assert out1.item() == pytest.approx(out0.item(), rel=1e-12)
    assert out1.item() == pytest.approx(want, rel=1e-12)

