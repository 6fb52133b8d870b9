"""A plain PyTorch FP32 restatement of the warm-start network (include/diva_cnn.h), the
reference its CUDA kernels are checked against: the same flat weight vector, the same
input and output channel definitions.  ``bf16=True`` rounds what the device keeps in
BF16 (inputs, 3x3 weights, every 3x3 layer's output) so that only the FP32
summation order differs."""
import numpy as np
import torch
import torch.nn.functional as F

from imau_ice_b200 import learned

VEL, TAU, VISC = 10.0, 1000.0, 8.0


def _r(t, bf16):
    return t.to(torch.bfloat16).float() if bf16 else t


def unflatten(w, bf16=False):
    """{name: (weight [cout][cin][3][3] or head [20][32], bias)} from the flat vector."""
    lay, total = learned.weight_layout()
    w = w if isinstance(w, torch.Tensor) else torch.as_tensor(np.asarray(w, np.float32))
    assert w.numel() == total
    out = {}
    for name, (wo, shape, bo, nb) in lay.items():
        ww = w[wo:wo + int(np.prod(shape))].reshape(shape)
        if name != "head":
            ww = _r(ww, bf16).permute(1, 2, 0).reshape(shape[1], shape[2], 3, 3)   # [tap][co][ci] -> [co][ci][3][3]
        out[name] = (ww, w[bo:bo + nb])
    return out


def forward(feat, w, bf16=False):
    """feat [n][Hp][Wp][16] (float) -> out [n][Hp][Wp][20] (float)."""
    p = unflatten(w, bf16)
    x = _r(torch.as_tensor(feat, dtype=torch.float32).permute(0, 3, 1, 2), bf16)

    def conv(name, t):
        ww, b = p[name]
        return _r(F.relu(F.conv2d(t, ww, b, padding=1)), bf16)

    def pool(t):
        return _r(F.avg_pool2d(t, 2), bf16)

    def up(t):
        return F.interpolate(t, scale_factor=2, mode="nearest")

    e1 = conv("e1b", conv("e1a", x))
    e2 = conv("e2b", conv("e2a", pool(e1)))
    b = conv("bb", conv("ba", pool(e2)))
    d2 = conv("d2b", conv("d2a", torch.cat([up(b), e2], 1)))
    d1 = conv("d1b", conv("d1a", torch.cat([up(d2), e1], 1)))
    wh, bh = p["head"]
    return (torch.einsum("oc,nchw->nhwo", wh, d1) + bh).contiguous()


def valid_mask(Hp, Wp, ny, nx, nz):
    m = np.zeros((Hp, Wp, learned.N_OUT), bool)
    m[:ny, :nx - 1, 0] = m[:ny, :nx - 1, 2] = True
    m[:ny - 1, :nx, 1] = m[:ny - 1, :nx, 3] = True
    m[:ny, :nx, 4:4 + nz] = True
    return m


def loss(out, tgt, mask, weights=None):
    """sum over valid entries of w_channel (out - tgt)^2, divided by the number of valid entries."""
    m = torch.as_tensor(np.array(mask), dtype=out.dtype)
    w = torch.ones(out.shape[-1]) if weights is None else torch.as_tensor(np.asarray(weights, np.float32))
    e = (out - tgt) * m
    return (w * e * e).sum() / float(mask.sum())


def features(f, Hp, Wp):
    """The input channels from downloaded fields ((ny, nx) arrays)."""
    ny, nx = f["Hi_a"].shape
    c = np.zeros((Hp, Wp, learned.IN_C), np.float32)
    c[:ny, :nx, 0] = f["Hi_a"] / 1000.0
    c[:ny, :nx, 1] = f["Hb_a"] / 1000.0
    c[:ny, :nx, 2] = f["dHs_dx_a"] * 100.0
    c[:ny, :nx, 3] = f["dHs_dy_a"] * 100.0
    c[:ny, :nx, 4] = np.log10(np.maximum(f["A_flow_vav_a"], 1e-30)) + 17.0
    c[:ny, :nx, 5] = np.log10(np.maximum(f["beta_sq_a"], 1e-30)) - 4.0
    c[:ny, :nx, 6] = f["mask_sheet_a"]
    c[:ny, :nx, 7] = f["mask_shelf_a"]
    return c


def targets(f, Hp, Wp):
    """The output channels of a converged state."""
    ny, nx = f["Hi_a"].shape
    nz = f["visc_eff_3D_a"].shape[0]
    t = np.zeros((Hp, Wp, learned.N_OUT), np.float32)
    t[:ny, :nx - 1, 0] = np.arcsinh(f["u_vav_cx"] / VEL)
    t[:ny - 1, :nx, 1] = np.arcsinh(f["v_vav_cy"] / VEL)
    t[:ny, :nx - 1, 2] = np.arcsinh(f["taub_cx"] / TAU)
    t[:ny - 1, :nx, 3] = np.arcsinh(f["taub_cy"] / TAU)
    t[:ny, :nx, 4:4 + nz] = np.moveaxis(np.log10(np.maximum(f["visc_eff_3D_a"], 1e-30)) - VISC, 0, -1)
    return t
