"""The operand staging of the tcgen05 convolution kernels (imau-ice_b200/csrc/cnn.cu),
restated on the CPU: each kernel's shared-memory byte offsets for the A and B tiles,
read back through the no-swizzle K-major canonical layout the kernels' matrix
descriptors describe (in 16-byte units ((8,n),2):((1,SBO),LBO), LBO between the two
8-element K halves, SBO between 8-row groups), must reproduce forward, dgrad and wgrad
of a 3x3 convolution as PyTorch autograd computes them.  This checks the index
arithmetic of the staging loops (tap mirroring, the transposed weight gather, the
ReLU gate, the pixel-slice layout and split partials) without a GPU; the device
forward pass itself is checked against the reference on a B200
(tests/test_gpu_cnn.py)."""
import numpy as np
import torch
import torch.nn.functional as F


def canon_read(smem, start, lbo, sbo, rows):
    """A[r][k] for k in [0,16) from a K-major no-swizzle tile: ((8,n),2):((1,SBO),LBO) in 16-byte units."""
    out = np.zeros((rows, 16), np.float32)
    for r in range(rows):
        for k in range(16):
            byte = start + 16 * ((r % 8) + (r // 8) * (sbo // 16) + (k // 8) * (lbo // 16)) + 2 * (k % 8)
            out[r, k] = smem[byte // 2]
    return out


def conv_kernel(x, gate, w, bias, KC, NO, dgrad, n, H, W):
    """k_conv3x3<KC, NO, dgrad>: x [n][H][W][KC]; w [9][NO][KC] (forward: W [9][COUT][CIN],
    dgrad: W^T [9][CIN][COUT] as k_transpose_w writes it); y [n][H][W][NO]
    (FP32 throughout: the BF16 roundings are not what this checks)."""
    npix = n * H * W
    y = np.zeros((npix, NO), np.float32)
    for blk in range((npix + 127) // 128):
        D = np.zeros((128, NO), np.float32)
        A_BYTES = 128 * KC * 2
        for t in range(9):
            sm = np.zeros((A_BYTES + NO * KC * 2) // 2, np.float32)   # element-addressed
            dy, dx = t // 3 - 1, t % 3 - 1
            if dgrad: dy, dx = -dy, -dx
            for tid in range(128):
                p = blk * 128 + tid
                pin = p < npix
                px = p % W; q = p // W; py = q % H; pb = q // H
                yy, xx = py + dy, px + dx
                inn = pin and 0 <= yy < H and 0 <= xx < W
                for kc in range(KC // 8):
                    v = np.zeros(8, np.float32)
                    if inn:
                        v = x[pb, yy, xx, kc * 8:kc * 8 + 8].copy()
                        if dgrad: v = v * (gate[pb, yy, xx, kc * 8:kc * 8 + 8] > 0)
                    base = (kc * 2048 + tid * 16) // 2
                    sm[base:base + 8] = v
            Bs = A_BYTES // 2
            for c in range(NO * (KC // 8)):
                nn_, kc = c % NO, c // NO
                v = w[t, nn_, kc * 8:kc * 8 + 8]          # forward: W; dgrad: the transposed copy
                base = Bs + (kc * (NO * 16) + nn_ * 16) // 2
                sm[base:base + 8] = v
            for k in range(KC // 16):
                A = canon_read(sm, 2 * k * 2048, 2048, 128, 128)
                B = canon_read(sm, A_BYTES + 2 * k * (NO * 16), NO * 16, 128, NO)
                D += A @ B.T
        for tid in range(128):
            p = blk * 128 + tid
            if p < npix:
                f = D[tid].copy()
                if not dgrad: f = np.maximum(f + bias, 0)
                y[p] = f
    return y.reshape(n, H, W, NO)


def wgrad_kernel(x, dy_, gate, CI, CO, n, H, W, nsplit, PIX=64):
    """k_conv3x3_wgrad<CI, CO> over nsplit pixel ranges, partials summed: [9][CO][CI]."""
    npix = n * H * W
    nchunk = (npix + PIX - 1) // PIX
    per = (nchunk + nsplit - 1) // nsplit
    part = np.zeros((nsplit, 9, CO, CI), np.float32)
    A_BYTES = 128 * PIX * 2
    for split in range(nsplit):
        c0 = split * per; c1 = min(c0 + per, nchunk)
        for t in range(9):
            ddy, ddx = t // 3 - 1, t % 3 - 1
            D = np.zeros((128, CI), np.float32)
            for c in range(max(0, c1 - c0)):
                sm = np.zeros((A_BYTES + CI * PIX * 2) // 2, np.float32)
                pbase = (c0 + c) * PIX
                for i in range(PIX * (CO // 8)):
                    kk, mc = i % PIX, i // PIX
                    p = pbase + kk
                    v = np.zeros(8, np.float32)
                    if p < npix:
                        b = p // (H * W); r = p % (H * W); yy, xx = r // W, r % W
                        v = dy_[b, yy, xx, mc * 8:mc * 8 + 8] * (gate[b, yy, xx, mc * 8:mc * 8 + 8] > 0)
                    for q in range(8):
                        sm[((kk >> 3) * 2048 + (mc * 8 + q) * 16 + (kk & 7) * 2) // 2] = v[q]
                for i in range(PIX * (CI // 8)):
                    kk, nc = i % PIX, i // PIX
                    p = pbase + kk
                    v = np.zeros(8, np.float32)
                    if p < npix:
                        px = p % W; q_ = p // W; py = q_ % H; pb = q_ // H
                        yy, xx = py + ddy, px + ddx
                        if 0 <= yy < H and 0 <= xx < W: v = x[pb, yy, xx, nc * 8:nc * 8 + 8]
                    for q in range(8):
                        sm[(A_BYTES + (kk >> 3) * (CI * 16) + (nc * 8 + q) * 16 + (kk & 7) * 2) // 2] = v[q]
                for k in range(PIX // 16):
                    A = canon_read(sm, 2 * k * 2048, 2048, 128, 128)
                    B = canon_read(sm, A_BYTES + 2 * k * (CI * 16), CI * 16, 128, CI)
                    D += A @ B.T
            part[split, t] = D[:CO]
    return part.sum(0)   # [9][CO][CI]


def test_staging_reproduces_forward_dgrad_and_wgrad():
    rng = np.random.default_rng(0)
    n, H, W, CI, CO = 1, 6, 10, 16, 32
    x = rng.normal(size=(n, H, W, CI)).astype(np.float32)
    w = rng.normal(size=(9, CO, CI)).astype(np.float32) * 0.2
    b = rng.normal(size=CO).astype(np.float32) * 0.1
    xt = torch.tensor(x).permute(0, 3, 1, 2).requires_grad_(True)
    wt = torch.tensor(w).permute(1, 2, 0).reshape(CO, CI, 3, 3).contiguous().requires_grad_(True)
    bt = torch.tensor(b)
    yt = F.relu(F.conv2d(xt, wt, bt, padding=1))
    gy = torch.tensor(rng.normal(size=yt.shape).astype(np.float32))
    yt.backward(gy)
    y = conv_kernel(x, None, w, b, CI, CO, False, n, H, W)
    np.testing.assert_allclose(y, yt.detach().permute(0, 2, 3, 1).numpy(), atol=1e-4)
    g = gy.permute(0, 2, 3, 1).numpy()
    w_tr = np.ascontiguousarray(w.transpose(0, 2, 1))      # k_transpose_w
    dx = conv_kernel(g, y, w_tr, None, CO, CI, True, n, H, W)
    np.testing.assert_allclose(dx, xt.grad.permute(0, 2, 3, 1).numpy(), atol=1e-4)
    dw = wgrad_kernel(x, g, y, CI, CO, n, H, W, nsplit=3, PIX=64)
    np.testing.assert_allclose(dw, wt.grad.reshape(CO, CI, 9).permute(2, 0, 1).numpy(), atol=1e-4)
