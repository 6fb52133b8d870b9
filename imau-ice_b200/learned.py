"""The learned warm start of solve_DIVA (include/diva_cnn.h) from Python.

``WarmStartNet`` owns one network for one grid size: it collects training samples
from contexts after converged solves (``add_sample``), trains on them on the device
(``train``: BF16 tensor-core convolutions with FP32 accumulation, Adam on FP32 master
weights), and warm-starts a context before its solve (``predict``): the predicted
velocities with the viscosity and basal stress completed from them, or the whole
predicted state (u_vav_cx, v_vav_cy, taub_cx, taub_cy, visc_eff_3D_a).
The viscosity iteration then runs to its own tolerance from there, so the prediction
changes the iteration count, not the converged velocities.

There is no host implementation: every call runs the kernels of libdiva_b200.so, and
the wrapper fails when the library or a GPU is missing.
"""
import ctypes as C

import numpy as np

from . import diva

N_OUT = 20      # head channels: u, v, taub_x, taub_y, log10 visc of up to 16 layers
IN_C = 16       # input channels (8 used)
# 3x3 layers in execution order: (name, cin, cout)
LAYERS = [("e1a", 16, 32), ("e1b", 32, 32), ("e2a", 32, 64), ("e2b", 64, 64), ("ba", 64, 128),
          ("bb", 128, 64), ("d2a", 128, 64), ("d2b", 64, 32), ("d1a", 64, 32), ("d1b", 32, 32)]
HEAD_C = 32


def weight_layout():
    """Offsets of the flat weight vector: {name: (w_off, w_shape, b_off, b_len)}, total."""
    out, off = {}, 0
    for name, ci, co in LAYERS:
        out[name] = (off, (9, co, ci), off + 9 * co * ci, co)
        off += 9 * co * ci + co
    out["head"] = (off, (N_OUT, HEAD_C), off + N_OUT * HEAD_C, N_OUT)
    off += N_OUT * HEAD_C + N_OUT
    return out, off


def _bind(lib):
    vp, i32, i64, f32p = C.c_void_p, C.c_int32, C.c_int64, C.POINTER(C.c_float)
    sig = {
        "create": [C.POINTER(vp), i32, i32, i32, i32, i32, C.c_uint64],
        "destroy": [vp],
        "num_weights": [vp, C.POINTER(i64)],
        "weights": [vp, f32p, i64, i32],
        "add_sample": [vp, vp],
        "num_samples": [vp, C.POINTER(i32)],
        "train": [vp, i32, C.c_float, C.c_uint64, f32p],
        "predict": [vp, vp, i32],
        "padded_shape": [vp, C.POINTER(i32), C.POINTER(i32)],
        "forward": [vp, vp, vp, i32],
        "train_step": [vp, vp, vp, i32, C.c_float, f32p],
        "grads": [vp, f32p, i64],
        "set_loss_weights": [vp, f32p, i32],
    }
    fns = {}
    for name, args in sig.items():
        f = getattr(lib, "diva_cnn_" + name)
        f.restype = C.c_int32
        f.argtypes = args
        fns[name] = f
    return fns


class WarmStartNet:
    """One network for contexts of ``grid``'s size (``nz`` <= 16 layers)."""

    def __init__(self, grid, batch=8, capacity=0, seed=0, backend=None):
        be = backend or diva.cuda_backend()
        if be.name != "cuda":
            raise diva.DivaError(7, "the warm-start network runs on the CUDA library only")
        self._f = _bind(be.lib)
        self.grid = grid
        self.batch = int(batch)
        self._h = C.c_void_p()
        self._check(self._f["create"](C.byref(self._h), grid.ny, grid.nx, grid.nz, self.batch,
                                      int(capacity), C.c_uint64(seed)), "create")
        hp, wp = C.c_int32(), C.c_int32()
        self._check(self._f["padded_shape"](self._h, C.byref(hp), C.byref(wp)), "padded_shape")
        self.padded_shape = (hp.value, wp.value)
        n = C.c_int64()
        self._check(self._f["num_weights"](self._h, C.byref(n)), "num_weights")
        self.num_weights = n.value

    def _check(self, st, what):
        if st != 0:
            raise diva.DivaError(st, f"diva_cnn_{what}")

    def close(self):
        if self._h:
            self._f["destroy"](self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # weights ---------------------------------------------------------------
    def get_weights(self):
        w = np.empty(self.num_weights, np.float32)
        self._check(self._f["weights"](self._h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size, 0), "weights")
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._check(self._f["weights"](self._h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size, 1), "weights")

    def grads(self):
        g = np.empty(self.num_weights, np.float32)
        self._check(self._f["grads"](self._h, g.ctypes.data_as(C.POINTER(C.c_float)), g.size), "grads")
        return g

    def save(self, path):
        np.savez(path, weights=self.get_weights(), ny=self.grid.ny, nx=self.grid.nx, nz=self.grid.nz)

    def load(self, path):
        d = np.load(path)
        if (int(d["ny"]), int(d["nx"]), int(d["nz"])) != (self.grid.ny, self.grid.nx, self.grid.nz):
            raise diva.DivaError(4, "weights were trained for another grid size")
        self.set_weights(d["weights"])

    # training set and training -----------------------------------------------
    def add_sample(self, ctx):
        """The context's fields and converged iteration state as one training sample."""
        self._check(self._f["add_sample"](self._h, ctx.h), "add_sample")

    @property
    def num_samples(self):
        n = C.c_int32()
        self._check(self._f["num_samples"](self._h, C.byref(n)), "num_samples")
        return n.value

    def set_loss_weights(self, w):
        """Loss weight of each of the N_OUT output channels (>= 0)."""
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._check(self._f["set_loss_weights"](self._h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size),
                    "set_loss_weights")

    def velocities_only(self):
        """Train on the velocity channels alone (what predict's default mode uses)."""
        w = np.zeros(N_OUT, np.float32)
        w[:2] = 1.0
        self.set_loss_weights(w)

    def train(self, epochs, lr=1e-3, seed=0):
        """Adam over the training set; returns the last epoch's mean squared error."""
        loss = C.c_float()
        self._check(self._f["train"](self._h, int(epochs), float(lr), C.c_uint64(seed), C.byref(loss)), "train")
        return loss.value

    def predict(self, ctx, complete_sweeps=10):
        """Warm-start ``ctx`` (call before solve_DIVA): the predicted velocities plus
        ``complete_sweeps`` state-completion sweeps, or with 0 the whole predicted state."""
        self._check(self._f["predict"](self._h, ctx.h, int(complete_sweeps)), "predict")

    # device-buffer forms (pointers to device memory) ----------------------------
    def forward(self, feat_ptr, out_ptr, n):
        self._check(self._f["forward"](self._h, C.c_void_p(feat_ptr), C.c_void_p(out_ptr), int(n)), "forward")

    def train_step(self, feat_ptr, tgt_ptr, n, lr):
        loss = C.c_float()
        self._check(self._f["train_step"](self._h, C.c_void_p(feat_ptr), C.c_void_p(tgt_ptr), int(n), float(lr),
                                          C.byref(loss)), "train_step")
        return loss.value
