"""The learned preconditioner's network through the C-ABI (include/lhi.h,
lhi_net_*).  No counterpart in the reference: it is the learned part of the
flexible PCG that LHI_PRECOND_LEARNED runs.

Layers (cin, cout), all 3x3x3 convolutions with zero padding:
  conv0 (4, 16)  full resolution      on [r / s, fluid, solid, air]
  conv1 (16, 32) half resolution      on avgpool(h0)
  conv2 (32, 64) quarter resolution   on avgpool(h1)
  conv3 (64, 32) half resolution      on upsample(h2), + h1
  conv4 (32, 16) full resolution      on upsample(u1), + h0
  conv5 (16, 1)  full resolution      -> z = s * conv5(u0) on fluid cells
"""
import ctypes as C

import numpy as np

from ._lib import call, lib

LAYERS = [(4, 16), (16, 32), (32, 64), (64, 32), (32, 16), (16, 1)]


def num_params():
    n = C.c_int64()
    call("lhi_net_num_params", C.byref(n))
    return n.value


def param_slices():
    """[(weight slice, bias slice, (27, cout, cin))] of the packed parameter vector."""
    out, off = [], 0
    for cin, cout in LAYERS:
        nw = 27 * cout * cin
        out.append((slice(off, off + nw), slice(off + nw, off + nw + cout), (27, cout, cin)))
        off += nw + cout
    return out


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class LearnedNet:
    """Owns one network on the GPU (FP32 master parameters, BF16 working
    copies, Adam state)."""

    def __init__(self, seed=0):
        h = C.c_void_p()
        call("lhi_net_create", int(seed), C.byref(h))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().lhi_net_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        out = np.empty(num_params(), np.float32)
        call("lhi_net_get_params", self._h, _p(out))
        return out

    def set_params(self, p):
        a = np.ascontiguousarray(p, np.float32)
        if a.size != num_params():
            raise ValueError(f"expected {num_params()} parameters, got {a.size}")
        call("lhi_net_set_params", self._h, _p(a))

    def set_relu(self, on):
        """ReLU between layers (default off: a linear multilevel operator)."""
        call("lhi_net_set_relu", self._h, 1 if on else 0)

    def set_sparse(self, on):
        """Evaluate each convolution only on the output tiles the cells with
        type != 0 depend on (default on; the result is the same, bit for bit)."""
        call("lhi_net_set_sparse", self._h, 1 if on else 0)

    def save(self, path):
        call("lhi_net_save", self._h, str(path).encode())

    def load(self, path):
        call("lhi_net_load", self._h, str(path).encode())

    def forward(self, r, type_, solid=None, scale=0.0):
        rr = np.ascontiguousarray(r, np.float32)
        tt = np.ascontiguousarray(type_, np.uint8)
        ss = None if solid is None else np.ascontiguousarray(solid, np.uint8)
        z = np.empty(rr.shape, np.float32)
        call("lhi_net_forward_host", self._h, (C.c_int32 * 3)(*rr.shape), _p(rr), _p(tt), _p(ss), float(scale), _p(z))
        return z

    def backward(self, r, type_, solid, dz, scale=0.0):
        rr = np.ascontiguousarray(r, np.float32)
        tt = np.ascontiguousarray(type_, np.uint8)
        ss = None if solid is None else np.ascontiguousarray(solid, np.uint8)
        d = np.ascontiguousarray(dz, np.float32)
        g = np.empty(num_params(), np.float32)
        call("lhi_net_backward_host", self._h, (C.c_int32 * 3)(*rr.shape), _p(rr), _p(tt), _p(ss), float(scale),
             _p(d), _p(g))
        return g

    def train(self, model, steps, batch=16, lr=1e-3, seed=0):
        """Adam steps on the residuals ``model`` recorded (its solver's
        RecordResiduals + Solve) with its level-0 matrix; returns the mean
        loss ||A M(r) - r||^2 / ||r||^2 of the first and the last step."""
        a, b = C.c_double(), C.c_double()
        call("lhi_net_train", self._h, model._h, int(steps), int(batch), float(lr), int(seed), C.byref(a), C.byref(b))
        return a.value, b.value

