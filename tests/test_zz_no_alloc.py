"""lhi_divergence_noalloc: the divergence diagnostic for callers that cannot
allocate device memory (a host that owns every device byte in its own pool,
or a frame loop that must not stall on cudaMalloc/cudaFree).  It must give
what the handle's
lhi_liquid_compute_divergence gives on the same fields: the max-norm exactly
(a maximum does not depend on order) and the mean within 1e-9 of the
max-norm (both are double sums of the same per-cell values, taken in another
block order).

The file is named so that pytest collects it last: a failure here leaves
every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

from liquidhairinteration_b200 import abi, scenes

from helpers import gpu_model

pytestmark = pytest.mark.gpu

FIELDS = ("liquidPhi", "liquidWx", "liquidWy", "liquidWz", "vx", "vy", "vz")
MEAN_TOL = 1e-9  # relative to the max-norm


def _device_fields(model, torch):
    return [torch.from_numpy(model.field(f).copy()).cuda() for f in FIELDS]


def _noalloc(lhi, dims, dx, precision, bufs):
    m, mx = C.c_double(), C.c_double()
    ptrs = [C.c_void_p(b.data_ptr()) for b in bufs]
    lhi.call("lhi_divergence_noalloc", (C.c_int32 * 3)(*dims), dx, precision, *ptrs, None, C.byref(m),
             C.byref(mx))
    return m.value, mx.value


def _handle(model):
    m, mx = C.c_double(), C.c_double()
    from liquidhairinteration_b200._lib import call
    call("lhi_liquid_compute_divergence", model._h, C.byref(m), C.byref(mx))
    return m.value, mx.value


def _check(got, want):
    mean, mx = got
    mean_h, mx_h = want
    assert mx == mx_h, (mx, mx_h)
    assert abs(mean - mean_h) <= MEAN_TOL * max(mx_h, 1e-30), (mean, mean_h)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_divergence_noalloc_matches_handle_twice(lhi, prec):
    torch = pytest.importorskip("torch")
    spec = scenes.dam(32)
    g = gpu_model(spec, prec)
    pos, vel = scenes.seed(spec, "fp64" if prec == "fp64" else "fp32")
    # seeded random particle velocities, so the field has divergence to measure
    vel = np.random.default_rng(21).uniform(-1.0, 1.0, size=vel.shape).astype(vel.dtype)
    g.GetParticleSystem().SetParticles(pos, vel)
    g.PreStep(spec.dt)
    g.Particle2Grid()
    g.ApplyGravity(spec.dt)
    dims = (spec.n,) * 3
    dx = C.c_double * 3
    d = dx()
    lhi.call("lhi_liquid_get_dx", g._h, d)
    code = {"mixed": abi.PRECISION_MIXED, "fp64": abi.PRECISION_FP64}[prec]

    # first call: the velocity field before the projection
    want = _handle(g)
    bufs = _device_fields(g, torch)
    torch.cuda.synchronize()
    got = _noalloc(lhi, dims, d[0], code, bufs)
    assert want[1] > 0
    _check(got, want)

    # second call in a row, on the projected field: nothing of the first
    # call's scratch may leak into it
    g.Projection(spec.dt)
    want2 = _handle(g)
    bufs2 = _device_fields(g, torch)
    torch.cuda.synchronize()
    got2 = _noalloc(lhi, dims, d[0], code, bufs2)
    _check(got2, want2)
    assert want2[1] < want[1]


def test_divergence_noalloc_rejects_grids_above_limit(lhi):
    torch = pytest.importorskip("torch")
    dummy = [torch.zeros(4, device="cuda") for _ in FIELDS]
    m, mx = C.c_double(), C.c_double()
    rc = lhi.lib().lhi_divergence_noalloc((C.c_int32 * 3)(257, 256, 256), 1.0 / 256, abi.PRECISION_FP32,
                                          *[C.c_void_p(b.data_ptr()) for b in dummy], None, C.byref(m),
                                          C.byref(mx))
    assert rc == abi.LHI_E_INVALID_ARG
    assert b"scratch limit" in lhi.lib().lhi_last_error()
