"""Builders shared by the parity tests: a GPU LiquidModel and an oracle
model on the same seeded scene, and array comparison helpers."""
import numpy as np

from liquidhairinteration_b200 import abi, scenes

ORACLE_PRECISION = {"fp32": False, "mixed": False, "fp64": True}


def gpu_model(spec, precision, solver=None):
    from liquidhairinteration_b200.model import LiquidModel
    from liquidhairinteration_b200._lib import call
    m = LiquidModel.from_params(spec.grid_desc(), solver or spec.solver_params(), spec.liquid_params(), precision)
    call("lhi_liquid_set_boundary", m._h, abi.boundary_array(spec.boundary), len(spec.boundary), 0)
    return m


def oracle_model(po, spec, precision, solver=None):
    o = po.Oracle(spec.grid_desc(), solver or spec.solver_params(), spec.liquid_params(),
                  dbl=ORACLE_PRECISION[precision])
    o.set_boundary(spec.boundary)
    return o


def pair(po, spec, precision, solver=None, with_particles=True):
    g = gpu_model(spec, precision, solver)
    o = oracle_model(po, spec, precision, solver)
    if with_particles:
        pos, vel = scenes.seed(spec, "fp64" if precision == "fp64" else "fp32")
        g.GetParticleSystem().SetParticles(pos, vel)
        o.set_particles(pos, vel)
    return g, o


def bits(a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.float32:
        return a.view(np.uint32)
    if a.dtype == np.float64:
        return a.view(np.uint64)
    return a


def assert_bitwise(a, b, what=""):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, f"{what}: shape {a.shape} vs {b.shape}"
    eq = bits(a) == bits(b)
    if not eq.all():
        idx = np.flatnonzero(~eq)
        i = idx[0]
        raise AssertionError(f"{what}: {idx.size} of {a.size} values differ; first at {i}: "
                             f"{a.reshape(-1)[i]!r} vs {b.reshape(-1)[i]!r}")


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def assert_close(a, b, rtol, atol, what=""):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    assert a.shape == b.shape, f"{what}: shape {a.shape} vs {b.shape}"
    bad = ~np.isclose(a, b, rtol=rtol, atol=atol)
    if bad.any():
        i = np.flatnonzero(bad)[0]
        raise AssertionError(f"{what}: {bad.sum()} of {a.size} values outside rtol={rtol} atol={atol}; "
                             f"first at {i}: {a.reshape(-1)[i]!r} vs {b.reshape(-1)[i]!r}; "
                             f"max abs diff {np.abs(a - b).max():.3e}")
