"""CorrectVolume (LiquidModel.cpp:1086-1132) with its neighbour search
(NeighborSearch.h:22-108) on the GPU against the oracle's restatement.

The oracle walks a particle's neighbours cell by cell in caller order; the
GPU walks the cell-sorted particles, whose order within a cell is the
caller order (the sort breaks ties by particle id), so the sums match bit
for bit on fresh particles and after steps.  Whole steps with the
correction on track the oracle within a tolerance (their P2G sums in
another order).  Coincident particles take the seeded counter-based random
numbers on both sides."""
import numpy as np
import pytest

from liquidhairinteration_b200 import abi, scenes

from helpers import assert_bitwise, gpu_model, oracle_model

pytestmark = pytest.mark.gpu


def _scene_particles(spec, prec):
    pos, vel = scenes.seed(spec, "fp64" if prec == "fp64" else "fp32")
    pos = pos.copy()
    # three particles on one spot and two more pairs: the coincident branch
    pos[101] = pos[100]
    pos[102] = pos[100]
    pos[2001] = pos[2000]
    pos[-1] = pos[-2]
    return pos, vel


def _pair(oracle_mod, spec, prec, **liquid):
    g = gpu_model(spec, prec) if not liquid else None
    if liquid:
        from liquidhairinteration_b200.model import LiquidModel
        from liquidhairinteration_b200._lib import call
        g = LiquidModel.from_params(spec.grid_desc(), spec.solver_params(), spec.liquid_params(**liquid), prec)
        call("lhi_liquid_set_boundary", g._h, abi.boundary_array(spec.boundary), len(spec.boundary), 0)
    o = oracle_mod.Oracle(spec.grid_desc(), spec.solver_params(), spec.liquid_params(**liquid), dbl=prec == "fp64")
    o.set_boundary(spec.boundary)
    return g, o


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_correct_volume_bitwise_on_fresh_particles(oracle_mod, lhi, prec):
    spec = scenes.dam(24)
    g, o = _pair(oracle_mod, spec, prec)
    pos, vel = _scene_particles(spec, prec)
    g.GetParticleSystem().SetParticles(pos, vel)
    o.set_particles(pos, vel)
    dt = 1.0 / 480.0
    for call_no in range(3):
        before = g.GetParticleSystem().GetPositions()
        g.CorrectVolume(dt)
        o.correct_volume(dt)
        after = g.GetParticleSystem().GetPositions()
        assert_bitwise(after, o.get_particles()[0], f"call {call_no}")
        moved = np.flatnonzero((after != before).any(axis=1))
        assert moved.size > 0
        assert (moved % 8 == call_no).all(), "only the particles of this step of the cycle move"


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_correct_volume_bitwise_after_steps(oracle_mod, lhi, prec):
    """After 3 steps the device holds the particles in the previous sort's
    order; the oracle gets the GPU's particles (caller order) and both
    correct them: bit for bit."""
    spec = scenes.dam(16)
    g, o = _pair(oracle_mod, spec, prec)
    pos, vel = scenes.seed(spec, "fp64" if prec == "fp64" else "fp32")
    g.GetParticleSystem().SetParticles(pos, vel)
    for _ in range(3):
        g.PreStep(spec.dt)
        g.Step(spec.dt)
    o.set_particles(*g.GetParticleSystem().GetParticles())
    for call_no in range(2):
        g.CorrectVolume(spec.dt)
        o.correct_volume(spec.dt)
        assert_bitwise(g.GetParticleSystem().GetPositions(), o.get_particles()[0], f"call {call_no}")


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_step_with_correct_volume_tracks_oracle(oracle_mod, lhi, prec):
    """Step ending with CorrectVolume (the call the reference's Step has
    commented out), 6 steps: GPU and oracle stay together."""
    spec = scenes.dam(16)
    g, o = _pair(oracle_mod, spec, prec, correct_volume=1)
    pos, vel = scenes.seed(spec, "fp64" if prec == "fp64" else "fp32")
    g.GetParticleSystem().SetParticles(pos, vel)
    o.set_particles(pos, vel)
    ref = oracle_model(oracle_mod, spec, prec)  # the same run without the correction
    ref.set_particles(pos, vel)
    for _ in range(6):
        g.PreStep(spec.dt)
        g.Step(spec.dt)
        o.pre_step(spec.dt)
        o.step(spec.dt)
        ref.pre_step(spec.dt)
        ref.step(spec.dt)
    p_g, p_o = g.GetParticleSystem().GetPositions(), o.get_particles()[0]
    d = np.abs(p_g - p_o).max()
    assert d < (1e-9 if prec == "fp64" else 1e-3) * spec.dx, d / spec.dx
    # and the correction did something
    assert np.abs(p_o - ref.get_particles()[0]).max() > 1e-3 * spec.dx
