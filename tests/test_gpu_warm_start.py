"""The PCG started from the previous step's solution (LHI_GUESS_PREVIOUS):
on the 64^3 dam break in mixed precision, stepped side by side with the
reference's zero guess, every solve still ends at ||r||/||b|| <= 1e-6 on
the true residual (measured against b here), takes no more iterations
than from zero (fewer in total), and the particles stay within 1e-4 dx."""
import numpy as np
import pytest

from liquidhairinteration_b200 import abi, scenes

from helpers import gpu_model

pytestmark = pytest.mark.gpu


def _b_norm(g):
    """||b|| over the cells with a matrix row (where the solve measures it)."""
    rhs = g.field("rhs").astype(np.float64)
    rows = g.field("liquidPhi") <= 0
    return float(np.sqrt((rhs[rows] ** 2).sum()))


def test_previous_guess_converges_with_fewer_iterations(lhi):
    spec = scenes.dam(64)
    spec.solver = dict(num_level=4, num_pre_smooth=2, num_post_smooth=2)
    cold = gpu_model(spec, "mixed", spec.solver_params())
    warm = gpu_model(spec, "mixed", spec.solver_params(initial_guess=abi.GUESS_PREVIOUS))
    pos, vel = scenes.seed(spec, "fp32")
    for m in (cold, warm):
        m.GetParticleSystem().SetParticles(pos, vel)
    its_c, its_w = [], []
    for step in range(12):
        for m, its in ((cold, its_c), (warm, its_w)):
            m.PreStep(spec.dt)
            m.Step(spec.dt)
            st = m.GetSolver().Stats()
            assert st["status"] == abi.LHI_OK, (step, st)
            its.append(st["iterations"])
        st = warm.GetSolver().Stats()
        assert st["true_residual"] <= 1e-6 * _b_norm(warm) * 1.0001, (step, st)
    assert all(w <= c + 1 for w, c in zip(its_w, its_c)), (its_w, its_c)
    assert sum(its_w) < sum(its_c), (its_w, its_c)
    d = np.abs(warm.GetParticleSystem().GetPositions() - cold.GetParticleSystem().GetPositions()).max()
    assert d <= 1e-4 * spec.dx, d / spec.dx
    cold.close()
    warm.close()
