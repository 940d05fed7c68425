"""Around the step: LiquidModel<3>::GetCFL (LiquidModel.h:49-55), the
reference's clamp of dx / max|v| over the particles' velocities, the same
after a step and after the same particles are set again; and the particle
checkpoint, which restores the exact particle state in a fresh model whose
next steps then track the uninterrupted run."""
import numpy as np
import pytest

from liquidhairinteration_b200 import scenes

from helpers import gpu_model

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_cfl_after_step_and_after_set_particles(lhi, prec):
    spec = scenes.dam(32)
    # FP32 keeps x in float: its true residual stalls near 1e-5 relative, so
    # the FP32 solve stops on the recursive residual alone
    m = gpu_model(spec, prec, spec.solver_params(coarse_cells=64, true_residual_every=0 if prec == "fp32" else 10))
    pos, vel = scenes.seed(spec, "fp64" if prec == "fp64" else "fp32")
    m.GetParticleSystem().SetParticles(pos, vel)
    for _ in range(3):
        m.PreStep(spec.dt)
        m.Step(spec.dt)
    after_step = m.GetCFL()
    p, v, a = m.GetParticleSystem().GetParticles()
    m.GetParticleSystem().SetParticles(p, v, a)
    full = m.GetCFL()
    assert after_step == full
    vmax = float(np.abs(v.astype(np.float64)).max())
    assert vmax > 0
    dx = 1.0 / spec.n
    assert abs(full - min(max(dx / vmax, 0.001), 0.1)) <= 1e-6 * full
    m.close()


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_checkpoint_restores_particles(lhi, prec, tmp_path):
    """ParticleSystem SaveCheckpoint / LoadCheckpoint through the C-ABI: a
    fresh model loaded from a checkpoint holds the same particle bits, in
    the caller's order, gets the counters back, and its next steps repeat
    the uninterrupted run bit for bit.  A model of another precision or
    grid refuses the file."""
    spec = scenes.dam(16)
    solver = spec.solver_params(coarse_cells=64, true_residual_every=0 if prec == "fp32" else 10)
    m = gpu_model(spec, prec, solver)
    pos, vel = scenes.seed(spec, "fp64" if prec == "fp64" else "fp32")
    m.GetParticleSystem().SetParticles(pos, vel)
    for _ in range(2):
        m.PreStep(spec.dt)
        m.Step(spec.dt)
    path = tmp_path / "ck.npz"
    m.GetParticleSystem().SaveCheckpoint(path, step=2, time=2 * spec.dt)
    saved = m.GetParticleSystem().GetParticles()
    m2 = gpu_model(spec, prec, solver)
    counters = m2.GetParticleSystem().LoadCheckpoint(path)
    assert counters == {"step": 2, "time": 2 * spec.dt}
    for a, b in zip(m2.GetParticleSystem().GetParticles(), saved):
        assert np.array_equal(a, b)
    # P2G's shared-memory and global atomic adds land in a run-dependent
    # order, so the resumed run tracks the uninterrupted one to rounding
    # (amplified by the solves' stopping rule), not bit for bit
    for step in range(2):
        its = []
        for x in (m, m2):
            x.PreStep(spec.dt)
            x.Step(spec.dt)
            its.append(x.GetSolver().Stats()["iterations"])
        assert abs(its[0] - its[1]) <= 1, its
        (p1, v1, a1), (p2, v2, a2) = m.GetParticleSystem().GetParticles(), m2.GetParticleSystem().GetParticles()
        assert np.abs(p2.astype(np.float64) - p1).max() <= 1e-4 * spec.dx, f"resumed step {step + 3}"
        for x1, x2 in ((v1, v2), (a1, a2)):
            assert np.abs(x2.astype(np.float64) - x1).max() <= 1e-3 * np.abs(x1).max(), f"resumed step {step + 3}"
    other = gpu_model(spec, "fp64" if prec != "fp64" else "fp32")
    with pytest.raises(ValueError, match="precision"):
        other.GetParticleSystem().LoadCheckpoint(path)
    spec24 = scenes.dam(24)
    other24 = gpu_model(spec24, prec)
    with pytest.raises(ValueError, match="grid_dim"):
        other24.GetParticleSystem().LoadCheckpoint(path)
    assert other24.GetParticleSystem().NumParticles() == 0
    for x in (m, m2, other, other24):
        x.close()
