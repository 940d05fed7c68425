"""Error behaviour of the C-ABI on the GPU: every failure is a status code
(the Python mirror raises LhiError), nothing traps the device."""
import ctypes as C

import numpy as np
import pytest

from liquidhairinteration_b200 import abi, scenes

from helpers import gpu_model

pytestmark = pytest.mark.gpu


def test_nan_particles_report_nan(lhi):
    spec = scenes.dam(16)
    g = gpu_model(spec, "fp32")
    pos, vel = scenes.seed(spec, "fp32")
    vel[5] = np.nan
    g.GetParticleSystem().SetParticles(pos, vel)
    g.PreStep(spec.dt)
    with pytest.raises(lhi.LhiError) as e:
        g.Step(spec.dt)
    assert e.value.code == abi.LHI_E_NAN


def test_iteration_cap_reports_not_converged(lhi):
    spec = scenes.dam(16)
    g = gpu_model(spec, "mixed", spec.solver_params(max_iterations=1))
    pos, vel = scenes.seed(spec, "fp32")
    g.GetParticleSystem().SetParticles(pos, vel)
    g.PreStep(spec.dt)
    g.Particle2Grid()
    g.ApplyGravity(spec.dt)
    with pytest.raises(lhi.LhiError) as e:
        g.GetSolver().Solve(spec.density, spec.dt, check=True)
    assert e.value.code == abi.LHI_E_NOT_CONVERGED
    assert g.GetSolver().Stats()["iterations"] == 1


def test_invalid_arguments(lhi):
    L = lhi.lib()
    spec = scenes.dam(8)
    h = C.c_void_p()
    grid, solver, liquid = spec.grid_desc(), spec.solver_params(), spec.liquid_params()
    assert L.lhi_liquid_create(C.byref(grid), C.byref(solver), C.byref(liquid), 7, C.byref(h)) == abi.LHI_E_INVALID_ARG
    bad = abi.make_grid_desc((0, 8, 8), (0, 0, 0), (1, 1, 1))
    assert L.lhi_liquid_create(C.byref(bad), C.byref(solver), C.byref(liquid), 0, C.byref(h)) == abi.LHI_E_INVALID_ARG
    assert L.lhi_liquid_step(None, 0.01) == abi.LHI_E_INVALID_ARG
    g = gpu_model(spec, "fp32")
    cnt, eb = C.c_int64(), C.c_int32()
    assert L.lhi_liquid_field_size(g._h, 999, 0, C.byref(cnt), C.byref(eb)) == abi.LHI_E_INVALID_ARG
    assert L.lhi_liquid_field_size(g._h, abi.FIELD_ADIAG, 99, C.byref(cnt), C.byref(eb)) == abi.LHI_E_INVALID_ARG
    nodes = abi.boundary_array([{"kind": abi.BOUNDARY_UNION, "left": 1, "right": 5}, scenes.walls(8)])
    assert L.lhi_liquid_set_boundary(g._h, nodes, 2, 0) == abi.LHI_E_INVALID_ARG
    assert b"boundary tree" in L.lhi_last_error()
    liquid_big = abi.make_liquid_params(particle_radius=10.0)
    h2 = C.c_void_p()
    assert L.lhi_liquid_create(C.byref(grid), C.byref(solver), C.byref(liquid_big), 0, C.byref(h2)) == abi.LHI_OK
    pos = np.full((4, 3), 0.5, np.float32)
    assert L.lhi_liquid_set_particles(h2, 4, pos.ctypes.data_as(C.c_void_p), None, None) == abi.LHI_OK
    assert L.lhi_liquid_pre_step(h2, 0.01) == abi.LHI_E_INVALID_ARG
    L.lhi_liquid_destroy(h2)


def test_empty_scene_steps(lhi):
    """No particles: every stage is a no-op, like the reference's early returns."""
    spec = scenes.dam(8)
    g = gpu_model(spec, "fp32")
    g.GetParticleSystem().SetParticles(np.zeros((0, 3), np.float32))
    g.PreStep(spec.dt)
    g.Step(spec.dt)
    g.PostStep(spec.dt)
    assert g.GetParticleSystem().NumParticles() == 0
