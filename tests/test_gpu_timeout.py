"""The bounded waits of the TMA-staged solver kernels run out (their limit
set to zero from the host): the solve reports LHI_E_TIMEOUT, every kernel
drains its own copies in flight before leaving, and the context stays
usable -- the next solve with the normal limit gives the same pressure as
a handle that never timed out."""
import ctypes as C

import numpy as np
import pytest

from liquidhairinteration_b200 import abi, scenes

from helpers import assert_bitwise, gpu_model

pytestmark = pytest.mark.gpu


def _loaded(spec):
    g = gpu_model(spec, "mixed")
    pos, vel = scenes.seed(spec, "fp32")
    g.GetParticleSystem().SetParticles(pos, vel)
    g.PreStep(spec.dt)
    g.Particle2Grid()
    g.ApplyGravity(spec.dt)
    return g


def test_stage_wait_timeout_is_reported_and_recovers(lhi):
    spec = scenes.dam(64)  # the fused sweep, TMA SpMV and restriction run on 64^3 and 32^3
    ref = _loaded(spec)
    st_ref = ref.GetSolver().Solve(spec.density, spec.dt)
    assert st_ref["status"] == abi.LHI_OK
    g = _loaded(spec)
    g.GetSolver().Solve(spec.density, spec.dt)  # host-driven first solve; the next ones replay the graph
    try:
        lhi.call("lhi_debug_set_stage_wait_limit", 0.0)
        st = abi.SolveStats()
        rc = lhi.lib().lhi_solver_solve(g._h, spec.density, spec.dt, C.byref(st))
        assert rc == abi.LHI_E_TIMEOUT and st.status == abi.LHI_E_TIMEOUT, (rc, st.as_dict())
    finally:
        lhi.call("lhi_debug_set_stage_wait_limit", 200.0)
    st2 = g.GetSolver().Solve(spec.density, spec.dt)
    assert st2["status"] == abi.LHI_OK and st2["iterations"] == st_ref["iterations"]
    assert_bitwise(g.field("pressure"), ref.field("pressure"), "pressure after the timed-out solve")


def test_network_pipeline_wait_timeout_is_reported_and_recovers(lhi):
    """The brick convolution's pipeline waits run out (limit 0): the forward
    reports LHI_E_TIMEOUT, the kernel drains its own brick loads and MMAs
    before leaving, and the next forward with the normal limit gives the
    same z, bit for bit, as before."""
    from liquidhairinteration_b200._lib import LhiError
    from liquidhairinteration_b200.net import LearnedNet
    from netcases import net_case
    net = LearnedNet(seed=5)
    r, t, s = net_case((24, 20, 36), seed=3)
    z_ref = net.forward(r, t, s)
    try:
        lhi.call("lhi_debug_set_stage_wait_limit", 0.0)
        with pytest.raises(LhiError) as e:
            net.forward(r, t, s)
        assert e.value.code == abi.LHI_E_TIMEOUT
    finally:
        lhi.call("lhi_debug_set_stage_wait_limit", 200.0)
    z = net.forward(r, t, s)
    assert np.array_equal(z.view(np.uint32), z_ref.view(np.uint32))
    net.close()


def test_learned_solve_reports_network_timeout_and_recovers(lhi):
    """An FPCG solve whose network and solver waits run out reports
    LHI_E_TIMEOUT; with the normal limit the next solve of the same handle
    gives the iterations and pressure of a handle that never timed out."""
    import os
    from liquidhairinteration_b200.net import LearnedNet
    spec = scenes.dam(64)
    net = LearnedNet(seed=0)
    net.load(os.path.join(os.path.dirname(abi.__file__), "weights", "fpcg.lhinet"))
    params = spec.solver_params(preconditioner=abi.PRECOND_LEARNED, coarse_cells=64)

    def loaded():
        g = gpu_model(spec, "mixed", params)
        pos, vel = scenes.seed(spec, "fp32")
        g.GetParticleSystem().SetParticles(pos, vel)
        g.PreStep(spec.dt)
        g.Particle2Grid()
        g.ApplyGravity(spec.dt)
        g.GetSolver().SetNetwork(net, fallbackIterations=0)
        return g

    ref = loaded()
    st_ref = ref.GetSolver().Solve(spec.density, spec.dt)
    assert st_ref["status"] == abi.LHI_OK
    g = loaded()
    try:
        lhi.call("lhi_debug_set_stage_wait_limit", 0.0)
        st = abi.SolveStats()
        rc = lhi.lib().lhi_solver_solve(g._h, spec.density, spec.dt, C.byref(st))
        assert rc == abi.LHI_E_TIMEOUT and st.status == abi.LHI_E_TIMEOUT, (rc, st.as_dict())
    finally:
        lhi.call("lhi_debug_set_stage_wait_limit", 200.0)
    st2 = g.GetSolver().Solve(spec.density, spec.dt)
    assert st2["status"] == abi.LHI_OK and st2["iterations"] == st_ref["iterations"], (st2, st_ref)
    assert_bitwise(g.field("pressure"), ref.field("pressure"), "pressure after the timed-out learned solve")
    ref.close()
    g.close()
    net.close()
