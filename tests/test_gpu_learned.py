"""Learned-preconditioner FPCG on the GPU: training on residuals that the
plain GPU MGPCG records, the gain over the method without a preconditioner,
and the V-cycle fallback."""
import numpy as np
import pytest

from liquidhairinteration_b200 import abi, scenes

from helpers import gpu_model, oracle_model, rel_l2

pytestmark = pytest.mark.gpu


def _scene_after_p2g(oracle_mod, spec, solver):
    """GPU model holding the scene's P2G velocity field and liquid SDF
    (computed by the FP32 oracle so every solver sees the same system)."""
    o = oracle_model(oracle_mod, spec, "fp32")
    pos, vel = scenes.seed(spec, "fp32")
    o.set_particles(pos, vel)
    o.pre_step(spec.dt)
    o.particle_to_grid()
    o.apply_gravity(spec.dt)
    g = gpu_model(spec, "mixed", solver)
    for f in ("vx", "vy", "vz", "liquidPhi"):
        g.set_field(f, o.field(f))
    return g


@pytest.fixture(scope="module")
def trained(lhi, oracle_mod):
    """A network trained on MGPCG residuals of the 32^3 dam break."""
    from liquidhairinteration_b200.net import LearnedNet
    spec = scenes.dam(32)
    g = _scene_after_p2g(oracle_mod, spec, spec.solver_params(coarse_cells=64))
    s = g.GetSolver()
    s.RecordResiduals(64)
    st = s.Solve(spec.density, spec.dt)
    assert st["status"] == abi.LHI_OK
    net = LearnedNet(seed=3)
    first, last = net.train(g, steps=300, batch=8, lr=2e-3, seed=5)
    yield net, first, last, st["iterations"]
    net.close()


def test_training_reduces_loss(trained):
    net, first, last, _ = trained
    assert np.isfinite(first) and np.isfinite(last)
    assert last < 0.5 * first, (first, last)


def test_fpcg_converges_and_gains_over_unpreconditioned_cg(oracle_mod, trained):
    net, _, _, mg_iters = trained
    spec = scenes.dam(32)
    learned = spec.solver_params(preconditioner=abi.PRECOND_LEARNED, coarse_cells=64, max_iterations=400)
    g = _scene_after_p2g(oracle_mod, spec, learned)
    s = g.GetSolver()
    s.SetNetwork(net, fallbackIterations=400)
    st = s.Solve(spec.density, spec.dt)
    net_iters, fallback_at = s.LearnedStats()
    assert st["status"] == abi.LHI_OK, st
    assert st["true_residual"] <= 1e-6 * st["initial_residual"] * 1.0001
    plain = spec.solver_params(preconditioner=abi.PRECOND_NONE, max_iterations=2000)
    gp = _scene_after_p2g(oracle_mod, spec, plain)
    stp = gp.GetSolver().Solve(spec.density, spec.dt)
    assert stp["status"] == abi.LHI_OK
    # the network is a real preconditioner: far fewer iterations than CG alone
    assert st["iterations"] < 0.5 * stp["iterations"], (st["iterations"], stp["iterations"], net_iters, fallback_at)
    # same answer as plain CG to the stopping tolerance, on every cell whose
    # row is not empty (cells walled in on all six faces have no equation:
    # their pressure is whatever the preconditioner leaves there)
    rows = np.abs(gp.field("Adiag", 0)) >= 1e-8
    assert rel_l2(g.field("pressure")[rows], gp.field("pressure")[rows]) < 1e-4
    print(f"FPCG {st['iterations']} iterations ({net_iters} with the network, fallback at {fallback_at}); "
          f"MGPCG {mg_iters}; CG without a preconditioner {stp['iterations']}")


def test_committed_network_gain_over_cg_without_preconditioner(oracle_mod, lhi):
    """What the shipped network (liquidhairinteration_b200/weights, made by
    liquidhairinteration_b200.train) gains over the method without it: after
    20 iterations FPCG with the network alone (no fallback) leaves a smaller
    relative residual than CG without a preconditioner on the 64^3 dam break.
    (It is a weak preconditioner: the V-cycle reaches 1e-6 in about 10.)"""
    import os
    from liquidhairinteration_b200.net import LearnedNet
    spec = scenes.dam(64)
    net = LearnedNet(seed=0)
    net.load(os.path.join(os.path.dirname(abi.__file__), "weights", "fpcg.lhinet"))
    out = {}
    for mode, over in (("net", dict(preconditioner=abi.PRECOND_LEARNED)), ("cg", dict(preconditioner=abi.PRECOND_NONE))):
        g = _scene_after_p2g(oracle_mod, spec, spec.solver_params(coarse_cells=64, max_iterations=20, **over))
        if mode == "net":
            g.GetSolver().SetNetwork(net, fallbackIterations=-1)
        st = g.GetSolver().Solve(spec.density, spec.dt)
        out[mode] = st["final_residual"] / st["initial_residual"]
    print(f"relative residual after 20 iterations: network-only FPCG {out['net']:.3f}, CG {out['cg']:.3f}")
    assert out["net"] < out["cg"], out
    net.close()


def test_untrained_network_falls_back_to_vcycle(oracle_mod, lhi):
    from liquidhairinteration_b200.net import LearnedNet
    spec = scenes.dam(32)
    net = LearnedNet(seed=11)
    net.set_params(np.zeros_like(net.params()))  # M(r) = 0: no progress at all
    learned = spec.solver_params(preconditioner=abi.PRECOND_LEARNED, coarse_cells=64, max_iterations=200)
    g = _scene_after_p2g(oracle_mod, spec, learned)
    s = g.GetSolver()
    s.SetNetwork(net, fallbackIterations=50)
    st = s.Solve(spec.density, spec.dt)
    net_iters, fallback_at = s.LearnedStats()
    assert st["status"] == abi.LHI_OK, st
    assert 0 <= fallback_at <= 3, fallback_at
    net.close()


def test_fpcg_tail_graph_matches_host_loop(oracle_mod, lhi):
    """After the fallback the rest of an FPCG solve replays a graph of the
    V-cycle loop; the same solves run host-driven all the way (eager) give
    the same iterations, fallback points and pressure, bit for bit.  Both
    start from the same fields (P2G's cross-tile sums land in a run-dependent
    order, so whole steps are compared elsewhere within tolerances); the first
    solve builds the tail graph, the second replays it again."""
    import os
    from liquidhairinteration_b200.net import LearnedNet
    spec = scenes.dam(64)
    net = LearnedNet(seed=0)
    net.load(os.path.join(os.path.dirname(abi.__file__), "weights", "fpcg.lhinet"))
    runs = {}
    for eager in (0, 1):
        g = _scene_after_p2g(oracle_mod, spec, spec.solver_params(preconditioner=abi.PRECOND_LEARNED,
                                                                  coarse_cells=64, eager=eager))
        s = g.GetSolver()
        s.SetNetwork(net, fallbackIterations=0)
        out = []
        for _ in range(2):
            st = s.Solve(spec.density, spec.dt)
            assert st["status"] == abi.LHI_OK, st
            out.append((st["iterations"], s.LearnedStats(), g.field("pressure").copy()))
        assert lhi.lib().lhi_solver_graph_error(g._h) in (b"", None), lhi.lib().lhi_solver_graph_error(g._h)
        runs[eager] = out
        g.close()
    for (it0, ls0, p0), (it1, ls1, p1) in zip(runs[0], runs[1]):
        assert it0 == it1 and ls0 == ls1, (it0, it1, ls0, ls1)
        assert ls0[1] >= 0  # the fallback happened, so the tail graph ran
        assert np.array_equal(p0.view(np.uint32), p1.view(np.uint32))
    net.close()
