"""Tile-sparse evaluation of the learned preconditioner's network: each
convolution runs only on the output tiles that the cells with type != 0
depend on, and z must equal the dense evaluation's bit for bit.

Every case first runs a dense forward on another residual over an all-fluid
grid, so that every activation buffer holds unrelated non-zero values where
the sparse pass does not write: a tile missing from the plan would then show
up as a difference."""
import numpy as np
import pytest

from liquidhairinteration_b200 import abi, scenes

from netcases import net_case, random_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def net(lhi, oracle_mod):
    from liquidhairinteration_b200.net import LearnedNet
    n = LearnedNet(seed=21)
    n.set_params(random_params(oracle_mod.net_num_params(), seed=22))
    yield n
    n.close()


def _poison(net, shape, seed):
    rng = np.random.default_rng(seed)
    r = rng.standard_normal(shape).astype(np.float32)
    net.set_sparse(False)
    net.forward(r, np.full(shape, 2, np.uint8), None, scale=1.0)


def _cases():
    out = []
    for shape, seed in (((16, 16, 32), 1), ((9, 6, 10), 2), ((37, 21, 13), 3), ((40, 34, 70), 4)):
        r, t, s = net_case(shape, seed)
        out.append((f"levelset{shape}", r, t, s))
    # a few small blobs in a mostly empty grid (most tiles skipped)
    shape = (48, 40, 56)
    rng = np.random.default_rng(5)
    t = np.zeros(shape, np.uint8)
    for _ in range(4):
        c = rng.integers(0, shape)
        sl = tuple(slice(max(0, c[a] - 2), c[a] + 3) for a in range(3))
        t[sl] = 2
    r = (rng.standard_normal(shape) * (t != 0)).astype(np.float32)
    out.append(("blobs", r, t, None))
    # one fluid cell in the last corner (ragged tiles on every axis)
    shape = (13, 19, 23)
    t = np.zeros(shape, np.uint8)
    t[-1, -1, -1] = 2
    r = np.zeros(shape, np.float32)
    r[-1, -1, -1] = 1.5
    out.append(("corner", r, t, None))
    # no fluid at all, and fluid everywhere
    shape = (12, 12, 12)
    out.append(("empty", np.zeros(shape, np.float32), np.zeros(shape, np.uint8), None))
    r = np.random.default_rng(6).standard_normal(shape).astype(np.float32)
    out.append(("full", r, np.full(shape, 2, np.uint8), None))
    return out


CASES = _cases()


@pytest.mark.parametrize("relu", [False, True])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_sparse_forward_is_bitwise_dense(net, case, relu):
    _, r, t, s = case
    net.set_relu(relu)
    _poison(net, r.shape, 7)
    net.set_sparse(True)
    z_sparse = net.forward(r, t, s)
    net.set_sparse(False)
    z_dense = net.forward(r, t, s)
    assert np.all(z_sparse[t == 0] == 0)
    assert np.array_equal(z_sparse.view(np.uint32), z_dense.view(np.uint32)), \
        int(np.count_nonzero(z_sparse != z_dense))
    net.set_sparse(True)


def _scene_after_p2g(oracle_mod, spec, solver):
    from helpers import gpu_model, oracle_model
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


def test_fpcg_solve_sparse_equals_dense(oracle_mod, lhi):
    """The solver's network applications with the tile plan give the same
    iterations and the same pressure, bit for bit, as the dense network."""
    import os
    from liquidhairinteration_b200.net import LearnedNet
    spec = scenes.dam(64)
    net = LearnedNet(seed=0)
    net.load(os.path.join(os.path.dirname(abi.__file__), "weights", "fpcg.lhinet"))
    out = {}
    for sparse in (True, False):
        net.set_sparse(sparse)
        params = spec.solver_params(preconditioner=abi.PRECOND_LEARNED, coarse_cells=64, max_iterations=60)
        g = _scene_after_p2g(oracle_mod, spec, params)
        s = g.GetSolver()
        s.SetNetwork(net, fallbackIterations=-1)
        st = s.Solve(spec.density, spec.dt)
        out[sparse] = (st["iterations"], st["final_residual"], g.field("pressure"))
    assert out[True][0] == out[False][0], (out[True][:2], out[False][:2])
    assert out[True][1] == out[False][1]
    assert np.array_equal(out[True][2].view(np.uint32), out[False][2].view(np.uint32))
    net.close()
