"""The learned preconditioner's network on the GPU (tcgen05 implicit-GEMM
convolutions, BF16 storage, FP32 accumulation) against the CPU network
oracle, which has the same BF16 storage points and accumulates in double.
Tolerances are relative L2: a BF16 rounding that flips on one side is one
BF16 unit (2^-8) of that value."""
import numpy as np
import pytest

from netcases import net_case, random_params

pytestmark = pytest.mark.gpu

LAYERS = [(4, 16), (16, 32), (32, 64), (64, 32), (32, 16), (16, 1)]
SHAPES = [(8, 8, 8), (9, 6, 10), (16, 16, 32), (24, 20, 36)]


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(np.asarray(b, np.float64)), 1e-30))


def _bf16_bits(a):
    u = np.ascontiguousarray(a, np.float32).view(np.uint32)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


@pytest.mark.parametrize("n,k", [(16, 16), (64, 64), (32, 48)])
def test_tensor_core_selftest(lhi, n, k):
    """One CTA, D = A B^T through the network's tcgen05 descriptors."""
    import ctypes as C
    rng = np.random.default_rng(n * 100 + k)
    a = _bf16_bits(rng.standard_normal((128, k)))
    b = _bf16_bits(rng.standard_normal((n, k)))
    d = np.zeros((128, n), np.float32)
    stage = C.c_int32()
    rc = lhi.lib().lhi_net_tensor_core_selftest(n, k, a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p),
                                                d.ctypes.data_as(C.c_void_p), C.byref(stage))
    assert rc == 0, (lhi.lib().lhi_last_error(), stage.value)
    af = (a.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    bf = (b.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    ref = af @ bf.T
    assert np.abs(d - ref).max() < 1e-3 * np.abs(ref).max(), (np.abs(d - ref).max(), stage.value)


@pytest.fixture(scope="module")
def net(lhi):
    from liquidhairinteration_b200.net import LearnedNet
    n = LearnedNet(seed=7)
    yield n
    n.close()


@pytest.mark.parametrize("relu", [False, True])
@pytest.mark.parametrize("shape", SHAPES)
def test_net_forward_matches_oracle(oracle_mod, net, shape, relu):
    r, t, s = net_case(shape, seed=11)
    params = random_params(oracle_mod.net_num_params(), seed=12)
    net.set_params(params)
    net.set_relu(relu)
    oracle_mod.net_set_relu(relu)
    z = net.forward(r, t, s)
    z_o = oracle_mod.net_forward(params, r, t, s)
    assert np.all(z[t == 0] == 0)
    assert rel(z, z_o) < 1e-2, rel(z, z_o)


@pytest.mark.parametrize("relu", [False, True])
@pytest.mark.parametrize("shape", SHAPES)
def test_net_gradients_match_oracle(oracle_mod, net, shape, relu):
    r, t, s = net_case(shape, seed=13)
    params = random_params(oracle_mod.net_num_params(), seed=14)
    net.set_params(params)
    net.set_relu(relu)
    oracle_mod.net_set_relu(relu)
    dz = np.random.default_rng(15).standard_normal(shape).astype(np.float32)
    g = net.backward(r, t, s, dz)
    g_o = oracle_mod.net_backward(params, r, t, s, dz)
    off = 0
    for cin, cout in LAYERS:
        nw = 27 * cout * cin
        assert rel(g[off:off + nw], g_o[off:off + nw]) < 3e-2, ("W", cin, cout, rel(g[off:off + nw], g_o[off:off + nw]))
        assert rel(g[off + nw:off + nw + cout], g_o[off + nw:off + nw + cout]) < 3e-2, ("b", cin, cout)
        off += nw + cout


def test_net_scale_invariance(net):
    """M(a r) = a M(r): the input is normalised by its RMS."""
    r, t, s = net_case((16, 16, 16), seed=17)
    z1 = net.forward(r, t, s)
    z2 = net.forward(np.float32(4.0) * r, t, s)
    assert rel(z2, 4.0 * z1) < 1e-6


def test_linear_network_is_linear(net):
    """The default (identity activation) network is linear in r: M(a + b) = M(a) + M(b) up to BF16 storage."""
    net.set_relu(False)
    r, t, s = net_case((16, 16, 16), seed=19)
    r2, _, _ = net_case((16, 16, 16), seed=20)
    za, zb, zab = net.forward(r, t, s, scale=1.0), net.forward(r2, t, s, scale=1.0), net.forward(r + r2, t, s, scale=1.0)
    assert rel(zab, za + zb) < 3e-2
