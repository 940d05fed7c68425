"""The network oracle (oracle/net_oracle.cpp) against an independent
restatement in torch on the CPU: float64 convolutions with the same BF16
storage points (forward) and autograd (backward).  The oracle rounds its
gradient tensors to BF16 where the GPU does and autograd does not, so the
gradient check uses a relative L2 tolerance per layer."""
import numpy as np
import pytest

from netcases import net_case, random_params

torch = pytest.importorskip("torch")
F = torch.nn.functional

LAYERS = [(4, 16), (16, 32), (32, 64), (64, 32), (32, 16), (16, 1)]


def bf(t):
    """BF16 rounding of the float32 value, identity gradient."""
    r = t.float().bfloat16().double()
    return t + (r - t).detach()


def torch_net(params, r, type_, solid, relu):
    p = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    ws, bs, off = [], [], 0
    for cin, cout in LAYERS:
        nw = 27 * cout * cin
        w = p[off:off + nw].reshape(3, 3, 3, cout, cin).permute(3, 4, 0, 1, 2)  # [cout, cin, dx, dy, dz]
        ws.append(bf(w))
        bs.append(p[off + nw:off + nw + cout])
        off += nw + cout
    fl = torch.tensor(type_ != 0)
    rr = torch.tensor(r, dtype=torch.float64)
    s = float(np.float32(np.sqrt(np.sum(r.astype(np.float64) ** 2 * (type_ != 0)) / max(1, (type_ != 0).sum()))))
    # neighbour classes: air (in-grid, type 0, not solid), solid (solid or outside)
    pad_t = np.pad(type_, 1, constant_values=0)
    pad_s = np.pad(solid, 1, constant_values=1)
    air = np.zeros(type_.shape, bool)
    sol = np.zeros(type_.shape, bool)
    nx, ny, nz = type_.shape
    for d in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
        sl = tuple(slice(1 + d[k], 1 + d[k] + type_.shape[k]) for k in range(3))
        sol |= pad_s[sl] != 0
        air |= (pad_s[sl] == 0) & (pad_t[sl] == 0)
    rh = bf(torch.where(fl, (rr.float() / np.float32(s)).double(), torch.zeros_like(rr)))
    a0 = torch.stack([rh, rh * torch.tensor(air), rh * torch.tensor(sol), torch.zeros_like(rh)])[None]

    def conv(x, l):
        return F.conv3d(x, ws[l], padding=1)

    def act(x, l, skip=None):
        v = x  # bias-free network
        if skip is not None:
            v = v + skip
        return bf(torch.relu(v) if relu else v)

    def pool(x):
        return bf(F.avg_pool3d(x, 2))

    def up(x, like):
        u = x.repeat_interleave(2, 2).repeat_interleave(2, 3).repeat_interleave(2, 4)
        out = torch.zeros_like(like)
        out[:, :u.shape[1], :u.shape[2], :u.shape[3], :u.shape[4]] = u[:, :, :like.shape[2], :like.shape[3],
                                                                        :like.shape[4]]
        return out

    h0 = act(conv(a0, 0), 0)
    h1 = act(conv(pool(h0), 1), 1)
    h2 = act(conv(pool(h1), 2), 2)
    u1 = act(conv(up(h2, torch.zeros(1, 64, *h1.shape[2:], dtype=torch.float64)), 3), 3, h1)
    u0 = act(conv(up(u1, torch.zeros(1, 32, *h0.shape[2:], dtype=torch.float64)), 4), 4, h0)
    y = conv(u0, 5)[0, 0]
    z = torch.where(fl, y * s, torch.zeros_like(y))
    return p, z


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("relu", [False, True])
@pytest.mark.parametrize("shape", [(8, 8, 8), (9, 6, 10)])
def test_net_oracle_matches_torch(oracle_mod, shape, relu):
    r, t, s = net_case(shape, seed=3)
    params = random_params(oracle_mod.net_num_params(), seed=4)
    oracle_mod.net_set_relu(relu)
    z_o = oracle_mod.net_forward(params, r, t, s)
    p, z_t = torch_net(params, r, t, s, relu)
    assert rel(z_o, z_t.detach().numpy()) < 1e-4
    dz = np.random.default_rng(5).standard_normal(shape).astype(np.float32)
    (z_t * torch.tensor(dz, dtype=torch.float64)).sum().backward()
    g_t = p.grad.numpy()
    g_o = oracle_mod.net_backward(params, r, t, s, dz)
    off = 0
    for cin, cout in LAYERS:
        nw = 27 * cout * cin
        assert rel(g_o[off:off + nw], g_t[off:off + nw]) < 3e-2, (cin, cout)
        assert rel(g_o[off + nw:off + nw + cout], g_t[off + nw:off + nw + cout]) < 3e-2, (cin, cout)
        off += nw + cout
