// net_oracle.cpp -- CPU oracle of the learned preconditioner's network.
// TEST INFRASTRUCTURE ONLY: loaded by tests/ as the checker, never by the
// product.
//
// The network has no counterpart in the reference (it is the learned part
// the GPU build adds); this file restates its definition independently of
// the CUDA kernels: 3x3x3 convolutions accumulated in double, with BF16
// rounding (round to nearest even) at exactly the points where the GPU
// stores BF16 tensors, so GPU and oracle agree to FP32 accumulation order.
//
//   a0 = bf16(r / s) x [1, next to air, next to solid, 0] on cells with
//        type != 0 (air neighbour: in-grid, type 0, not solid; solid
//        neighbour: solid or outside the grid)
//   h0 = bf16(act(conv0(a0)))                       16 ch, N
//   p0 = bf16(avg8(h0))                             16 ch, N/2
//   h1 = bf16(act(conv1(p0)))                       32 ch, N/2
//   p1 = bf16(avg8(h1))                             32 ch, N/4
//   h2 = bf16(act(conv2(p1)))                       64 ch, N/4
//   u1 = bf16(act(conv3(up(h2)) + h1))              32 ch, N/2
//   u0 = bf16(act(conv4(up(u1)) + h0))              16 ch, N
// act = identity (default) or ReLU (lho_net_set_relu).
//   z  = fluid ? s * conv5(u0) : 0                  1 ch,  N
// No biases: the packed bias entries are ignored and get zero gradient.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

bool g_relu = false;  // activation: ReLU or identity (the GPU default)

constexpr int L = 6;
constexpr int CIN[L] = {4, 16, 32, 64, 32, 16};
constexpr int COUT[L] = {16, 32, 64, 32, 16, 1};

uint16_t bf_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu)) return uint16_t((u >> 16) | 0x40u);
    u += 0x7fffu + ((u >> 16) & 1u);
    return uint16_t(u >> 16);
}
float bf(float f) {
    uint32_t u = uint32_t(bf_bits(f)) << 16;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

long long poff(int l) {
    long long n = 0;
    for (int k = 0; k < l; ++k) n += 27LL * COUT[k] * CIN[k] + COUT[k];
    return n;
}

struct Grid {
    int n[3];
    long long vox() const { return (long long)n[0] * n[1] * n[2]; }
    long long idx(int x, int y, int z) const { return ((long long)x * n[1] + y) * n[2] + z; }
    bool in(int x, int y, int z) const { return x >= 0 && x < n[0] && y >= 0 && y < n[1] && z >= 0 && z < n[2]; }
};

using Vec = std::vector<double>;  // channels-last [vox][C]

// out[v][co] = sum_tap sum_ci in[v + off][ci] * w[tap][co][ci] (double sum)
Vec conv(const Grid& g, const Vec& in, int cin, const std::vector<float>& w, int cout) {
    Vec out(size_t(g.vox()) * cout, 0.0);
    for (int x = 0; x < g.n[0]; ++x)
        for (int y = 0; y < g.n[1]; ++y)
            for (int z = 0; z < g.n[2]; ++z) {
                double* o = &out[size_t(g.idx(x, y, z)) * cout];
                for (int tap = 0; tap < 27; ++tap) {
                    const int xx = x + tap / 9 - 1, yy = y + (tap / 3) % 3 - 1, zz = z + tap % 3 - 1;
                    if (!g.in(xx, yy, zz)) continue;
                    const double* a = &in[size_t(g.idx(xx, yy, zz)) * cin];
                    for (int co = 0; co < cout; ++co) {
                        const float* wr = &w[(size_t(tap) * cout + co) * cin];
                        double acc = 0.0;
                        for (int ci = 0; ci < cin; ++ci) acc += a[ci] * double(wr[ci]);
                        o[co] += acc;
                    }
                }
            }
    return out;
}

// dW[tap][co][ci] += sum_v g[v][co] * in[v + off][ci]
void wgrad(const Grid& g, const Vec& gr, int cout, const Vec& in, int cin, double* dw) {
    for (int x = 0; x < g.n[0]; ++x)
        for (int y = 0; y < g.n[1]; ++y)
            for (int z = 0; z < g.n[2]; ++z) {
                const double* gv = &gr[size_t(g.idx(x, y, z)) * cout];
                for (int tap = 0; tap < 27; ++tap) {
                    const int xx = x + tap / 9 - 1, yy = y + (tap / 3) % 3 - 1, zz = z + tap % 3 - 1;
                    if (!g.in(xx, yy, zz)) continue;
                    const double* a = &in[size_t(g.idx(xx, yy, zz)) * cin];
                    for (int co = 0; co < cout; ++co)
                        for (int ci = 0; ci < cin; ++ci) dw[(size_t(tap) * cout + co) * cin + ci] += gv[co] * a[ci];
                }
            }
}

// input gradient: dx[v][ci] = sum_tap sum_co g[v - off][co] * w[tap][co][ci]
Vec conv_t(const Grid& g, const Vec& gr, int cout, const std::vector<float>& w, int cin) {
    Vec out(size_t(g.vox()) * cin, 0.0);
    for (int x = 0; x < g.n[0]; ++x)
        for (int y = 0; y < g.n[1]; ++y)
            for (int z = 0; z < g.n[2]; ++z) {
                double* o = &out[size_t(g.idx(x, y, z)) * cin];
                for (int tap = 0; tap < 27; ++tap) {
                    const int xx = x - (tap / 9 - 1), yy = y - ((tap / 3) % 3 - 1), zz = z - (tap % 3 - 1);
                    if (!g.in(xx, yy, zz)) continue;
                    const double* gv = &gr[size_t(g.idx(xx, yy, zz)) * cout];
                    for (int co = 0; co < cout; ++co) {
                        const float* wr = &w[(size_t(tap) * cout + co) * cin];
                        for (int ci = 0; ci < cin; ++ci) o[ci] += gv[co] * double(wr[ci]);
                    }
                }
            }
    return out;
}

Grid half(const Grid& g) { return Grid{{g.n[0] / 2, g.n[1] / 2, g.n[2] / 2}}; }

Vec pool(const Grid& f, const Grid& c, const Vec& in, int C) {
    Vec out(size_t(c.vox()) * C);
    for (int x = 0; x < c.n[0]; ++x)
        for (int y = 0; y < c.n[1]; ++y)
            for (int z = 0; z < c.n[2]; ++z)
                for (int ch = 0; ch < C; ++ch) {
                    float acc = 0.f;
                    for (int k = 0; k < 8; ++k)
                        acc += float(in[size_t(f.idx(2 * x + (k >> 2), 2 * y + ((k >> 1) & 1), 2 * z + (k & 1))) * C + ch]);
                    out[size_t(c.idx(x, y, z)) * C + ch] = bf(acc * 0.125f);
                }
    return out;
}

Vec upsample(const Grid& c, const Grid& f, const Vec& in, int C) {
    Vec out(size_t(f.vox()) * C, 0.0);
    for (int x = 0; x < f.n[0]; ++x)
        for (int y = 0; y < f.n[1]; ++y)
            for (int z = 0; z < f.n[2]; ++z)
                if (c.in(x >> 1, y >> 1, z >> 1))
                    for (int ch = 0; ch < C; ++ch)
                        out[size_t(f.idx(x, y, z)) * C + ch] = in[size_t(c.idx(x >> 1, y >> 1, z >> 1)) * C + ch];
    return out;
}

// bf16(relu(float(acc) + b + skip))
Vec act(const Vec& acc, int C, const float* b, const Vec* skip) {
    Vec out(acc.size());
    for (size_t i = 0; i < acc.size(); ++i) {
        float v = float(acc[i]) + b[i % C];
        if (skip) v += float((*skip)[i]);
        out[i] = bf((!g_relu || v > 0.f) ? v : 0.f);
    }
    return out;
}

struct Fwd {
    Grid g0, g1, g2;
    float s;
    std::vector<uint8_t> fluid;
    Vec a0, h0, p0, h1, p1, h2, q1, u1, q0, u0;
    std::vector<float> y;
};

std::vector<float> wslice(const float* p, int l) {
    const long long o = poff(l);
    return std::vector<float>(p + o, p + o + 27LL * COUT[l] * CIN[l]);
}
std::vector<float> wbf(const float* p, int l) {
    std::vector<float> w = wslice(p, l);
    for (float& v : w) v = bf(v);
    return w;
}
const float kZeroBias[64] = {};
const float* bias(const float* p, int l) {
    (void)p, (void)l;
    return kZeroBias;  // bias-free network
}

Fwd forward(const float* params, const int dims[3], const float* r, const uint8_t* type, const uint8_t* solid,
            double scale) {
    Fwd f;
    f.g0 = Grid{{dims[0], dims[1], dims[2]}};
    f.g1 = half(f.g0);
    f.g2 = half(f.g1);
    const long long V0 = f.g0.vox();
    f.fluid.resize(size_t(V0));
    double ss = 0.0, cnt = 0.0;
    for (long long v = 0; v < V0; ++v) {
        f.fluid[size_t(v)] = type[v] != 0;
        if (type[v] != 0) {
            ss += double(r[v]) * double(r[v]);
            cnt += 1.0;
        }
    }
    f.s = scale > 0 ? float(scale) : float((cnt > 0 && ss > 0) ? std::sqrt(ss / cnt) : 1.0);
    f.a0.assign(size_t(V0) * 4, 0.0);
    const Grid& g0 = f.g0;
    for (int x = 0; x < g0.n[0]; ++x)
        for (int y = 0; y < g0.n[1]; ++y)
            for (int z = 0; z < g0.n[2]; ++z) {
                const long long v = g0.idx(x, y, z);
                if (!f.fluid[size_t(v)]) continue;
                bool air = false, sol = false;
                const int d[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
                for (int k = 0; k < 6; ++k) {
                    const int xx = x + d[k][0], yy = y + d[k][1], zz = z + d[k][2];
                    if (!g0.in(xx, yy, zz)) {
                        sol = true;
                        continue;
                    }
                    const long long u = g0.idx(xx, yy, zz);
                    if (solid && solid[u]) sol = true;
                    else if (type[u] == 0) air = true;
                }
                const double rh = bf(r[v] / f.s);
                f.a0[size_t(v) * 4 + 0] = rh;
                f.a0[size_t(v) * 4 + 1] = air ? rh : 0.0;
                f.a0[size_t(v) * 4 + 2] = sol ? rh : 0.0;
            }
    f.h0 = act(conv(f.g0, f.a0, 4, wbf(params, 0), 16), 16, bias(params, 0), nullptr);
    f.p0 = pool(f.g0, f.g1, f.h0, 16);
    f.h1 = act(conv(f.g1, f.p0, 16, wbf(params, 1), 32), 32, bias(params, 1), nullptr);
    f.p1 = pool(f.g1, f.g2, f.h1, 32);
    f.h2 = act(conv(f.g2, f.p1, 32, wbf(params, 2), 64), 64, bias(params, 2), nullptr);
    f.q1 = upsample(f.g2, f.g1, f.h2, 64);
    f.u1 = act(conv(f.g1, f.q1, 64, wbf(params, 3), 32), 32, bias(params, 3), &f.h1);
    f.q0 = upsample(f.g1, f.g0, f.u1, 32);
    f.u0 = act(conv(f.g0, f.q0, 32, wbf(params, 4), 16), 16, bias(params, 4), &f.h0);
    Vec y = conv(f.g0, f.u0, 16, wbf(params, 5), 1);
    f.y.resize(size_t(V0));
    for (long long v = 0; v < V0; ++v) f.y[size_t(v)] = float(y[size_t(v)]);
    return f;
}

// bf16(d * relu'(u))
Vec relu_grad(const Vec& d, const Vec& u) {
    Vec g(d.size());
    for (size_t i = 0; i < d.size(); ++i) g[i] = bf((!g_relu || u[i] > 0.0) ? float(d[i]) : 0.f);
    return g;
}

Vec sum_children(const Grid& f, const Grid& c, const Vec& d, int C) {
    Vec out(size_t(c.vox()) * C);
    for (int x = 0; x < c.n[0]; ++x)
        for (int y = 0; y < c.n[1]; ++y)
            for (int z = 0; z < c.n[2]; ++z)
                for (int ch = 0; ch < C; ++ch) {
                    float acc = 0.f;
                    for (int k = 0; k < 8; ++k)
                        acc += float(d[size_t(f.idx(2 * x + (k >> 2), 2 * y + ((k >> 1) & 1), 2 * z + (k & 1))) * C + ch]);
                    out[size_t(c.idx(x, y, z)) * C + ch] = acc;
                }
    return out;
}

// bf16((skip + 0.125 * dcoarse[parent]) * relu'(u))
Vec relu_grad_unpool(const Grid& f, const Grid& c, const Vec& skip, const Vec& dc, const Vec& u, int C) {
    Vec g(size_t(f.vox()) * C);
    for (int x = 0; x < f.n[0]; ++x)
        for (int y = 0; y < f.n[1]; ++y)
            for (int z = 0; z < f.n[2]; ++z)
                for (int ch = 0; ch < C; ++ch) {
                    const size_t i = size_t(f.idx(x, y, z)) * C + ch;
                    float d = float(skip[i]);
                    if (c.in(x >> 1, y >> 1, z >> 1)) d += 0.125f * float(dc[size_t(c.idx(x >> 1, y >> 1, z >> 1)) * C + ch]);
                    g[i] = bf((!g_relu || u[i] > 0.0) ? d : 0.f);
                }
    return g;
}

Vec to_float(const Vec& v) {
    Vec o(v.size());
    for (size_t i = 0; i < v.size(); ++i) o[i] = double(float(v[i]));
    return o;
}

void bgrad(const Vec& g, int C, double* db) {
    (void)g, (void)C, (void)db;  // bias-free network: zero bias gradients
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) long long lho_net_num_params() { return poff(L); }

// relu = 1: ReLU between layers; 0: identity (the GPU network's default)
__attribute__((visibility("default"))) void lho_net_set_relu(int relu) { g_relu = relu != 0; }

__attribute__((visibility("default"))) int lho_net_forward(const float* params, const int32_t dims[3], const float* r,
                                                           const uint8_t* type, const uint8_t* solid, double scale,
                                                           float* z) {
    const int d[3] = {dims[0], dims[1], dims[2]};
    Fwd f = forward(params, d, r, type, solid, scale);
    for (long long v = 0; v < f.g0.vox(); ++v) z[v] = f.fluid[size_t(v)] ? f.y[size_t(v)] * f.s : 0.f;
    return 0;
}

// gradient of sum(dz * z) with respect to the packed parameters
__attribute__((visibility("default"))) int lho_net_backward(const float* params, const int32_t dims[3], const float* r,
                                                            const uint8_t* type, const uint8_t* solid, double scale,
                                                            const float* dz, float* grad) {
    const int d[3] = {dims[0], dims[1], dims[2]};
    Fwd f = forward(params, d, r, type, solid, scale);
    const long long np = poff(L);
    std::vector<double> G(size_t(np), 0.0);
    auto GW = [&](int l) { return &G[size_t(poff(l))]; };
    auto GB = [&](int l) { return &G[size_t(poff(l) + 27LL * COUT[l] * CIN[l])]; };
    const long long V0 = f.g0.vox();
    Vec g5(static_cast<size_t>(V0), 0.0);
    for (long long v = 0; v < V0; ++v) g5[size_t(v)] = bf(f.fluid[size_t(v)] ? dz[v] * f.s : 0.f);
    wgrad(f.g0, g5, 1, f.u0, 16, GW(5));
    bgrad(g5, 1, GB(5));
    Vec du0 = to_float(conv_t(f.g0, g5, 1, wbf(params, 5), 16));
    Vec g4 = relu_grad(du0, f.u0);
    wgrad(f.g0, g4, 16, f.q0, 32, GW(4));
    bgrad(g4, 16, GB(4));
    Vec dq0 = to_float(conv_t(f.g0, g4, 16, wbf(params, 4), 32));
    Vec du1 = sum_children(f.g0, f.g1, dq0, 32);
    Vec g3 = relu_grad(du1, f.u1);
    wgrad(f.g1, g3, 32, f.q1, 64, GW(3));
    bgrad(g3, 32, GB(3));
    Vec dq1 = to_float(conv_t(f.g1, g3, 32, wbf(params, 3), 64));
    Vec dh2 = sum_children(f.g1, f.g2, dq1, 64);
    Vec g2 = relu_grad(dh2, f.h2);
    wgrad(f.g2, g2, 64, f.p1, 32, GW(2));
    bgrad(g2, 64, GB(2));
    Vec dp1 = to_float(conv_t(f.g2, g2, 64, wbf(params, 2), 32));
    Vec g1 = relu_grad_unpool(f.g1, f.g2, g3, dp1, f.h1, 32);
    wgrad(f.g1, g1, 32, f.p0, 16, GW(1));
    bgrad(g1, 32, GB(1));
    Vec dp0 = to_float(conv_t(f.g1, g1, 32, wbf(params, 1), 16));
    Vec g0 = relu_grad_unpool(f.g0, f.g1, g4, dp0, f.h0, 16);
    wgrad(f.g0, g0, 16, f.a0, 4, GW(0));
    bgrad(g0, 16, GB(0));
    for (long long i = 0; i < np; ++i) grad[i] = float(G[size_t(i)]);
    return 0;
}

}  // extern "C"
