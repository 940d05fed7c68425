// scene.cpp -- host-side scene building: boundary SDF evaluation, the seeded
// particle generator and the reference's lattice spawner.  Pure C++ (no
// device code); exported through the C-ABI in include/lhi.h.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "lhi.h"

namespace lhi {
namespace scene {

template <class S> inline S mac_min(S a, S b) { return (a < b) ? a : b; }
template <class S> inline S mac_max(S a, S b) { return (a > b) ? a : b; }
template <class S> inline S eig_maxi(S a, S b) { return (a < b) ? b : a; }

// RectBoundary / OperatorBoundary / SolidBoundary::Compute (Boundary.h:38-90),
// in the reference's evaluation order for Scalar S.
template <class S>
S boundary_compute(const lhi_boundary_node* nodes, int32_t count, int32_t idx, const S p[3], int depth = 0) {
    if (idx < 0 || idx >= count || depth > 64) throw std::invalid_argument("boundary tree: bad child index");
    const lhi_boundary_node& n = nodes[idx];
    switch (n.kind) {
        case LHI_BOUNDARY_RECT: {
            S q[3], qm[3];
            for (int i = 0; i < 3; ++i) {
                q[i] = std::abs(p[i] - S(n.center[i])) - S(n.half_extent[i]);
                qm[i] = eig_maxi(q[i], S(0));
            }
            S outside = std::sqrt(qm[0] * qm[0] + (qm[1] * qm[1] + qm[2] * qm[2]));
            S inside = mac_min(eig_maxi(q[0], eig_maxi(q[1], q[2])), S(0));
            return n.use_inside ? -outside - inside : outside + inside;
        }
        case LHI_BOUNDARY_SOLID: return S(1.0);
        case LHI_BOUNDARY_UNION:
            return mac_min(boundary_compute(nodes, count, n.left, p, depth + 1),
                           boundary_compute(nodes, count, n.right, p, depth + 1));
        case LHI_BOUNDARY_INTERSECTION:
            return mac_max(boundary_compute(nodes, count, n.left, p, depth + 1),
                           boundary_compute(nodes, count, n.right, p, depth + 1));
        case LHI_BOUNDARY_SUBTRACT:
            return mac_max(boundary_compute(nodes, count, n.left, p, depth + 1),
                           -boundary_compute(nodes, count, n.right, p, depth + 1));
        case LHI_BOUNDARY_NONE: return boundary_compute(nodes, count, n.left, p, depth + 1);
        default: throw std::invalid_argument("boundary tree: unknown node kind");
    }
}

// splitmix64 finaliser: a counter-based generator, so every particle's jitter
// depends only on (seed, cell, sub-cell, axis).
inline uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
inline double uniform01(uint64_t seed, uint64_t counter) {
    uint64_t h = mix64(seed ^ mix64(counter));
    return double(h >> 40) * (1.0 / 16777216.0);  // 24 random bits in [0, 1)
}

bool inside_prim(const lhi_fluid_prim& p, const double c[3]) {
    if (p.kind == LHI_FLUID_BOX) {
        for (int i = 0; i < 3; ++i)
            if (!(c[i] >= p.a[i] && c[i] < p.b[i])) return false;
        return true;
    }
    if (p.kind == LHI_FLUID_SPHERE) {
        double d2 = 0;
        for (int i = 0; i < 3; ++i) d2 += (c[i] - p.a[i]) * (c[i] - p.a[i]);
        return d2 < p.b[0] * p.b[0];
    }
    throw std::invalid_argument("unknown fluid primitive kind");
}

template <class S>
int64_t seed(const lhi_grid_desc& g, const lhi_boundary_node* nodes, int32_t count, int32_t root,
             const lhi_fluid_prim* prims, int32_t nprims, uint64_t seedv, S* pos, S* vel) {
    double dx[3];
    for (int i = 0; i < 3; ++i) dx[i] = (g.max_coord[i] - g.min_coord[i]) / g.dim[i];
    int64_t n = 0;
    for (int x = 0; x < g.dim[0]; ++x)
        for (int y = 0; y < g.dim[1]; ++y)
            for (int z = 0; z < g.dim[2]; ++z) {
                int idx[3] = {x, y, z};
                double c[3];
                for (int i = 0; i < 3; ++i) c[i] = g.min_coord[i] + (idx[i] + 0.5) * dx[i];
                int which = -1;
                for (int k = 0; k < nprims && which < 0; ++k)
                    if (inside_prim(prims[k], c)) which = k;
                if (which < 0) continue;
                if (count > 0 && boundary_compute<double>(nodes, count, root, c) < 0.0) continue;
                if (pos) {
                    uint64_t cell = (uint64_t(x) * g.dim[1] + y) * g.dim[2] + z;
                    for (int s = 0; s < 8; ++s) {
                        int sub[3] = {(s >> 2) & 1, (s >> 1) & 1, s & 1};
                        for (int i = 0; i < 3; ++i) {
                            double u = uniform01(seedv, (cell * 8 + s) * 3 + i);
                            double j = (u - 0.5) * 0.5;  // +-0.25 sub-cell
                            pos[3 * (n + s) + i] = S(g.min_coord[i] + dx[i] * (idx[i] + (sub[i] + 0.5 + j) * 0.5));
                            if (vel) vel[3 * (n + s) + i] = S(prims[which].velocity[i]);
                        }
                    }
                }
                n += 8;
            }
    return n;
}

// ParticleSystem<3>::SpawnParticles (ParticleSystem.cpp:45-64)
template <class S>
int64_t spawn(const double mn[3], const double mx[3], double default_radius, int64_t max_count, S* out) {
    S minc[3] = {S(mn[0]), S(mn[1]), S(mn[2])}, maxc[3] = {S(mx[0]), S(mx[1]), S(mx[2])};
    S r = S(default_radius);
    S interval = S(0.5 * double(r));
    int d[3];
    for (int i = 0; i < 3; ++i) d[i] = int((maxc[i] - minc[i]) / interval);
    int64_t total = std::min<int64_t>(max_count, int64_t(d[0]) * d[1] * d[2]);
    if (!out) return total;
    for (int xi = 0; xi < d[0]; ++xi)
        for (int yi = 0; yi < d[1]; ++yi)
            for (int zi = 0; zi < d[2]; ++zi) {
                int64_t index = int64_t(xi) * d[1] * d[2] + int64_t(yi) * d[2] + zi;
                if (index >= total) break;
                out[3 * index + 0] = S(xi) * interval + minc[0];
                out[3 * index + 1] = S(yi) * interval + minc[1];
                out[3 * index + 2] = S(zi) * interval + minc[2];
            }
    return total;
}

}  // namespace scene
}  // namespace lhi

extern "C" void lhi_set_error_message(const char* msg);

extern "C" {

LHI_API int lhi_boundary_eval(const lhi_boundary_node* nodes, int32_t count, int32_t root, int32_t precision,
                              const void* points, int64_t n, void* out) {
    try {
        if (!nodes || count <= 0 || (n > 0 && (!points || !out))) throw std::invalid_argument("null argument");
        if (precision == LHI_PRECISION_FP64) {
            const double* p = static_cast<const double*>(points);
            double* o = static_cast<double*>(out);
            for (int64_t i = 0; i < n; ++i) o[i] = lhi::scene::boundary_compute<double>(nodes, count, root, p + 3 * i);
        } else {
            const float* p = static_cast<const float*>(points);
            float* o = static_cast<float*>(out);
            for (int64_t i = 0; i < n; ++i) o[i] = lhi::scene::boundary_compute<float>(nodes, count, root, p + 3 * i);
        }
        return LHI_OK;
    } catch (const std::exception& e) {
        lhi_set_error_message(e.what());
        return LHI_E_INVALID_ARG;
    }
}

LHI_API int lhi_scene_seed_particles(const lhi_grid_desc* grid, const lhi_boundary_node* nodes, int32_t count,
                                     int32_t root, const lhi_fluid_prim* prims, int32_t nprims, uint64_t seed,
                                     int32_t precision, int64_t* n_out, void* pos, void* vel) {
    try {
        if (!grid || !n_out || (nprims > 0 && !prims)) throw std::invalid_argument("null argument");
        for (int i = 0; i < 3; ++i)
            if (grid->dim[i] < 1) throw std::invalid_argument("grid dimensions must be >= 1");
        if (precision == LHI_PRECISION_FP64)
            *n_out = lhi::scene::seed<double>(*grid, nodes, count, root, prims, nprims, seed,
                                              static_cast<double*>(pos), static_cast<double*>(vel));
        else
            *n_out = lhi::scene::seed<float>(*grid, nodes, count, root, prims, nprims, seed, static_cast<float*>(pos),
                                             static_cast<float*>(vel));
        return LHI_OK;
    } catch (const std::exception& e) {
        lhi_set_error_message(e.what());
        return LHI_E_INVALID_ARG;
    }
}

LHI_API int lhi_scene_spawn_lattice(const double min_coord[3], const double max_coord[3], double default_radius,
                                    int64_t max_count, int32_t precision, int64_t* n_out, void* pos) {
    try {
        if (!min_coord || !max_coord || !n_out) throw std::invalid_argument("null argument");
        if (!(default_radius > 0)) throw std::invalid_argument("default_radius must be > 0");
        if (precision == LHI_PRECISION_FP64)
            *n_out = lhi::scene::spawn<double>(min_coord, max_coord, default_radius, max_count,
                                               static_cast<double*>(pos));
        else
            *n_out = lhi::scene::spawn<float>(min_coord, max_coord, default_radius, max_count, static_cast<float*>(pos));
        return LHI_OK;
    } catch (const std::exception& e) {
        lhi_set_error_message(e.what());
        return LHI_E_INVALID_ARG;
    }
}

}  // extern "C"
