// lhi_oracle.cpp -- CPU oracle of the liquid step.  TEST INFRASTRUCTURE ONLY:
// the checker for the CUDA path, never part of it.
//
// Restates the reference's 3D liquid path in plain C++ (float = the
// reference's Scalar, or double), deterministic.  The
// arithmetic follows the reference expression by expression, including:
//   * Eigen's fixed-size reductions: squaredNorm/dot of a 3-vector evaluate
//     as a0 + (a1 + a2) (Eigen redux_novec_unroller splits the range in half);
//     maxCoeff as maxi(a0, maxi(a1, a2)) with maxi(a, b) = (a < b) ? b : a.
//   * windows.h min/max macros (Definition.h:22): min(a,b) = (a < b) ? a : b,
//     max(a,b) = (a > b) ? a : b, evaluated in the promoted type (double when
//     one operand is a double literal) and then narrowed.
//   * double-literal promotion, e.g. (1. - w) * z + w * term in Smooth.
// Built with -ffp-contract=off so no multiply-add is fused.
//
// The reference's own data races (its OpenMP loops add into shared sums and
// flags without ordering) are replaced by deterministic
// semantics: serial sums in PCG; extrapolation flags either Jacobi (GPU
// semantics) or serial x-y-z order (the reference with one OpenMP thread).
//
// Threads: only loops whose result cannot depend on the thread count run in
// parallel (OpenMP, lho_set_threads):
//   * loops whose iterations write disjoint cells, faces, nodes or particles
//     (one colour of a red-black sweep, restriction, prolongation, matrix and
//     right-hand side, G2P, advection, Jacobi extrapolation, ...);
//   * scatters (P2G sums, the liquid SDF's minimum) split into x slabs of the
//     target grid: each thread walks every particle in the serial order and
//     keeps the window nodes of its own slab, so every node receives the same
//     terms in the same order as in the serial loop;
//   * every reduction (dot products, residual norms) is a serial pass in the
//     serial loop's order over values the parallel pass stored.
// So the results are bit-identical for any thread count.
#include "lhi_oracle.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

namespace {

int g_threads = 0;  // 0: every processor
inline int nthreads() { return g_threads > 0 ? g_threads : omp_get_num_procs(); }
// [lo, hi) of n split into nt near-equal parts, part t
inline void slab(int n, int t, int nt, int& lo, int& hi) {
    lo = int((long long)n * t / nt);
    hi = int((long long)n * (t + 1) / nt);
}

template <class S> S eps_of() { return S(1e-8); }  // EPSILON (Definition.h:88)

template <class S> inline S mac_min(S a, S b) { return (a < b) ? a : b; }
template <class S> inline S mac_max(S a, S b) { return (a > b) ? a : b; }
template <class S> inline S eig_maxi(S a, S b) { return (a < b) ? b : a; }

// MathUtils::IsSmall (MathUtils.h:8)
template <class S> inline bool is_small(S v) { return std::abs(v) < eps_of<S>(); }

// MathUtils::Clamp (MathUtils.h:10) with Scalar arguments
template <class S> inline S clampS(S v, S lo, S hi) { return mac_min(hi, mac_max(lo, v)); }

// MathUtils::Lerp / Bilerp / Trilerp (MathUtils.h:12-33)
template <class S> inline S lerp(S v0, S v1, S f) { return v0 + clampS(f, S(0.0), S(1.0)) * (v1 - v0); }
template <class S> inline S bilerp(S v00, S v10, S v01, S v11, S f1, S f2) {
    S a = lerp(v00, v10, f1);
    S b = lerp(v01, v11, f1);
    return lerp(a, b, clampS(f2, S(0.0), S(1.0)));
}
template <class S>
inline S trilerp(S v000, S v100, S v010, S v110, S v001, S v101, S v011, S v111, S f1, S f2, S f3) {
    S a = bilerp(v000, v100, v010, v110, f1, f2);
    S b = bilerp(v001, v101, v011, v111, f1, f2);
    return lerp(a, b, clampS(f3, S(0.0), S(1.0)));
}

// MathUtils::FractionInRegion(left, right) (MathUtils.cpp:29-35)
template <class S> inline S fraction_in_region(S l, S r) {
    S ans = S(0.0);
    if (l < S(0.0) && r < S(0.0)) ans = S(1.0);
    else if (l < S(0.0) && S(0.0) < r) ans = l / (l - r);
    else if (l > S(0.0) && S(0.0) > r) ans = r / (r - l);
    return ans;
}

// max(0.1, FractionInRegion(a, b)) with the windows.h macro: the comparison
// and the selected value are double, then narrowed to Scalar.
template <class S> inline S frac_floor(S f) {
    double v = (0.1 > double(f)) ? 0.1 : double(f);
    return S(v);
}

// MathUtils::Clamp(1.0 - FractionInRegion(a, b), 0.0, 1.0): the argument is
// evaluated in double and narrowed on binding to the Scalar parameter.
template <class S> inline S open_fraction(S a, S b) {
    S val = S(1.0 - double(fraction_in_region(a, b)));
    return clampS(val, S(0.0), S(1.0));
}

// MathUtils::GetBarycentricCoord (MathUtils.cpp:75-88)
template <class S> inline void barycentric(S x, int minI, int maxI, int& index, S& frac) {
    index = int(std::floor(x));
    frac = x - S(index);
    if (index < minI) {
        index = minI;
        frac = S(0.0);
    } else if (index > maxI - 2) {
        index = maxI - 2;
        frac = S(1.0);
    }
}

// BSplineKernel::QuadraticWeight / GradQuadraticWeight (Kernel.h:12-31)
template <class S> inline S qweight(S d) {
    d = std::abs(d);
    if (d < S(0.5f)) return S(0.75f) - d * d;
    else if (d < S(1.5f)) return S(0.5f) * (S(1.5f) - d) * (S(1.5f) - d);
    return S(0.0f);
}
template <class S> inline S gqweight(S d) {
    d = std::abs(d);
    if (d < S(0.5f)) return S(-2.f) * d;
    else if (d < S(1.5f)) return d - S(1.5f);
    return S(0.f);
}

// Eigen 3-vector reductions
template <class S> inline S sqnorm3(S a, S b, S c) { return a * a + (b * b + c * c); }
template <class S> inline S dot3(S a0, S a1, S a2, S b0, S b1, S b2) { return a0 * b0 + (a1 * b1 + a2 * b2); }

// ------------------------------------------------------------ boundary tree
// RectBoundary / OperatorBoundary / SolidBoundary::Compute (Boundary.h:38-90)
template <class S>
S boundary_compute(const lhi_boundary_node* nodes, int32_t count, int32_t idx, const S p[3]) {
    if (idx < 0 || idx >= count) return S(1.0);
    const lhi_boundary_node& n = nodes[idx];
    switch (n.kind) {
        case LHI_BOUNDARY_RECT: {
            S q[3], qm[3];
            for (int i = 0; i < 3; ++i) {
                S c = S(n.center[i]);
                S h = S(n.half_extent[i]);
                q[i] = std::abs(p[i] - c) - h;
                qm[i] = eig_maxi(q[i], S(0));  // cwiseMax(Scalar(0))
            }
            S outside = std::sqrt(sqnorm3(qm[0], qm[1], qm[2]));
            S mc = eig_maxi(q[0], eig_maxi(q[1], q[2]));
            S inside = mac_min(mc, S(0));
            return n.use_inside ? -outside - inside : outside + inside;
        }
        case LHI_BOUNDARY_SOLID: return S(1.0);
        case LHI_BOUNDARY_UNION:
            return mac_min(boundary_compute(nodes, count, n.left, p), boundary_compute(nodes, count, n.right, p));
        case LHI_BOUNDARY_INTERSECTION:
            return mac_max(boundary_compute(nodes, count, n.left, p), boundary_compute(nodes, count, n.right, p));
        case LHI_BOUNDARY_SUBTRACT:
            return mac_max(boundary_compute(nodes, count, n.left, p), -boundary_compute(nodes, count, n.right, p));
        case LHI_BOUNDARY_NONE: return boundary_compute(nodes, count, n.left, p);
        default: return S(1.0);
    }
}

struct Dims {
    int nx, ny, nz;
};

template <class S> struct Field {
    int ax = 0, ay = 0, az = 0;
    std::vector<S> d;
    void resize(int x, int y, int z) {
        ax = x;
        ay = y;
        az = z;
        d.assign(size_t(x) * y * z, S(0));
    }
    inline S& operator()(int x, int y, int z) { return d[(size_t(x) * ay + y) * az + z]; }
    inline const S& operator()(int x, int y, int z) const { return d[(size_t(x) * ay + y) * az + z]; }
    void fill(S v) { std::fill(d.begin(), d.end(), v); }
};

template <class S> struct Model {
    // grid (Grid.h:146-171)
    int nx, ny, nz;
    S minc[3], maxc[3], dx[3];
    Field<S> vx, vy, vz, tvx, tvy, tvz, wx, wy, wz, lwx, lwy, lwz, pressure, liquidPhi, solidPhi;
    Field<uint8_t> isValid;
    // particles
    int64_t np = 0;
    std::vector<S> pos, vel, aff;  // pos/vel xyz AoS, aff 9 column-major
    S radius;
    // parameters
    S density, gravity;
    int extrap_iters;
    // CorrectVolume (LiquidModel.cpp:1086-1132)
    int correct_cycle = 8, correct_step = 0;
    bool correct_in_step = false;
    unsigned long long correct_calls = 0;
    // solver (PressureSolver.h:121-145)
    lhi_solver_params sp;
    int maxLevel;
    S tolerance, smoothFactor;
    Field<S> rhs, p, x, tmp;  // tmp: the true residual when r is not overwritten
    std::vector<Field<S>> r, z, Adiag;
    std::vector<std::vector<S>> Acoef;  // 6 per cell
    std::vector<Dims> ldims;
    S oldRZ = 0, newRZ = 0, alpha = 0, beta = 0;
    lhi_solve_stats last{};

    Model(const lhi_grid_desc& g, const lhi_solver_params& s, const lhi_liquid_params& lp) {
        nx = g.dim[0];
        ny = g.dim[1];
        nz = g.dim[2];
        for (int i = 0; i < 3; ++i) {
            minc[i] = S(g.min_coord[i]);
            maxc[i] = S(g.max_coord[i]);
        }
        // Grid<3>::Grid (Grid.cpp:94-97): dx = Scalar(interval / dimension)
        int dims[3] = {nx, ny, nz};
        for (int i = 0; i < 3; ++i) dx[i] = S((maxc[i] - minc[i]) / S(dims[i]));
        vx.resize(nx + 1, ny, nz);
        vy.resize(nx, ny + 1, nz);
        vz.resize(nx, ny, nz + 1);
        tvx.resize(nx + 1, ny, nz);
        tvy.resize(nx, ny + 1, nz);
        tvz.resize(nx, ny, nz + 1);
        wx.resize(nx + 1, ny, nz);
        wy.resize(nx, ny + 1, nz);
        wz.resize(nx, ny, nz + 1);
        lwx.resize(nx + 1, ny, nz);
        lwy.resize(nx, ny + 1, nz);
        lwz.resize(nx, ny, nz + 1);
        pressure.resize(nx, ny, nz);
        liquidPhi.resize(nx, ny, nz);
        solidPhi.resize(nx + 1, ny + 1, nz + 1);
        isValid.resize(nx + 1, ny + 1, nz + 1);
        // ParticleSystem(numParticles, m_grid.dx.x()): radius = 2 * dx.x
        radius = lp.particle_radius > 0 ? S(lp.particle_radius) : S(2 * dx[0]);
        density = S(lp.density);
        gravity = S(lp.gravity);
        extrap_iters = lp.extrapolate_iterations > 0 ? lp.extrapolate_iterations : 5;
        correct_cycle = lp.correct_cycle > 0 ? lp.correct_cycle : 8;
        correct_in_step = lp.correct_volume != 0;
        // CGSolver<3>::CGSolver (PressureSolver.cpp:422-447)
        sp = s;
        tolerance = S(s.tolerance);
        smoothFactor = S(s.smoothing_factor);
        maxLevel = std::max(1, s.num_level);
        if (s.preconditioner != LHI_PRECOND_MULTIGRID) maxLevel = 1;
        r.resize(maxLevel);
        z.resize(maxLevel);
        Adiag.resize(maxLevel);
        Acoef.resize(maxLevel);
        ldims.resize(maxLevel);
        for (int l = 0; l < maxLevel; ++l) {
            Dims d{nx / (1 << l), ny / (1 << l), nz / (1 << l)};
            ldims[l] = d;
            r[l].resize(d.nx, d.ny, d.nz);
            z[l].resize(d.nx, d.ny, d.nz);
            Adiag[l].resize(d.nx, d.ny, d.nz);
            Acoef[l].assign(size_t(d.nx) * d.ny * d.nz * 6, S(0));
        }
        rhs.resize(nx, ny, nz);
        p.resize(nx, ny, nz);
        x.resize(nx, ny, nz);
        tmp.resize(nx, ny, nz);
    }

    // ---------------------------------------------------------- Grid helpers
    // Grid<3>::Clear (Grid.cpp:157-169); isValid is not reset.
    void clear() {
        pressure.fill(S(0.0));
        liquidPhi.fill(S(3 * dx[0]));
        vx.fill(S(0.0));
        wx.fill(S(0.0));
        tvx.fill(S(0.0));
        vy.fill(S(0.0));
        wy.fill(S(0.0));
        tvy.fill(S(0.0));
        vz.fill(S(0.0));
        wz.fill(S(0.0));
        tvz.fill(S(0.0));
    }

    bool in_grid(S x_, S y_, S z_) const {
        return minc[0] <= x_ && minc[1] <= y_ && minc[2] <= z_ && x_ <= maxc[0] && y_ <= maxc[1] &&
               z_ <= maxc[2];
    }

    // Grid<3>::GetSolidPhi (Grid.cpp:128-155)
    S solid_phi_at(S x_, S y_, S z_) const {
        if (!in_grid(x_, y_, z_)) {
            S vX = clampS(x_, S(minc[0] + dx[0]), S(maxc[0] - dx[0]));
            S vY = clampS(y_, S(minc[1] + dx[1]), S(maxc[1] - dx[1]));
            S vZ = clampS(z_, S(minc[2] + dx[2]), S(maxc[2] - dx[2]));
            if (!in_grid(vX, vY, vZ)) return std::numeric_limits<S>::quiet_NaN();  // NaN input
            S g[3];
            solid_gradient(vX, vY, vZ, g);
            return solid_phi_at(vX, vY, vZ) + g[0] * (x_ - vX) + g[1] * (y_ - vY) + g[2] * (z_ - vZ);
        }
        S lx = (x_ - minc[0]) / dx[0];
        S ly = (y_ - minc[1]) / dx[1];
        S lz = (z_ - minc[2]) / dx[2];
        int xi, yi, zi;
        S fx, fy, fz;
        barycentric(lx, 0, nx + 1, xi, fx);
        barycentric(ly, 0, ny + 1, yi, fy);
        barycentric(lz, 0, nz + 1, zi, fz);
        const Field<S>& sp_ = solidPhi;
        return trilerp(sp_(xi, yi, zi), sp_(xi + 1, yi, zi), sp_(xi, yi + 1, zi), sp_(xi + 1, yi + 1, zi),
                       sp_(xi, yi, zi + 1), sp_(xi + 1, yi, zi + 1), sp_(xi, yi + 1, zi + 1),
                       sp_(xi + 1, yi + 1, zi + 1), fx, fy, fz);
    }

    // Grid<3>::GetSolidGradient (Grid.cpp:175-192)
    void solid_gradient(S x_, S y_, S z_, S g[3]) const {
        if (!in_grid(x_, y_, z_)) {
            S vX = clampS(x_, S(minc[0] + dx[0]), S(maxc[0] - dx[0]));
            S vY = clampS(y_, S(minc[1] + dx[1]), S(maxc[1] - dx[1]));
            S vZ = clampS(z_, S(minc[2] + dx[2]), S(maxc[2] - dx[2]));
            if (!in_grid(vX, vY, vZ)) {  // NaN coordinates: the reference recurses without end here
                g[0] = g[1] = g[2] = std::numeric_limits<S>::quiet_NaN();
                return;
            }
            solid_gradient(vX, vY, vZ, g);
            return;
        }
        S eps = S(1e-4);
        S left = solid_phi_at(x_ - eps, y_, z_);
        S right = solid_phi_at(x_ + eps, y_, z_);
        S bottom = solid_phi_at(x_, y_ - eps, z_);
        S top = solid_phi_at(x_, y_ + eps, z_);
        S front = solid_phi_at(x_, y_, z_ + eps);
        S back = solid_phi_at(x_, y_, z_ - eps);
        S div = S(2.0 * double(eps));  // Vector3 / double: the double is narrowed to Scalar
        S v0 = (right - left) / div, v1 = (top - bottom) / div, v2 = (front - back) / div;
        S n2 = sqnorm3(v0, v1, v2);  // normalized(): n / sqrt(squaredNorm) if > 0
        if (n2 > S(0)) {
            S n = std::sqrt(n2);
            g[0] = v0 / n;
            g[1] = v1 / n;
            g[2] = v2 / n;
        } else {
            g[0] = v0;
            g[1] = v1;
            g[2] = v2;
        }
    }

    // ------------------------------------------------------- solid / liquid
    void set_boundary(const lhi_boundary_node* nodes, int32_t count, int32_t root) {
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (int xi = 0; xi < nx + 1; ++xi)
            for (int yi = 0; yi < ny + 1; ++yi)
                for (int zi = 0; zi < nz + 1; ++zi) {
                    // Vector3(xi, yi, zi).cwiseProduct(dx) + minCoord
                    S pp[3] = {S(xi) * dx[0] + minc[0], S(yi) * dx[1] + minc[1], S(zi) * dx[2] + minc[2]};
                    solidPhi(xi, yi, zi) = boundary_compute<S>(nodes, count, root, pp);
                }
        compute_face_fractions();
    }

    // LiquidModel<3>::ComputeSolidPhi face fractions (LiquidModel.cpp:574-610):
    // liquidWx uses the y-edge, liquidWy and liquidWz both use the x-edge.
    void compute_face_fractions() {
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (int xi = 0; xi < nx + 1; ++xi)
            for (int yi = 0; yi < ny; ++yi)
                for (int zi = 0; zi < nz; ++zi)
                    lwx(xi, yi, zi) = open_fraction(solidPhi(xi, yi, zi), solidPhi(xi, yi + 1, zi));
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (int xi = 0; xi < nx; ++xi)
            for (int yi = 0; yi < ny + 1; ++yi)
                for (int zi = 0; zi < nz; ++zi)
                    lwy(xi, yi, zi) = open_fraction(solidPhi(xi, yi, zi), solidPhi(xi + 1, yi, zi));
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (int xi = 0; xi < nx; ++xi)
            for (int yi = 0; yi < ny; ++yi)
                for (int zi = 0; zi < nz + 1; ++zi)
                    lwz(xi, yi, zi) = open_fraction(solidPhi(xi, yi, zi), solidPhi(xi + 1, yi, zi));
    }

    // Grid<3>::Point2Index (Grid.h:127-133)
    void point2index(const S* q, int c[3]) const {
        for (int i = 0; i < 3; ++i) c[i] = int((q[i] - minc[i]) / dx[i]);
    }

    // LiquidModel<3>::ComputeLiquidPhi (LiquidModel.cpp:540-560)
    void compute_liquid_phi() {
        if (np == 0) return;
        int dX = int(std::ceil(radius / dx[0]));
        int dY = int(std::ceil(radius / dx[1]));
        int dZ = int(std::ceil(radius / dx[2]));
        // x slabs of the cells; every thread walks all particles in order
#pragma omp parallel num_threads(nthreads())
        {
            int xlo, xhi;
            slab(nx, omp_get_thread_num(), omp_get_num_threads(), xlo, xhi);
            liquid_phi_slab(dX, dY, dZ, xlo, xhi);
        }
    }
    void liquid_phi_slab(int dX, int dY, int dZ, int xlo, int xhi) {
        for (int64_t pi = 0; pi < np; ++pi) {
            const S* q = &pos[3 * pi];
            int c[3];
            point2index(q, c);
            for (int xi = std::max(xlo, c[0] - dX); xi <= std::min(xhi - 1, c[0] + dX); ++xi)
                for (int yi = std::max(0, c[1] - dY); yi <= std::min(ny - 1, c[1] + dY); ++yi)
                    for (int zi = std::max(0, c[2] - dZ); zi <= std::min(nz - 1, c[2] + dZ); ++zi) {
                        // Index2Point: (index + 0.5) * dx + minCoord
                        S cx = (S(xi) + S(0.5)) * dx[0] + minc[0];
                        S cy = (S(yi) + S(0.5)) * dx[1] + minc[1];
                        S cz = (S(zi) + S(0.5)) * dx[2] + minc[2];
                        S phi = std::sqrt(sqnorm3(S(cx - q[0]), S(cy - q[1]), S(cz - q[2]))) - radius;
                        S& cur = liquidPhi(xi, yi, zi);
                        cur = mac_min(cur, phi);
                    }
        }
    }

    // ------------------------------------------------------------------ P2G
    // LiquidModel<3>::Particle2Grid (LiquidModel.cpp:614-721), serial
    // particle order; zero-weight nodes add +-0 and are skipped.
    template <int A>
    void p2g_component(const S* q, const S* v, const S* C, const S g[3], const int ci[3], const int del[3],
                       int xlo, int xhi) {
        Field<S>& wf = (A == 0) ? wx : (A == 1) ? wy : wz;
        Field<S>& vf = (A == 0) ? vx : (A == 1) ? vy : vz;
        int hx = nx - 1 + (A == 0), hy = ny - 1 + (A == 1), hz = nz - 1 + (A == 2);
        // window columns in this thread's slab, in the serial order
        const int d0 = std::max(-del[0], xlo - ci[0]), d1 = std::min(del[0], xhi - 1 - ci[0]);
        for (int ddx = d0; ddx <= d1; ++ddx)
            for (int ddy = -del[1]; ddy <= del[1]; ++ddy)
                for (int ddz = -del[2]; ddz <= del[2]; ++ddz) {
                    int xi = ci[0] + ddx, yi = ci[1] + ddy, zi = ci[2] + ddz;
                    if (xi < 0 || xi > hx || yi < 0 || yi > hy || zi < 0 || zi > hz) continue;
                    S cc[3] = {A == 0 ? S(xi) : S(S(xi) + S(0.5)), A == 1 ? S(yi) : S(S(yi) + S(0.5)),
                               A == 2 ? S(zi) : S(S(zi) + S(0.5))};
                    S e0 = S(g[0] - cc[0]), e1 = S(g[1] - cc[1]), e2 = S(g[2] - cc[2]);
                    // |e| >= 1.5 on any axis gives weight 0: that node adds +-0
                    if (std::abs(e0) >= S(1.5f) || std::abs(e1) >= S(1.5f) || std::abs(e2) >= S(1.5f)) continue;
                    S w0 = qweight(e0), w1 = qweight(e1), w2 = qweight(e2);
                    S weight = w0 * w1 * w2;
                    S d0 = q[0] - (cc[0] * dx[0] + minc[0]);
                    S d1 = q[1] - (cc[1] * dx[1] + minc[1]);
                    S d2 = q[2] - (cc[2] * dx[2] + minc[2]);
                    S dt_ = dot3(C[3 * A + 0], C[3 * A + 1], C[3 * A + 2], d0, d1, d2);
                    wf(xi, yi, zi) += weight;
                    vf(xi, yi, zi) += weight * (v[A] + dt_);
                }
    }

    void particle_to_grid() {
        if (np == 0) return;
        int del[3];
        for (int i = 0; i < 3; ++i) del[i] = int(std::ceil(radius / dx[i]));
        // x slabs of each component's faces; every thread walks all particles in order
#pragma omp parallel num_threads(nthreads())
        {
            const int t = omp_get_thread_num(), nt = omp_get_num_threads();
            int lo[3], hi[3];
            slab(nx + 1, t, nt, lo[0], hi[0]);
            slab(nx, t, nt, lo[1], hi[1]);
            slab(nx, t, nt, lo[2], hi[2]);
            const int lmin = std::min(lo[0], lo[1]), hmax = std::max(hi[0], hi[1]);
            for (int64_t pi = 0; pi < np; ++pi) {
                const S* q = &pos[3 * pi];
                const S* v = &vel[3 * pi];
                const S* C = &aff[9 * pi];
                S g[3];
                int ci[3];
                for (int i = 0; i < 3; ++i) {
                    g[i] = (q[i] - minc[i]) / dx[i];  // cwiseQuotient
                    ci[i] = int(g[i]);                // cast<Integer>
                }
                if (ci[0] + del[0] < lmin || ci[0] - del[0] >= hmax) continue;  // no node in this slab
                p2g_component<0>(q, v, C, g, ci, del, lo[0], hi[0]);
                p2g_component<1>(q, v, C, g, ci, del, lo[1], hi[1]);
                p2g_component<2>(q, v, C, g, ci, del, lo[2], hi[2]);
            }
        }
        normalize(vx, wx);
        normalize(vy, wy);
        normalize(vz, wz);
    }
    void normalize(Field<S>& v, const Field<S>& w) {
        const long long n = (long long)v.d.size();
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (long long i = 0; i < n; ++i) v.d[i] = !is_small(w.d[i]) ? v.d[i] / w.d[i] : S(0.0);
    }

    // LiquidModel<3>::ApplyGravity (LiquidModel.cpp:899-910)
    void apply_gravity(S dt) {
        S gdt = gravity * dt;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (int xi = 1; xi < nx - 1; ++xi)
            for (int yi = 1; yi < ny; ++yi)
                for (int zi = 1; zi < nz - 1; ++zi) vy(xi, yi, zi) += gdt;
    }

    // ------------------------------------------------------------------ G2P
    // LiquidModel<3>::Grid2Particle (LiquidModel.cpp:724-823)
    template <int A>
    void g2p_component(const S g[3], const int ci[3], const int del[3], S& velA, S col[3]) {
        const Field<S>& vf = (A == 0) ? vx : (A == 1) ? vy : vz;
        int hx = nx - 1 + (A == 0), hy = ny - 1 + (A == 1), hz = nz - 1 + (A == 2);
        for (int ddx = -del[0]; ddx <= del[0]; ++ddx)
            for (int ddy = -del[1]; ddy <= del[1]; ++ddy)
                for (int ddz = -del[2]; ddz <= del[2]; ++ddz) {
                    int xi = ci[0] + ddx, yi = ci[1] + ddy, zi = ci[2] + ddz;
                    if (xi < 0 || xi > hx || yi < 0 || yi > hy || zi < 0 || zi > hz) continue;
                    S cc[3] = {A == 0 ? S(xi) : S(S(xi) + S(0.5)), A == 1 ? S(yi) : S(S(yi) + S(0.5)),
                               A == 2 ? S(zi) : S(S(zi) + S(0.5))};
                    S e0 = S(g[0] - cc[0]), e1 = S(g[1] - cc[1]), e2 = S(g[2] - cc[2]);
                    // |e| >= 1.5 on any axis zeroes weight and gradient of this node
                    if (std::abs(e0) >= S(1.5f) || std::abs(e1) >= S(1.5f) || std::abs(e2) >= S(1.5f)) continue;
                    S wX = qweight(e0), wY = qweight(e1), wZ = qweight(e2);
                    S gX = gqweight(e0), gY = gqweight(e1), gZ = gqweight(e2);
                    S weight = wX * wY * wZ;
                    S gw0 = gX * wY * wZ, gw1 = wX * gY * wZ, gw2 = wX * wY * gZ;
                    S val = vf(xi, yi, zi);
                    velA += val * weight;
                    col[0] += val * gw0;
                    col[1] += val * gw1;
                    col[2] += val * gw2;
                }
    }

    void grid_to_particle() {
        if (np == 0) return;
        int del[3];
        for (int i = 0; i < 3; ++i) del[i] = int(std::ceil(radius / dx[i]));
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (int64_t pi = 0; pi < np; ++pi) {
            const S* q = &pos[3 * pi];
            S g[3];
            int ci[3];
            for (int i = 0; i < 3; ++i) {
                g[i] = (q[i] - minc[i]) / dx[i];
                ci[i] = int(g[i]);
            }
            S v[3] = {S(0.0), S(0.0), S(0.0)};
            S C[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            g2p_component<0>(g, ci, del, v[0], &C[0]);
            g2p_component<1>(g, ci, del, v[1], &C[3]);
            g2p_component<2>(g, ci, del, v[2], &C[6]);
            for (int i = 0; i < 3; ++i) vel[3 * pi + i] = v[i];
            for (int i = 0; i < 9; ++i) aff[9 * pi + i] = C[i];
        }
    }

    // LiquidModel<3>::AdvectParticle (LiquidModel.cpp:913-935); the mirrored
    // velocity is never stored by the reference, so only positions change.
    void advect(S dt) {
        if (np == 0) return;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (int64_t pi = 0; pi < np; ++pi) {
            S* q = &pos[3 * pi];
            const S* v = &vel[3 * pi];
            for (int i = 0; i < 3; ++i) q[i] += v[i] * dt;
            S sphi = solid_phi_at(q[0], q[1], q[2]);
            if (sphi < S(0.0)) {
                S g[3];
                solid_gradient(q[0], q[1], q[2], g);
                S s = sphi + eps_of<S>();
                for (int i = 0; i < 3; ++i) q[i] -= s * g[i];
            }
        }
    }

    // ------------------------------------------------------- CorrectVolume
    // Uniform number in [0, 1): SplitMix64 (Steele, Lea and Flood, 2014) of
    // the call count, both particles' indices, the visit and the axis; top
    // 24 bits.  Stands in for the reference's unseeded std::mt19937.
    static float cv_uniform(unsigned long long call, long long i, long long j, int visit, int axis) {
        unsigned long long z = call * 0x9E3779B97F4A7C15ull + (unsigned long long)i * 0xBF58476D1CE4E5B9ull +
                               (unsigned long long)j * 0x94D049BB133111EBull + (unsigned long long)(visit * 3 + axis);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return float(z >> 40) * (1.0f / 16777216.0f);
    }
    // HashNeighborSearch::GetImpactRegion (NeighborSearch.h:87-95)
    void cv_region(const S* q, int lo[3], int hi[3]) const {
        int c[3];
        point2index(q, c);
        const int n[3] = {nx, ny, nz};
        for (int i = 0; i < 3; ++i) {
            lo[i] = std::min(std::max(c[i] - 1, 0), n[i] - 1);
            hi[i] = std::min(std::max(c[i] + 1, 0), n[i] - 1);
        }
    }
    // LiquidModel<3>::CorrectVolume (LiquidModel.cpp:1086-1132) with the
    // neighbour lists of the current positions: a neighbour within one
    // radius counts once per cell its impact region shares with the
    // particle's (HashNeighborSearch lists a particle once per cell of its
    // region, NeighborSearch.h:62-83, and the query walks the cells of the
    // particle's region, :22-50).  Neighbours are visited cell by cell (x, y,
    // z over the region grown by one cell), in caller order within a cell.
    void correct_volume(S dt) {
        if (np == 0) return;
        const S weightFactor = std::sqrt(dx[0] * dx[1] * dx[2]);
        // cell lists, stable in caller order
        const int64_t ncell = int64_t(nx) * ny * nz;
        std::vector<int32_t> start(ncell + 1, 0), ids(np);
        std::vector<int64_t> key(np);
        for (int64_t i = 0; i < np; ++i) {
            int c[3];
            point2index(&pos[3 * i], c);
            c[0] = std::min(std::max(c[0], 0), nx - 1);
            c[1] = std::min(std::max(c[1], 0), ny - 1);
            c[2] = std::min(std::max(c[2], 0), nz - 1);
            key[i] = (int64_t(c[0]) * ny + c[1]) * nz + c[2];
            start[key[i] + 1]++;
        }
        for (int64_t c = 0; c < ncell; ++c) start[c + 1] += start[c];
        {
            std::vector<int32_t> fill(start.begin(), start.end() - 1);
            for (int64_t i = 0; i < np; ++i) ids[fill[key[i]]++] = int32_t(i);
        }
        std::vector<S> buffer(3 * np);
#pragma omp parallel for num_threads(nthreads()) schedule(dynamic, 256)
        for (int64_t pi = 0; pi < np; ++pi) {
            if (pi % correct_cycle != correct_step) continue;
            const S* p = &pos[3 * pi];
            const S r = radius, r2 = r * r;
            int lo[3], hi[3];
            cv_region(p, lo, hi);
            S repel[3] = {S(0), S(0), S(0)};
            for (int cx = std::max(lo[0] - 1, 0); cx <= std::min(hi[0] + 1, nx - 1); ++cx)
                for (int cy = std::max(lo[1] - 1, 0); cy <= std::min(hi[1] + 1, ny - 1); ++cy)
                    for (int cz = std::max(lo[2] - 1, 0); cz <= std::min(hi[2] + 1, nz - 1); ++cz) {
                        const int64_t c = (int64_t(cx) * ny + cy) * nz + cz;
                        for (int32_t s = start[c]; s < start[c + 1]; ++s) {
                            const int64_t npi = ids[s];
                            if (npi == pi) continue;
                            const S* q = &pos[3 * npi];
                            const S dir[3] = {S(p[0] - q[0]), S(p[1] - q[1]), S(p[2] - q[2])};
                            const S d2 = sqnorm3(dir[0], dir[1], dir[2]);
                            if (d2 >= r2) continue;
                            int lj[3], hj[3];
                            cv_region(q, lj, hj);
                            int mult = 1;
                            for (int i = 0; i < 3; ++i)
                                mult *= std::max(0, std::min(hi[i], hj[i]) - std::max(lo[i], lj[i]) + 1);
                            if (mult == 0) continue;
                            const S dist = std::sqrt(d2);
                            const S weight = weightFactor * qweight(S(dist / r));
                            if (double(dist) > 1e-4 * double(r)) {
                                const S wr = weight * r;
                                const S t[3] = {S(wr * S(dir[0] / dist)), S(wr * S(dir[1] / dist)),
                                                S(wr * S(dir[2] / dist))};
                                for (int v = 0; v < mult; ++v)
                                    for (int i = 0; i < 3; ++i) repel[i] += t[i];
                            } else {
                                const S rdt = r / dt;
                                for (int v = 0; v < mult; ++v)
                                    for (int i = 0; i < 3; ++i)
                                        repel[i] += rdt * S(cv_uniform(correct_calls, pi, npi, v, i));
                            }
                        }
                    }
            S np3[3];
            for (int i = 0; i < 3; ++i) np3[i] = p[i] + repel[i] * dt;
            const S sphi = solid_phi_at(np3[0], np3[1], np3[2]);
            if (sphi < S(0.0)) {
                S g[3];
                solid_gradient(np3[0], np3[1], np3[2], g);
                for (int i = 0; i < 3; ++i) np3[i] -= sphi * g[i];
            }
            for (int i = 0; i < 3; ++i) buffer[3 * pi + i] = np3[i];
        }
        for (int64_t pi = 0; pi < np; ++pi) {
            if (pi % correct_cycle != correct_step) continue;
            for (int i = 0; i < 3; ++i) pos[3 * pi + i] = buffer[3 * pi + i];
        }
        correct_step = (correct_step + 1) % correct_cycle;
        ++correct_calls;
    }

    // --------------------------------------------------------- extrapolation
    // LiquidModel<3>::Extrapolate (LiquidModel.cpp:938-1063) for one face
    // component.  Ranges are the reference's; vx/tempVx are swapped after
    // every sweep exactly like std::swap there.
    template <int A> void extrapolate_component(int mode) {
        Field<S>* v = (A == 0) ? &vx : (A == 1) ? &vy : &vz;
        Field<S>* t = (A == 0) ? &tvx : (A == 1) ? &tvy : &tvz;
        const Field<S>& lw = (A == 0) ? lwx : (A == 1) ? lwy : lwz;
        int x0 = 1, x1 = (A == 0) ? nx : nx - 1;  // exclusive upper bounds
        int y0 = 1, y1 = (A == 1) ? ny : ny - 1;
        int z0 = 1, z1 = (A == 2) ? nz : nz - 1;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (int xi = x0; xi < x1; ++xi)
            for (int yi = y0; yi < y1; ++yi)
                for (int zi = z0; zi < z1; ++zi) isValid(xi, yi, zi) = (lw(xi, yi, zi) > S(0.0)) ? 1 : 0;
        Field<uint8_t> prev;
        // Jacobi flags: every face reads the previous sweep's flags only, so
        // x planes are independent; serial flags keep the x-y-z order.
        const int nt = (mode == LHO_EXTRAP_JACOBI) ? nthreads() : 1;
        for (int iter = 0; iter < extrap_iters; ++iter) {
            if (mode == LHO_EXTRAP_JACOBI) prev = isValid;
            const Field<uint8_t>& rv = (mode == LHO_EXTRAP_JACOBI) ? prev : isValid;
#pragma omp parallel for num_threads(nt) schedule(static)
            for (int xi = x0; xi < x1; ++xi)
                for (int yi = y0; yi < y1; ++yi)
                    for (int zi = z0; zi < z1; ++zi) {
                        (*t)(xi, yi, zi) = (*v)(xi, yi, zi);
                        if (rv(xi, yi, zi)) continue;
                        S sum = S(0.0);
                        int count = 0;
                        for (int a = -1; a <= 1; ++a)
                            for (int b = -1; b <= 1; ++b)
                                for (int c = -1; c <= 1; ++c)
                                    if (rv(xi + a, yi + b, zi + c)) {
                                        sum += (*v)(xi + a, yi + b, zi + c);
                                        ++count;
                                    }
                        if (count > 0) {
                            (*t)(xi, yi, zi) = sum / S(count);
                            isValid(xi, yi, zi) = 1;
                        }
                    }
            std::swap(v->d, t->d);
        }
    }
    void extrapolate(int mode) {
        if (np == 0) return;
        extrapolate_component<0>(mode);
        extrapolate_component<1>(mode);
        extrapolate_component<2>(mode);
    }

    // LiquidModel<3>::ComputeDivergence (LiquidModel.cpp:1066-1083)
    void divergence(double* mean, double* max_abs) {
        S divergence = S(0.0);
        int count = 0;
        double mx = 0.0;
        for (int xi = 0; xi < nx; ++xi)
            for (int yi = 0; yi < ny; ++yi)
                for (int zi = 0; zi < nz; ++zi) {
                    if (liquidPhi(xi, yi, zi) > S(0.0)) continue;
                    ++count;
                    S div = lwx(xi + 1, yi, zi) * vx(xi + 1, yi, zi) - lwx(xi, yi, zi) * vx(xi, yi, zi);
                    div += lwy(xi, yi + 1, zi) * vy(xi, yi + 1, zi) - lwy(xi, yi, zi) * vy(xi, yi, zi);
                    div += lwz(xi, yi, zi + 1) * vz(xi, yi, zi + 1) - lwz(xi, yi, zi) * vz(xi, yi, zi);
                    div /= dx[0];
                    divergence += div;
                    // max-norm only over cells whose six faces the projection updates
                    if (xi >= 1 && xi <= nx - 3 && yi >= 1 && yi <= ny - 3 && zi >= 1 && zi <= nz - 3)
                        mx = std::max(mx, std::abs(double(div)));
                }
        if (mean) *mean = double(divergence / S(count));
        if (max_abs) *max_abs = mx;
    }

    // LiquidModel::GetCFL (LiquidModel.h:49-55)
    double cfl() {
        S maxVel = S(0.0);
        for (int64_t pi = 0; pi < np; ++pi) {
            const S* v = &vel[3 * pi];
            S m = eig_maxi(std::abs(v[0]), eig_maxi(std::abs(v[1]), std::abs(v[2])));
            maxVel = mac_max(maxVel, m);
        }
        return double(clampS(S(dx[0] / maxVel), S(0.001), S(0.1)));
    }

    // ---------------------------------------------------------------- solver
    void solver_init() {  // PressureSolver.cpp:666-680
        oldRZ = newRZ = alpha = beta = S(0.0);
        p.fill(S(0.0));
        x.fill(S(0.0));
        rhs.fill(S(0.0));
        for (int l = 0; l < maxLevel; ++l) {
            r[l].fill(S(0.0));
            z[l].fill(S(0.0));
            Adiag[l].fill(S(0.0));
            std::fill(Acoef[l].begin(), Acoef[l].end(), S(0));
        }
    }

    void build_rhs() {  // PressureSolver.cpp:682-698
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (int xi = 0; xi < nx; ++xi)
            for (int yi = 0; yi < ny; ++yi)
                for (int zi = 0; zi < nz; ++zi) {
                    S& b = rhs(xi, yi, zi);
                    b = S(0.0);
                    if (liquidPhi(xi, yi, zi) > S(0.0)) continue;
                    b -= lwx(xi + 1, yi, zi) * vx(xi + 1, yi, zi) / dx[0];
                    b += lwx(xi, yi, zi) * vx(xi, yi, zi) / dx[0];
                    b -= lwy(xi, yi + 1, zi) * vy(xi, yi + 1, zi) / dx[1];
                    b += lwy(xi, yi, zi) * vy(xi, yi, zi) / dx[1];
                    b -= lwz(xi, yi, zi + 1) * vz(xi, yi, zi + 1) / dx[2];
                    b += lwz(xi, yi, zi) * vz(xi, yi, zi) / dx[2];
                }
    }

    // GetApproxLiquidPhi / Wx / Wy / Wz (PressureSolver.cpp:476-542)
    S approx_phi(int xi, int yi, int zi, int level) const {
        if (level == 0) return liquidPhi(xi, yi, zi);
        int f = 1 << level, h = (1 << (level - 1)) - 1;
        int bx = f * xi + h, by = f * yi + h, bz = f * zi + h;
        const Field<S>& L = liquidPhi;
        return trilerp(L(bx, by, bz), L(bx + 1, by, bz), L(bx, by + 1, bz), L(bx + 1, by + 1, bz),
                       L(bx, by, bz + 1), L(bx + 1, by, bz + 1), L(bx, by + 1, bz + 1),
                       L(bx + 1, by + 1, bz + 1), S(0.5), S(0.5), S(0.5));
    }
    S approx_wx(int xi, int yi, int zi, int level) const {
        if (level == 0) return lwx(xi, yi, zi);
        int f = 1 << level, h = (1 << (level - 1)) - 1;
        int bx = f * xi, by = f * yi + h, bz = f * zi + h;
        return bilerp(lwx(bx, by, bz), lwx(bx, by + 1, bz), lwx(bx, by, bz + 1), lwx(bx, by + 1, bz + 1),
                      S(0.5), S(0.5));
    }
    S approx_wy(int xi, int yi, int zi, int level) const {
        if (level == 0) return lwy(xi, yi, zi);
        int f = 1 << level, h = (1 << (level - 1)) - 1;
        int bx = f * xi + h, by = f * yi, bz = f * zi + h;
        return bilerp(lwy(bx, by, bz), lwy(bx + 1, by, bz), lwy(bx, by, bz + 1), lwy(bx + 1, by, bz + 1),
                      S(0.5), S(0.5));
    }
    S approx_wz(int xi, int yi, int zi, int level) const {
        if (level == 0) return lwz(xi, yi, zi);
        int f = 1 << level, h = (1 << (level - 1)) - 1;
        int bx = f * xi + h, by = f * yi + h, bz = f * zi;
        return bilerp(lwz(bx, by, bz), lwz(bx + 1, by, bz), lwz(bx, by + 1, bz), lwz(bx + 1, by + 1, bz),
                      S(0.5), S(0.5));
    }

    // CGSolver<3>::BuildLHS (PressureSolver.cpp:544-664)
    void build_lhs(S rho, S dt) {
        for (int level = 0; level < maxLevel; ++level) {
            int factor = 1 << level;
            Dims d = ldims[level];
            S ldx[3] = {S(factor) * dx[0], S(factor) * dx[1], S(factor) * dx[2]};
            Field<S>& D = Adiag[level];
            std::vector<S>& Cf = Acoef[level];
#pragma omp parallel for num_threads(nthreads()) schedule(static)
            for (int xi = 0; xi < d.nx; ++xi)
                for (int yi = 0; yi < d.ny; ++yi)
                    for (int zi = 0; zi < d.nz; ++zi) {
                        S centerPhi = approx_phi(xi, yi, zi, level);
                        if (centerPhi > S(0.0)) continue;
                        size_t ci = (size_t(xi) * d.ny + yi) * d.nz + zi;
                        S* coef = &Cf[6 * ci];
                        S& diag = D(xi, yi, zi);
                        auto face = [&](bool exists, S w, S h, int nbx, int nby, int nbz, int slot) {
                            if (!exists) return;
                            if (w > S(0.0)) {
                                S term = w * dt / (rho * h * h);
                                S phi = approx_phi(nbx, nby, nbz, level);
                                if (phi < S(0.0)) {
                                    coef[slot] -= term;
                                    diag += term;
                                } else {
                                    S frac = frac_floor(fraction_in_region(centerPhi, phi));
                                    diag += term / frac;
                                }
                            }
                        };
                        face(xi + 1 < d.nx, xi + 1 < d.nx ? approx_wx(xi + 1, yi, zi, level) : S(0), ldx[0],
                             xi + 1, yi, zi, 0);
                        face(xi - 1 >= 0, xi - 1 >= 0 ? approx_wx(xi, yi, zi, level) : S(0), ldx[0], xi - 1, yi,
                             zi, 1);
                        face(yi + 1 < d.ny, yi + 1 < d.ny ? approx_wy(xi, yi + 1, zi, level) : S(0), ldx[1], xi,
                             yi + 1, zi, 2);
                        face(yi - 1 >= 0, yi - 1 >= 0 ? approx_wy(xi, yi, zi, level) : S(0), ldx[1], xi, yi - 1,
                             zi, 3);
                        face(zi + 1 < d.nz, zi + 1 < d.nz ? approx_wz(xi, yi, zi + 1, level) : S(0), ldx[2], xi,
                             yi, zi + 1, 4);
                        face(zi - 1 >= 0, zi - 1 >= 0 ? approx_wz(xi, yi, zi, level) : S(0), ldx[2], xi, yi,
                             zi - 1, 5);
                    }
        }
    }

    // CGSolver<3>::GetAx (PressureSolver.cpp:700-717)
    S get_ax(const Field<S>& g, int xi, int yi, int zi, int level) const {
        const Dims& d = ldims[level];
        const S* coef = &Acoef[level][6 * ((size_t(xi) * d.ny + yi) * d.nz + zi)];
        S result = g(xi, yi, zi) * Adiag[level](xi, yi, zi);
        if (xi + 1 < d.nx) result += g(xi + 1, yi, zi) * coef[0];
        if (xi - 1 >= 0) result += g(xi - 1, yi, zi) * coef[1];
        if (yi + 1 < d.ny) result += g(xi, yi + 1, zi) * coef[2];
        if (yi - 1 >= 0) result += g(xi, yi - 1, zi) * coef[3];
        if (zi + 1 < d.nz) result += g(xi, yi, zi + 1) * coef[4];
        if (zi - 1 >= 0) result += g(xi, yi, zi - 1) * coef[5];
        return result;
    }

    // CGSolver<3>::Smooth (PressureSolver.cpp:821-837): (1. - w) is double.
    void smooth(int level, int phase) {
        const Dims& d = ldims[level];
        Field<S>& zl = z[level];
        // one colour: its cells are not each other's neighbours
#pragma omp parallel for num_threads(d.nx >= 16 ? nthreads() : 1) schedule(static)
        for (int xi = 0; xi < d.nx; ++xi)
            for (int yi = 0; yi < d.ny; ++yi)
                for (int zi = 0; zi < d.nz; ++zi) {
                    if (((xi + yi + zi) & 1) != phase) continue;
                    S dg = Adiag[level](xi, yi, zi);
                    if (is_small(dg)) continue;
                    S term = (r[level](xi, yi, zi) - get_ax(zl, xi, yi, zi, level)) / dg;
                    if (sp.smoother == LHI_SMOOTHER_DAMPED_GS)
                        zl(xi, yi, zi) = zl(xi, yi, zi) + smoothFactor * term;
                    else
                        zl(xi, yi, zi) =
                            S((1. - double(smoothFactor)) * double(zl(xi, yi, zi)) + double(S(smoothFactor * term)));
                }
    }

    // CGSolver<3>::Restrict (PressureSolver.cpp:796-819): 0.125 is double.
    void restrict_(int toLevel) {
        int from = toLevel - 1;
        const Dims& d = ldims[toLevel];
#pragma omp parallel for num_threads(d.nx >= 8 ? nthreads() : 1) schedule(static)
        for (int xi = 0; xi < d.nx; ++xi)
            for (int yi = 0; yi < d.ny; ++yi)
                for (int zi = 0; zi < d.nz; ++zi) {
                    S& rc = r[toLevel](xi, yi, zi);
                    rc = S(0.0);
                    z[toLevel](xi, yi, zi) = S(0.0);
                    int bx = xi << 1, by = yi << 1, bz = zi << 1;
                    const int off[8][3] = {{0, 0, 0}, {0, 0, 1}, {0, 1, 0}, {0, 1, 1},
                                           {1, 0, 0}, {1, 0, 1}, {1, 1, 0}, {1, 1, 1}};
                    for (int k = 0; k < 8; ++k) {
                        int fx = bx + off[k][0], fy = by + off[k][1], fz = bz + off[k][2];
                        S res = r[from](fx, fy, fz) - get_ax(z[from], fx, fy, fz, from);
                        rc = S(double(rc) + 0.125 * double(res));
                    }
                }
    }

    // CGSolver<3>::Prolong (PressureSolver.cpp:774-794)
    void prolong(int toLevel) {
        int from = toLevel + 1;
        const Dims& d = ldims[from];
#pragma omp parallel for num_threads(d.nx >= 8 ? nthreads() : 1) schedule(static)
        for (int xi = 0; xi < d.nx; ++xi)
            for (int yi = 0; yi < d.ny; ++yi)
                for (int zi = 0; zi < d.nz; ++zi) {
                    S v = z[from](xi, yi, zi);
                    int bx = xi << 1, by = yi << 1, bz = zi << 1;
                    for (int a = 0; a < 2; ++a)
                        for (int b = 0; b < 2; ++b)
                            for (int c = 0; c < 2; ++c) z[toLevel](bx + a, by + b, bz + c) += v;
                }
    }

    // CGSolver<3>::ApplyPreconditioner (PressureSolver.cpp:719-772)
    void apply_preconditioner() {
        switch (sp.preconditioner) {
            case LHI_PRECOND_NONE:
                for (size_t i = 0; i < z[0].d.size(); ++i)
                    if (!(liquidPhi.d[i] > S(0.0))) z[0].d[i] = r[0].d[i];
                break;
            case LHI_PRECOND_JACOBI:
                for (size_t i = 0; i < z[0].d.size(); ++i) {
                    S dn = Adiag[0].d[i];
                    if (is_small(dn)) continue;
                    z[0].d[i] = r[0].d[i] / dn;
                }
                break;
            default: {
                for (int level = 1; level < maxLevel; ++level) {
                    for (int it = 0; it < sp.num_pre_smooth; ++it) {
                        smooth(level - 1, 0);
                        smooth(level - 1, 1);
                    }
                    restrict_(level);
                }
                for (int it = 0; it < sp.num_final_smooth; ++it) {
                    smooth(maxLevel - 1, 0);
                    smooth(maxLevel - 1, 1);
                }
                for (int level = maxLevel - 2; level >= 0; --level) {
                    prolong(level);
                    for (int it = 0; it < sp.num_post_smooth; ++it) {
                        smooth(level, 0);
                        smooth(level, 1);
                    }
                }
            }
        }
    }

    static S reduce(const Field<S>& a, const Field<S>& b) {  // Array3::Reduce (Array.h:111-122)
        S sum = S();
        for (size_t i = 0; i < a.d.size(); ++i) sum += a.d[i] * b.d[i];
        return sum;
    }

    // cells where PCG updates x, r and takes p.Ap / ||r||: the fluid cells
    // of [1, N-2]^3 as the reference (PressureSolver.cpp:874-899), or every
    // fluid cell with LHI_REGION_FLUID.
    int lo() const { return sp.update_region == LHI_REGION_FLUID ? 0 : 1; }
    int hx() const { return sp.update_region == LHI_REGION_FLUID ? nx : nx - 1; }
    int hy() const { return sp.update_region == LHI_REGION_FLUID ? ny : ny - 1; }
    int hz() const { return sp.update_region == LHI_REGION_FLUID ? nz : nz - 1; }
    bool interior_fluid(int xi, int yi, int zi) const { return !(liquidPhi(xi, yi, zi) > S(0.0)); }

    // ||b - A x|| over interior fluid cells; optionally stores it into r[0].
    S true_residual(bool store) {
        Field<S>& out = store ? r[0] : tmp;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (int xi = lo(); xi < hx(); ++xi)
            for (int yi = lo(); yi < hy(); ++yi)
                for (int zi = lo(); zi < hz(); ++zi) {
                    if (!interior_fluid(xi, yi, zi)) continue;
                    out(xi, yi, zi) = rhs(xi, yi, zi) - get_ax(x, xi, yi, zi, 0);
                }
        S acc = S(0.0);
        for (int xi = lo(); xi < hx(); ++xi)
            for (int yi = lo(); yi < hy(); ++yi)
                for (int zi = lo(); zi < hz(); ++zi) {
                    if (!interior_fluid(xi, yi, zi)) continue;
                    S rr = out(xi, yi, zi);
                    acc += rr * rr;
                }
        return std::sqrt(acc);
    }

    // CGSolver<3>::Solve (PressureSolver.cpp:839-934) plus the new options:
    // relative tolerance, Polak-Ribiere beta, periodic true residual.
    void solve(S rho, S dt) {
        solver_init();
        build_rhs();
        build_lhs(rho, dt);
        const long long ncells = (long long)rhs.d.size();
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (long long i = 0; i < ncells; ++i)
            if (!(liquidPhi.d[i] > S(0.0))) r[0].d[i] = rhs.d[i];
        apply_preconditioner();
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (long long i = 0; i < ncells; ++i)
            if (!(liquidPhi.d[i] > S(0.0))) p.d[i] = z[0].d[i];
        oldRZ = reduce(r[0], z[0]);
        S residual = std::sqrt(reduce(r[0], r[0]));
        S residual0 = residual;
        S threshold = (sp.tolerance_mode == LHI_TOL_RELATIVE) ? S(tolerance * residual0) : tolerance;
        int iters = 0;
        Field<S> Ap;  // A p of the iteration (p does not change between its two uses)
        Ap.resize(nx, ny, nz);
        for (int iter = 0; iter < sp.max_iterations; ++iter) {
            if (residual < threshold) break;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
            for (int xi = lo(); xi < hx(); ++xi)
                for (int yi = lo(); yi < hy(); ++yi)
                    for (int zi = lo(); zi < hz(); ++zi) {
                        if (liquidPhi(xi, yi, zi) > S(0.0)) continue;
                        Ap(xi, yi, zi) = get_ax(p, xi, yi, zi, 0);
                    }
            S denom = S(0.0);
            for (int xi = lo(); xi < hx(); ++xi)
                for (int yi = lo(); yi < hy(); ++yi)
                    for (int zi = lo(); zi < hz(); ++zi) {
                        if (liquidPhi(xi, yi, zi) > S(0.0)) continue;
                        denom += p(xi, yi, zi) * Ap(xi, yi, zi);
                    }
            alpha = oldRZ / denom;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
            for (int xi = lo(); xi < hx(); ++xi)
                for (int yi = lo(); yi < hy(); ++yi)
                    for (int zi = lo(); zi < hz(); ++zi) {
                        if (liquidPhi(xi, yi, zi) > S(0.0)) continue;
                        x(xi, yi, zi) += alpha * p(xi, yi, zi);
                        r[0](xi, yi, zi) -= alpha * Ap(xi, yi, zi);
                    }
            residual = S(0.0);
            for (int xi = lo(); xi < hx(); ++xi)
                for (int yi = lo(); yi < hy(); ++yi)
                    for (int zi = lo(); zi < hz(); ++zi) {
                        if (liquidPhi(xi, yi, zi) > S(0.0)) continue;
                        residual += r[0](xi, yi, zi) * r[0](xi, yi, zi);
                    }
            residual = std::sqrt(residual);
            ++iters;
            if (sp.true_residual_every > 0 && iters % sp.true_residual_every == 0) residual = true_residual(true);
            apply_preconditioner();
            newRZ = reduce(r[0], z[0]);
            if (sp.cg_variant == LHI_CG_FLEXIBLE) {
                // beta = r_new . (z_new - z_old) / rz_old = -alpha (Ap . z_new) / rz_old
                S apz = S(0.0);
                for (int xi = lo(); xi < hx(); ++xi)
                    for (int yi = lo(); yi < hy(); ++yi)
                        for (int zi = lo(); zi < hz(); ++zi) {
                            if (liquidPhi(xi, yi, zi) > S(0.0)) continue;
                            apz += Ap(xi, yi, zi) * z[0](xi, yi, zi);
                        }
                beta = -alpha * apz / oldRZ;
            } else {
                beta = newRZ / oldRZ;
            }
#pragma omp parallel for num_threads(nthreads()) schedule(static)
            for (long long i = 0; i < ncells; ++i)
                if (!(liquidPhi.d[i] > S(0.0))) p.d[i] = z[0].d[i] + beta * p.d[i];
            oldRZ = newRZ;
        }
        pressure.d = x.d;  // m_grid.pressure.CopyFrom(m_x)
        last.iterations = iters;
        last.initial_residual = double(residual0);
        last.final_residual = double(residual);
        last.true_residual = double(true_residual(false));
        bool ok = residual < threshold;
        last.status = std::isfinite(double(residual)) ? (ok ? LHI_OK : LHI_E_NOT_CONVERGED) : LHI_E_NAN;
        last.solve_ms = 0.0;
    }

    // LiquidModel<3>::SolvePressure velocity update (LiquidModel.cpp:834-889)
    void velocity_update(S dt) {
        S rho = density;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
        for (int xi = 1; xi < nx - 1; ++xi)
            for (int yi = 1; yi < ny - 1; ++yi)
                for (int zi = 1; zi < nz - 1; ++zi) {
                    S centerPhi = liquidPhi(xi, yi, zi);
                    auto upd = [&](const Field<S>& lw, Field<S>& v, S phi, S pn, S h) {
                        if (lw(xi, yi, zi) > S(0.0)) {
                            if (centerPhi < S(0.0) || phi < S(0.0)) {
                                S frac = S(1.0);
                                if (centerPhi >= S(0.0) || phi >= S(0.0))
                                    frac = frac_floor(fraction_in_region(centerPhi, phi));
                                S grad = (pressure(xi, yi, zi) - pn) / (h * frac);
                                v(xi, yi, zi) -= grad * dt / rho;
                            }
                        } else {
                            v(xi, yi, zi) = S(0.0);
                        }
                    };
                    upd(lwx, vx, liquidPhi(xi - 1, yi, zi), pressure(xi - 1, yi, zi), dx[0]);
                    upd(lwy, vy, liquidPhi(xi, yi - 1, zi), pressure(xi, yi - 1, zi), dx[1]);
                    upd(lwz, vz, liquidPhi(xi, yi, zi - 1), pressure(xi, yi, zi - 1), dx[2]);
                }
    }

    void projection(S dt) {  // LiquidModel<3>::Projection -> SolvePressure
        if (np == 0) return;
        solve(density, dt);
        velocity_update(dt);
    }

    // ------------------------------------------------------------ fields
    Field<S>* scalar_field(int f, int level) {
        switch (f) {
            case LHI_FIELD_VX: return &vx;
            case LHI_FIELD_VY: return &vy;
            case LHI_FIELD_VZ: return &vz;
            case LHI_FIELD_WX: return &wx;
            case LHI_FIELD_WY: return &wy;
            case LHI_FIELD_WZ: return &wz;
            case LHI_FIELD_LIQUID_WX: return &lwx;
            case LHI_FIELD_LIQUID_WY: return &lwy;
            case LHI_FIELD_LIQUID_WZ: return &lwz;
            case LHI_FIELD_TEMP_VX: return &tvx;
            case LHI_FIELD_TEMP_VY: return &tvy;
            case LHI_FIELD_TEMP_VZ: return &tvz;
            case LHI_FIELD_PRESSURE: return &pressure;
            case LHI_FIELD_LIQUID_PHI: return &liquidPhi;
            case LHI_FIELD_SOLID_PHI: return &solidPhi;
            case LHI_FIELD_RHS: return &rhs;
            case LHI_FIELD_X: return &x;
            case LHI_FIELD_P: return &p;
            case LHI_FIELD_R: return (level >= 0 && level < maxLevel) ? &r[level] : nullptr;
            case LHI_FIELD_Z: return (level >= 0 && level < maxLevel) ? &z[level] : nullptr;
            case LHI_FIELD_ADIAG: return (level >= 0 && level < maxLevel) ? &Adiag[level] : nullptr;
            default: return nullptr;
        }
    }
};

struct AnyModel {
    int dbl;
    std::unique_ptr<Model<float>> f;
    std::unique_ptr<Model<double>> d;
};

template <class S> Model<S>* get(lho_model* m);
template <> Model<float>* get<float>(lho_model* m) { return reinterpret_cast<AnyModel*>(m)->f.get(); }
template <> Model<double>* get<double>(lho_model* m) { return reinterpret_cast<AnyModel*>(m)->d.get(); }

#define DISPATCH(m, EXPR)                                  \
    do {                                                   \
        AnyModel* am_ = reinterpret_cast<AnyModel*>(m);    \
        if (!am_) return LHI_E_INVALID_ARG;                \
        if (am_->dbl) {                                    \
            auto* M = am_->d.get();                        \
            using S = double;                              \
            (void)sizeof(S);                               \
            EXPR;                                          \
        } else {                                           \
            auto* M = am_->f.get();                        \
            using S = float;                               \
            (void)sizeof(S);                               \
            EXPR;                                          \
        }                                                  \
    } while (0)

template <class S> int field_size_t(Model<S>* M, int f, int level, int64_t* count, int32_t* eb) {
    if (f == LHI_FIELD_IS_VALID) {
        *count = int64_t(M->isValid.d.size());
        *eb = 1;
        return 0;
    }
    if (f == LHI_FIELD_ACOEF) {
        if (level < 0 || level >= M->maxLevel) return LHI_E_INVALID_ARG;
        *count = int64_t(M->Acoef[level].size());
        *eb = sizeof(S);
        return 0;
    }
    Field<S>* fp = M->scalar_field(f, level);
    if (!fp) return LHI_E_INVALID_ARG;
    *count = int64_t(fp->d.size());
    *eb = sizeof(S);
    return 0;
}

}  // namespace

namespace {
// ParticleSystem<3>::SpawnParticles (ParticleSystem.cpp:45-64)
template <class S>
int64_t spawn_t(const double mn[3], const double mx[3], double defr, int64_t max_count, S* out) {
    S minc[3] = {S(mn[0]), S(mn[1]), S(mn[2])}, maxc[3] = {S(mx[0]), S(mx[1]), S(mx[2])};
    S defaultRadius = S(defr);
    S interval = S(0.5 * double(defaultRadius));
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

}  // namespace

extern "C" {

// Error text of the scene generator compiled into this library (the CUDA
// library keeps its own copy of the same function).
static thread_local std::string g_scene_error;
extern "C" void lhi_set_error_message(const char* msg) { g_scene_error = msg ? msg : ""; }
const char* lho_last_error(void) { return g_scene_error.c_str(); }

void lho_set_threads(int32_t n) { g_threads = n > 0 ? n : 0; }

// LiquidModel<3>::Render (LiquidModel.cpp:1138-1159) restated without GL:
// Shader/Scene3D_vertex.glsl:9 in float, then the fixed-function point
// rasterisation the reference relies on (clip to [-1, 1]^3, viewport
// x_w = (x + 1) * width / 2, pixels whose centres lie in the square of side
// pointSize around the point, one colour, no depth test).
int lho_render(const float* pos, int64_t n, const float mn[3], const float mx[3], const lhi_render_params* rp,
               float* ndc, uint8_t* rgba) {
    if (!rp || rp->width < 1 || rp->height < 1) return LHI_E_INVALID_ARG;
    const int64_t npix = int64_t(rp->width) * rp->height;
    if (rgba)
        for (int64_t i = 0; i < npix; ++i) std::memcpy(rgba + 4 * i, rp->background, 4);
    auto cover = [](float v, int extent, float size, int& lo, int& hi) {
        const float xw = (v + 1.0f) * (0.5f * float(extent));
        const float h = size * 0.5f;
        lo = int(std::ceil((xw - h) - 0.5f));
        hi = int(std::ceil((xw + h) - 0.5f)) - 1;
        lo = std::max(lo, 0);
        hi = std::min(hi, extent - 1);
    };
    for (int64_t k = 0; k < n; ++k) {
        float p[3];
        for (int i = 0; i < 3; ++i) {
            const float a = pos[3 * k + i] - mn[i];
            const float b = mx[i] - mn[i];
            p[i] = (a / b) * 2.0f - 1.0f;
        }
        if (ndc)
            for (int i = 0; i < 3; ++i) ndc[3 * k + i] = p[i];
        if (!rgba) continue;
        if (!(p[0] >= -1.f && p[0] <= 1.f && p[1] >= -1.f && p[1] <= 1.f && p[2] >= -1.f && p[2] <= 1.f)) continue;
        int x0, x1, y0, y1;
        cover(p[0], rp->width, rp->point_size, x0, x1);
        cover(p[1], rp->height, rp->point_size, y0, y1);
        for (int j = y0; j <= y1; ++j)
            for (int i = x0; i <= x1; ++i) std::memcpy(rgba + 4 * (int64_t(j) * rp->width + i), rp->color, 4);
    }
    return LHI_OK;
}

void lho_set_omp_default_threads(int32_t n) {
    if (n > 0) omp_set_num_threads(n);
}

int32_t lho_get_threads(void) { return nthreads(); }

lho_model* lho_create(const lhi_grid_desc* grid, const lhi_solver_params* solver,
                      const lhi_liquid_params* liquid, int32_t dbl) {
    if (!grid || !solver || !liquid) return nullptr;
    auto* am = new AnyModel();
    am->dbl = dbl ? 1 : 0;
    if (am->dbl) am->d.reset(new Model<double>(*grid, *solver, *liquid));
    else am->f.reset(new Model<float>(*grid, *solver, *liquid));
    return reinterpret_cast<lho_model*>(am);
}

void lho_destroy(lho_model* m) { delete reinterpret_cast<AnyModel*>(m); }

void lho_get_dx(const lho_model* m, double dx[3]) {
    auto* am = reinterpret_cast<const AnyModel*>(m);
    for (int i = 0; i < 3; ++i) dx[i] = am->dbl ? am->d->dx[i] : double(am->f->dx[i]);
}

int lho_set_boundary(lho_model* m, const lhi_boundary_node* nodes, int32_t count, int32_t root) {
    DISPATCH(m, M->set_boundary(nodes, count, root));
    return 0;
}

int lho_set_solid_phi(lho_model* m, const void* node_phi) {
    DISPATCH(m, {
        std::memcpy(M->solidPhi.d.data(), node_phi, M->solidPhi.d.size() * sizeof(S));
        M->compute_face_fractions();
    });
    return 0;
}

int lho_boundary_eval(const lhi_boundary_node* nodes, int32_t count, int32_t root, int32_t dbl,
                      const void* points, int64_t n, void* out) {
    if (dbl) {
        const double* pp = static_cast<const double*>(points);
        double* o = static_cast<double*>(out);
        for (int64_t i = 0; i < n; ++i) o[i] = boundary_compute<double>(nodes, count, root, pp + 3 * i);
    } else {
        const float* pp = static_cast<const float*>(points);
        float* o = static_cast<float*>(out);
        for (int64_t i = 0; i < n; ++i) o[i] = boundary_compute<float>(nodes, count, root, pp + 3 * i);
    }
    return 0;
}

int lho_set_particles(lho_model* m, int64_t n, const void* pos, const void* vel, const void* affine) {
    DISPATCH(m, {
        M->np = n;
        M->pos.assign(static_cast<const S*>(pos), static_cast<const S*>(pos) + 3 * n);
        if (vel) M->vel.assign(static_cast<const S*>(vel), static_cast<const S*>(vel) + 3 * n);
        else M->vel.assign(3 * n, S(0));
        if (affine) M->aff.assign(static_cast<const S*>(affine), static_cast<const S*>(affine) + 9 * n);
        else M->aff.assign(9 * n, S(0));
    });
    return 0;
}

int lho_get_particles(lho_model* m, void* pos, void* vel, void* affine) {
    DISPATCH(m, {
        if (pos) std::memcpy(pos, M->pos.data(), M->pos.size() * sizeof(S));
        if (vel) std::memcpy(vel, M->vel.data(), M->vel.size() * sizeof(S));
        if (affine) std::memcpy(affine, M->aff.data(), M->aff.size() * sizeof(S));
    });
    return 0;
}

int64_t lho_num_particles(const lho_model* m) {
    auto* am = reinterpret_cast<const AnyModel*>(m);
    return am->dbl ? am->d->np : am->f->np;
}

int lho_field_size(const lho_model* m, int32_t field, int32_t level, int64_t* count, int32_t* elem_bytes) {
    auto* am = reinterpret_cast<AnyModel*>(const_cast<lho_model*>(m));
    if (am->dbl) return field_size_t(am->d.get(), field, level, count, elem_bytes);
    return field_size_t(am->f.get(), field, level, count, elem_bytes);
}

int lho_get_field(lho_model* m, int32_t field, int32_t level, void* out) {
    int rc = 0;
    DISPATCH(m, {
        if (field == LHI_FIELD_IS_VALID) {
            std::memcpy(out, M->isValid.d.data(), M->isValid.d.size());
        } else if (field == LHI_FIELD_ACOEF) {
            if (level < 0 || level >= M->maxLevel) return LHI_E_INVALID_ARG;
            std::memcpy(out, M->Acoef[level].data(), M->Acoef[level].size() * sizeof(S));
        } else {
            auto* fp = M->scalar_field(field, level);
            if (!fp) return LHI_E_INVALID_ARG;
            std::memcpy(out, fp->d.data(), fp->d.size() * sizeof(S));
        }
    });
    return rc;
}

int lho_set_field(lho_model* m, int32_t field, int32_t level, const void* in) {
    DISPATCH(m, {
        if (field == LHI_FIELD_IS_VALID) {
            std::memcpy(M->isValid.d.data(), in, M->isValid.d.size());
        } else if (field == LHI_FIELD_ACOEF) {
            if (level < 0 || level >= M->maxLevel) return LHI_E_INVALID_ARG;
            std::memcpy(M->Acoef[level].data(), in, M->Acoef[level].size() * sizeof(S));
        } else {
            auto* fp = M->scalar_field(field, level);
            if (!fp) return LHI_E_INVALID_ARG;
            std::memcpy(fp->d.data(), in, fp->d.size() * sizeof(S));
        }
    });
    return 0;
}

int lho_clear(lho_model* m) {
    DISPATCH(m, M->clear());
    return 0;
}
int lho_compute_liquid_phi(lho_model* m) {
    DISPATCH(m, M->compute_liquid_phi());
    return 0;
}
int lho_particle_to_grid(lho_model* m) {
    DISPATCH(m, M->particle_to_grid());
    return 0;
}
int lho_apply_gravity(lho_model* m, double dt) {
    DISPATCH(m, M->apply_gravity(S(dt)));
    return 0;
}
int lho_velocity_update(lho_model* m, double dt) {
    DISPATCH(m, M->velocity_update(S(dt)));
    return 0;
}
int lho_projection(lho_model* m, double dt, lhi_solve_stats* stats) {
    DISPATCH(m, {
        M->projection(S(dt));
        if (stats) *stats = M->last;
    });
    return 0;
}
int lho_extrapolate(lho_model* m, int32_t mode) {
    DISPATCH(m, M->extrapolate(mode));
    return 0;
}
int lho_grid_to_particle(lho_model* m) {
    DISPATCH(m, M->grid_to_particle());
    return 0;
}
int lho_advect_particles(lho_model* m, double dt) {
    DISPATCH(m, M->advect(S(dt)));
    return 0;
}
int lho_pre_step(lho_model* m, double dt) {
    (void)dt;
    DISPATCH(m, {
        M->clear();
        M->compute_liquid_phi();
    });
    return 0;
}
int lho_step(lho_model* m, double dt, int32_t extrap_mode, lhi_solve_stats* stats) {
    DISPATCH(m, {
        S sdt = S(dt);
        M->particle_to_grid();
        M->apply_gravity(sdt);
        M->projection(sdt);
        M->extrapolate(extrap_mode);
        M->grid_to_particle();
        M->advect(sdt);
        if (M->correct_in_step) M->correct_volume(sdt);
        if (stats) *stats = M->last;
    });
    return 0;
}
int lho_correct_volume(lho_model* m, double dt) {
    DISPATCH(m, M->correct_volume(S(dt)));
    return 0;
}
int lho_compute_divergence(lho_model* m, double* mean, double* max_abs) {
    DISPATCH(m, M->divergence(mean, max_abs));
    return 0;
}
int lho_get_cfl(lho_model* m, double* dt_out) {
    DISPATCH(m, *dt_out = M->cfl());
    return 0;
}
int lho_solver_init(lho_model* m) {
    DISPATCH(m, M->solver_init());
    return 0;
}
int lho_solver_build_rhs(lho_model* m) {
    DISPATCH(m, M->build_rhs());
    return 0;
}
int lho_solver_build_lhs(lho_model* m, double density, double dt) {
    DISPATCH(m, M->build_lhs(S(density), S(dt)));
    return 0;
}
int lho_solver_apply_preconditioner(lho_model* m) {
    DISPATCH(m, M->apply_preconditioner());
    return 0;
}
int lho_solver_solve(lho_model* m, double density, double dt, lhi_solve_stats* stats) {
    DISPATCH(m, {
        M->solve(S(density), S(dt));
        if (stats) *stats = M->last;
    });
    return 0;
}
int lho_solver_get_ax(lho_model* m, int32_t level, const void* xin, void* out) {
    DISPATCH(m, {
        if (level < 0 || level >= M->maxLevel) return LHI_E_INVALID_ARG;
        const Dims d = M->ldims[level];
        Field<S> g;
        g.resize(d.nx, d.ny, d.nz);
        std::memcpy(g.d.data(), xin, g.d.size() * sizeof(S));
        S* o = static_cast<S*>(out);
        for (int xi = 0; xi < d.nx; ++xi)
            for (int yi = 0; yi < d.ny; ++yi)
                for (int zi = 0; zi < d.nz; ++zi)
                    o[(size_t(xi) * d.ny + yi) * d.nz + zi] = M->get_ax(g, xi, yi, zi, level);
    });
    return 0;
}

int lho_cell_keys(lho_model* m, int32_t* keys) {
    DISPATCH(m, {
        for (int64_t i = 0; i < M->np; ++i) {
            int c[3];
            M->point2index(&M->pos[3 * i], c);
            c[0] = std::min(std::max(c[0], 0), M->nx - 1);
            c[1] = std::min(std::max(c[1], 0), M->ny - 1);
            c[2] = std::min(std::max(c[2], 0), M->nz - 1);
            keys[i] = int32_t((int64_t(c[0]) * M->ny + c[1]) * M->nz + c[2]);
        }
    });
    return 0;
}

int lho_sort_by_cell(lho_model* m, int32_t* sorted_ids, int32_t* cell_start) {
    int64_t n = lho_num_particles(m);
    std::vector<int32_t> keys(n);
    lho_cell_keys(m, keys.data());
    std::vector<int32_t> ids(n);
    for (int64_t i = 0; i < n; ++i) ids[i] = int32_t(i);
    std::stable_sort(ids.begin(), ids.end(), [&](int32_t a, int32_t b) { return keys[a] < keys[b]; });
    std::memcpy(sorted_ids, ids.data(), n * sizeof(int32_t));
    if (cell_start) {
        auto* am = reinterpret_cast<AnyModel*>(m);
        int64_t ncell = am->dbl ? int64_t(am->d->nx) * am->d->ny * am->d->nz
                                : int64_t(am->f->nx) * am->f->ny * am->f->nz;
        std::vector<int32_t> cnt(ncell + 1, 0);
        for (int64_t i = 0; i < n; ++i) cnt[keys[i] + 1]++;
        for (int64_t c = 0; c < ncell; ++c) cnt[c + 1] += cnt[c];
        std::memcpy(cell_start, cnt.data(), (ncell + 1) * sizeof(int32_t));
    }
    return 0;
}

int64_t lho_spawn_lattice(const double min_coord[3], const double max_coord[3], double default_radius,
                          int64_t max_count, int32_t dbl, void* pos) {
    if (dbl) return spawn_t<double>(min_coord, max_coord, default_radius, max_count, static_cast<double*>(pos));
    return spawn_t<float>(min_coord, max_coord, default_radius, max_count, static_cast<float*>(pos));
}

}  // extern "C"
