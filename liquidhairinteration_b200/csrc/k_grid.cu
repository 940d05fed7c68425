// k_grid.cu -- MAC-grid side of the liquid step: allocation, Clear, the solid
// SDF and face fractions, gravity, the ghost-fluid velocity update,
// extrapolation, divergence, field access and the step orchestration.
#include <algorithm>
#include <cstring>

#include "impl.cuh"

namespace lhi {

namespace {

template <class T> struct G3 {
    int nx, ny, nz;
    T mn[3], dx[3];
};

template <class T> __global__ void k_fill(T* __restrict__ p, long long n, T v) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// RectBoundary / OperatorBoundary / SolidBoundary::Compute (Boundary.h:38-90)
// at node (xi, yi, zi): Vector3(xi, yi, zi).cwiseProduct(dx) + minCoord.
template <class T> __global__ void k_boundary(BoundaryProgram prog, G3<T> g, T* __restrict__ sp) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int fy = g.ny + 1, fz = g.nz + 1;
    long long n = (long long)(g.nx + 1) * fy * fz;
    if (i >= n) return;
    int xi, yi, zi;
    idx3(i, fy, fz, xi, yi, zi);
    T p[3] = {X<T>::add(X<T>::mul(T(xi), g.dx[0]), g.mn[0]), X<T>::add(X<T>::mul(T(yi), g.dx[1]), g.mn[1]),
              X<T>::add(X<T>::mul(T(zi), g.dx[2]), g.mn[2])};
    T val[kMaxBoundaryNodes];
    for (int k = 0; k < prog.count; ++k) {
        T r;
        switch (prog.kind[k]) {
            case LHI_BOUNDARY_RECT: {
                T q[3], qm[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    q[a] = X<T>::sub(fabs(X<T>::sub(p[a], T(prog.center[k][a]))), T(prog.half[k][a]));
                    qm[a] = eig_maxi(q[a], T(0));
                }
                T outside = X<T>::sqrt(sqnorm3(qm[0], qm[1], qm[2]));
                T inside = mac_min(eig_maxi(q[0], eig_maxi(q[1], q[2])), T(0));
                r = prog.use_inside[k] ? X<T>::sub(-outside, inside) : X<T>::add(outside, inside);
                break;
            }
            case LHI_BOUNDARY_UNION: r = mac_min(val[prog.left[k]], val[prog.right[k]]); break;
            case LHI_BOUNDARY_INTERSECTION: r = mac_max(val[prog.left[k]], val[prog.right[k]]); break;
            case LHI_BOUNDARY_SUBTRACT: r = mac_max(val[prog.left[k]], -val[prog.right[k]]); break;
            case LHI_BOUNDARY_NONE: r = val[prog.left[k]]; break;
            default: r = T(1); break;  // SolidBoundary::Compute
        }
        val[k] = r;
    }
    sp[i] = val[prog.root];
}

// LiquidModel<3>::ComputeSolidPhi face fractions (LiquidModel.cpp:574-610).
// liquidWx uses the y-edge of the face; liquidWy and liquidWz both use the
// x-edge, exactly as the reference does.
template <class T>
__global__ void k_face_fractions(const T* __restrict__ sp, int nx, int ny, int nz, int comp, T* __restrict__ lw) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int fx = nx + (comp == 0), fy = ny + (comp == 1), fz = nz + (comp == 2);
    long long n = (long long)fx * fy * fz;
    if (i >= n) return;
    int xi, yi, zi;
    idx3(i, fy, fz, xi, yi, zi);
    const long long sy = nz + 1, sx = (long long)(ny + 1) * (nz + 1);
    long long a = xi * sx + yi * sy + zi;
    long long b = (comp == 0) ? a + sy : a + sx;
    lw[i] = open_fraction(sp[a], sp[b]);
}

// LiquidModel<3>::ApplyGravity (LiquidModel.cpp:899-910)
template <class T> __global__ void k_gravity(T* __restrict__ vy, int nx, int ny, int nz, T gdt) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int fy = ny + 1;
    long long n = (long long)nx * fy * nz;
    if (i >= n) return;
    int x, y, z;
    idx3(i, fy, nz, x, y, z);
    if (x >= 1 && x < nx - 1 && y >= 1 && y < ny && z >= 1 && z < nz - 1) vy[i] = X<T>::add(vy[i], gdt);
}

// LiquidModel<3>::SolvePressure velocity update (LiquidModel.cpp:834-889):
// ghost-fluid pressure gradient on the interior cells' low faces.
template <class T>
__global__ void k_velocity_update(int nx, int ny, int nz, T hx, T hy, T hz, T dt, T rho, const T* __restrict__ phi,
                                  const T* __restrict__ pr, const T* __restrict__ lwx, const T* __restrict__ lwy,
                                  const T* __restrict__ lwz, T* __restrict__ vx, T* __restrict__ vy,
                                  T* __restrict__ vz) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int ix = nx - 2, iy = ny - 2, iz = nz - 2;
    if (ix <= 0 || iy <= 0 || iz <= 0) return;
    long long n = (long long)ix * iy * iz;
    if (i >= n) return;
    // 32-bit index arithmetic: the interior has fewer than 2^31 cells
    const unsigned u = unsigned(i), t = u / unsigned(iz);
    const int z = 1 + int(u - t * unsigned(iz)), y = 1 + int(t % unsigned(iy)), x = 1 + int(t / unsigned(iy));
    long long c = ((long long)x * ny + y) * nz + z;
    const long long sx = (long long)ny * nz, sy = nz;
    const long long fx = ((long long)x * ny + y) * nz + z;        // face (x, y, z) of vx
    const long long fy = ((long long)x * (ny + 1) + y) * nz + z;  // of vy
    const long long fz = ((long long)x * ny + y) * (nz + 1) + z;  // of vz
    // the operands of the tests first (all in bounds for an interior cell),
    // so the loads overlap instead of waiting on one another behind branches
    const T center = phi[c], pc = pr[c];
    const T nphi[3] = {phi[c - sx], phi[c - sy], phi[c - 1]};
    const T npr[3] = {pr[c - sx], pr[c - sy], pr[c - 1]};
    const T lw[3] = {lwx[fx], lwy[fy], lwz[fz]};
    T* const vv[3] = {vx + fx, vy + fy, vz + fz};
    const T hh[3] = {hx, hy, hz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (lw[a] > T(0)) {
            if (center < T(0) || nphi[a] < T(0)) {
                T frac = T(1);
                if (center >= T(0) || nphi[a] >= T(0)) frac = frac_floor(fraction_in_region(center, nphi[a]));
                T grad = X<T>::div(X<T>::sub(pc, npr[a]), X<T>::mul(hh[a], frac));
                *vv[a] = X<T>::sub(*vv[a], X<T>::div(X<T>::mul(grad, dt), rho));
            }
        } else {
            *vv[a] = T(0);
        }
    }
}

// ------------------------------------------------------------ extrapolation
// LiquidModel<3>::Extrapolate (LiquidModel.cpp:938-1063).  Validity is kept
// as a level per node of the (N+1)^3 isValid array: 255 = invalid, otherwise
// the sweep before which it became valid.  In sweep k a node counts as valid
// iff its level <= k, so flags are read as of the previous sweep (Jacobi),
// which makes the result independent of thread order.
struct ExtRange {
    int x0, x1, y0, y1, z0, z1;  // inclusive in-range box of the component
    int fy, fz;                  // face-array extents
    int ny1, nz1;                // isValid extents (ny+1, nz+1)
};

// Face (x, y, z) of this thread inside the range (32-bit index arithmetic:
// every face array has fewer than 2^31 entries).
// Faces (x, y, z .. z+3) of this thread inside the range: 4 consecutive
// faces along z per thread (32-bit index arithmetic: every face array has
// fewer than 2^31 entries).
__device__ __forceinline__ bool ext_cell4(const ExtRange& r, int& x, int& y, int& z) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    const int ey = r.y1 - r.y0 + 1, ez4 = (r.z1 - r.z0 + 1 + 3) / 4;
    if (ey <= 0 || ez4 <= 0 || i >= unsigned(r.x1 - r.x0 + 1) * unsigned(ey) * unsigned(ez4)) return false;
    const unsigned t = i / unsigned(ez4);
    z = r.z0 + 4 * int(i - t * unsigned(ez4));
    y = r.y0 + int(t % unsigned(ey));
    x = r.x0 + int(t / unsigned(ey));
    return true;
}
inline long long ext_threads(const ExtRange& r) {
    return (long long)std::max(r.x1 - r.x0 + 1, 0) * std::max(r.y1 - r.y0 + 1, 0) *
           std::max((r.z1 - r.z0 + 1 + 3) / 4, 0);
}

template <class T> __global__ void k_extrap_init(ExtRange r, const T* __restrict__ lw, uint8_t* __restrict__ valid) {
    int x, y, z0;
    if (!ext_cell4(r, x, y, z0)) return;
    for (int z = z0; z < z0 + 4 && z <= r.z1; ++z) {
        long long f = ((long long)x * r.fy + y) * r.fz + z;
        valid[((long long)x * r.ny1 + y) * r.nz1 + z] = (lw[f] > T(0)) ? 0 : 255;
    }
}

// With t == v the sweep runs in place: it writes only faces that were not
// valid before sweep k, and it reads only faces that were, so the values
// equal those of the sweep into a separate buffer (the same holds between
// a thread's own 4 faces).
template <class T>
__global__ void k_extrap_sweep(ExtRange r, int k, const T* v, T* t, uint8_t* __restrict__ valid) {
    int x, y, z0;
    if (!ext_cell4(r, x, y, z0)) return;
    for (int z = z0; z < z0 + 4 && z <= r.z1; ++z) {
        long long f = ((long long)x * r.fy + y) * r.fz + z;
        long long vi = ((long long)x * r.ny1 + y) * r.nz1 + z;
        if (t != v) t[f] = v[f];
        if (valid[vi] <= k) continue;
        T sum = T(0);
        int count = 0;
        for (int a = -1; a <= 1; ++a)
            for (int b = -1; b <= 1; ++b)
                for (int c = -1; c <= 1; ++c) {
                    long long nv = ((long long)(x + a) * r.ny1 + (y + b)) * r.nz1 + (z + c);
                    if (valid[nv] <= k) {
                        sum = X<T>::add(sum, v[((long long)(x + a) * r.fy + (y + b)) * r.fz + (z + c)]);
                        ++count;
                    }
                }
        if (count > 0) {
            t[f] = X<T>::div(sum, T(count));
            valid[vi] = uint8_t(k + 1);
        }
    }
}

__global__ void k_extrap_finish(ExtRange r, uint8_t* __restrict__ valid) {
    int x, y, z0;
    if (!ext_cell4(r, x, y, z0)) return;
    for (int z = z0; z < z0 + 4 && z <= r.z1; ++z) {
        long long vi = ((long long)x * r.ny1 + y) * r.nz1 + z;
        uint8_t v = valid[vi];
        valid[vi] = (v == 255) ? 255 : 0;
    }
}

// The same three stages over a list of isValid nodes of the range (the
// nodes whose flag can be other than 0 there; every other node of the
// range holds 0 before and after, so skipping it changes nothing).
__device__ __forceinline__ void ext_node(const ExtRange& r, int32_t vi, int& x, int& y, int& z) {
    const int yz = r.ny1 * r.nz1;
    x = vi / yz;
    const int rem = vi - x * yz;
    y = rem / r.nz1;
    z = rem - y * r.nz1;
}

template <class T>
__global__ void k_extrap_init_l(ExtRange r, const int32_t* __restrict__ list, long long n, const T* __restrict__ lw,
                                uint8_t* __restrict__ valid) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int x, y, z;
    ext_node(r, list[i], x, y, z);
    valid[list[i]] = (lw[((long long)x * r.fy + y) * r.fz + z] > T(0)) ? 0 : 255;
}

// In place (sweeps before the ones through tempV), as k_extrap_sweep with t == v.
template <class T>
__global__ void k_extrap_sweep_l(ExtRange r, const int32_t* __restrict__ list, long long n, int k, T* v,
                                 uint8_t* __restrict__ valid) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t vi = list[i];
    if (valid[vi] <= k) return;
    int x, y, z;
    ext_node(r, vi, x, y, z);
    T sum = T(0);
    int count = 0;
    for (int a = -1; a <= 1; ++a)
        for (int b = -1; b <= 1; ++b)
            for (int c = -1; c <= 1; ++c) {
                long long nv = ((long long)(x + a) * r.ny1 + (y + b)) * r.nz1 + (z + c);
                if (valid[nv] <= k) {
                    sum = X<T>::add(sum, v[((long long)(x + a) * r.fy + (y + b)) * r.fz + (z + c)]);
                    ++count;
                }
            }
    if (count > 0) {
        v[((long long)x * r.fy + y) * r.fz + z] = X<T>::div(sum, T(count));
        valid[vi] = uint8_t(k + 1);
    }
}

__global__ void k_extrap_finish_l(const int32_t* __restrict__ list, long long n, uint8_t* __restrict__ valid) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t v = valid[list[i]];
    valid[list[i]] = (v == 255) ? 255 : 0;
}

// Builds the lists: node (x, y, z) of component a's range goes to U_a when
// some component b has it in its range with liquidW_b = 0 there, and to S_a
// when component a does.  count_only: counts alone.
struct ExtRanges {
    ExtRange r[3];
};
__device__ __forceinline__ bool ext_in(const ExtRange& r, int x, int y, int z) {
    return x >= r.x0 && x <= r.x1 && y >= r.y0 && y <= r.y1 && z >= r.z0 && z <= r.z1;
}
template <class T>
__global__ void k_extrap_lists(ExtRanges rs, long long nnode, const T* __restrict__ lw0, const T* __restrict__ lw1,
                               const T* __restrict__ lw2, unsigned long long* __restrict__ counts,
                               int32_t* __restrict__ u0, int32_t* __restrict__ u1, int32_t* __restrict__ u2,
                               int32_t* __restrict__ s0, int32_t* __restrict__ s1, int32_t* __restrict__ s2) {
    const long long vi = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (vi >= nnode) return;
    int x, y, z;
    ext_node(rs.r[0], int32_t(vi), x, y, z);
    const T* lw[3] = {lw0, lw1, lw2};
    int32_t* u[3] = {u0, u1, u2};
    int32_t* sl[3] = {s0, s1, s2};
    bool in[3], solid[3], any = false;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        const ExtRange& r = rs.r[b];
        in[b] = ext_in(r, x, y, z);
        solid[b] = in[b] && !(lw[b][((long long)x * r.fy + y) * r.fz + z] > T(0));
        any |= solid[b];
    }
    if (!any) return;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (!in[a]) continue;
        const unsigned long long iu = atomicAdd(&counts[a], 1ull);
        if (u[a]) u[a][iu] = int32_t(vi);
        if (solid[a]) {
            const unsigned long long is = atomicAdd(&counts[3 + a], 1ull);
            if (sl[a]) sl[a][is] = int32_t(vi);
        }
    }
}

// LiquidModel<3>::ComputeDivergence (LiquidModel.cpp:1066-1083): per fluid
// cell divergence in Scalar, summed in double together with the cell count.
template <class T>
__global__ void k_divergence(int nx, int ny, int nz, T h, const T* __restrict__ phi, const T* __restrict__ lwx,
                             const T* __restrict__ lwy, const T* __restrict__ lwz, const T* __restrict__ vx,
                             const T* __restrict__ vy, const T* __restrict__ vz, double* __restrict__ partials,
                             unsigned* __restrict__ counter, double* __restrict__ out) {
    double s = 0.0, cnt = 0.0;
    long long n = (long long)nx * ny * nz;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        if (phi[c] > T(0)) continue;
        int x, y, z;
        idx3(c, ny, nz, x, y, z);
        long long fxi = ((long long)x * ny + y) * nz + z, fxs = (long long)ny * nz;
        long long fyi = ((long long)x * (ny + 1) + y) * nz + z, fys = nz;
        long long fzi = ((long long)x * ny + y) * (nz + 1) + z;
        T d = X<T>::sub(X<T>::mul(lwx[fxi + fxs], vx[fxi + fxs]), X<T>::mul(lwx[fxi], vx[fxi]));
        d = X<T>::add(d, X<T>::sub(X<T>::mul(lwy[fyi + fys], vy[fyi + fys]), X<T>::mul(lwy[fyi], vy[fyi])));
        d = X<T>::add(d, X<T>::sub(X<T>::mul(lwz[fzi + 1], vz[fzi + 1]), X<T>::mul(lwz[fzi], vz[fzi])));
        d = X<T>::div(d, h);
        s += double(d);
        cnt += 1.0;
    }
    double v2[2] = {s, cnt};
    grid_sum_finish<2>(v2, partials, counter, out);
}

template <class T>
__global__ void k_divergence_max(int nx, int ny, int nz, T h, const T* __restrict__ phi, const T* __restrict__ lwx,
                                 const T* __restrict__ lwy, const T* __restrict__ lwz, const T* __restrict__ vx,
                                 const T* __restrict__ vy, const T* __restrict__ vz, double* __restrict__ partials,
                                 unsigned* __restrict__ counter, double* __restrict__ out) {
    double mx = 0.0;
    long long n = (long long)nx * ny * nz;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        if (phi[c] > T(0)) continue;
        int x, y, z;
        idx3(c, ny, nz, x, y, z);
        // only cells whose six faces the velocity update touches: [1, N-3]^3
        if (x < 1 || x > nx - 3 || y < 1 || y > ny - 3 || z < 1 || z > nz - 3) continue;
        long long fxi = ((long long)x * ny + y) * nz + z, fxs = (long long)ny * nz;
        long long fyi = ((long long)x * (ny + 1) + y) * nz + z, fys = nz;
        long long fzi = ((long long)x * ny + y) * (nz + 1) + z;
        T d = X<T>::sub(X<T>::mul(lwx[fxi + fxs], vx[fxi + fxs]), X<T>::mul(lwx[fxi], vx[fxi]));
        d = X<T>::add(d, X<T>::sub(X<T>::mul(lwy[fyi + fys], vy[fyi + fys]), X<T>::mul(lwy[fyi], vy[fyi])));
        d = X<T>::add(d, X<T>::sub(X<T>::mul(lwz[fzi + 1], vz[fzi + 1]), X<T>::mul(lwz[fzi], vz[fzi])));
        d = X<T>::div(d, h);
        mx = fmax(mx, fabs(double(d)));
    }
    mx = block_max(mx);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = mx;
        __threadfence();
        last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double a = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) a = fmax(a, ((volatile double*)partials)[b]);
    a = block_max(a);
    if (threadIdx.x == 0) {
        *out = a;
        *counter = 0u;
    }
}

}  // namespace

// ------------------------------------------------------------- lifecycle
template <class T, class TX>
LiquidImpl<T, TX>::LiquidImpl(const lhi_grid_desc& g, const lhi_solver_params& sp, const lhi_liquid_params& lp,
                              int precision)
    : precision_(precision) {
    nx_ = g.dim[0];
    ny_ = g.dim[1];
    nz_ = g.dim[2];
    if (nx_ < 1 || ny_ < 1 || nz_ < 1) throw std::invalid_argument("grid dimensions must be >= 1");
    if ((long long)(nx_ + 1) * (ny_ + 1) * (nz_ + 1) >= (1LL << 31))
        throw std::invalid_argument("grid too large: (nx+1)(ny+1)(nz+1) must be < 2^31");
    int dims[3] = {nx_, ny_, nz_};
    for (int i = 0; i < 3; ++i) {
        min_[i] = T(g.min_coord[i]);
        max_[i] = T(g.max_coord[i]);
        // Grid<3>::Grid (Grid.cpp:94-97): Scalar(interval / dimension)
        T interval = max_[i] - min_[i];
        dx_[i] = T(interval / T(dims[i]));
        if (!(dx_[i] > T(0))) throw std::invalid_argument("max_coord must exceed min_coord");
        dxd_[i] = (g.max_coord[i] - g.min_coord[i]) / double(dims[i]);
    }
    radius_ = lp.particle_radius > 0 ? T(lp.particle_radius) : T(2 * dx_[0]);
    density_ = T(lp.density);
    gravity_ = T(lp.gravity);
    extrap_iters_ = lp.extrapolate_iterations > 0 ? lp.extrapolate_iterations : 5;
    correct_in_step_ = lp.correct_volume != 0;
    correct_cycle_ = lp.correct_cycle > 0 ? lp.correct_cycle : 8;
    if (extrap_iters_ > 250) throw std::invalid_argument("extrapolate_iterations must be <= 250");
    sp_ = sp;
    if (sp.max_iterations < 0 || sp.num_pre_smooth < 0 || sp.num_post_smooth < 0 || sp.num_final_smooth < 0)
        throw std::invalid_argument("negative solver parameter");
    if (sp.preconditioner < LHI_PRECOND_NONE || sp.preconditioner > LHI_PRECOND_LEARNED)
        throw std::invalid_argument("unknown preconditioner");
    if (sp.update_region != LHI_REGION_INTERIOR && sp.update_region != LHI_REGION_FLUID)
        throw std::invalid_argument("unknown update_region");
    if (sp.smoother != LHI_SMOOTHER_REFERENCE && sp.smoother != LHI_SMOOTHER_DAMPED_GS)
        throw std::invalid_argument("unknown smoother");
    if (sp.tolerance_mode != LHI_TOL_ABSOLUTE && sp.tolerance_mode != LHI_TOL_RELATIVE)
        throw std::invalid_argument("unknown tolerance_mode");
    if (sp.cg_variant != LHI_CG_REFERENCE && sp.cg_variant != LHI_CG_FLEXIBLE)
        throw std::invalid_argument("unknown cg_variant");
    if (sp.coarse_operator != LHI_COARSE_REFERENCE && sp.coarse_operator != LHI_COARSE_GALERKIN)
        throw std::invalid_argument("unknown coarse_operator");
    if (sp.initial_guess != LHI_GUESS_ZERO && sp.initial_guess != LHI_GUESS_PREVIOUS)
        throw std::invalid_argument("unknown initial_guess");
    nlev_ = std::max(1, sp.num_level);
    if (sp.preconditioner != LHI_PRECOND_MULTIGRID && sp.preconditioner != LHI_PRECOND_LEARNED) nlev_ = 1;
    if (sp.preconditioner == LHI_PRECOND_LEARNED && precision == LHI_PRECISION_FP64)
        throw std::invalid_argument("the learned preconditioner needs an FP32 or MIXED handle");
    if (nlev_ > kMaxLevels) throw std::invalid_argument("num_level above 10 is not supported");

    ncell_ = (long long)nx_ * ny_ * nz_;
    nface_[0] = (long long)(nx_ + 1) * ny_ * nz_;
    nface_[1] = (long long)nx_ * (ny_ + 1) * nz_;
    nface_[2] = (long long)nx_ * ny_ * (nz_ + 1);
    nnode_ = (long long)(nx_ + 1) * (ny_ + 1) * (nz_ + 1);

    LHI_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    LHI_CUDA(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
    cur_ = stream_;
    LHI_CUDA(cudaEventCreate(&ev0_));
    LHI_CUDA(cudaEventCreate(&ev1_));
    for (int a = 0; a < 3; ++a) {
        LHI_CUDA(cudaMalloc(&v_[a], sizeof(T) * nface_[a]));
        LHI_CUDA(cudaMalloc(&tv_[a], sizeof(T) * nface_[a]));
        LHI_CUDA(cudaMalloc(&w_[a], sizeof(T) * nface_[a]));
        LHI_CUDA(cudaMalloc(&lw_[a], sizeof(T) * nface_[a]));
        LHI_CUDA(cudaMemsetAsync(v_[a], 0, sizeof(T) * nface_[a], stream_));
        LHI_CUDA(cudaMemsetAsync(tv_[a], 0, sizeof(T) * nface_[a], stream_));
        LHI_CUDA(cudaMemsetAsync(w_[a], 0, sizeof(T) * nface_[a], stream_));
        LHI_CUDA(cudaMemsetAsync(lw_[a], 0, sizeof(T) * nface_[a], stream_));
    }
    LHI_CUDA(cudaMalloc(&pressure_, sizeof(T) * ncell_));
    LHI_CUDA(cudaMalloc(&liquid_phi_, sizeof(T) * ncell_));
    LHI_CUDA(cudaMalloc(&solid_phi_, sizeof(T) * nnode_));
    LHI_CUDA(cudaMalloc(&valid_, nnode_));
    LHI_CUDA(cudaMemsetAsync(pressure_, 0, sizeof(T) * ncell_, stream_));
    LHI_CUDA(cudaMemsetAsync(liquid_phi_, 0, sizeof(T) * ncell_, stream_));
    LHI_CUDA(cudaMemsetAsync(solid_phi_, 0, sizeof(T) * nnode_, stream_));
    LHI_CUDA(cudaMemsetAsync(valid_, 255, nnode_, stream_));  // std::vector<bool>: all false
    for (int i = 0; i < 3; ++i) occ_dim_[i] = (dims[i] + 3) / 4;
    LHI_CUDA(cudaMalloc(&occ_, size_t(occ_dim_[0]) * occ_dim_[1] * occ_dim_[2]));
    build_liquid_phi_table();
    LHI_CUDA(cudaMalloc(&cell_count_, sizeof(int32_t) * (ncell_ + 1)));
    LHI_CUDA(cudaMalloc(&cell_start_, sizeof(int32_t) * (ncell_ + 1)));
    LHI_CUDA(cudaMemsetAsync(cell_start_, 0, sizeof(int32_t) * (ncell_ + 1), stream_));
    scan_tmp_bytes_ = scan_tmp_bytes(ncell_ + 1);
    LHI_CUDA(cudaMalloc(&scan_tmp_, size_t(scan_tmp_bytes_)));

    // solver levels: dimension / (1 << level) (PressureSolver.cpp:433-440)
    for (int l = 0; l < nlev_; ++l) {
        LevelDev<T>& L = lv_[l];
        L.nx = nx_ >> l;
        L.ny = ny_ >> l;
        L.nz = nz_ >> l;
        L.n = (long long)L.nx * L.ny * L.nz;
        for (int i = 0; i < 3; ++i) L.h[i] = T(1 << l) * dx_[i];
        size_t n = size_t(std::max<long long>(L.n, 1));
        LHI_CUDA(cudaMalloc(&L.diag, sizeof(T) * n));
        for (int a = 0; a < 3; ++a) LHI_CUDA(cudaMalloc(&L.cf[a], sizeof(T) * n));
        LHI_CUDA(cudaMalloc(&L.type, n));
        LHI_CUDA(cudaMalloc(&L.phi, sizeof(T) * n));
        LHI_CUDA(cudaMalloc(&L.r, sizeof(T) * n));
        LHI_CUDA(cudaMalloc(&L.z, sizeof(T) * n));
        LHI_CUDA(cudaMemsetAsync(L.diag, 0, sizeof(T) * n, stream_));
        for (int a = 0; a < 3; ++a) LHI_CUDA(cudaMemsetAsync(L.cf[a], 0, sizeof(T) * n, stream_));
        LHI_CUDA(cudaMemsetAsync(L.type, 0, n, stream_));
        LHI_CUDA(cudaMemsetAsync(L.phi, 0, sizeof(T) * n, stream_));
        LHI_CUDA(cudaMemsetAsync(L.r, 0, sizeof(T) * n, stream_));
        LHI_CUDA(cudaMemsetAsync(L.z, 0, sizeof(T) * n, stream_));
        L.tdim[0] = (L.nx + kTileX - 1) / kTileX;
        L.tdim[1] = (L.ny + kTileY - 1) / kTileY;
        L.tdim[2] = (L.nz + kTileZ - 1) / kTileZ;
        L.ntiles = (L.n > 0) ? L.tdim[0] * L.tdim[1] * L.tdim[2] : 0;
        size_t nt = size_t(std::max(L.ntiles, 1));
        LHI_CUDA(cudaMalloc(&L.tile_flag, nt));
        LHI_CUDA(cudaMalloc(&L.tiles, sizeof(int32_t) * nt));
        LHI_CUDA(cudaMemsetAsync(L.tile_flag, 0, nt, stream_));
        LHI_CUDA(cudaMemsetAsync(L.tiles, 0, sizeof(int32_t) * nt, stream_));
    }
    setup_coarse();
    setup_fused();
    tile_grid_ = kSMs * 6;
    LHI_CUDA(cudaMalloc(&rhs_, sizeof(T) * ncell_));
    LHI_CUDA(cudaMalloc(&x_, sizeof(TX) * ncell_));
    LHI_CUDA(cudaMalloc(&p_, sizeof(T) * ncell_));
    LHI_CUDA(cudaMalloc(&ap_, sizeof(T) * ncell_));
    LHI_CUDA(cudaMemsetAsync(rhs_, 0, sizeof(T) * ncell_, stream_));
    LHI_CUDA(cudaMemsetAsync(x_, 0, sizeof(TX) * ncell_, stream_));
    LHI_CUDA(cudaMemsetAsync(p_, 0, sizeof(T) * ncell_, stream_));
    LHI_CUDA(cudaMemsetAsync(ap_, 0, sizeof(T) * ncell_, stream_));
    if constexpr (kHiResidual) {
        LHI_CUDA(cudaMalloc(&rhs_hi_, sizeof(double) * ncell_));
        LHI_CUDA(cudaMalloc(&diag_hi_, sizeof(double) * ncell_));
        LHI_CUDA(cudaMemsetAsync(rhs_hi_, 0, sizeof(double) * ncell_, stream_));
        LHI_CUDA(cudaMemsetAsync(diag_hi_, 0, sizeof(double) * ncell_, stream_));
        for (int a = 0; a < 3; ++a) {
            LHI_CUDA(cudaMalloc(&cf_hi_[a], sizeof(double) * ncell_));
            LHI_CUDA(cudaMemsetAsync(cf_hi_[a], 0, sizeof(double) * ncell_, stream_));
        }
    }
    setup_spmv();
    LHI_CUDA(cudaMalloc(&sc_, sizeof(SolveScalars)));
    LHI_CUDA(cudaMemsetAsync(sc_, 0, sizeof(SolveScalars), stream_));
    LHI_CUDA(cudaHostAlloc(&sc_host_, sizeof(SolveScalars), cudaHostAllocDefault));
    std::memset(sc_host_, 0, sizeof(SolveScalars));
    sum_blocks_ = 4 * kSMs;
    LHI_CUDA(cudaMalloc(&partials_, sizeof(double) * 8 * 4096));
    LHI_CUDA(cudaMalloc(&counter_, sizeof(unsigned) * 16));
    LHI_CUDA(cudaMemsetAsync(counter_, 0, sizeof(unsigned) * 16, stream_));
    alloc_particles(1);
    LHI_CUDA(cudaStreamSynchronize(stream_));
}

template <class T, class TX> LiquidImpl<T, TX>::~LiquidImpl() {
    if (stream_) cudaStreamSynchronize(stream_);
    auto F = [](void* p) {
        if (p) cudaFree(p);
    };
    for (int a = 0; a < 3; ++a) {
        F(v_[a]);
        F(tv_[a]);
        F(w_[a]);
        F(lw_[a]);
    }
    F(image_);
    F(ndc_);
    F(pressure_);
    F(liquid_phi_);
    F(solid_phi_);
    F(valid_);
    for (int a = 0; a < 3; ++a) {
        F(ext_u_[a]);
        F(ext_s_[a]);
    }
    F(occ_);
    F(lphi_tab_);
    F(cell_count_);
    F(cell_start_);
    F(scan_tmp_);
    for (int b = 0; b < 2; ++b) {
        F(pdata_[b]);
        F(pid_[b]);
        F(keys_[b]);
        F(vals_[b]);
    }
    for (int l = 0; l < nlev_; ++l) {
        F(lv_[l].diag);
        for (int a = 0; a < 3; ++a) F(lv_[l].cf[a]);
        F(lv_[l].type);
        F(lv_[l].phi);
        F(lv_[l].r);
        F(lv_[l].z);
        F(lv_[l].zb);
        F(lv_[l].mask);
        F(lv_[l].tile_flag);
        F(lv_[l].tiles);
    }
    F(coarse_list_);
    F(coarse_counts_);
    if (solve_exec_) cudaGraphExecDestroy(solve_exec_);
    if (tail_exec_) cudaGraphExecDestroy(tail_exec_);
    F(solid_cell_);
    F(net_type_);
    F(snaps_);
    F(train_z_);
    F(train_dz_);
    F(train_e_);
    F(train_red_);
    if (side_) cudaStreamDestroy(side_);
    F(rhs_);
    F(rhs_hi_);
    F(diag_hi_);
    for (int a = 0; a < 3; ++a) F(cf_hi_[a]);
    F(x_);
    F(p_);
    F(ap_);
    F(sc_);
    F(partials_);
    F(counter_);
    if (sc_host_) cudaFreeHost(sc_host_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (stream_) cudaStreamDestroy(stream_);
}

// ------------------------------------------------------------------ stages
// Grid<3>::Clear (Grid.cpp:157-169); isValid is left as it is.
template <class T, class TX> void LiquidImpl<T, TX>::clear() {
    auto ps_ = scope(LHI_KERNEL_GRID);
    LHI_CUDA(cudaMemsetAsync(pressure_, 0, sizeof(T) * ncell_, stream_));
    k_fill<T><<<blocks_for(ncell_, 256), 256, 0, stream_>>>(liquid_phi_, ncell_, T(3 * dx_[0]));
    LHI_LAUNCH_CHECK();
    for (int a = 0; a < 3; ++a) {
        LHI_CUDA(cudaMemsetAsync(v_[a], 0, sizeof(T) * nface_[a], stream_));
        LHI_CUDA(cudaMemsetAsync(w_[a], 0, sizeof(T) * nface_[a], stream_));
        LHI_CUDA(cudaMemsetAsync(tv_[a], 0, sizeof(T) * nface_[a], stream_));
    }
}

template <class T, class TX> void LiquidImpl<T, TX>::set_boundary(const BoundaryProgram& prog) {
    solid_cell_fresh_ = false;
    ext_dirty_ = true;
    G3<T> g{nx_, ny_, nz_, {min_[0], min_[1], min_[2]}, {dx_[0], dx_[1], dx_[2]}};
    k_boundary<T><<<blocks_for(nnode_, 256), 256, 0, stream_>>>(prog, g, solid_phi_);
    LHI_LAUNCH_CHECK();
    for (int a = 0; a < 3; ++a) {
        k_face_fractions<T><<<blocks_for(nface_[a], 256), 256, 0, stream_>>>(solid_phi_, nx_, ny_, nz_, a, lw_[a]);
        LHI_LAUNCH_CHECK();
    }
}

template <class T, class TX> void LiquidImpl<T, TX>::set_solid_phi(const void* host) {
    solid_cell_fresh_ = false;
    ext_dirty_ = true;
    LHI_CUDA(cudaMemcpyAsync(solid_phi_, host, sizeof(T) * nnode_, cudaMemcpyHostToDevice, stream_));
    for (int a = 0; a < 3; ++a) {
        k_face_fractions<T><<<blocks_for(nface_[a], 256), 256, 0, stream_>>>(solid_phi_, nx_, ny_, nz_, a, lw_[a]);
        LHI_LAUNCH_CHECK();
    }
    LHI_CUDA(cudaStreamSynchronize(stream_));
}

template <class T, class TX> void LiquidImpl<T, TX>::apply_gravity(double dt) {
    auto ps_ = scope(LHI_KERNEL_GRID);
    T gdt = gravity_ * T(dt);
    k_gravity<T><<<blocks_for(nface_[1], 256), 256, 0, stream_>>>(v_[1], nx_, ny_, nz_, gdt);
    LHI_LAUNCH_CHECK();
}

template <class T, class TX> void LiquidImpl<T, TX>::velocity_update(double dt) {
    long long n = (long long)std::max(nx_ - 2, 0) * std::max(ny_ - 2, 0) * std::max(nz_ - 2, 0);
    if (n == 0) return;
    auto ps_ = scope(LHI_KERNEL_GRID);
    k_velocity_update<T><<<blocks_for(n, 256), 256, 0, stream_>>>(nx_, ny_, nz_, dx_[0], dx_[1], dx_[2], T(dt),
                                                                   density_, liquid_phi_, pressure_, lw_[0], lw_[1],
                                                                   lw_[2], v_[0], v_[1], v_[2]);
    LHI_LAUNCH_CHECK();
}

// LiquidModel<3>::Projection -> SolvePressure (LiquidModel.cpp:826-896)
template <class T, class TX> int LiquidImpl<T, TX>::projection(double dt) {
    if (np_ == 0) return LHI_OK;
    int st = solve(double(density_), dt);
    velocity_update(dt);
    return st;
}

// The extrapolation range of face component a (LiquidModel.cpp:949-953).
static ExtRange ext_range(int a, int nx, int ny, int nz) {
    ExtRange r;
    r.x0 = 1;
    r.x1 = (a == 0) ? nx - 1 : nx - 2;
    r.y0 = 1;
    r.y1 = (a == 1) ? ny - 1 : ny - 2;
    r.z0 = 1;
    r.z1 = (a == 2) ? nz - 1 : nz - 2;
    r.fy = ny + (a == 1);
    r.fz = nz + (a == 2);
    r.ny1 = ny + 1;
    r.nz1 = nz + 1;
    return r;
}

template <class T, class TX> void LiquidImpl<T, TX>::build_extrapolation_lists() {
    ExtRanges rs;
    for (int a = 0; a < 3; ++a) {
        rs.r[a] = ext_range(a, nx_, ny_, nz_);
        if (ext_u_[a]) cudaFree(ext_u_[a]);
        if (ext_s_[a]) cudaFree(ext_s_[a]);
        ext_u_[a] = ext_s_[a] = nullptr;
    }
    unsigned long long* counts = reinterpret_cast<unsigned long long*>(partials_);  // 6 counters, scratch
    unsigned long long hc[6];
    for (int pass = 0; pass < 2; ++pass) {
        LHI_CUDA(cudaMemsetAsync(counts, 0, sizeof(hc), stream_));
        k_extrap_lists<T><<<blocks_for(nnode_, 256), 256, 0, stream_>>>(rs, nnode_, lw_[0], lw_[1], lw_[2], counts,
                                                                       ext_u_[0], ext_u_[1], ext_u_[2], ext_s_[0],
                                                                       ext_s_[1], ext_s_[2]);
        LHI_LAUNCH_CHECK();
        LHI_CUDA(cudaMemcpyAsync(hc, counts, sizeof(hc), cudaMemcpyDeviceToHost, stream_));
        LHI_CUDA(cudaStreamSynchronize(stream_));
        if (pass == 1) break;
        for (int a = 0; a < 3; ++a) {  // first pass counted: allocate, then fill
            ext_nu_[a] = (long long)hc[a];
            ext_ns_[a] = (long long)hc[3 + a];
            LHI_CUDA(cudaMalloc(&ext_u_[a], sizeof(int32_t) * size_t(std::max(ext_nu_[a], 1LL))));
            LHI_CUDA(cudaMalloc(&ext_s_[a], sizeof(int32_t) * size_t(std::max(ext_ns_[a], 1LL))));
        }
    }
    ext_dirty_ = false;
}

// LiquidModel<3>::Extrapolate.  After the first call (or a change of the
// solid fractions or of isValid, which run the full passes again) the init,
// the in-place sweeps and the finish walk the node lists; the sweeps through
// tempV keep their full pass, which also copies every face of the range.
template <class T, class TX> void LiquidImpl<T, TX>::extrapolate() {
    if (np_ == 0) return;
    auto ps_ = scope(LHI_KERNEL_EXTRAPOLATE);
    const bool full = ext_dirty_;
    for (int a = 0; a < 3; ++a) {
        const ExtRange r = ext_range(a, nx_, ny_, nz_);
        const long long n = ext_threads(r);  // 4 faces along z per thread
        if (full && n > 0) {
            k_extrap_init<T><<<blocks_for(n, 256), 256, 0, stream_>>>(r, lw_[a], valid_);
            LHI_LAUNCH_CHECK();
        } else if (ext_nu_[a] > 0) {
            k_extrap_init_l<T><<<blocks_for(ext_nu_[a], 256), 256, 0, stream_>>>(r, ext_u_[a], ext_nu_[a], lw_[a],
                                                                                 valid_);
            LHI_LAUNCH_CHECK();
        }
        // The reference sweeps into tempV and swaps (std::swap(m_grid.tempVx,
        // m_grid.vx)) after every sweep.  The first sweeps run in place on vx;
        // the last one (odd count) or two (even count) go through tempV with
        // the swaps, which leaves vx and tempVx holding the reference's last
        // two states in the reference's buffers (faces outside the range keep
        // each buffer's own values).
        const int jacobi_from = extrap_iters_ - ((extrap_iters_ % 2) ? 1 : 2);
        for (int k = 0; k < extrap_iters_; ++k) {
            const bool swap = k >= jacobi_from;
            if (!full && !swap) {
                if (ext_ns_[a] > 0) {
                    k_extrap_sweep_l<T><<<blocks_for(ext_ns_[a], 256), 256, 0, stream_>>>(r, ext_s_[a], ext_ns_[a], k,
                                                                                         v_[a], valid_);
                    LHI_LAUNCH_CHECK();
                }
                continue;
            }
            if (n > 0) {
                k_extrap_sweep<T><<<blocks_for(n, 256), 256, 0, stream_>>>(r, k, v_[a], swap ? tv_[a] : v_[a],
                                                                         valid_);
                LHI_LAUNCH_CHECK();
            }
            if (swap) std::swap(v_[a], tv_[a]);
        }
        if (full && n > 0) {
            k_extrap_finish<<<blocks_for(n, 256), 256, 0, stream_>>>(r, valid_);
            LHI_LAUNCH_CHECK();
        } else if (ext_ns_[a] > 0) {
            k_extrap_finish_l<<<blocks_for(ext_ns_[a], 256), 256, 0, stream_>>>(ext_s_[a], ext_ns_[a], valid_);
            LHI_LAUNCH_CHECK();
        }
    }
    if (full) build_extrapolation_lists();
}

template <class T, class TX> void LiquidImpl<T, TX>::divergence(double* mean, double* max_abs) {
    unsigned nb = std::min<unsigned>(blocks_for(ncell_, 256), unsigned(sum_blocks_));
    k_divergence<T><<<nb, 256, 0, stream_>>>(nx_, ny_, nz_, dx_[0], liquid_phi_, lw_[0], lw_[1], lw_[2], v_[0],
                                             v_[1], v_[2], partials_, counter_, &sc_->div[0]);
    LHI_LAUNCH_CHECK();
    k_divergence_max<T><<<nb, 256, 0, stream_>>>(nx_, ny_, nz_, dx_[0], liquid_phi_, lw_[0], lw_[1], lw_[2], v_[0],
                                                 v_[1], v_[2], partials_, counter_, &sc_->div[2]);
    LHI_LAUNCH_CHECK();
    read_scalars();
    double s = sc_host_->div[0], c = sc_host_->div[1];
    if (mean) *mean = (c > 0) ? s / c : std::nan("");
    if (max_abs) *max_abs = sc_host_->div[2];
}

template <class T, class TX> int LiquidImpl<T, TX>::pre_step(double dt) {
    (void)dt;
    clear();
    compute_liquid_phi();
    return LHI_OK;
}

// LiquidModel<3>::Step (LiquidModel.cpp:520-528)
template <class T, class TX> int LiquidImpl<T, TX>::step(double dt) {
    if (np_ == 0) return LHI_OK;
    p2g_accumulate();
    p2g_normalize(true, gravity_ * T(dt));  // Particle2Grid normalisation + ApplyGravity
    int st = projection(dt);
    extrapolate();
    g2p(true, T(dt));  // Grid2Particle + AdvectParticle
    if (correct_in_step_) correct_volume(dt);
    return st;
}

// ------------------------------------------------------------------ fields
template <class T, class TX> int LiquidImpl<T, TX>::field_size(int f, int level, int64_t* count, int32_t* eb) {
    *eb = sizeof(T);
    switch (f) {
        case LHI_FIELD_VX:
        case LHI_FIELD_WX:
        case LHI_FIELD_LIQUID_WX:
        case LHI_FIELD_TEMP_VX: *count = nface_[0]; return 0;
        case LHI_FIELD_VY:
        case LHI_FIELD_WY:
        case LHI_FIELD_LIQUID_WY:
        case LHI_FIELD_TEMP_VY: *count = nface_[1]; return 0;
        case LHI_FIELD_VZ:
        case LHI_FIELD_WZ:
        case LHI_FIELD_LIQUID_WZ:
        case LHI_FIELD_TEMP_VZ: *count = nface_[2]; return 0;
        case LHI_FIELD_PRESSURE:
        case LHI_FIELD_LIQUID_PHI:
        case LHI_FIELD_RHS:
        case LHI_FIELD_X:
        case LHI_FIELD_P:
        case LHI_FIELD_AP: *count = ncell_; return 0;
        case LHI_FIELD_SOLID_PHI: *count = nnode_; return 0;
        case LHI_FIELD_IS_VALID:
            *count = nnode_;
            *eb = 1;
            return 0;
        case LHI_FIELD_R:
        case LHI_FIELD_Z:
        case LHI_FIELD_ADIAG:
        case LHI_FIELD_ACOEF:
            if (level < 0 || level >= nlev_) return LHI_E_INVALID_ARG;
            *count = lv_[level].n * (f == LHI_FIELD_ACOEF ? 6 : 1);
            return 0;
        case LHI_FIELD_CELL_KEY:
        case LHI_FIELD_PARTICLE_ID:
            *count = np_;
            *eb = 4;
            return 0;
        case LHI_FIELD_CELL_START:
            *count = ncell_ + 1;
            *eb = 4;
            return 0;
        default: return LHI_E_INVALID_ARG;
    }
}

template <class T, class TX> static T* grid_ptr(LiquidImpl<T, TX>& s, int f, int level) {
    switch (f) {
        case LHI_FIELD_VX: return s.v_[0];
        case LHI_FIELD_VY: return s.v_[1];
        case LHI_FIELD_VZ: return s.v_[2];
        case LHI_FIELD_WX: return s.w_[0];
        case LHI_FIELD_WY: return s.w_[1];
        case LHI_FIELD_WZ: return s.w_[2];
        case LHI_FIELD_LIQUID_WX: return s.lw_[0];
        case LHI_FIELD_LIQUID_WY: return s.lw_[1];
        case LHI_FIELD_LIQUID_WZ: return s.lw_[2];
        case LHI_FIELD_TEMP_VX: return s.tv_[0];
        case LHI_FIELD_TEMP_VY: return s.tv_[1];
        case LHI_FIELD_TEMP_VZ: return s.tv_[2];
        case LHI_FIELD_PRESSURE: return s.pressure_;
        case LHI_FIELD_LIQUID_PHI: return s.liquid_phi_;
        case LHI_FIELD_SOLID_PHI: return s.solid_phi_;
        case LHI_FIELD_RHS: return s.rhs_;
        case LHI_FIELD_P: return s.p_;
        case LHI_FIELD_AP: return s.ap_;
        case LHI_FIELD_R: return s.lv_[level].r;
        case LHI_FIELD_Z: return s.lv_[level].z;
        case LHI_FIELD_ADIAG: return s.lv_[level].diag;
        default: return nullptr;
    }
}

template <class T, class TX> void LiquidImpl<T, TX>::get_field(int f, int level, void* out) {
    int64_t count;
    int32_t eb;
    if (field_size(f, level, &count, &eb)) throw std::invalid_argument("unknown field or level");
    if (count == 0) return;
    if (f == LHI_FIELD_IS_VALID) {
        LHI_CUDA(cudaMemcpyAsync(out, valid_, count, cudaMemcpyDeviceToHost, stream_));
        LHI_CUDA(cudaStreamSynchronize(stream_));
        uint8_t* o = static_cast<uint8_t*>(out);
        for (int64_t i = 0; i < count; ++i) o[i] = (o[i] == 255) ? 0 : 1;
        return;
    }
    if (f == LHI_FIELD_CELL_KEY || f == LHI_FIELD_CELL_START) {
        ensure_sorted();
        const void* src = (f == LHI_FIELD_CELL_KEY) ? (const void*)keys_[0] : (const void*)cell_start_;
        LHI_CUDA(cudaMemcpyAsync(out, src, count * 4, cudaMemcpyDeviceToHost, stream_));
        LHI_CUDA(cudaStreamSynchronize(stream_));
        return;
    }
    if (f == LHI_FIELD_PARTICLE_ID) {
        apply_order();  // the ids in the current (cell-sorted, once sorted) order
        LHI_CUDA(cudaMemcpyAsync(out, pid_[pcur_], count * 4, cudaMemcpyDeviceToHost, stream_));
        LHI_CUDA(cudaStreamSynchronize(stream_));
        return;
    }
    if (f == LHI_FIELD_X) {
        std::vector<TX> tmp(count);
        LHI_CUDA(cudaMemcpyAsync(tmp.data(), x_, sizeof(TX) * count, cudaMemcpyDeviceToHost, stream_));
        LHI_CUDA(cudaStreamSynchronize(stream_));
        T* o = static_cast<T*>(out);
        for (int64_t i = 0; i < count; ++i) o[i] = T(tmp[i]);
        return;
    }
    if (f == LHI_FIELD_ACOEF) {
        get_acoef(level, static_cast<T*>(out));
        return;
    }
    T* src = grid_ptr(*this, f, level);
    LHI_CUDA(cudaMemcpyAsync(out, src, sizeof(T) * count, cudaMemcpyDeviceToHost, stream_));
    LHI_CUDA(cudaStreamSynchronize(stream_));
}

template <class T, class TX> void LiquidImpl<T, TX>::set_field(int f, int level, const void* in) {
    int64_t count;
    int32_t eb;
    if (field_size(f, level, &count, &eb)) throw std::invalid_argument("unknown field or level");
    if (count == 0) return;
    if (f == LHI_FIELD_CELL_KEY || f == LHI_FIELD_PARTICLE_ID || f == LHI_FIELD_CELL_START ||
        f == LHI_FIELD_ACOEF)
        throw std::invalid_argument("field is read-only");
    if (f == LHI_FIELD_IS_VALID || f == LHI_FIELD_LIQUID_WX || f == LHI_FIELD_LIQUID_WY ||
        f == LHI_FIELD_LIQUID_WZ)
        ext_dirty_ = true;  // the extrapolation's node lists follow these
    if (f == LHI_FIELD_IS_VALID) {
        std::vector<uint8_t> tmp(count);
        const uint8_t* p = static_cast<const uint8_t*>(in);
        for (int64_t i = 0; i < count; ++i) tmp[i] = p[i] ? 0 : 255;
        LHI_CUDA(cudaMemcpyAsync(valid_, tmp.data(), count, cudaMemcpyHostToDevice, stream_));
        LHI_CUDA(cudaStreamSynchronize(stream_));
        return;
    }
    if (f == LHI_FIELD_X) {
        std::vector<TX> tmp(count);
        const T* p = static_cast<const T*>(in);
        for (int64_t i = 0; i < count; ++i) tmp[i] = TX(p[i]);
        LHI_CUDA(cudaMemcpyAsync(x_, tmp.data(), sizeof(TX) * count, cudaMemcpyHostToDevice, stream_));
        LHI_CUDA(cudaStreamSynchronize(stream_));
        return;
    }
    T* dst = grid_ptr(*this, f, level);
    LHI_CUDA(cudaMemcpyAsync(dst, in, sizeof(T) * count, cudaMemcpyHostToDevice, stream_));
    LHI_CUDA(cudaStreamSynchronize(stream_));
}

template class LiquidImpl<float, float>;
template class LiquidImpl<float, double>;
template class LiquidImpl<double, double>;

}  // namespace lhi
