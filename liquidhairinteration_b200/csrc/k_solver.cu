// k_solver.cu -- CGSolver<3> on the device: per-level ghost-fluid matrix
// assembly, SpMV, damped red-black Gauss-Seidel, restriction/prolongation,
// the V-cycle preconditioner and the PCG loop with device-resident scalars.
//
// Matrix storage: per level, diag plus one coefficient per +x/+y/+z face and
// a cell type byte (0: phi > 0, 1: phi == 0, 2: phi < 0).  The reference's
// per-row coefficient (PressureSolver.cpp:556-662) is -term when the
// neighbour has phi < 0 and 0 otherwise, and rows with phi > 0 are empty; the
// face term is the same expression seen from both rows, so
//   A(i, j) = [type_i >= 1] [type_j == 2] * face_coef(i, j).
#include <algorithm>

#include "impl.cuh"

namespace lhi {

namespace {

template <class T> struct LevelK {
    int nx, ny, nz;
    const T* diag;
    const T* cx;
    const T* cy;
    const T* cz;
    const uint8_t* type;
};

template <class T> LevelK<T> lk(const LevelDev<T>& L) {
    return LevelK<T>{L.nx, L.ny, L.nz, L.diag, L.cf[0], L.cf[1], L.cf[2], L.type};
}

__device__ __forceinline__ void decode(long long i, int ny, int nz, int& x, int& y, int& z) {
    z = int(i % nz);
    long long t = i / nz;
    y = int(t % ny);
    x = int(t / ny);
}

// CGSolver<3>::GetAx (PressureSolver.cpp:700-717), computed in C
template <class C, class T, class V>
__device__ __forceinline__ C ax_at(const LevelK<T>& L, const V* __restrict__ x, long long i, int xi, int yi, int zi) {
    if (L.type[i] == 0) return C(0);
    const long long sy = L.nz, sx = (long long)L.ny * L.nz;
    C r = C(x[i]) * C(L.diag[i]);
    if (xi + 1 < L.nx && L.type[i + sx] == 2) r += C(x[i + sx]) * C(L.cx[i]);
    if (xi - 1 >= 0 && L.type[i - sx] == 2) r += C(x[i - sx]) * C(L.cx[i - sx]);
    if (yi + 1 < L.ny && L.type[i + sy] == 2) r += C(x[i + sy]) * C(L.cy[i]);
    if (yi - 1 >= 0 && L.type[i - sy] == 2) r += C(x[i - sy]) * C(L.cy[i - sy]);
    if (zi + 1 < L.nz && L.type[i + 1] == 2) r += C(x[i + 1]) * C(L.cz[i]);
    if (zi - 1 >= 0 && L.type[i - 1] == 2) r += C(x[i - 1]) * C(L.cz[i - 1]);
    return r;
}

// PCG update region: fluid cells of [1, N-2]^3 (PressureSolver.cpp:874-899)
// or, with LHI_REGION_FLUID, every fluid cell.
__device__ __forceinline__ bool in_region(int x, int y, int z, int nx, int ny, int nz, int region) {
    return region == LHI_REGION_FLUID || (x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2 && z >= 1 && z <= nz - 2);
}

// ------------------------------------------------------------- assembly
struct LevelGeom {
    int nx, ny, nz;     // this level
    int fnx, fny, fnz;  // level 0
    int level;
};

// GetApproxLiquidPhi (PressureSolver.cpp:476-493): trilerp of the 2x2x2
// central fine cells with factors 0.5.
template <class T> __device__ __forceinline__ T approx_phi(const T* __restrict__ f, LevelGeom g, int xi, int yi, int zi) {
    if (g.level == 0) return f[((long long)xi * g.fny + yi) * g.fnz + zi];
    const int fac = 1 << g.level, h = (1 << (g.level - 1)) - 1;
    const int bx = fac * xi + h, by = fac * yi + h, bz = fac * zi + h;
    const long long sy = g.fnz, sx = (long long)g.fny * g.fnz;
    const T* b = f + bx * sx + by * sy + bz;
    return trilerp(b[0], b[sx], b[sy], b[sx + sy], b[1], b[sx + 1], b[sy + 1], b[sx + sy + 1], T(0.5), T(0.5), T(0.5));
}
// GetApproxWx / Wy / Wz (PressureSolver.cpp:495-542)
template <class T> __device__ __forceinline__ T approx_w(const T* __restrict__ w, LevelGeom g, int a, int xi, int yi, int zi) {
    const int fy = g.fny + (a == 1), fz = g.fnz + (a == 2);
    if (g.level == 0) return w[((long long)xi * fy + yi) * fz + zi];
    const int fac = 1 << g.level, h = (1 << (g.level - 1)) - 1;
    const long long sy = fz, sx = (long long)fy * fz;
    if (a == 0) {
        const T* b = w + (long long)(fac * xi) * sx + (long long)(fac * yi + h) * sy + (fac * zi + h);
        return bilerp(b[0], b[sy], b[1], b[sy + 1], T(0.5), T(0.5));
    } else if (a == 1) {
        const T* b = w + (long long)(fac * xi + h) * sx + (long long)(fac * yi) * sy + (fac * zi + h);
        return bilerp(b[0], b[sx], b[1], b[sx + 1], T(0.5), T(0.5));
    }
    const T* b = w + (long long)(fac * xi + h) * sx + (long long)(fac * yi + h) * sy + (fac * zi);
    return bilerp(b[0], b[sx], b[sy], b[sx + sy], T(0.5), T(0.5));
}

template <class T>
__global__ void k_level_phi(LevelGeom g, const T* __restrict__ fine_phi, T* __restrict__ phi, uint8_t* __restrict__ type) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)g.nx * g.ny * g.nz;
    if (i >= n) return;
    int x, y, z;
    decode(i, g.ny, g.nz, x, y, z);
    T ph = approx_phi(fine_phi, g, x, y, z);
    if (g.level > 0) phi[i] = ph;
    type[i] = (ph > T(0)) ? 0 : ((ph < T(0)) ? 2 : 1);
}

// CGSolver<3>::BuildLHS for one level (PressureSolver.cpp:544-664).
template <class T>
__global__ void k_level_matrix(LevelGeom g, const T* __restrict__ phi, const T* __restrict__ lwx,
                               const T* __restrict__ lwy, const T* __restrict__ lwz, T h0, T h1, T h2, T dt, T rho,
                               T* __restrict__ diag, T* __restrict__ cx, T* __restrict__ cy, T* __restrict__ cz) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)g.nx * g.ny * g.nz;
    if (i >= n) return;
    int x, y, z;
    decode(i, g.ny, g.nz, x, y, z);
    const long long sy = g.nz, sx = (long long)g.ny * g.nz;
    const T* lw[3] = {lwx, lwy, lwz};
    const T hh[3] = {h0, h1, h2};
    auto term_of = [&](int a, T w) -> T {
        return X<T>::div(X<T>::mul(w, dt), X<T>::mul(X<T>::mul(rho, hh[a]), hh[a]));
    };
    // own +x/+y/+z face coefficients
    T c[3] = {T(0), T(0), T(0)};
    {
        int cc[3] = {x, y, z};
        int dd[3] = {g.nx, g.ny, g.nz};
        for (int a = 0; a < 3; ++a) {
            if (cc[a] + 1 < dd[a]) {
                T w = approx_w(lw[a], g, a, x + (a == 0), y + (a == 1), z + (a == 2));
                if (w > T(0)) c[a] = -term_of(a, w);
            }
        }
    }
    cx[i] = c[0];
    cy[i] = c[1];
    cz[i] = c[2];
    const T center = phi[i];
    T d = T(0);
    if (!(center > T(0))) {
        // right, left, top, bottom, front, back
        const int xs[6] = {x + 1, x, x, x, x, x};
        const int ys[6] = {y, y, y + 1, y, y, y};
        const int zs[6] = {z, z, z, z, z + 1, z};
        const int ax[6] = {0, 0, 1, 1, 2, 2};
        const long long off[6] = {sx, -sx, sy, -sy, 1, -1};
        const bool exists[6] = {x + 1 < g.nx, x - 1 >= 0, y + 1 < g.ny, y - 1 >= 0, z + 1 < g.nz, z - 1 >= 0};
        for (int k = 0; k < 6; ++k) {
            if (!exists[k]) continue;
            const int a = ax[k];
            T w = approx_w(lw[a], g, a, xs[k], ys[k], zs[k]);
            if (w > T(0)) {
                T term = term_of(a, w);
                T nphi = phi[i + off[k]];
                if (nphi < T(0)) d = X<T>::add(d, term);
                else d = X<T>::add(d, X<T>::div(term, frac_floor(fraction_in_region(center, nphi))));
            }
        }
    }
    diag[i] = d;
}

// CGSolver<3>::BuildRHS (PressureSolver.cpp:682-698)
template <class T>
__global__ void k_build_rhs(int nx, int ny, int nz, T h0, T h1, T h2, const T* __restrict__ phi,
                            const T* __restrict__ lwx, const T* __restrict__ lwy, const T* __restrict__ lwz,
                            const T* __restrict__ vx, const T* __restrict__ vy, const T* __restrict__ vz,
                            T* __restrict__ rhs) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)nx * ny * nz;
    if (i >= n) return;
    T b = T(0);
    if (!(phi[i] > T(0))) {
        int x, y, z;
        decode(i, ny, nz, x, y, z);
        long long fxi = ((long long)x * ny + y) * nz + z, fxs = (long long)ny * nz;
        long long fyi = ((long long)x * (ny + 1) + y) * nz + z, fys = nz;
        long long fzi = ((long long)x * ny + y) * (nz + 1) + z;
        b = X<T>::sub(b, X<T>::div(X<T>::mul(lwx[fxi + fxs], vx[fxi + fxs]), h0));
        b = X<T>::add(b, X<T>::div(X<T>::mul(lwx[fxi], vx[fxi]), h0));
        b = X<T>::sub(b, X<T>::div(X<T>::mul(lwy[fyi + fys], vy[fyi + fys]), h1));
        b = X<T>::add(b, X<T>::div(X<T>::mul(lwy[fyi], vy[fyi]), h1));
        b = X<T>::sub(b, X<T>::div(X<T>::mul(lwz[fzi + 1], vz[fzi + 1]), h2));
        b = X<T>::add(b, X<T>::div(X<T>::mul(lwz[fzi], vz[fzi]), h2));
    }
    rhs[i] = b;
}

// ----------------------------------------------------------- V-cycle
// CGSolver<3>::Smooth (PressureSolver.cpp:821-837): one colour of damped
// red-black Gauss-Seidel; (1. - w) * z + w * term evaluated in double.
template <class T>
__device__ __forceinline__ void smooth_cell(const LevelK<T>& L, const T* __restrict__ r, T* __restrict__ z, T w,
                                            int variant, long long i, int x, int y, int zz) {
    T dg = L.diag[i];
    if (is_small(dg)) return;
    T term = (r[i] - ax_at<T>(L, z, i, x, y, zz)) / dg;
    if (variant == LHI_SMOOTHER_DAMPED_GS) z[i] = z[i] + w * term;
    else z[i] = T((1.0 - double(w)) * double(z[i]) + double(T(w * term)));
}

template <class T>
__global__ void __launch_bounds__(256) k_smooth(LevelK<T> L, const T* __restrict__ r, T* __restrict__ z, T w,
                                               int variant, int phase) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)L.nx * L.ny * L.nz;
    if (i >= n) return;
    int x, y, zz;
    decode(i, L.ny, L.nz, x, y, zz);
    if (((x + y + zz) & 1) != phase) return;
    smooth_cell(L, r, z, w, variant, i, x, y, zz);
}

// All sweeps of a small level inside one CTA (the level is L2-resident).
template <class T>
__global__ void __launch_bounds__(1024) k_smooth_block(LevelK<T> L, const T* __restrict__ r, T* __restrict__ z, T w,
                                                       int variant, int sweeps) {
    long long n = (long long)L.nx * L.ny * L.nz;
    for (int s = 0; s < sweeps; ++s)
        for (int phase = 0; phase < 2; ++phase) {
            for (long long i = threadIdx.x; i < n; i += blockDim.x) {
                int x, y, zz;
                decode(i, L.ny, L.nz, x, y, zz);
                if (((x + y + zz) & 1) != phase) continue;
                smooth_cell(L, r, z, w, variant, i, x, y, zz);
            }
            __syncthreads();
        }
}

// CGSolver<3>::Restrict (PressureSolver.cpp:796-819): the coarse residual is
// accumulated in Scalar with 0.125 * (...) evaluated in double; z_c = 0.
template <class T>
__global__ void k_restrict(LevelK<T> F, const T* __restrict__ rf, const T* __restrict__ zf, int cnx, int cny, int cnz,
                           T* __restrict__ rc, T* __restrict__ zc) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)cnx * cny * cnz;
    if (i >= n) return;
    int x, y, z;
    decode(i, cny, cnz, x, y, z);
    const long long sy = F.nz, sx = (long long)F.ny * F.nz;
    const int bx = x << 1, by = y << 1, bz = z << 1;
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        int a = (k >> 2) & 1, b = (k >> 1) & 1, c = k & 1;  // (0,0,0) (0,0,1) (0,1,0) ... as the reference
        long long f = (long long)(bx + a) * sx + (by + b) * sy + (bz + c);
        T res = rf[f] - ax_at<T>(F, zf, f, bx + a, by + b, bz + c);
        acc = T(double(acc) + 0.125 * double(res));
    }
    rc[i] = acc;
    zc[i] = T(0);
}

// CGSolver<3>::Prolong (PressureSolver.cpp:774-794): piecewise-constant.
template <class T>
__global__ void k_prolong(int cnx, int cny, int cnz, const T* __restrict__ zc, int fny, int fnz, T* __restrict__ zf) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)cnx * cny * cnz;
    if (i >= n) return;
    int x, y, z;
    decode(i, cny, cnz, x, y, z);
    const long long sy = fnz, sx = (long long)fny * fnz;
    const T v = zc[i];
    const long long b = (long long)(x << 1) * sx + (y << 1) * sy + (z << 1);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        long long f = b + ((k >> 2) & 1) * sx + ((k >> 1) & 1) * sy + (k & 1);
        zf[f] = zf[f] + v;
    }
}

template <class T> __global__ void k_precond_none(long long n, const uint8_t* __restrict__ type, const T* __restrict__ r, T* __restrict__ z) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && type[i] != 0) z[i] = r[i];
}
template <class T> __global__ void k_precond_jacobi(long long n, const T* __restrict__ diag, const T* __restrict__ r, T* __restrict__ z) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T d = diag[i];
    if (!is_small(d)) z[i] = r[i] / d;
}

// ---------------------------------------------------------------- PCG
// r0 = rhs on fluid cells (PressureSolver.cpp:847-856)
template <class T> __global__ void k_init_r(long long n, const uint8_t* __restrict__ type, const T* __restrict__ rhs, T* __restrict__ r) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && type[i] != 0) r[i] = rhs[i];
}

// p = z on fluid cells; rz_old = r.z, rr_all = r.r over all cells
// (PressureSolver.cpp:858-868)
template <class T>
__global__ void k_init_p(long long n, const uint8_t* __restrict__ type, const T* __restrict__ r, const T* __restrict__ z,
                         T* __restrict__ p, double* __restrict__ partials, unsigned* __restrict__ counter,
                         SolveScalars* __restrict__ sc) {
    double v[2] = {0.0, 0.0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        T zi = z[i], ri = r[i];
        if (type[i] != 0) p[i] = zi;
        v[0] += double(ri) * double(zi);
        v[1] += double(ri) * double(ri);
    }
    grid_sum_finish<2>(v, partials, counter, &sc->pad[1]);
}

// Ap = A p; denom = sum p.Ap over interior fluid cells; alpha = rz_old/denom
// (PressureSolver.cpp:873-883)
template <class T, class TX>
__global__ void __launch_bounds__(256) k_spmv_dot(LevelK<T> L, int region, const T* __restrict__ p, T* __restrict__ ap,
                                                  double* __restrict__ partials, unsigned* __restrict__ counter,
                                                  SolveScalars* __restrict__ sc) {
    double v[1] = {0.0};
    long long n = (long long)L.nx * L.ny * L.nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        decode(i, L.ny, L.nz, x, y, z);
        T a = ax_at<T>(L, p, i, x, y, z);
        ap[i] = a;
        if (L.type[i] != 0 && in_region(x, y, z, L.nx, L.ny, L.nz, region)) v[0] += double(p[i]) * double(a);
    }
    grid_sum_finish<1>(v, partials, counter, &sc->pad[1]);
}

// x += alpha p; r -= alpha Ap; res2 = sum r^2 on interior fluid cells
// (PressureSolver.cpp:889-902)
template <class T, class TX>
__global__ void __launch_bounds__(256) k_update_xr(LevelK<T> L, int region, const T* __restrict__ p, const T* __restrict__ ap,
                                                   TX* __restrict__ x, T* __restrict__ r, double* __restrict__ partials,
                                                   unsigned* __restrict__ counter, SolveScalars* __restrict__ sc) {
    const double alpha = sc->rz_old / sc->denom;
    double v[1] = {0.0};
    long long n = (long long)L.nx * L.ny * L.nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int xi, yi, zi;
        decode(i, L.ny, L.nz, xi, yi, zi);
        if (L.type[i] == 0 || !in_region(xi, yi, zi, L.nx, L.ny, L.nz, region)) continue;
        x[i] = TX(double(x[i]) + alpha * double(p[i]));
        T rn = T(double(r[i]) - alpha * double(ap[i]));
        r[i] = rn;
        v[0] += double(rn) * double(rn);
    }
    grid_sum_finish<1>(v, partials, counter, &sc->pad[1]);
}

// r = b - A x on interior fluid cells (optionally stored), sum of squares
template <class T, class TX>
__global__ void __launch_bounds__(256) k_true_residual(LevelK<T> L, int region, const T* __restrict__ b, const TX* __restrict__ x,
                                                       T* __restrict__ r, int store, double* __restrict__ partials,
                                                       unsigned* __restrict__ counter, double* __restrict__ out) {
    double v[1] = {0.0};
    long long n = (long long)L.nx * L.ny * L.nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int xi, yi, zi;
        decode(i, L.ny, L.nz, xi, yi, zi);
        if (L.type[i] == 0 || !in_region(xi, yi, zi, L.nx, L.ny, L.nz, region)) continue;
        double res = double(b[i]) - ax_at<double>(L, x, i, xi, yi, zi);
        if (store) r[i] = T(res);
        v[0] += res * res;
    }
    grid_sum_finish<1>(v, partials, counter, out);
}

// rz_new = r.z over all cells (Array3::Reduce); apz = Ap.z over interior fluid
template <class T>
__global__ void __launch_bounds__(256) k_dot_rz(LevelK<T> L, int region, const T* __restrict__ r, const T* __restrict__ z,
                                                const T* __restrict__ ap, double* __restrict__ partials,
                                                unsigned* __restrict__ counter, double* __restrict__ out) {
    double v[2] = {0.0, 0.0};
    long long n = (long long)L.nx * L.ny * L.nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        T zi = z[i];
        v[0] += double(r[i]) * double(zi);
        int xi, yi, zz;
        decode(i, L.ny, L.nz, xi, yi, zz);
        if (L.type[i] != 0 && in_region(xi, yi, zz, L.nx, L.ny, L.nz, region)) v[1] += double(ap[i]) * double(zi);
    }
    grid_sum_finish<2>(v, partials, counter, out);
}

// p = z + beta p on fluid cells (PressureSolver.cpp:913-921)
template <class T>
__global__ void k_update_p(long long n, const uint8_t* __restrict__ type, const T* __restrict__ z, T* __restrict__ p,
                           const SolveScalars* __restrict__ sc) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || type[i] == 0) return;
    const double beta = sc->pad[0];
    p[i] = T(double(z[i]) + beta * double(p[i]));
}

// single-thread scalar bookkeeping between kernels
__global__ void k_scalars_after_init(SolveScalars* sc) {
    sc->rz_old = sc->pad[1];
    sc->rr_all = sc->pad[2];
}
__global__ void k_scalars_alpha(SolveScalars* sc) { sc->denom = sc->pad[1]; }
__global__ void k_scalars_res(SolveScalars* sc) { sc->res2 = sc->pad[1]; }
__global__ void k_scalars_beta(SolveScalars* sc, int flexible) {
    double rz_new = sc->pad[1], apz = sc->pad[2];
    double alpha = sc->rz_old / sc->denom;
    double beta = flexible ? (-alpha * apz / sc->rz_old) : (rz_new / sc->rz_old);
    sc->rz_new = rz_new;
    sc->apz = apz;
    sc->pad[0] = beta;
    sc->rz_old = rz_new;
}

template <class T, class TX> __global__ void k_x_to_pressure(long long n, const TX* __restrict__ x, T* __restrict__ pr) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pr[i] = T(x[i]);
}

template <class T>
__global__ void k_get_ax(LevelK<T> L, const T* __restrict__ x, T* __restrict__ out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)L.nx * L.ny * L.nz;
    if (i >= n) return;
    int xi, yi, zi;
    decode(i, L.ny, L.nz, xi, yi, zi);
    out[i] = ax_at<T>(L, x, i, xi, yi, zi);
}

// m_Acoef[level] expanded to 6 per cell: right, left, top, bottom, front, back
template <class T> __global__ void k_expand_acoef(LevelK<T> L, T* __restrict__ out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)L.nx * L.ny * L.nz;
    if (i >= n) return;
    int x, y, z;
    decode(i, L.ny, L.nz, x, y, z);
    const long long sy = L.nz, sx = (long long)L.ny * L.nz;
    T c[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    if (L.type[i] != 0) {
        if (x + 1 < L.nx && L.type[i + sx] == 2) c[0] = L.cx[i];
        if (x - 1 >= 0 && L.type[i - sx] == 2) c[1] = L.cx[i - sx];
        if (y + 1 < L.ny && L.type[i + sy] == 2) c[2] = L.cy[i];
        if (y - 1 >= 0 && L.type[i - sy] == 2) c[3] = L.cy[i - sy];
        if (z + 1 < L.nz && L.type[i + 1] == 2) c[4] = L.cz[i];
        if (z - 1 >= 0 && L.type[i - 1] == 2) c[5] = L.cz[i - 1];
    }
    for (int k = 0; k < 6; ++k) out[6 * i + k] = c[k];
}

constexpr long long kBlockSmoothMax = 4096;

}  // namespace

// ------------------------------------------------------------- host side
template <class T, class TX> double LiquidImpl<T, TX>::read_scalar(const double* dptr) {
    double v;
    LHI_CUDA(cudaMemcpyAsync(&v, dptr, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    LHI_CUDA(cudaStreamSynchronize(stream_));
    return v;
}

template <class T, class TX> void LiquidImpl<T, TX>::read_scalars() {
    LHI_CUDA(cudaMemcpyAsync(sc_host_, sc_, sizeof(SolveScalars), cudaMemcpyDeviceToHost, stream_));
    LHI_CUDA(cudaStreamSynchronize(stream_));
}

// CGSolver<3>::Init (PressureSolver.cpp:666-680)
template <class T, class TX> void LiquidImpl<T, TX>::solver_init() {
    LHI_CUDA(cudaMemsetAsync(p_, 0, sizeof(T) * ncell_, stream_));
    LHI_CUDA(cudaMemsetAsync(x_, 0, sizeof(TX) * ncell_, stream_));
    LHI_CUDA(cudaMemsetAsync(rhs_, 0, sizeof(T) * ncell_, stream_));
    for (int l = 0; l < nlev_; ++l) {
        LevelDev<T>& L = lv_[l];
        if (L.n == 0) continue;
        LHI_CUDA(cudaMemsetAsync(L.r, 0, sizeof(T) * L.n, stream_));
        LHI_CUDA(cudaMemsetAsync(L.z, 0, sizeof(T) * L.n, stream_));
        LHI_CUDA(cudaMemsetAsync(L.diag, 0, sizeof(T) * L.n, stream_));
        for (int a = 0; a < 3; ++a) LHI_CUDA(cudaMemsetAsync(L.cf[a], 0, sizeof(T) * L.n, stream_));
    }
    LHI_CUDA(cudaMemsetAsync(sc_, 0, sizeof(SolveScalars), stream_));
}

template <class T, class TX> void LiquidImpl<T, TX>::build_rhs() {
    auto ps_ = scope(LHI_KERNEL_GRID);
    k_build_rhs<T><<<blocks_for(ncell_, 256), 256, 0, stream_>>>(nx_, ny_, nz_, dx_[0], dx_[1], dx_[2], liquid_phi_,
                                                                 lw_[0], lw_[1], lw_[2], v_[0], v_[1], v_[2], rhs_);
    LHI_LAUNCH_CHECK();
}

template <class T, class TX> void LiquidImpl<T, TX>::build_lhs(double rho, double dt) {
    auto ps_ = scope(LHI_KERNEL_LHS);
    for (int l = 0; l < nlev_; ++l) {
        LevelDev<T>& L = lv_[l];
        if (L.n == 0) continue;
        LevelGeom g{L.nx, L.ny, L.nz, nx_, ny_, nz_, l};
        k_level_phi<T><<<blocks_for(L.n, 256), 256, 0, stream_>>>(g, liquid_phi_, L.phi, L.type);
        LHI_LAUNCH_CHECK();
        const T* phi = (l == 0) ? liquid_phi_ : L.phi;
        k_level_matrix<T><<<blocks_for(L.n, 256), 256, 0, stream_>>>(g, phi, lw_[0], lw_[1], lw_[2], L.h[0], L.h[1],
                                                                     L.h[2], T(dt), T(rho), L.diag, L.cf[0],
                                                                     L.cf[1], L.cf[2]);
        LHI_LAUNCH_CHECK();
    }
}

template <class T, class TX> void LiquidImpl<T, TX>::smooth(int level, int sweeps) {
    LevelDev<T>& L = lv_[level];
    if (L.n == 0 || sweeps <= 0) return;
    T w = T(sp_.smoothing_factor);
    const int cat = (level == 0) ? LHI_KERNEL_SMOOTH_FINE : LHI_KERNEL_SMOOTH_COARSE;
    if (L.n <= kBlockSmoothMax) {
        auto ps_ = scope(cat);
        k_smooth_block<T><<<1, 1024, 0, stream_>>>(lk(L), L.r, L.z, w, sp_.smoother, sweeps);
        LHI_LAUNCH_CHECK();
        return;
    }
    for (int s = 0; s < sweeps; ++s)
        for (int phase = 0; phase < 2; ++phase) {
            auto ps_ = scope(cat);
            k_smooth<T><<<blocks_for(L.n, 256), 256, 0, stream_>>>(lk(L), L.r, L.z, w, sp_.smoother, phase);
            LHI_LAUNCH_CHECK();
        }
}

template <class T, class TX> void LiquidImpl<T, TX>::restrict_to(int level) {
    LevelDev<T>& C = lv_[level];
    LevelDev<T>& F = lv_[level - 1];
    if (C.n == 0) return;
    auto ps_ = scope(LHI_KERNEL_RESTRICT);
    k_restrict<T><<<blocks_for(C.n, 256), 256, 0, stream_>>>(lk(F), F.r, F.z, C.nx, C.ny, C.nz, C.r, C.z);
    LHI_LAUNCH_CHECK();
}

template <class T, class TX> void LiquidImpl<T, TX>::prolong_to(int level) {
    LevelDev<T>& C = lv_[level + 1];
    LevelDev<T>& F = lv_[level];
    if (C.n == 0) return;
    auto ps_ = scope(LHI_KERNEL_PROLONG);
    k_prolong<T><<<blocks_for(C.n, 256), 256, 0, stream_>>>(C.nx, C.ny, C.nz, C.z, F.ny, F.nz, F.z);
    LHI_LAUNCH_CHECK();
}

template <class T, class TX> void LiquidImpl<T, TX>::vcycle() {
    for (int l = 1; l < nlev_; ++l) {
        smooth(l - 1, sp_.num_pre_smooth);
        restrict_to(l);
    }
    smooth(nlev_ - 1, sp_.num_final_smooth);
    for (int l = nlev_ - 2; l >= 0; --l) {
        prolong_to(l);
        smooth(l, sp_.num_post_smooth);
    }
}

// CGSolver<3>::ApplyPreconditioner (PressureSolver.cpp:719-772)
template <class T, class TX> void LiquidImpl<T, TX>::apply_preconditioner() {
    LevelDev<T>& L0 = lv_[0];
    switch (sp_.preconditioner) {
        case LHI_PRECOND_NONE:
            k_precond_none<T><<<blocks_for(ncell_, 256), 256, 0, stream_>>>(ncell_, L0.type, L0.r, L0.z);
            LHI_LAUNCH_CHECK();
            break;
        case LHI_PRECOND_JACOBI:
            k_precond_jacobi<T><<<blocks_for(ncell_, 256), 256, 0, stream_>>>(ncell_, L0.diag, L0.r, L0.z);
            LHI_LAUNCH_CHECK();
            break;
        default: vcycle();
    }
}

template <class T, class TX> void LiquidImpl<T, TX>::spmv(int level, const T* x, T* y) {
    LevelDev<T>& L = lv_[level];
    if (L.n == 0) return;
    k_get_ax<T><<<blocks_for(L.n, 256), 256, 0, stream_>>>(lk(L), x, y);
    LHI_LAUNCH_CHECK();
}

// CGSolver<3>::Solve (PressureSolver.cpp:839-934)
template <class T, class TX> int LiquidImpl<T, TX>::solve(double rho, double dt) {
    LHI_CUDA(cudaEventRecord(ev0_, stream_));
    solver_init();
    build_rhs();
    build_lhs(rho, dt);
    LevelDev<T>& L0 = lv_[0];
    const LevelK<T> K0 = lk(L0);
    const unsigned nb = std::min<unsigned>(blocks_for(ncell_, 256), unsigned(sum_blocks_));
    {
        auto ps_ = scope(LHI_KERNEL_CG_VECTOR);
        k_init_r<T><<<blocks_for(ncell_, 256), 256, 0, stream_>>>(ncell_, L0.type, rhs_, L0.r);
        LHI_LAUNCH_CHECK();
    }
    apply_preconditioner();
    {
        auto ps_ = scope(LHI_KERNEL_CG_VECTOR);
        k_init_p<T><<<nb, 256, 0, stream_>>>(ncell_, L0.type, L0.r, L0.z, p_, partials_, counter_, sc_);
        LHI_LAUNCH_CHECK();
        k_scalars_after_init<<<1, 1, 0, stream_>>>(sc_);
        LHI_LAUNCH_CHECK();
    }
    read_scalars();
    const double residual0 = std::sqrt(sc_host_->rr_all);
    double residual = residual0;
    const T tol = T(sp_.tolerance);
    const double threshold =
        (sp_.tolerance_mode == LHI_TOL_RELATIVE) ? double(T(tol * T(residual0))) : double(tol);
    const bool flexible = sp_.cg_variant == LHI_CG_FLEXIBLE;
    const int region = sp_.update_region;
    const int every = sp_.true_residual_every;
    int iters = 0;
    bool converged = false;
    for (int it = 0; it < sp_.max_iterations; ++it) {
        if (residual < threshold) {
            if (every > 0 && iters > 0) {  // final check on the true residual
                {
                    auto ps_ = scope(LHI_KERNEL_CG_VECTOR);
                    k_true_residual<T, TX><<<nb, 256, 0, stream_>>>(K0, region, rhs_, x_, L0.r, 1, partials_,
                                                                    counter_, &sc_->pad[1]);
                    LHI_LAUNCH_CHECK();
                    k_scalars_res<<<1, 1, 0, stream_>>>(sc_);
                    LHI_LAUNCH_CHECK();
                }
                read_scalars();
                residual = std::sqrt(sc_host_->res2);
                if (residual < threshold) {
                    converged = true;
                    break;
                }
            } else {
                converged = true;
                break;
            }
        }
        {
            auto ps_ = scope(LHI_KERNEL_SPMV);
            k_spmv_dot<T, TX><<<nb, 256, 0, stream_>>>(K0, region, p_, ap_, partials_, counter_, sc_);
            LHI_LAUNCH_CHECK();
        }
        {
            auto ps_ = scope(LHI_KERNEL_CG_VECTOR);
            k_scalars_alpha<<<1, 1, 0, stream_>>>(sc_);
            LHI_LAUNCH_CHECK();
            k_update_xr<T, TX><<<nb, 256, 0, stream_>>>(K0, region, p_, ap_, x_, L0.r, partials_, counter_, sc_);
            LHI_LAUNCH_CHECK();
            k_scalars_res<<<1, 1, 0, stream_>>>(sc_);
            LHI_LAUNCH_CHECK();
        }
        ++iters;
        if (every > 0 && iters % every == 0) {
            auto ps_ = scope(LHI_KERNEL_CG_VECTOR);
            k_true_residual<T, TX><<<nb, 256, 0, stream_>>>(K0, region, rhs_, x_, L0.r, 1, partials_, counter_,
                                                            &sc_->pad[1]);
            LHI_LAUNCH_CHECK();
            k_scalars_res<<<1, 1, 0, stream_>>>(sc_);
            LHI_LAUNCH_CHECK();
        }
        apply_preconditioner();
        {
            auto ps_ = scope(LHI_KERNEL_CG_VECTOR);
            k_dot_rz<T><<<nb, 256, 0, stream_>>>(K0, region, L0.r, L0.z, ap_, partials_, counter_, &sc_->pad[1]);
            LHI_LAUNCH_CHECK();
            k_scalars_beta<<<1, 1, 0, stream_>>>(sc_, flexible ? 1 : 0);
            LHI_LAUNCH_CHECK();
            k_update_p<T><<<blocks_for(ncell_, 256), 256, 0, stream_>>>(ncell_, L0.type, L0.z, p_, sc_);
            LHI_LAUNCH_CHECK();
        }
        read_scalars();
        residual = std::sqrt(sc_host_->res2);
        if (!std::isfinite(residual)) break;
    }
    if (!converged && residual < threshold) converged = true;
    {
        auto ps_ = scope(LHI_KERNEL_CG_VECTOR);
        k_x_to_pressure<T, TX><<<blocks_for(ncell_, 256), 256, 0, stream_>>>(ncell_, x_, pressure_);
        LHI_LAUNCH_CHECK();
        k_true_residual<T, TX><<<nb, 256, 0, stream_>>>(K0, region, rhs_, x_, L0.r, 0, partials_, counter_,
                                                        &sc_->true2);
        LHI_LAUNCH_CHECK();
    }
    LHI_CUDA(cudaEventRecord(ev1_, stream_));
    read_scalars();
    float ms = 0.f;
    LHI_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    stats_.iterations = iters;
    stats_.initial_residual = residual0;
    stats_.final_residual = residual;
    stats_.true_residual = std::sqrt(sc_host_->true2);
    stats_.solve_ms = ms;
    stats_.status = !std::isfinite(residual) ? LHI_E_NAN : (converged ? LHI_OK : LHI_E_NOT_CONVERGED);
    return stats_.status;
}

template <class T, class TX> void LiquidImpl<T, TX>::get_ax(int level, const void* x, void* out) {
    if (level < 0 || level >= nlev_) throw std::invalid_argument("bad level");
    LevelDev<T>& L = lv_[level];
    if (L.n == 0) return;
    T *dx = nullptr, *dy = nullptr;
    LHI_CUDA(cudaMalloc(&dx, sizeof(T) * L.n));
    LHI_CUDA(cudaMalloc(&dy, sizeof(T) * L.n));
    LHI_CUDA(cudaMemcpyAsync(dx, x, sizeof(T) * L.n, cudaMemcpyHostToDevice, stream_));
    spmv(level, dx, dy);
    LHI_CUDA(cudaMemcpyAsync(out, dy, sizeof(T) * L.n, cudaMemcpyDeviceToHost, stream_));
    LHI_CUDA(cudaStreamSynchronize(stream_));
    cudaFree(dx);
    cudaFree(dy);
}

template <class T, class TX> void LiquidImpl<T, TX>::get_acoef(int level, T* host_out) {
    LevelDev<T>& L = lv_[level];
    if (L.n == 0) return;
    T* d = nullptr;
    LHI_CUDA(cudaMalloc(&d, sizeof(T) * 6 * L.n));
    k_expand_acoef<T><<<blocks_for(L.n, 256), 256, 0, stream_>>>(lk(L), d);
    LHI_LAUNCH_CHECK();
    LHI_CUDA(cudaMemcpyAsync(host_out, d, sizeof(T) * 6 * L.n, cudaMemcpyDeviceToHost, stream_));
    LHI_CUDA(cudaStreamSynchronize(stream_));
    cudaFree(d);
}

template class LiquidImpl<float, float>;
template class LiquidImpl<float, double>;
template class LiquidImpl<double, double>;

}  // namespace lhi
