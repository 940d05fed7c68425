// k_solver.cu -- CGSolver<3> on the device: per-level ghost-fluid matrix
// assembly, SpMV, damped red-black Gauss-Seidel, restriction/prolongation,
// the V-cycle preconditioner and the PCG loop, which runs on the device.
//
// Matrix storage: per level, diag plus one coefficient per +x/+y/+z face and
// a cell type byte (0: phi > 0, 1: phi == 0, 2: phi < 0).  The reference's
// per-row coefficient (PressureSolver.cpp:556-662) is -term when the
// neighbour has phi < 0 and 0 otherwise, and rows with phi > 0 are empty; the
// face term is the same expression seen from both rows, so
//   A(i, j) = [type_i >= 1] [type_j == 2] * face_coef(i, j).
//
// Sparsity: rows with phi > 0 are empty, so every sweep visits only the
// level's active 8 x 8 x 32 tiles (cells with phi <= 0, plus tiles covering
// an active finer tile so that restricted residuals are carried down).  Cells
// outside active tiles are air cells whose values no row ever reads.
//
// Levels below the finest with at most coarse_cells cells (default 16^3)
// are solved by one CTA in one launch, staged in shared memory: their
// pre-smoothing, restriction, coarsest sweeps, prolongation, post-smoothing.
//
// The PCG loop keeps every scalar on the device.  By default one solve is
// one CUDA graph: the initial V-cycle, then a conditional while node whose
// body is one PCG iteration; the kernel that applies the stopping rule sets
// the loop condition.  With eager = 1 the host drives the same kernels and
// reads the stop flag after every iteration.
#include <algorithm>
#include <random>
#include <string>
#include <type_traits>

#include "impl.cuh"
#include "layouts.cuh"

namespace lhi {

namespace {

constexpr int kGraphIterationCap = 100000;  // hard stop of the device-side loop

// Limit of the solver kernels' waits on their TMA staging copies (200 ms;
// lhi_debug_set_stage_wait_limit lowers it to test the timeout path).  On
// a timeout a CTA records it, waits (200 ms at most) for every copy of its
// own still in flight, and leaves.
__device__ unsigned long long g_stage_wait_ns = kWaitLimitNs;

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

// the mixed mode's FP64 finest-level matrix with the level's cell types
template <class T, class TX> LevelK<double> lk_hi(const LiquidImpl<T, TX>& s) {
    const LevelDev<T>& L = s.lv_[0];
    return LevelK<double>{L.nx, L.ny, L.nz, s.diag_hi_, s.cf_hi_[0], s.cf_hi_[1], s.cf_hi_[2], L.type};
}

__device__ __forceinline__ void decode(long long i, int ny, int nz, int& x, int& y, int& z) { idx3(i, ny, nz, x, y, z); }

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

// The 7-point row of one cell, loaded without data-dependent branches so a
// thread can put the loads of several cells in flight before any arithmetic.
// Out-of-range neighbours read the cell itself and are masked by `in`.
template <class T, class V> struct Cell7 {
    V zc, zn[6];
    T d, cf[6];
    unsigned m;  // bit k: neighbour k exists and has phi < 0
    uint8_t tc;
};

template <class T, class V>
__device__ __forceinline__ void load7(const LevelK<T>& L, const V* __restrict__ x, long long i, int xi, int yi, int zi,
                                      Cell7<T, V>& s) {
    const long long sy = L.nz, sx = (long long)L.ny * L.nz;
    const bool in[6] = {xi + 1 < L.nx, xi > 0, yi + 1 < L.ny, yi > 0, zi + 1 < L.nz, zi > 0};
    const long long j[6] = {in[0] ? i + sx : i, in[1] ? i - sx : i, in[2] ? i + sy : i,
                            in[3] ? i - sy : i, in[4] ? i + 1 : i,  in[5] ? i - 1 : i};
    s.tc = L.type[i];
    s.d = L.diag[i];
    s.zc = x[i];
    uint8_t tn[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        tn[k] = L.type[j[k]];
        s.zn[k] = x[j[k]];
    }
    s.cf[0] = L.cx[i];
    s.cf[1] = L.cx[j[1]];
    s.cf[2] = L.cy[i];
    s.cf[3] = L.cy[j[3]];
    s.cf[4] = L.cz[i];
    s.cf[5] = L.cz[j[5]];
    unsigned m = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) m |= (in[k] && tn[k] == 2) ? (1u << k) : 0u;
    s.m = m;
}

// ax_at on a loaded row: same terms in the same order (+x, -x, +y, -y, +z, -z)
template <class C, class T, class V> __device__ __forceinline__ C ax7(const Cell7<T, V>& s) {
    if (s.tc == 0) return C(0);
    C r = C(s.zc) * C(s.d);
#pragma unroll
    for (int k = 0; k < 6; ++k)
        if (s.m & (1u << k)) r += C(s.zn[k]) * C(s.cf[k]);
    return r;
}

// CGSolver<3>::Smooth update of one cell from its loaded row (PressureSolver.cpp:830-834)
template <class T>
__device__ __forceinline__ bool smooth7(const Cell7<T, T>& s, T rv, T w, int variant, T& out) {
    if (is_small(s.d)) return false;
    const T term = (rv - ax7<T>(s)) / s.d;
    if (variant == LHI_SMOOTHER_DAMPED_GS) out = s.zc + w * term;
    else out = T((1.0 - double(w)) * double(s.zc) + double(T(w * term)));
    return true;
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

// Also marks the level's tile of every cell with phi <= 0 as active.
template <class T>
__global__ void k_level_phi(LevelGeom g, const T* __restrict__ fine_phi, T* __restrict__ phi, uint8_t* __restrict__ type,
                            uint8_t* __restrict__ tile_flag, int tdy, int tdz) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)g.nx * g.ny * g.nz;
    if (i >= n) return;
    int x, y, z;
    decode(i, g.ny, g.nz, x, y, z);
    T ph = approx_phi(fine_phi, g, x, y, z);
    if (g.level > 0) phi[i] = ph;
    const uint8_t t = (ph > T(0)) ? 0 : ((ph < T(0)) ? 2 : 1);
    type[i] = t;
    if (t != 0) tile_flag[((long long)(x / kTileX) * tdy + y / kTileY) * tdz + z / kTileZ] = 1;
}

// CGSolver<3>::BuildLHS for one level (PressureSolver.cpp:544-664), in T
// from fields of type TI (TI = float, T = double: the FP64 finest-level
// matrix the mixed mode's outer residual uses).
template <class T, class TI = T>
__device__ __forceinline__ void level_matrix_cell(long long i, LevelGeom g, const TI* __restrict__ phi,
                                                  const TI* __restrict__ lwx, const TI* __restrict__ lwy,
                                                  const TI* __restrict__ lwz, T h0, T h1, T h2, T dt, T rho,
                                                  T* __restrict__ diag, T* __restrict__ cx, T* __restrict__ cy,
                                                  T* __restrict__ cz, uint8_t* __restrict__ type,
                                                  uint8_t* __restrict__ tile_flag, int tdy, int tdz,
                                                  uint8_t* __restrict__ mask, int mpitch) {
    // the FP64 copy is read only on rows with phi <= 0 (and their fluid
    // neighbours): air cells need no entries
    if constexpr (!std::is_same<T, TI>::value)
        if (T(phi[i]) > T(0)) return;
    int x, y, z;
    decode(i, g.ny, g.nz, x, y, z);
    const long long sy = g.nz, sx = (long long)g.ny * g.nz;
    const TI* lw[3] = {lwx, lwy, lwz};
    const T hh[3] = {h0, h1, h2};
    auto term_of = [&](int a, T w) -> T {
        return X<T>::div(X<T>::mul(w, dt), X<T>::mul(X<T>::mul(rho, hh[a]), hh[a]));
    };
    // The six faces (right, left, top, bottom, front, back) and the
    // neighbours' phi, loaded up front so the loads overlap; each face's term
    // w dt / (rho h^2) is formed once (the +x/+y/+z terms serve both this
    // cell's couplings and its diagonal), in the reference's arithmetic.
    const int xs[6] = {x + 1, x, x, x, x, x};
    const int ys[6] = {y, y, y + 1, y, y, y};
    const int zs[6] = {z, z, z, z, z + 1, z};
    const int ax[6] = {0, 0, 1, 1, 2, 2};
    const long long off[6] = {sx, -sx, sy, -sy, 1, -1};
    const bool exists[6] = {x + 1 < g.nx, x - 1 >= 0, y + 1 < g.ny, y - 1 >= 0, z + 1 < g.nz, z - 1 >= 0};
    const T center = T(phi[i]);
    const bool row = !(center > T(0));
    T w6[6], nphi6[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        w6[k] = exists[k] ? T(approx_w(lw[ax[k]], g, ax[k], xs[k], ys[k], zs[k])) : T(0);
        nphi6[k] = exists[k] ? T(phi[i + off[k]]) : T(0);
    }
    T term6[6];
#pragma unroll
    for (int k = 0; k < 6; ++k)  // the -x/-y/-z terms only for a row of the matrix
        term6[k] = (w6[k] > T(0) && ((k & 1) == 0 || row)) ? term_of(ax[k], w6[k]) : T(0);
    // own +x/+y/+z face coefficients
    cx[i] = (w6[0] > T(0)) ? -term6[0] : T(0);
    cy[i] = (w6[2] > T(0)) ? -term6[2] : T(0);
    cz[i] = (w6[4] > T(0)) ? -term6[4] : T(0);
    // the finest level (type != nullptr) also classifies the cell, marks its
    // tile active (k_level_phi's work) and, where the fused sweep runs, writes
    // its neighbour mask (k_level_mask's), from the phi values at hand
    if (type) {
        const uint8_t t = (center > T(0)) ? 0 : ((center < T(0)) ? 2 : 1);
        type[i] = t;
        if (t != 0) tile_flag[((long long)(x / kTileX) * tdy + y / kTileY) * tdz + z / kTileZ] = 1;
        if (mask) {
            unsigned m = t != 0 ? 64u : 0u;
#pragma unroll
            for (int k = 0; k < 6; ++k)
                if (exists[k] && nphi6[k] < T(0)) m |= 1u << k;  // right, left, top, bottom, front, back
            mask[((long long)x * g.ny + y) * mpitch + z] = uint8_t(m);
        }
    }
    T d = T(0);
    if (row) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            if (!exists[k] || !(w6[k] > T(0))) continue;
            const T term = term6[k];
            const T nphi = nphi6[k];
            if (nphi < T(0)) d = X<T>::add(d, term);
            else d = X<T>::add(d, X<T>::div(term, frac_floor(fraction_in_region(center, nphi))));
        }
    }
    diag[i] = d;
}

template <class T, class TI = T>
__global__ void k_level_matrix(LevelGeom g, const TI* __restrict__ phi, const TI* __restrict__ lwx,
                               const TI* __restrict__ lwy, const TI* __restrict__ lwz, T h0, T h1, T h2, T dt, T rho,
                               T* __restrict__ diag, T* __restrict__ cx, T* __restrict__ cy, T* __restrict__ cz,
                               uint8_t* __restrict__ type, uint8_t* __restrict__ tile_flag, int tdy, int tdz,
                               uint8_t* __restrict__ mask, int mpitch) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)g.nx * g.ny * g.nz) return;
    level_matrix_cell<T, TI>(i, g, phi, lwx, lwy, lwz, h0, h1, h2, dt, rho, diag, cx, cy, cz, type, tile_flag, tdy,
                             tdz, mask, mpitch);
}

// The mixed mode's finest level: the FP32 matrix (with the cell classes,
// tile flags and neighbour mask) and the FP64 matrix of the outer residual
// from one read of the fields, each in its own arithmetic (the same bits as
// two k_level_matrix launches).
template <class T>
__global__ void k_level_matrix_mixed(LevelGeom g, const T* __restrict__ phi, const T* __restrict__ lwx,
                                     const T* __restrict__ lwy, const T* __restrict__ lwz, T h0, T h1, T h2, T dt,
                                     T rho, T* __restrict__ diag, T* __restrict__ cx, T* __restrict__ cy,
                                     T* __restrict__ cz, uint8_t* __restrict__ type, uint8_t* __restrict__ tile_flag,
                                     int tdy, int tdz, uint8_t* __restrict__ mask, int mpitch, double hd0, double hd1,
                                     double hd2, double dtd, double rhod, double* __restrict__ diag_hi,
                                     double* __restrict__ cx_hi, double* __restrict__ cy_hi,
                                     double* __restrict__ cz_hi) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)g.nx * g.ny * g.nz) return;
    level_matrix_cell<T, T>(i, g, phi, lwx, lwy, lwz, h0, h1, h2, dt, rho, diag, cx, cy, cz, type, tile_flag, tdy,
                            tdz, mask, mpitch);
    level_matrix_cell<double, T>(i, g, phi, lwx, lwy, lwz, hd0, hd1, hd2, dtd, rhod, diag_hi, cx_hi, cy_hi, cz_hi,
                                 nullptr, nullptr, 0, 0, nullptr, 0);
}

// Galerkin coarse level (LHI_COARSE_GALERKIN): A_c = P^T A P / 8 of the
// finer level f under the V-cycle's transfers (constant injection P, the
// 1/8 averaging restriction), with A_ij = [type_i >= 1][type_j == 2] c_ij as
// every kernel of the solver applies it.  Coarse cell I takes its 8
// children's diagonals and the couplings between them; the coupling of I
// with its +x / +y / +z neighbour is the sum over the 4 child pairs across
// that face.  type_I = 2 if a child is fluid, else 1 if a child has phi = 0.
template <class T>
__global__ void k_level_galerkin(LevelK<T> F, int cnx, int cny, int cnz, T* __restrict__ diag, T* __restrict__ cx,
                                 T* __restrict__ cy, T* __restrict__ cz, uint8_t* __restrict__ type,
                                 uint8_t* __restrict__ tile_flag, int tdy, int tdz) {
    long long I = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)cnx * cny * cnz;
    if (I >= n) return;
    int X, Y, Z;
    decode(I, cny, cnz, X, Y, Z);
    const long long fsy = F.nz, fsx = (long long)F.ny * F.nz;
    auto fi = [&](int x, int y, int z) -> long long { return ((long long)x * F.ny + y) * F.nz + z; };
    // A_ij of fine cells i and its +axis neighbour j = i + step: rows couple to fluid columns only
    auto a_ij = [&](long long i, long long j, T c) -> T {
        return (F.type[i] >= 1 && F.type[j] == 2) ? c : T(0);
    };
    T d = T(0);
    uint8_t t = 0;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 2; ++c) {
                const long long i = fi(2 * X + a, 2 * Y + b, 2 * Z + c);
                const uint8_t ti = F.type[i];
                t = (ti == 2 || t == 2) ? 2 : (ti == 1 ? uint8_t(1) : t);
                if (ti >= 1) d += F.diag[i];
                // couplings inside the coarse cell, both directions
                if (a == 0) d += a_ij(i, i + fsx, F.cx[i]) + a_ij(i + fsx, i, F.cx[i]);
                if (b == 0) d += a_ij(i, i + fsy, F.cy[i]) + a_ij(i + fsy, i, F.cy[i]);
                if (c == 0) d += a_ij(i, i + 1, F.cz[i]) + a_ij(i + 1, i, F.cz[i]);
            }
    T ccx = T(0), ccy = T(0), ccz = T(0);
    for (int u = 0; u < 2; ++u)
        for (int v = 0; v < 2; ++v) {
            if (X + 1 < cnx) {
                const long long i = fi(2 * X + 1, 2 * Y + u, 2 * Z + v);
                ccx += a_ij(i, i + fsx, F.cx[i]);
            }
            if (Y + 1 < cny) {
                const long long i = fi(2 * X + u, 2 * Y + 1, 2 * Z + v);
                ccy += a_ij(i, i + fsy, F.cy[i]);
            }
            if (Z + 1 < cnz) {
                const long long i = fi(2 * X + u, 2 * Y + v, 2 * Z + 1);
                ccz += a_ij(i, i + 1, F.cz[i]);
            }
        }
    const T s = T(0.125);
    diag[I] = d * s;
    cx[I] = ccx * s;
    cy[I] = ccy * s;
    cz[I] = ccz * s;
    type[I] = t;
    if (t != 0) tile_flag[((long long)(X / kTileX) * tdy + Y / kTileY) * tdz + Z / kTileZ] = 1;
}

// CGSolver<3>::BuildRHS (PressureSolver.cpp:682-698)
// (TI = float, T = double: the FP64 right-hand side of the mixed mode's
// outer residual, from the same float fields)
template <class T, class TI = T>
__device__ __forceinline__ void build_rhs_cell(long long i, int nx, int ny, int nz, T h0, T h1, T h2,
                                               const TI* __restrict__ phi, const TI* __restrict__ lwx,
                                               const TI* __restrict__ lwy, const TI* __restrict__ lwz,
                                               const TI* __restrict__ vx, const TI* __restrict__ vy,
                                               const TI* __restrict__ vz, T* __restrict__ rhs) {
    (void)nx;
    if constexpr (!std::is_same<T, TI>::value)  // the FP64 copy is read only where phi <= 0
        if (T(phi[i]) > T(0)) return;
    T b = T(0);
    if (!(T(phi[i]) > T(0))) {
        int x, y, z;
        decode(i, ny, nz, x, y, z);
        long long fxi = ((long long)x * ny + y) * nz + z, fxs = (long long)ny * nz;
        long long fyi = ((long long)x * (ny + 1) + y) * nz + z, fys = nz;
        long long fzi = ((long long)x * ny + y) * (nz + 1) + z;
        b = X<T>::sub(b, X<T>::div(X<T>::mul(T(lwx[fxi + fxs]), T(vx[fxi + fxs])), h0));
        b = X<T>::add(b, X<T>::div(X<T>::mul(T(lwx[fxi]), T(vx[fxi])), h0));
        b = X<T>::sub(b, X<T>::div(X<T>::mul(T(lwy[fyi + fys]), T(vy[fyi + fys])), h1));
        b = X<T>::add(b, X<T>::div(X<T>::mul(T(lwy[fyi]), T(vy[fyi])), h1));
        b = X<T>::sub(b, X<T>::div(X<T>::mul(T(lwz[fzi + 1]), T(vz[fzi + 1])), h2));
        b = X<T>::add(b, X<T>::div(X<T>::mul(T(lwz[fzi]), T(vz[fzi])), h2));
    }
    rhs[i] = b;
}

template <class T, class TI = T>
__global__ void k_build_rhs(int nx, int ny, int nz, T h0, T h1, T h2, const TI* __restrict__ phi,
                            const TI* __restrict__ lwx, const TI* __restrict__ lwy, const TI* __restrict__ lwz,
                            const TI* __restrict__ vx, const TI* __restrict__ vy, const TI* __restrict__ vz,
                            T* __restrict__ rhs) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nx * ny * nz) return;
    build_rhs_cell<T, TI>(i, nx, ny, nz, h0, h1, h2, phi, lwx, lwy, lwz, vx, vy, vz, rhs);
}

// The mixed mode's two right-hand sides (FP32 for the loop, FP64 for the
// outer residual) from one read of the fields, each in its own arithmetic.
template <class T>
__global__ void k_build_rhs_mixed(int nx, int ny, int nz, T h0, T h1, T h2, double hd0, double hd1, double hd2,
                                  const T* __restrict__ phi, const T* __restrict__ lwx, const T* __restrict__ lwy,
                                  const T* __restrict__ lwz, const T* __restrict__ vx, const T* __restrict__ vy,
                                  const T* __restrict__ vz, T* __restrict__ rhs, double* __restrict__ rhs_hi) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nx * ny * nz) return;
    build_rhs_cell<T, T>(i, nx, ny, nz, h0, h1, h2, phi, lwx, lwy, lwz, vx, vy, vz, rhs);
    build_rhs_cell<double, T>(i, nx, ny, nz, hd0, hd1, hd2, phi, lwx, lwy, lwz, vx, vy, vz, rhs_hi);
}

// ------------------------------------------------------------ active tiles
struct TileK {
    const int32_t* ids;
    const int* count;
    int tdy, tdz;
    int ysplit;  // work units per tile: each takes every ysplit-th row
};

// Visits every in-grid cell of the active tiles.  A work unit is (tile, row
// subset); persistent CTAs take units blockIdx.x, blockIdx.x + gridDim.x, ...;
// warp w takes x = x0 + w and lane l takes z = z0 + l.  Small levels use
// ysplit = 8 (one row per thread) so their few tiles still fill the GPU.
template <class F> __device__ __forceinline__ void for_tiles(const TileK& tk, int nx, int ny, int nz, F&& f) {
    const int units = *tk.count * tk.ysplit;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int u = blockIdx.x; u < units; u += gridDim.x) {
        const int t = u / tk.ysplit, sub = u - t * tk.ysplit;
        const int id = tk.ids[t];
        const int tz = id % tk.tdz, rest = id / tk.tdz;
        const int ty = rest % tk.tdy, tx = rest / tk.tdy;
        const int x = tx * kTileX + w, z = tz * kTileZ + lane;
        if (x >= nx || z >= nz) continue;
        const int y0 = ty * kTileY, y1 = min(y0 + kTileY, ny);
        for (int y = y0 + sub; y < y1; y += tk.ysplit) f(x, y, z, ((long long)x * ny + y) * nz + z);
    }
}

// for_tiles with a thread's rows of a work unit handed over together:
// f(x, z, i0, rows, ys) where row k < rows is cell i0 + k * ys * nz (y
// ascending).  Kernels load every row before using any, so a thread keeps
// up to 8 rows of loads in flight; per-thread sums keep for_tiles' order.
template <class F> __device__ __forceinline__ void for_tile_cols(const TileK& tk, int nx, int ny, int nz, F&& f) {
    const int units = *tk.count * tk.ysplit;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int u = blockIdx.x; u < units; u += gridDim.x) {
        const int t = u / tk.ysplit, sub = u - t * tk.ysplit;
        const int id = tk.ids[t];
        const int tz = id % tk.tdz, rest = id / tk.tdz;
        const int ty = rest % tk.tdy, tx = rest / tk.tdy;
        const int x = tx * kTileX + w, z = tz * kTileZ + lane;
        if (x >= nx || z >= nz) continue;
        const int yb = ty * kTileY + sub, ye = min(ty * kTileY + kTileY, ny);
        const int rows = yb < ye ? (ye - yb + tk.ysplit - 1) / tk.ysplit : 0;
        f(x, z, ((long long)x * ny + yb) * nz + z, yb, rows, tk.ysplit);
    }
}

struct TileLevels {
    int nlev;
    int tdim[kMaxLevels][3];
    uint8_t* flag[kMaxLevels];
    int32_t* ids[kMaxLevels];
};

// One CTA: level l's flags |= its 2x2x2 child tiles' flags at level l - 1
// (finest first), then each level's active tiles are listed in increasing
// order (deterministic) with their count in counts[l].
__global__ void __launch_bounds__(1024) k_tiles_finalize(TileLevels tl, int* __restrict__ counts) {
    __shared__ int warp_tot[32];
    __shared__ int base;
    for (int l = 0; l < tl.nlev; ++l) {
        const int ax = tl.tdim[l][0], ay = tl.tdim[l][1], az = tl.tdim[l][2];
        const int n = ax * ay * az;
        if (l > 0) {
            const int fx = tl.tdim[l - 1][0], fy = tl.tdim[l - 1][1], fz = tl.tdim[l - 1][2];
            for (int t = threadIdx.x; t < n; t += blockDim.x) {
                const int tz = t % az, ty = (t / az) % ay, tx = t / (az * ay);
                uint8_t f = tl.flag[l][t];
                for (int c = 0; c < 8 && !f; ++c) {
                    const int cx = 2 * tx + (c >> 2), cy = 2 * ty + ((c >> 1) & 1), cz = 2 * tz + (c & 1);
                    if (cx < fx && cy < fy && cz < fz) f |= tl.flag[l - 1][(cx * fy + cy) * fz + cz];
                }
                tl.flag[l][t] = f;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) base = 0;
        __syncthreads();
        for (int c0 = 0; c0 < n; c0 += blockDim.x) {
            const int t = c0 + threadIdx.x;
            const int f = (t < n && tl.flag[l][t]) ? 1 : 0;
            const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
            const unsigned m = __ballot_sync(0xffffffffu, f);
            if (lane == 0) warp_tot[w] = __popc(m);
            __syncthreads();
            int off = 0;
            for (int k = 0; k < w; ++k) off += warp_tot[k];
            const int rank = base + off + __popc(m & ((1u << lane) - 1u));
            if (f) tl.ids[l][rank] = t;
            __syncthreads();
            if (threadIdx.x == 0) {
                int tot = 0;
                for (int k = 0; k < int(blockDim.x >> 5); ++k) tot += warp_tot[k];
                base += tot;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) counts[l] = base;
        __syncthreads();
    }
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

// One colour of one level over its active tiles.  A thread owns (x, z) of a
// tile and the 4 rows y of that colour; a work unit takes every ysplit-th of
// them.  All loads of a thread's rows are issued before any update.
template <class T>
__global__ void __launch_bounds__(kTileThreads, 2) k_sweep(LevelK<T> L, TileK tk, const T* __restrict__ r, T* __restrict__ z,
                                                        T w, int variant, int phase, const int* __restrict__ stop) {
    if (*stop) return;
    const int units = *tk.count * tk.ysplit;
    const int wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int u = blockIdx.x; u < units; u += gridDim.x) {
        const int t = u / tk.ysplit, sub = u - t * tk.ysplit;
        const int id = tk.ids[t];
        const int tz = id % tk.tdz, rest = id / tk.tdz;
        const int ty = rest % tk.tdy, tx = rest / tk.tdy;
        const int x = tx * kTileX + wp, zz = tz * kTileZ + lane;
        if (x >= L.nx || zz >= L.nz) continue;
        const int y0 = ty * kTileY;
        const int yf = y0 + ((phase + x + zz + y0) & 1);
        Cell7<T, T> c[4];
        T rv[4];
        bool act[4];
        long long idx[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int y = yf + 2 * k;
            act[k] = (k % tk.ysplit == sub) && y < L.ny;
            if (act[k]) {
                idx[k] = ((long long)x * L.ny + y) * L.nz + zz;
                load7(L, z, idx[k], x, y, zz, c[k]);
                rv[k] = r[idx[k]];
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            T out;
            if (act[k] && smooth7(c[k], rv[k], w, variant, out)) z[idx[k]] = out;
        }
    }
}

// ------------------------------------------------- fused red-black sweep
// One damped red-black Gauss-Seidel sweep (both colours) of an FP32 level in
// one pass.  A CTA takes an active 8 x 8 x 32 tile T and stages by TMA:
//   Z  (z_in)    T grown by 2 cells in x and y, z from z0-4: 12 x 12 x 40
//   R, D, CZ     T grown by 1 in x and y:                    10 x 10 x 40
//   CX           as R with x from x0-2:                      11 x 10 x 40
//   CY           as R with y from y0-2:                      10 x 11 x 40
//   M (bytes)    T grown by 1, z from z0-16:                 10 x 10 x 64
// It updates colour 0 on T grown by one cell (the ring recomputes exactly
// what the neighbouring tiles compute), then colour 1 on T, in place in
// shared memory, and writes T to z_out.  Reading z_in and writing z_out
// keeps the neighbours' halo reads on the old values.  Each cell's update is
// the arithmetic of smooth7 in the same order, so the values equal those of
// two k_sweep launches.  Cells outside the grid read diag 0 and are skipped.
namespace rb {
constexpr int kZW = layout::kZW;
constexpr int kZ = layout::kZBox;
constexpr int kR = layout::kRBox;
constexpr int kC = layout::kCBox;
constexpr int kMW = layout::kMW;
constexpr int kM = layout::kMBox;
constexpr uint32_t kTx = uint32_t((kZ + 3 * kR + 2 * kC) * 4 + kM);  // bytes the 7 boxes deliver
constexpr int al(int b) { return (b + 127) & ~127; }
// offsets inside one stage
constexpr int oZ = 0;
constexpr int oR = oZ + al(kZ * 4);
constexpr int oD = oR + al(kR * 4);
constexpr int oCZ = oD + al(kR * 4);
constexpr int oCX = oCZ + al(kR * 4);
constexpr int oCY = oCX + al(kC * 4);
constexpr int oM = oCY + al(kC * 4);
constexpr int kStage = oM + al(kM);
constexpr int kBase = 128;  // two mbarriers, then two stages
constexpr int kSmem = kBase + 2 * kStage;
constexpr int kThreads = 512;
}  // namespace rb

// Mask bits of a cell: 0..5 neighbour +x, -x, +y, -y, +z, -z exists with phi < 0;
// 6: the cell's own type is not 0.
__device__ __forceinline__ bool rb_eval(const float* __restrict__ Zs, const float* __restrict__ Rs,
                                        const float* __restrict__ Ds, const float* __restrict__ CZs,
                                        const float* __restrict__ CXs, const float* __restrict__ CYs,
                                        const uint8_t* __restrict__ Ms, int lx, int ly, int lz, float w, int variant,
                                        int& zi, float& out) {
    const int ri = layout::rb_r(lx, ly, lz);
    zi = layout::rb_z(lx, ly, lz);
    const float d = Ds[ri];
    if (is_small(d)) return false;
    const unsigned m = Ms[layout::rb_m(lx, ly, lz)];
    const float zc = Zs[zi];
    float ax = 0.f;
    if (m & 64u) {
        const int xi = layout::rb_cx(lx, ly, lz);
        const int yi = layout::rb_cy(lx, ly, lz);
        ax = zc * d;
        if (m & 1u) ax += Zs[zi + layout::kZStepX] * CXs[xi];
        if (m & 2u) ax += Zs[zi - layout::kZStepX] * CXs[xi - layout::kCXStepX];
        if (m & 4u) ax += Zs[zi + layout::kZStepY] * CYs[yi];
        if (m & 8u) ax += Zs[zi - layout::kZStepY] * CYs[yi - layout::kCYStepY];
        if (m & 16u) ax += Zs[zi + 1] * CZs[ri];
        if (m & 32u) ax += Zs[zi - 1] * CZs[ri - 1];
    }
    const float term = (Rs[ri] - ax) / d;
    if (variant == LHI_SMOOTHER_DAMPED_GS) out = zc + w * term;
    else out = float((1.0 - double(w)) * double(zc) + double(float(w * term)));
    return true;
}

// Tile id u of the active list -> origin of its 8 x 8 x 32 cells.
__device__ __forceinline__ void tile_origin(const int32_t* __restrict__ ids, int u, int tdy, int tdz, int& x0, int& y0,
                                            int& z0) {
    const int id = ids[u];
    const int tz = id % tdz, rest = id / tdz;
    z0 = tz * kTileZ;
    y0 = (rest % tdy) * kTileY;
    x0 = (rest / tdy) * kTileX;
}

__device__ __forceinline__ void rb_issue(unsigned char* st, uint64_t* bar, const CUtensorMap* mz, const CUtensorMap* mr,
                                         const CUtensorMap* md, const CUtensorMap* mcx, const CUtensorMap* mcy,
                                         const CUtensorMap* mcz, const CUtensorMap* mm, int x0, int y0, int z0) {
    fence_proxy_async();
    bar_expect_tx(bar, rb::kTx);
    tma_load_box(st + rb::oZ, mz, z0 - 4, y0 - 2, x0 - 2, bar);
    tma_load_box(st + rb::oR, mr, z0 - 4, y0 - 1, x0 - 1, bar);
    tma_load_box(st + rb::oD, md, z0 - 4, y0 - 1, x0 - 1, bar);
    tma_load_box(st + rb::oCZ, mcz, z0 - 4, y0 - 1, x0 - 1, bar);
    tma_load_box(st + rb::oCX, mcx, z0 - 4, y0 - 1, x0 - 2, bar);
    tma_load_box(st + rb::oCY, mcy, z0 - 4, y0 - 2, x0 - 1, bar);
    tma_load_box(st + rb::oM, mm, z0 - 16, y0 - 1, x0 - 1, bar);
}

// One CTA per SM walks its tiles through two shared-memory stages: the
// boxes of the next tile are in flight while the current one is smoothed.
__global__ void __launch_bounds__(rb::kThreads, 1)
    k_rb_fused(const __grid_constant__ CUtensorMap mz, const __grid_constant__ CUtensorMap mr,
               const __grid_constant__ CUtensorMap md, const __grid_constant__ CUtensorMap mcx,
               const __grid_constant__ CUtensorMap mcy, const __grid_constant__ CUtensorMap mcz,
               const __grid_constant__ CUtensorMap mm, int nx, int ny, int nz, const int32_t* __restrict__ ids,
               const int* __restrict__ count, int tdy, int tdz, float* __restrict__ zout, float w, int variant,
               SolveScalars* __restrict__ sc, const float* __restrict__ ap, double* __restrict__ partials,
               unsigned* __restrict__ counter, int final_dot, int region, int flexible) {
    if (sc->stop) return;
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm);
    double v[2] = {0.0, 0.0};  // r.z and Ap.z of the swept tiles (final_dot)
    if (threadIdx.x == 0) {
        bar_init(&bar[0], 1);
        bar_init(&bar[1], 1);
    }
    __syncthreads();
    const int units = *count;
    if (threadIdx.x == 0 && int(blockIdx.x) < units) {
        int a, b, c;
        tile_origin(ids, blockIdx.x, tdy, tdz, a, b, c);
        rb_issue(sm + rb::kBase, &bar[0], &mz, &mr, &md, &mcx, &mcy, &mcz, &mm, a, b, c);
    }
    int it = 0;
    for (int u = blockIdx.x; u < units; u += gridDim.x, ++it) {
        const int s = it & 1;
        unsigned char* st = sm + rb::kBase + s * rb::kStage;
        int x0, y0, z0;
        tile_origin(ids, u, tdy, tdz, x0, y0, z0);
        const int un = u + int(gridDim.x);
        if (threadIdx.x == 0 && un < units) {  // the other stage was released by the last barrier
            int a, b, c;
            tile_origin(ids, un, tdy, tdz, a, b, c);
            rb_issue(sm + rb::kBase + (s ^ 1) * rb::kStage, &bar[s ^ 1], &mz, &mr, &md, &mcx, &mcy, &mcz, &mm, a, b,
                     c);
        }
        if (__syncthreads_or(!bar_wait(&bar[s], (it >> 1) & 1, g_stage_wait_ns))) {  // every thread leaves together
            if (threadIdx.x == 0) {
                sc->timeout = 1;
                sc->status = LHI_E_TIMEOUT;
                sc->stop = 1;
                // no copy of this CTA may still be landing when it exits: the one given up on and the prefetch
                bar_wait(&bar[s], (it >> 1) & 1);
                if (un < units) bar_wait(&bar[s ^ 1], ((it + 1) >> 1) & 1);
            }
            break;  // a CTA that gave up still takes part in the grid-wide sum below
        }
        // final_dot: this thread's float4 of Ap (the tile's 512 float4s, one
        // per thread), loaded now so the load overlaps the two colour phases
        static_assert(64 * 8 == rb::kThreads, "one float4 of the tile per thread");
        float4 apv = make_float4(0.f, 0.f, 0.f, 0.f);
        if (final_dot) {
            const int row = threadIdx.x >> 3, c = threadIdx.x & 7;
            const int x = x0 + (row >> 3), y = y0 + (row & 7), z = z0 + 4 * c;
            if (x < nx && y < ny && z < nz) apv = *reinterpret_cast<const float4*>(ap + ((long long)x * ny + y) * nz + z);
        }
        float* Zs = reinterpret_cast<float*>(st + rb::oZ);
        const float* Rs = reinterpret_cast<const float*>(st + rb::oR);
        const float* Ds = reinterpret_cast<const float*>(st + rb::oD);
        const float* CZs = reinterpret_cast<const float*>(st + rb::oCZ);
        const float* CXs = reinterpret_cast<const float*>(st + rb::oCX);
        const float* CYs = reinterpret_cast<const float*>(st + rb::oCY);
        const uint8_t* Ms = st + rb::oM;
        // colour 0 ((x + y + z) even) on T grown by one cell: 10 x 10 rows of 17
        // a colour's updates read only the other colour: a thread evaluates
        // all of its cells before storing any, so their loads overlap
        {
            constexpr int kN = (layout::kRbColour0Items + rb::kThreads - 1) / rb::kThreads;
            int zi[kN];
            float out[kN];
            bool upd[kN];
#pragma unroll
            for (int n = 0; n < kN; ++n) {
                const int q = threadIdx.x + n * rb::kThreads;
                upd[n] = false;
                if (q < layout::kRbColour0Items) {
                    int lx, ly, lz;
                    layout::rb_colour0(q, x0, y0, z0, lx, ly, lz);
                    upd[n] = rb_eval(Zs, Rs, Ds, CZs, CXs, CYs, Ms, lx, ly, lz, w, variant, zi[n], out[n]);
                }
            }
#pragma unroll
            for (int n = 0; n < kN; ++n)
                if (upd[n]) Zs[zi[n]] = out[n];
        }
        __syncthreads();
        // colour 1 on T: 8 x 8 rows of 16
        {
            constexpr int kN = layout::kRbColour1Items / rb::kThreads;
            int zi[kN];
            float out[kN];
            bool upd[kN];
#pragma unroll
            for (int n = 0; n < kN; ++n) {
                const int q = threadIdx.x + n * rb::kThreads;
                int lx, ly, lz;
                layout::rb_colour1(q, x0, y0, z0, lx, ly, lz);
                upd[n] = rb_eval(Zs, Rs, Ds, CZs, CXs, CYs, Ms, lx, ly, lz, w, variant, zi[n], out[n]);
            }
#pragma unroll
            for (int n = 0; n < kN; ++n)
                if (upd[n]) Zs[zi[n]] = out[n];
        }
        __syncthreads();
        for (int q = threadIdx.x; q < layout::kRbOutItems; q += rb::kThreads) {
            int lx, ly, c;
            const int zo = layout::rb_out(q, lx, ly, c);
            const int x = x0 + lx, y = y0 + ly, z = z0 + 4 * c;
            if (x < nx && y < ny && z < nz) {
                const float4 zv = *reinterpret_cast<const float4*>(Zs + zo);
                *reinterpret_cast<float4*>(zout + ((long long)x * ny + y) * nz + z) = zv;
                if (final_dot) {  // k_cg_dot_rz's sums over the swept cells
                    const float zz[4] = {zv.x, zv.y, zv.z, zv.w}, aa[4] = {apv.x, apv.y, apv.z, apv.w};
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int lz = 4 * c + j;
                        const float rv = Rs[layout::rb_r(lx, ly, lz)];
                        v[0] += double(rv) * double(zz[j]);
                        const unsigned m = Ms[layout::rb_m(lx, ly, lz)];
                        if ((m & 64u) && in_region(x, y, z + j, nx, ny, nz, region))
                            v[1] += double(aa[j]) * double(zz[j]);
                    }
                }
            }
        }
        __syncthreads();
    }
    if (!final_dot) return;
    double tot[2];
    if (!grid_sum_last<2>(v, partials, counter, tot)) return;
    const double rz_new = tot[0], apz = tot[1];
    sc->rz_new = rz_new;
    sc->apz = apz;
    sc->beta = flexible ? (-sc->alpha * apz / sc->rz_old) : (rz_new / sc->rz_old);
    sc->rz_old = rz_new;
}

// Neighbour masks of one level for the fused sweep (bits as rb_eval reads them).
template <class T>
__global__ void k_level_mask(LevelK<T> L, uint8_t* __restrict__ mask, int pitch) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)L.nx * L.ny * L.nz;
    if (i >= n) return;
    int x, y, z;
    decode(i, L.ny, L.nz, x, y, z);
    const long long sy = L.nz, sx = (long long)L.ny * L.nz;
    unsigned m = L.type[i] != 0 ? 64u : 0u;
    if (x + 1 < L.nx && L.type[i + sx] == 2) m |= 1u;
    if (x > 0 && L.type[i - sx] == 2) m |= 2u;
    if (y + 1 < L.ny && L.type[i + sy] == 2) m |= 4u;
    if (y > 0 && L.type[i - sy] == 2) m |= 8u;
    if (z + 1 < L.nz && L.type[i + 1] == 2) m |= 16u;
    if (z > 0 && L.type[i - 1] == 2) m |= 32u;
    mask[((long long)x * L.ny + y) * pitch + z] = uint8_t(m);
}

// CGSolver<3>::Restrict (PressureSolver.cpp:796-819) at one coarse cell: the
// coarse residual is accumulated in Scalar with 0.125 * (...) evaluated in
// double; z_c = 0.
template <class T>
__device__ __forceinline__ void restrict_cell(const LevelK<T>& F, const T* __restrict__ rf, const T* __restrict__ zf,
                                              int x, int y, int z, long long i, T* __restrict__ rc,
                                              T* __restrict__ zc) {
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

// restrict_cell with the 8 children's rows loaded 4 at a time before use;
// the children are still summed in the reference's order.
template <class T>
__device__ __forceinline__ void restrict_cell_batched(const LevelK<T>& F, const T* __restrict__ rf,
                                                      const T* __restrict__ zf, int x, int y, int z, long long i,
                                                      T* __restrict__ rc, T* __restrict__ zc) {
    const long long sy = F.nz, sx = (long long)F.ny * F.nz;
    const int bx = x << 1, by = y << 1, bz = z << 1;
    T acc = T(0);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        Cell7<T, T> c[4];
        T rv[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int a = h, b = (k >> 1) & 1, cc = k & 1;
            const long long f = (long long)(bx + a) * sx + (by + b) * sy + (bz + cc);
            load7(F, zf, f, bx + a, by + b, bz + cc, c[k]);
            rv[k] = rf[f];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const T res = rv[k] - ax7<T>(c[k]);
            acc = T(double(acc) + 0.125 * double(res));
        }
    }
    rc[i] = acc;
    zc[i] = T(0);
}

template <class T>
__global__ void __launch_bounds__(kTileThreads, 2) k_restrict_t(LevelK<T> F, const T* __restrict__ rf, const T* __restrict__ zf,
                                                             int cnx, int cny, int cnz, TileK tk, T* __restrict__ rc,
                                                             T* __restrict__ zc, const int* __restrict__ stop) {
    if (*stop) return;
    for_tiles(tk, cnx, cny, cnz,
              [&](int x, int y, int z, long long i) { restrict_cell_batched(F, rf, zf, x, y, z, i, rc, zc); });
}

template <class T>
__global__ void k_restrict_dense(LevelK<T> F, const T* __restrict__ rf, const T* __restrict__ zf, int cnx, int cny,
                                 int cnz, T* __restrict__ rc, T* __restrict__ zc, const int* __restrict__ stop) {
    if (*stop) return;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)cnx * cny * cnz;
    if (i >= n) return;
    int x, y, z;
    decode(i, cny, cnz, x, y, z);
    restrict_cell(F, rf, zf, x, y, z, i, rc, zc);
}

// CGSolver<3>::Prolong (PressureSolver.cpp:774-794): piecewise-constant,
// written per fine cell (fine cells beyond 2 * coarse extent get nothing).
template <class T>
__global__ void __launch_bounds__(kTileThreads) k_prolong_t(int fnx, int fny, int fnz, TileK tk, const T* __restrict__ zc,
                                                            int cnx, int cny, int cnz, T* __restrict__ zf,
                                                            const int* __restrict__ stop) {
    if (*stop) return;
    for_tile_cols(tk, fnx, fny, fnz, [&](int x, int z, long long i0, int yb, int rows, int ys) {
        const long long st = (long long)ys * fnz;
        const int cx = x >> 1, cz = z >> 1;
        bool on[kTileY];
        T fv[kTileY], cv[kTileY];
#pragma unroll
        for (int k = 0; k < kTileY; ++k) {
            const int cy = (yb + k * ys) >> 1;
            on[k] = k < rows && cx < cnx && cy < cny && cz < cnz;
            if (on[k]) {
                fv[k] = zf[i0 + k * st];
                cv[k] = zc[((long long)cx * cny + cy) * cnz + cz];
            }
        }
#pragma unroll
        for (int k = 0; k < kTileY; ++k)
            if (on[k]) zf[i0 + k * st] = fv[k] + cv[k];
    });
}

// The coarse levels [first, last] of one V-cycle in a single CTA.
template <class T> struct CoarseLevels {
    int first, last;
    LevelK<T> L[kMaxLevels];
    T* r[kMaxLevels];
    T* z[kMaxLevels];
    const uint32_t* list[kMaxLevels];
    const int* counts;
};

// Per-colour lists of the cells a coarse sweep updates (diag not small), one
// 32-bit entry per cell: index (low 16 bits) | neighbour mask << 16 (bits as
// the fused sweep's masks).  Built once per BuildLHS by one CTA; counts[2l]
// ends colour 0 of level l and counts[2l + 1] ends colour 1.
struct CoarseLists {
    uint32_t* list[kMaxLevels];
    int* counts;
};

template <class T>
__global__ void __launch_bounds__(1024) k_coarse_lists(CoarseLevels<T> c, CoarseLists cl) {
    __shared__ int warp_tot[32];
    __shared__ int base;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    for (int l = c.first; l <= c.last; ++l) {
        const LevelK<T>& L = c.L[l];
        const int n = L.nx * L.ny * L.nz;
        const int sy = L.nz, sx = L.ny * L.nz;
        if (threadIdx.x == 0) base = 0;
        __syncthreads();
        for (int colour = 0; colour < 2; ++colour) {
            for (int c0 = 0; c0 < n; c0 += blockDim.x) {
                const int i = c0 + threadIdx.x;
                uint32_t ent = 0;
                int f = 0;
                if (i < n) {
                    const int zz = i % L.nz, y = (i / L.nz) % L.ny, x = i / sx;
                    if (((x + y + zz) & 1) == colour && !is_small(L.diag[i])) {
                        unsigned m = L.type[i] != 0 ? 64u : 0u;
                        if (x + 1 < L.nx && L.type[i + sx] == 2) m |= 1u;
                        if (x > 0 && L.type[i - sx] == 2) m |= 2u;
                        if (y + 1 < L.ny && L.type[i + sy] == 2) m |= 4u;
                        if (y > 0 && L.type[i - sy] == 2) m |= 8u;
                        if (zz + 1 < L.nz && L.type[i + 1] == 2) m |= 16u;
                        if (zz > 0 && L.type[i - 1] == 2) m |= 32u;
                        ent = uint32_t(i) | (m << 16);
                        f = 1;
                    }
                }
                const unsigned bal = __ballot_sync(0xffffffffu, f);
                if (lane == 0) warp_tot[wp] = __popc(bal);
                __syncthreads();
                int off = base;
                for (int k = 0; k < wp; ++k) off += warp_tot[k];
                if (f) cl.list[l][off + __popc(bal & ((1u << lane) - 1u))] = ent;
                __syncthreads();
                if (threadIdx.x == 0)
                    for (int k = 0; k < int(blockDim.x >> 5); ++k) base += warp_tot[k];
                __syncthreads();
            }
            if (threadIdx.x == 0) cl.counts[2 * l + colour] = base;
            __syncthreads();
        }
    }
}

// Sweeps of one level inside the CTA over its colour lists: smooth7's
// arithmetic in the same order on shared-memory rows.
template <class T>
__device__ __forceinline__ void cta_smooth(const LevelK<T>& L, const T* r, T* z, const uint32_t* list, int n0,
                                           int n01, T w, int variant, int sweeps) {
    const int sy = L.nz, sx = L.ny * L.nz;
    constexpr int K = 1;  // cells per colour per thread kept in registers
    if (n0 <= K * int(blockDim.x) && n01 - n0 <= K * int(blockDim.x)) {
        // Every thread's cells (at most K per colour) keep diag, r, their six
        // coefficients and mask in registers for all sweeps; a pass loads
        // only the neighbours' z.
        int ci[2][K];
        unsigned cm[2][K];
        T cd[2][K], cr[2][K], cf[2][K][6];
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int e = (c ? n0 : 0) + int(threadIdx.x) + k * int(blockDim.x);
                ci[c][k] = -1;
                if (e < (c ? n01 : n0)) {
                    const uint32_t ent = list[e];
                    const int i = int(ent & 0xffffu);
                    ci[c][k] = i;
                    cm[c][k] = ent >> 16;
                    cd[c][k] = L.diag[i];
                    cr[c][k] = r[i];
                    const unsigned m = cm[c][k];
                    cf[c][k][0] = (m & 1u) ? L.cx[i] : T(0);
                    cf[c][k][1] = (m & 2u) ? L.cx[i - sx] : T(0);
                    cf[c][k][2] = (m & 4u) ? L.cy[i] : T(0);
                    cf[c][k][3] = (m & 8u) ? L.cy[i - sy] : T(0);
                    cf[c][k][4] = (m & 16u) ? L.cz[i] : T(0);
                    cf[c][k][5] = (m & 32u) ? L.cz[i - 1] : T(0);
                }
            }
        for (int s = 0; s < sweeps; ++s)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                T out[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const int i = ci[c][k];
                    if (i < 0) continue;
                    const unsigned m = cm[c][k];
                    const T d = cd[c][k];
                    const T zc = z[i];
                    T ax = T(0);
                    if (m & 64u) {
                        ax = zc * d;
                        if (m & 1u) ax += z[i + sx] * cf[c][k][0];
                        if (m & 2u) ax += z[i - sx] * cf[c][k][1];
                        if (m & 4u) ax += z[i + sy] * cf[c][k][2];
                        if (m & 8u) ax += z[i - sy] * cf[c][k][3];
                        if (m & 16u) ax += z[i + 1] * cf[c][k][4];
                        if (m & 32u) ax += z[i - 1] * cf[c][k][5];
                    }
                    const T term = (cr[c][k] - ax) / d;
                    if (variant == LHI_SMOOTHER_DAMPED_GS) out[k] = zc + w * term;
                    else out[k] = T((1.0 - double(w)) * double(zc) + double(T(w * term)));
                }
#pragma unroll
                for (int k = 0; k < K; ++k)
                    if (ci[c][k] >= 0) z[ci[c][k]] = out[k];
                __syncthreads();
            }
        return;
    }
    for (int s = 0; s < sweeps; ++s)
        for (int colour = 0; colour < 2; ++colour) {
            const int end = colour ? n01 : n0;
            for (int e = (colour ? n0 : 0) + int(threadIdx.x); e < end; e += blockDim.x) {
                const uint32_t ent = list[e];
                const int i = int(ent & 0xffffu);
                const unsigned m = ent >> 16;
                const T d = L.diag[i];
                const T zc = z[i];
                T ax = T(0);
                if (m & 64u) {
                    ax = zc * d;
                    if (m & 1u) ax += z[i + sx] * L.cx[i];
                    if (m & 2u) ax += z[i - sx] * L.cx[i - sx];
                    if (m & 4u) ax += z[i + sy] * L.cy[i];
                    if (m & 8u) ax += z[i - sy] * L.cy[i - sy];
                    if (m & 16u) ax += z[i + 1] * L.cz[i];
                    if (m & 32u) ax += z[i - 1] * L.cz[i - 1];
                }
                const T term = (r[i] - ax) / d;
                T out;
                if (variant == LHI_SMOOTHER_DAMPED_GS) out = zc + w * term;
                else out = T((1.0 - double(w)) * double(zc) + double(T(w * term)));
                z[i] = out;
            }
            __syncthreads();
        }
}

// The whole coarse V-cycle in one CTA with every coarse level staged in
// shared memory: r, z, diag, cx, cy, cz (Scalar) and type per level.
template <class T>
__global__ void __launch_bounds__(kCoarseThreads) k_coarse_cycle(CoarseLevels<T> c, T w, int variant, int pre, int post,
                                                                   int fin, const int* __restrict__ stop) {
    if (*stop) return;
    extern __shared__ __align__(16) unsigned char smem[];
    LevelK<T> S[kMaxLevels];
    T* r[kMaxLevels];
    T* z[kMaxLevels];
    uint32_t* lst[kMaxLevels];
    int n0[kMaxLevels], n01[kMaxLevels];
    size_t off = 0;
    for (int l = c.first; l <= c.last; ++l) {
        const LevelK<T>& G = c.L[l];
        const int n = G.nx * G.ny * G.nz;
        T* base = reinterpret_cast<T*>(smem + off);
        r[l] = base;
        z[l] = base + n;
        T* d = base + 2 * n;
        T* ax = base + 3 * n;
        T* ay = base + 4 * n;
        T* az = base + 5 * n;
        off += size_t(6) * n * sizeof(T);
        uint8_t* ty = smem + off;
        off += (size_t(n) + 15) & ~size_t(15);
        lst[l] = reinterpret_cast<uint32_t*>(smem + off);
        off += size_t(n) * 4;
        S[l] = LevelK<T>{G.nx, G.ny, G.nz, d, ax, ay, az, ty};
        n0[l] = c.counts[2 * l];
        n01[l] = c.counts[2 * l + 1];
        for (int e = threadIdx.x; e < n01[l]; e += blockDim.x) lst[l][e] = c.list[l][e];
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            d[i] = G.diag[i];
            ax[i] = G.cx[i];
            ay[i] = G.cy[i];
            az[i] = G.cz[i];
            ty[i] = G.type[i];
            r[l][i] = (l == c.first) ? c.r[l][i] : T(0);
            z[l][i] = (l == c.first) ? c.z[l][i] : T(0);
        }
    }
    __syncthreads();
    for (int l = c.first; l < c.last; ++l) {
        cta_smooth(S[l], r[l], z[l], lst[l], n0[l], n01[l], w, variant, pre);
        const LevelK<T>& C = S[l + 1];
        const int n = C.nx * C.ny * C.nz;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int zz = i % C.nz, y = (i / C.nz) % C.ny, x = i / (C.nz * C.ny);
            restrict_cell(S[l], r[l], z[l], x, y, zz, i, r[l + 1], z[l + 1]);
        }
        __syncthreads();
    }
    cta_smooth(S[c.last], r[c.last], z[c.last], lst[c.last], n0[c.last], n01[c.last], w, variant, fin);
    for (int l = c.last - 1; l >= c.first; --l) {
        const LevelK<T>& C = S[l + 1];
        const LevelK<T>& F = S[l];
        const int n = C.nx * C.ny * C.nz;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int zz = i % C.nz, y = (i / C.nz) % C.ny, x = i / (C.nz * C.ny);
            const T v = z[l + 1][i];
            const int b = ((x << 1) * F.ny + (y << 1)) * F.nz + (zz << 1);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int f = b + ((k >> 2) & 1) * F.ny * F.nz + ((k >> 1) & 1) * F.nz + (k & 1);
                z[l][f] = z[l][f] + v;
            }
        }
        __syncthreads();
        cta_smooth(F, r[l], z[l], lst[l], n0[l], n01[l], w, variant, post);
    }
    for (int l = c.first; l <= c.last; ++l) {
        const int n = S[l].nx * S[l].ny * S[l].nz;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            c.r[l][i] = r[l][i];
            c.z[l][i] = z[l][i];
        }
    }
}

template <class T>
__global__ void __launch_bounds__(kTileThreads) k_precond_none_t(LevelK<T> L, TileK tk, const T* __restrict__ r,
                                                                 T* __restrict__ z, const int* __restrict__ stop) {
    if (*stop) return;
    for_tiles(tk, L.nx, L.ny, L.nz, [&](int x, int y, int zz, long long i) {
        if (L.type[i] != 0) z[i] = r[i];
    });
}
template <class T>
__global__ void __launch_bounds__(kTileThreads) k_precond_jacobi_t(LevelK<T> L, TileK tk, const T* __restrict__ r,
                                                                   T* __restrict__ z, const int* __restrict__ stop) {
    if (*stop) return;
    for_tiles(tk, L.nx, L.ny, L.nz, [&](int x, int y, int zz, long long i) {
        T d = L.diag[i];
        if (!is_small(d)) z[i] = r[i] / d;
    });
}

// ---------------------------------------------------------------- PCG
struct CgConf {
    int region;
    int maxit;
    int every;       // true residual every k iterations (0 = never)
    int flexible;
    int rel;         // LHI_TOL_RELATIVE
    double tol;
    cudaGraphConditionalHandle cond;
    int use_cond;
    int warm;        // LHI_GUESS_PREVIOUS: the relative threshold comes from ||b||, not ||r0||
};

// Stopping rule after an update of r (PressureSolver.cpp:889-902): with a
// true-residual period, every k-th iteration and every apparent convergence
// is decided on r = b - A x instead (the next kernel computes it).
__device__ void cg_decide(SolveScalars* sc, double res2, const CgConf& cf, bool after_true) {
    const double residual = sqrt(res2);
    sc->residual = residual;
    if (!after_true) {
        sc->iter += 1;
        if (cf.every > 0 && (sc->iter % cf.every == 0 || residual < sc->threshold)) {
            sc->true_now = 1;
            return;
        }
    } else {
        sc->true_now = 0;
    }
    const bool conv = residual < sc->threshold;
    const bool bad = !isfinite(residual);
    const bool stop = conv || bad || sc->iter >= cf.maxit || sc->iter >= kGraphIterationCap;
    sc->status = bad ? LHI_E_NAN : (conv ? LHI_OK : LHI_E_NOT_CONVERGED);
    if (stop) sc->stop = 1;
    if (cf.use_cond) cudaGraphSetConditional(cf.cond, stop ? 0u : 1u);
}

// A loop-body kernel that finds the solve stopped by another kernel (a
// bounded wait that ran out) ends the graph's while loop: the iteration that
// set the conditional to continue did so before the stop.
__device__ __forceinline__ void cg_end_loop(const CgConf& cf) {
    if (cf.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(cf.cond, 0u);
}

// r0 = rhs on fluid cells (PressureSolver.cpp:847-856)
template <class T>
__global__ void __launch_bounds__(kTileThreads) k_cg_init_r(LevelK<T> L, TileK tk, const T* __restrict__ rhs, T* __restrict__ r) {
    for_tiles(tk, L.nx, L.ny, L.nz, [&](int x, int y, int z, long long i) {
        if (L.type[i] != 0) r[i] = rhs[i];
    });
}

// LHI_GUESS_PREVIOUS: x keeps the last solve's values on the cells that are
// fluid now and is 0 elsewhere (so the pressure written from it is 0 off
// the liquid, as the reference's cleared grid has it).
template <class TX>
__global__ void k_x_fluid_only(long long n, const uint8_t* __restrict__ type, TX* __restrict__ x) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && type[i] != 2) x[i] = TX(0);
}

// LHI_GUESS_PREVIOUS: r0 = b - A x0 on the cells with a row (where the
// reference's r0 = b is set), and sum b^2 over them into red[0]: the
// relative stopping rule's reference norm.
template <class T, class TX>
__global__ void __launch_bounds__(kTileThreads) k_cg_init_warm(LevelK<T> L, TileK tk, const T* __restrict__ b,
                                                               const TX* __restrict__ x, T* __restrict__ r,
                                                               double* __restrict__ partials,
                                                               unsigned* __restrict__ counter,
                                                               SolveScalars* __restrict__ sc) {
    double v[1] = {0.0};
    for_tiles(tk, L.nx, L.ny, L.nz, [&](int xi, int yi, int zi, long long i) {
        if (L.type[i] == 0) return;
        r[i] = T(double(b[i]) - ax_at<double>(L, x, i, xi, yi, zi));
        v[0] += double(b[i]) * double(b[i]);
    });
    double tot[1];
    if (!grid_sum_last<1>(v, partials, counter, tot)) return;
    sc->red[0] = tot[0];
}

// p = z on fluid cells; rz = r.z and rr = r.r over all cells; the stopping
// threshold from ||r0|| (PressureSolver.cpp:858-871)
template <class T>
__global__ void __launch_bounds__(kTileThreads) k_cg_init_p(LevelK<T> L, TileK tk, const T* __restrict__ r,
                                                            const T* __restrict__ z, T* __restrict__ p,
                                                            double* __restrict__ partials, unsigned* __restrict__ counter,
                                                            SolveScalars* __restrict__ sc, CgConf cf) {
    double v[2] = {0.0, 0.0};
    for_tiles(tk, L.nx, L.ny, L.nz, [&](int x, int y, int zz, long long i) {
        const T zi = z[i], ri = r[i];
        if (L.type[i] != 0) p[i] = zi;
        v[0] += double(ri) * double(zi);
        v[1] += double(ri) * double(ri);
    });
    double tot[2];
    if (!grid_sum_last<2>(v, partials, counter, tot)) return;
    sc->rz_old = tot[0];
    sc->rr_all = tot[1];
    const double r0 = sqrt(tot[1]);
    const T t = T(cf.tol);
    sc->residual0 = r0;
    sc->residual = r0;
    // with a previous solution as the guess, ||r|| is measured against ||b|| (k_cg_init_warm)
    const double ref = cf.warm ? sqrt(sc->red[0]) : r0;
    sc->threshold = cf.rel ? double(T(t * T(ref))) : double(t);
    sc->iter = 0;
    sc->true_now = 0;
    // a zero right-hand side is solved by x = 0 (under the relative rule the
    // threshold is then 0 as well, and r0 < threshold never holds)
    const bool conv = r0 < sc->threshold || r0 == 0.0;
    const bool stop = conv || cf.maxit <= 0;
    sc->status = conv ? LHI_OK : LHI_E_NOT_CONVERGED;
    sc->stop = stop ? 1 : 0;
    if (cf.use_cond) cudaGraphSetConditional(cf.cond, stop ? 0u : 1u);
}

// ------------------------------------------------- TMA-staged SpMV
// Ap = A p with p.Ap for the finest level, one 8 x 8 x 32 tile per step: p
// grown by one cell in x and y (z from z0-4), diag, the coefficients with
// the -x / -y / -z neighbours' faces, and the neighbour mask staged by TMA.
// A thread owns (x0 + warp, z0 + lane) and the tile's 8 rows, as k_cg_spmv
// does; the CTAs take other tiles than k_cg_spmv's, so p.Ap is grouped
// differently in its last bits.
namespace sp {
constexpr int kP = layout::kPBox, kD = layout::kDBox, kCX = layout::kCXBox, kCY = layout::kCYBox,
              kCZ = layout::kCZBox, kM = kD;
constexpr uint32_t kTx = uint32_t((kP + kD + kCX + kCY + kCZ) * 4 + kM);
// offsets inside one stage; two mbarriers, then two stages
constexpr int oP = 0, oD = oP + kP * 4, oCX = oD + kD * 4, oCY = oCX + kCX * 4, oCZ = oCY + kCY * 4,
              oM = oCZ + kCZ * 4, kStage = oM + kM;
constexpr int kBase = 128, kSmem = kBase + 2 * kStage;
static_assert(kP * 4 % 128 == 0 && kCX * 4 % 128 == 0 && kCZ * 4 % 128 == 0 && kStage % 128 == 0,
              "128-byte aligned boxes");
}  // namespace sp

__device__ __forceinline__ void sp_issue(unsigned char* st, uint64_t* bar, const CUtensorMap* mp, const CUtensorMap* md,
                                         const CUtensorMap* mcx, const CUtensorMap* mcy, const CUtensorMap* mcz,
                                         const CUtensorMap* mm, int x0, int y0, int z0) {
    fence_proxy_async();
    bar_expect_tx(bar, sp::kTx);
    tma_load_box(st + sp::oP, mp, z0 - 4, y0 - 1, x0 - 1, bar);
    tma_load_box(st + sp::oD, md, z0, y0, x0, bar);
    tma_load_box(st + sp::oCX, mcx, z0, y0, x0 - 1, bar);
    tma_load_box(st + sp::oCY, mcy, z0, y0 - 1, x0, bar);
    tma_load_box(st + sp::oCZ, mcz, z0 - 4, y0, x0, bar);
    tma_load_box(st + sp::oM, mm, z0, y0, x0, bar);
}

// Two CTAs per SM, each walking its tiles through two stages (the next
// tile's boxes in flight while the current one is multiplied).
__global__ void __launch_bounds__(kTileThreads, 2)
    k_spmv_tma(const __grid_constant__ CUtensorMap mp, const __grid_constant__ CUtensorMap md,
               const __grid_constant__ CUtensorMap mcx, const __grid_constant__ CUtensorMap mcy,
               const __grid_constant__ CUtensorMap mcz, const __grid_constant__ CUtensorMap mm, int nx, int ny, int nz,
               const int32_t* __restrict__ ids, const int* __restrict__ count, int tdy, int tdz, float* __restrict__ ap,
               double* __restrict__ partials, unsigned* __restrict__ counter, SolveScalars* __restrict__ sc,
               CgConf cf) {
    if (sc->stop) return;
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm);
    if (threadIdx.x == 0) {
        bar_init(&bar[0], 1);
        bar_init(&bar[1], 1);
    }
    __syncthreads();
    double v[1] = {0.0};
    const int units = *count;
    const int wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0 && int(blockIdx.x) < units) {
        int a, b, c;
        tile_origin(ids, blockIdx.x, tdy, tdz, a, b, c);
        sp_issue(sm + sp::kBase, &bar[0], &mp, &md, &mcx, &mcy, &mcz, &mm, a, b, c);
    }
    bool failed = false;
    int it = 0;
    for (int u = blockIdx.x; u < units; u += gridDim.x, ++it) {
        const int s = it & 1;
        const unsigned char* st = sm + sp::kBase + s * sp::kStage;
        int x0, y0, z0;
        tile_origin(ids, u, tdy, tdz, x0, y0, z0);
        const int un = u + int(gridDim.x);
        if (threadIdx.x == 0 && un < units) {  // the other stage was released by the last barrier
            int a, b, c;
            tile_origin(ids, un, tdy, tdz, a, b, c);
            sp_issue(sm + sp::kBase + (s ^ 1) * sp::kStage, &bar[s ^ 1], &mp, &md, &mcx, &mcy, &mcz, &mm, a, b, c);
        }
        if (__syncthreads_or(!bar_wait(&bar[s], (it >> 1) & 1, g_stage_wait_ns))) {  // every thread leaves together
            if (threadIdx.x == 0) {  // drain this CTA's copies in flight (the one given up on, the prefetch)
                bar_wait(&bar[s], (it >> 1) & 1);
                if (un < units) bar_wait(&bar[s ^ 1], ((it + 1) >> 1) & 1);
            }
            failed = true;
            break;
        }
        const float* Ps = reinterpret_cast<const float*>(st + sp::oP);
        const float* Ds = reinterpret_cast<const float*>(st + sp::oD);
        const float* CXs = reinterpret_cast<const float*>(st + sp::oCX);
        const float* CYs = reinterpret_cast<const float*>(st + sp::oCY);
        const float* CZs = reinterpret_cast<const float*>(st + sp::oCZ);
        const uint8_t* Ms = st + sp::oM;
        const int x = x0 + wp, zz = z0 + lane;
        if (x < nx && zz < nz) {
#pragma unroll
            for (int ly = 0; ly < kTileY; ++ly) {
                const int y = y0 + ly;
                if (y >= ny) break;
                const int pi = layout::sp_p(wp, ly, lane);
                const int ci = layout::sp_c(wp, ly, lane);
                const unsigned m = Ms[ci];
                const float pc = Ps[pi];
                float a = 0.f;
                if (m & 64u) {
                    a = pc * Ds[ci];
                    if (m & 1u) a += Ps[pi + layout::kPStepX] * CXs[layout::sp_cx(wp, ly, lane)];
                    if (m & 2u) a += Ps[pi - layout::kPStepX] * CXs[layout::sp_cx_minus(wp, ly, lane)];
                    if (m & 4u) a += Ps[pi + layout::kPStepY] * CYs[layout::sp_cy(wp, ly, lane)];
                    if (m & 8u) a += Ps[pi - layout::kPStepY] * CYs[layout::sp_cy_minus(wp, ly, lane)];
                    if (m & 16u) a += Ps[pi + 1] * CZs[layout::sp_cz(wp, ly, lane)];
                    if (m & 32u) a += Ps[pi - 1] * CZs[layout::sp_cz_minus(wp, ly, lane)];
                }
                ap[((long long)x * ny + y) * nz + zz] = a;
                if ((m & 64u) && in_region(x, y, zz, nx, ny, nz, cf.region)) v[0] += double(pc) * double(a);
            }
        }
        __syncthreads();
    }
    if (failed && threadIdx.x == 0) {
        sc->timeout = 1;
        sc->status = LHI_E_TIMEOUT;
        sc->stop = 1;
    }
    // every CTA takes part in the grid-wide sum, a failed one too
    double tot[1];
    if (!grid_sum_last<1>(v, partials, counter, tot)) return;
    sc->denom = tot[0];
    sc->alpha = sc->rz_old / tot[0];
}

// ------------------------------------------------- TMA restriction
// CGSolver<3>::Restrict from one active fine tile: z grown by one cell, r,
// diag, coefficients and mask staged by TMA; the residual r - A z of the
// tile's 2048 cells goes to shared memory, then each of its 4 x 4 x 16
// coarse cells sums its 8 children in the reference's order (restrict_cell).
// Coarse cells whose children all lie in inactive fine tiles are air cells
// whose restriction is 0, which they already hold.
namespace rs {
constexpr int kR = 8 * 8 * 32;
constexpr int oP = 128, oR = oP + sp::kP * 4, oD = oR + kR * 4, oCX = oD + sp::kD * 4, oCY = oCX + sp::kCX * 4,
              oCZ = oCY + sp::kCY * 4, oM = oCZ + sp::kCZ * 4, oRes = oM + sp::kM, kSmem = oRes + kR * 4;
constexpr uint32_t kTx = sp::kTx + kR * 4;
}  // namespace rs

__global__ void __launch_bounds__(kTileThreads, 3)
    k_restrict_tma(const __grid_constant__ CUtensorMap mz, const __grid_constant__ CUtensorMap mr,
                   const __grid_constant__ CUtensorMap md, const __grid_constant__ CUtensorMap mcx,
                   const __grid_constant__ CUtensorMap mcy, const __grid_constant__ CUtensorMap mcz,
                   const __grid_constant__ CUtensorMap mm, int nx, int ny, int nz, const int32_t* __restrict__ ids,
                   const int* __restrict__ count, int tdy, int tdz, int cnx, int cny, int cnz, float* __restrict__ rc,
                   float* __restrict__ zc, SolveScalars* __restrict__ sc) {
    if (sc->stop) return;
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm);
    const float* Ps = reinterpret_cast<const float*>(sm + rs::oP);
    const float* Rs = reinterpret_cast<const float*>(sm + rs::oR);
    const float* Ds = reinterpret_cast<const float*>(sm + rs::oD);
    const float* CXs = reinterpret_cast<const float*>(sm + rs::oCX);
    const float* CYs = reinterpret_cast<const float*>(sm + rs::oCY);
    const float* CZs = reinterpret_cast<const float*>(sm + rs::oCZ);
    const uint8_t* Ms = sm + rs::oM;
    float* Res = reinterpret_cast<float*>(sm + rs::oRes);
    if (threadIdx.x == 0) bar_init(bar, 1);
    __syncthreads();
    const int units = *count;
    const int wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned parity = 0;
    for (int u = blockIdx.x; u < units; u += gridDim.x) {
        int x0, y0, z0;
        tile_origin(ids, u, tdy, tdz, x0, y0, z0);
        if (threadIdx.x == 0) {
            fence_proxy_async();
            bar_expect_tx(bar, rs::kTx);
            tma_load_box(sm + rs::oP, &mz, z0 - 4, y0 - 1, x0 - 1, bar);
            tma_load_box(sm + rs::oR, &mr, z0, y0, x0, bar);
            tma_load_box(sm + rs::oD, &md, z0, y0, x0, bar);
            tma_load_box(sm + rs::oCX, &mcx, z0, y0, x0 - 1, bar);
            tma_load_box(sm + rs::oCY, &mcy, z0, y0 - 1, x0, bar);
            tma_load_box(sm + rs::oCZ, &mcz, z0 - 4, y0, x0, bar);
            tma_load_box(sm + rs::oM, &mm, z0, y0, x0, bar);
        }
        if (__syncthreads_or(!bar_wait(bar, parity, g_stage_wait_ns))) {  // every thread leaves together
            if (threadIdx.x == 0) {
                sc->timeout = 1;
                sc->status = LHI_E_TIMEOUT;
                sc->stop = 1;
                bar_wait(bar, parity);  // the copy given up on lands before the CTA exits
            }
            __syncthreads();
            return;
        }
        parity ^= 1u;
        float res[kTileY];  // all rows first, then the stores: their loads overlap
#pragma unroll
        for (int ly = 0; ly < kTileY; ++ly) {
            const int pi = layout::sp_p(wp, ly, lane);
            const int ci = layout::sp_c(wp, ly, lane);
            const unsigned m = Ms[ci];
            const float zc0 = Ps[pi];
            float a = 0.f;
            if (m & 64u) {
                a = zc0 * Ds[ci];
                if (m & 1u) a += Ps[pi + layout::kPStepX] * CXs[layout::sp_cx(wp, ly, lane)];
                if (m & 2u) a += Ps[pi - layout::kPStepX] * CXs[layout::sp_cx_minus(wp, ly, lane)];
                if (m & 4u) a += Ps[pi + layout::kPStepY] * CYs[layout::sp_cy(wp, ly, lane)];
                if (m & 8u) a += Ps[pi - layout::kPStepY] * CYs[layout::sp_cy_minus(wp, ly, lane)];
                if (m & 16u) a += Ps[pi + 1] * CZs[layout::sp_cz(wp, ly, lane)];
                if (m & 32u) a += Ps[pi - 1] * CZs[layout::sp_cz_minus(wp, ly, lane)];
            }
            res[ly] = Rs[ci] - a;
        }
#pragma unroll
        for (int ly = 0; ly < kTileY; ++ly) Res[layout::sp_c(wp, ly, lane)] = res[ly];
        __syncthreads();
        {
            int i, j, k;
            layout::rs_coarse(threadIdx.x, i, j, k);
            const int cx = (x0 >> 1) + i, cy = (y0 >> 1) + j, cz = (z0 >> 1) + k;
            if (cx < cnx && cy < cny && cz < cnz) {
                float acc = 0.f;
#pragma unroll
                for (int c8 = 0; c8 < 8; ++c8) {
                    const float res = Res[layout::rs_child(i, j, k, c8)];
                    acc = float(double(acc) + 0.125 * double(res));
                }
                const long long o = ((long long)cx * cny + cy) * cnz + cz;
                rc[o] = acc;
                zc[o] = 0.f;
            }
        }
        __syncthreads();
    }
}

// Ap = A p; p.Ap over the update region; alpha = rz / p.Ap (PressureSolver.cpp:873-888).
// A thread owns (x, z) of a tile and 8 rows, loaded 4 rows at a time.
template <class T>
__global__ void __launch_bounds__(kTileThreads, 2) k_cg_spmv(LevelK<T> L, TileK tk, const T* __restrict__ p, T* __restrict__ ap,
                                                          double* __restrict__ partials, unsigned* __restrict__ counter,
                                                          SolveScalars* __restrict__ sc, CgConf cf) {
    if (sc->stop) return;
    double v[1] = {0.0};
    const int units = *tk.count * tk.ysplit;
    const int wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int u = blockIdx.x; u < units; u += gridDim.x) {
        const int t = u / tk.ysplit, sub = u - t * tk.ysplit;
        const int id = tk.ids[t];
        const int tz = id % tk.tdz, rest = id / tk.tdz;
        const int ty = rest % tk.tdy, tx = rest / tk.tdy;
        const int x = tx * kTileX + wp, zz = tz * kTileZ + lane;
        if (x >= L.nx || zz >= L.nz) continue;
        const int y0 = ty * kTileY;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            Cell7<T, T> c[4];
            bool act[4];
            long long idx[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int yy = 4 * h + k, y = y0 + yy;
                act[k] = (yy % tk.ysplit == sub) && y < L.ny;
                if (act[k]) {
                    idx[k] = ((long long)x * L.ny + y) * L.nz + zz;
                    load7(L, p, idx[k], x, y, zz, c[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (!act[k]) continue;
                const T a = ax7<T>(c[k]);
                ap[idx[k]] = a;
                if (c[k].tc != 0 && in_region(x, y0 + 4 * h + k, zz, L.nx, L.ny, L.nz, cf.region))
                    v[0] += double(c[k].zc) * double(a);
            }
        }
    }
    double tot[1];
    if (!grid_sum_last<1>(v, partials, counter, tot)) return;
    sc->denom = tot[0];
    sc->alpha = sc->rz_old / tot[0];
}

// x += alpha p; r -= alpha Ap; ||r||^2 over the update region; then the
// stopping rule (PressureSolver.cpp:889-902)
template <class T, class TX>
__global__ void __launch_bounds__(kTileThreads) k_cg_update_xr(LevelK<T> L, TileK tk, const T* __restrict__ p,
                                                               const T* __restrict__ ap, TX* __restrict__ x,
                                                               T* __restrict__ r, double* __restrict__ partials,
                                                               unsigned* __restrict__ counter,
                                                               SolveScalars* __restrict__ sc, CgConf cf) {
    if (sc->stop) {
        cg_end_loop(cf);
        return;
    }
    const double alpha = sc->alpha;
    double v[1] = {0.0};
    for_tile_cols(tk, L.nx, L.ny, L.nz, [&](int xi, int zi, long long i0, int yb, int rows, int ys) {
        const long long st = (long long)ys * L.nz;
        bool on[kTileY];
        TX xv[kTileY];
        T pv[kTileY], rv[kTileY], av[kTileY];
#pragma unroll
        for (int k = 0; k < kTileY; ++k)
            on[k] = k < rows && L.type[i0 + k * st] != 0 && in_region(xi, yb + k * ys, zi, L.nx, L.ny, L.nz, cf.region);
#pragma unroll
        for (int k = 0; k < kTileY; ++k)
            if (on[k]) {
                xv[k] = x[i0 + k * st];
                pv[k] = p[i0 + k * st];
                rv[k] = r[i0 + k * st];
                av[k] = ap[i0 + k * st];
            }
#pragma unroll
        for (int k = 0; k < kTileY; ++k)
            if (on[k]) {
                x[i0 + k * st] = TX(double(xv[k]) + alpha * double(pv[k]));
                const T rn = T(double(rv[k]) - alpha * double(av[k]));
                r[i0 + k * st] = rn;
                v[0] += double(rn) * double(rn);
            }
    });
    double tot[1];
    if (!grid_sum_last<1>(v, partials, counter, tot)) return;
    sc->res2 = tot[0];
    cg_decide(sc, tot[0], cf, false);
}

// r = b - A x on the update region (stored when `store`, as TR), summed
// squares.  The mixed mode passes its FP64 finest-level matrix and
// right-hand side here (T = double) with the FP32 residual (TR = float).
template <class T, class TX, class TR>
__device__ __forceinline__ void true_residual_sweep(const LevelK<T>& L, const TileK& tk, int region, const T* __restrict__ b,
                                                    const TX* __restrict__ x, TR* __restrict__ r, bool store, double& acc) {
    for_tiles(tk, L.nx, L.ny, L.nz, [&](int xi, int yi, int zi, long long i) {
        if (L.type[i] == 0 || !in_region(xi, yi, zi, L.nx, L.ny, L.nz, region)) return;
        const double res = double(b[i]) - ax_at<double>(L, x, i, xi, yi, zi);
        if (store) r[i] = TR(res);
        acc += res * res;
    });
}

template <class T, class TX, class TR = T>
__global__ void __launch_bounds__(kTileThreads) k_cg_true_residual(LevelK<T> L, TileK tk, const T* __restrict__ b,
                                                                   const TX* __restrict__ x, TR* __restrict__ r,
                                                                   double* __restrict__ partials,
                                                                   unsigned* __restrict__ counter,
                                                                   SolveScalars* __restrict__ sc, CgConf cf) {
    if (sc->stop) {
        cg_end_loop(cf);
        return;
    }
    if (!sc->true_now) return;
    double v[1] = {0.0};
    true_residual_sweep(L, tk, cf.region, b, x, r, true, v[0]);
    double tot[1];
    if (!grid_sum_last<1>(v, partials, counter, tot)) return;
    sc->res2 = tot[0];
    sc->true2 = tot[0];
    cg_decide(sc, tot[0], cf, true);
}

// ||b - A x||^2 of the final iterate (not stored)
template <class T, class TX>
__global__ void __launch_bounds__(kTileThreads) k_true_residual_final(LevelK<T> L, TileK tk, int region,
                                                                      const T* __restrict__ b, const TX* __restrict__ x,
                                                                      double* __restrict__ partials,
                                                                      unsigned* __restrict__ counter,
                                                                      double* __restrict__ out) {
    double v[1] = {0.0};
    true_residual_sweep<T, TX, T>(L, tk, region, b, x, nullptr, false, v[0]);
    grid_sum_finish<1>(v, partials, counter, out);
}

// rz_new = r.z over all cells (Array3::Reduce); Ap.z over the update region;
// beta (PressureSolver.cpp:905-912): Fletcher-Reeves, or Polak-Ribiere
// -alpha Ap.z / rz_old when flexible
template <class T>
__global__ void __launch_bounds__(kTileThreads) k_cg_dot_rz(LevelK<T> L, TileK tk, const T* __restrict__ r,
                                                            const T* __restrict__ z, const T* __restrict__ ap,
                                                            double* __restrict__ partials, unsigned* __restrict__ counter,
                                                            SolveScalars* __restrict__ sc, CgConf cf) {
    if (sc->stop) return;
    double v[2] = {0.0, 0.0};
    for_tile_cols(tk, L.nx, L.ny, L.nz, [&](int xi, int zz, long long i0, int yb, int rows, int ys) {
        const long long st = (long long)ys * L.nz;
        bool on[kTileY];
        T zv[kTileY], rv[kTileY], av[kTileY];
#pragma unroll
        for (int k = 0; k < kTileY; ++k) {
            on[k] = k < rows && L.type[i0 + k * st] != 0 && in_region(xi, yb + k * ys, zz, L.nx, L.ny, L.nz, cf.region);
            if (k < rows) {
                zv[k] = z[i0 + k * st];
                rv[k] = r[i0 + k * st];
            }
        }
#pragma unroll
        for (int k = 0; k < kTileY; ++k)
            if (on[k]) av[k] = ap[i0 + k * st];
#pragma unroll
        for (int k = 0; k < kTileY; ++k) {
            if (k >= rows) break;
            v[0] += double(rv[k]) * double(zv[k]);
            if (on[k]) v[1] += double(av[k]) * double(zv[k]);
        }
    });
    double tot[2];
    if (!grid_sum_last<2>(v, partials, counter, tot)) return;
    const double rz_new = tot[0], apz = tot[1];
    sc->rz_new = rz_new;
    sc->apz = apz;
    sc->beta = cf.flexible ? (-sc->alpha * apz / sc->rz_old) : (rz_new / sc->rz_old);
    sc->rz_old = rz_new;
}

// p = z + beta p on fluid cells (PressureSolver.cpp:913-921)
template <class T>
__global__ void __launch_bounds__(kTileThreads) k_cg_update_p(LevelK<T> L, TileK tk, const T* __restrict__ z,
                                                              T* __restrict__ p, const SolveScalars* __restrict__ sc) {
    if (sc->stop) return;
    const double beta = sc->beta;
    for_tile_cols(tk, L.nx, L.ny, L.nz, [&](int x, int zz, long long i0, int yb, int rows, int ys) {
        const long long st = (long long)ys * L.nz;
        bool on[kTileY];
        T zv[kTileY], pv[kTileY];
#pragma unroll
        for (int k = 0; k < kTileY; ++k) on[k] = k < rows && L.type[i0 + k * st] != 0;
#pragma unroll
        for (int k = 0; k < kTileY; ++k)
            if (on[k]) {
                zv[k] = z[i0 + k * st];
                pv[k] = p[i0 + k * st];
            }
#pragma unroll
        for (int k = 0; k < kTileY; ++k)
            if (on[k]) p[i0 + k * st] = T(double(zv[k]) + beta * double(pv[k]));
    });
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

// --------------------------------------------------- learned preconditioner
// Cell-centre solid flag: mean of the cell's 8 node SDF values < 0.
template <class T>
__global__ void k_solid_cells(const T* __restrict__ sp, int nx, int ny, int nz, uint8_t* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)nx * ny * nz;
    if (i >= n) return;
    int x, y, z;
    decode(i, ny, nz, x, y, z);
    const long long sy = nz + 1, sx = (long long)(ny + 1) * (nz + 1);
    const T* b = sp + x * sx + y * sy + z;
    const double m = double(b[0]) + b[1] + b[sy] + b[sy + 1] + b[sx] + b[sx + 1] + b[sx + sy] + b[sx + sy + 1];
    out[i] = m < 0.0 ? 1 : 0;
}

// The network's cell classes: the level-0 type, with rows that the solver
// skips (diagonal below EPSILON: cells cut off by solid walls) marked 0.
template <class T>
__global__ void k_net_type(const uint8_t* __restrict__ type, const T* __restrict__ diag, long long n,
                           uint8_t* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = is_small(diag[i]) ? 0 : type[i];
}

// e = A z - r; sums of e^2 and r^2 over all cells
template <class T>
__global__ void k_loss_residual(LevelK<T> L, const float* __restrict__ z, const T* __restrict__ r, float* __restrict__ e,
                                double* __restrict__ partials, unsigned* __restrict__ counter, double* __restrict__ out) {
    double v[2] = {0.0, 0.0};
    const long long n = (long long)L.nx * L.ny * L.nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int x, y, zz;
        decode(i, L.ny, L.nz, x, y, zz);
        const double ei = ax_at<double>(L, z, i, x, y, zz) - double(r[i]);
        e[i] = float(ei);
        v[0] += ei * ei;
        v[1] += double(r[i]) * double(r[i]);
    }
    grid_sum_finish<2>(v, partials, counter, out);
}

// dz = 2 A^T e / (sum r^2 * batch); the loss sum e^2 / sum r^2 / batch is added to out[2]
template <class T>
__global__ void k_loss_grad(LevelK<T> L, const float* __restrict__ e, int batch, float* __restrict__ dz,
                            double* __restrict__ red) {
    const long long n = (long long)L.nx * L.ny * L.nz;
    const double rr = red[1] > 0 ? red[1] : 1.0;
    const double scale = 2.0 / (rr * batch);
    const long long sy = L.nz, sx = (long long)L.ny * L.nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        decode(i, L.ny, L.nz, x, y, z);
        const uint8_t ti = L.type[i];
        double acc = 0.0;
        if (ti != 0) acc = double(L.diag[i]) * e[i];
        if (ti == 2) {  // A(j, i) = [t_j >= 1][t_i == 2] c_ij
            if (x + 1 < L.nx && L.type[i + sx] != 0) acc += double(L.cx[i]) * e[i + sx];
            if (x > 0 && L.type[i - sx] != 0) acc += double(L.cx[i - sx]) * e[i - sx];
            if (y + 1 < L.ny && L.type[i + sy] != 0) acc += double(L.cy[i]) * e[i + sy];
            if (y > 0 && L.type[i - sy] != 0) acc += double(L.cy[i - sy]) * e[i - sy];
            if (z + 1 < L.nz && L.type[i + 1] != 0) acc += double(L.cz[i]) * e[i + 1];
            if (z > 0 && L.type[i - 1] != 0) acc += double(L.cz[i - 1]) * e[i - 1];
        }
        dz[i] = float(scale * acc);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) red[2] += red[0] / rr / batch;
}

// The coarse kernel's view of levels [first, nlev): pointers and lists.
template <class T>
CoarseLevels<T> coarse_levels_of(const LevelDev<T>* lv, int nlev, int first, uint32_t* list, const long long* off,
                                 int* counts) {
    CoarseLevels<T> c{};
    c.first = first;
    c.last = nlev - 1;
    for (int l = first; l < nlev; ++l) {
        c.L[l] = lk(lv[l]);
        c.r[l] = lv[l].r;
        c.z[l] = lv[l].z;
        c.list[l] = list + off[l];
    }
    c.counts = counts;
    return c;
}

}  // namespace

// ------------------------------------------------------------- host side
// Work units per tile: enough units to fill `grid` CTAs, at most max_split
// (4 for the colour sweeps, whose threads own 4 rows; 8 otherwise).
static int ysplit_for(int ntiles, int grid, int max_split = kTileY) {
    int s = 1;
    while (s < max_split && ntiles * s * 2 <= grid) s *= 2;
    return s;
}
template <class T> static TileK tile_k(const LevelDev<T>& L, const int* count, int grid, int max_split = kTileY) {
    return TileK{L.tiles, count, L.tdim[1], L.tdim[2], ysplit_for(L.ntiles, grid, max_split)};
}
// persistent CTAs for a tile kernel on level L (0 when the level is empty)
template <class T> static unsigned tile_blocks(const LevelDev<T>& L, int grid, int max_split = kTileY) {
    const long long units = (long long)L.ntiles * ysplit_for(L.ntiles, grid, max_split);
    return unsigned(std::min<long long>(units, grid));
}

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
    LHI_CUDA(cudaMemsetAsync(p_, 0, sizeof(T) * ncell_, cur_));
    if (sp_.initial_guess != LHI_GUESS_PREVIOUS)  // else the last solution is the guess (k_x_fluid_only)
        LHI_CUDA(cudaMemsetAsync(x_, 0, sizeof(TX) * ncell_, cur_));
    LHI_CUDA(cudaMemsetAsync(rhs_, 0, sizeof(T) * ncell_, cur_));
    for (int l = 0; l < nlev_; ++l) {
        LevelDev<T>& L = lv_[l];
        if (L.n == 0) continue;
        LHI_CUDA(cudaMemsetAsync(L.r, 0, sizeof(T) * L.n, cur_));
        LHI_CUDA(cudaMemsetAsync(L.z, 0, sizeof(T) * L.n, cur_));
        LHI_CUDA(cudaMemsetAsync(L.diag, 0, sizeof(T) * L.n, cur_));
        for (int a = 0; a < 3; ++a) LHI_CUDA(cudaMemsetAsync(L.cf[a], 0, sizeof(T) * L.n, cur_));
    }
    LHI_CUDA(cudaMemsetAsync(sc_, 0, sizeof(SolveScalars), cur_));
}

template <class T, class TX> void LiquidImpl<T, TX>::build_rhs() {
    auto ps_ = scope(LHI_KERNEL_GRID);
    if constexpr (kHiResidual) {
        k_build_rhs_mixed<T><<<blocks_for(ncell_, 256), 256, 0, cur_>>>(
            nx_, ny_, nz_, dx_[0], dx_[1], dx_[2], dxd_[0], dxd_[1], dxd_[2], liquid_phi_, lw_[0], lw_[1], lw_[2],
            v_[0], v_[1], v_[2], rhs_, rhs_hi_);
    } else {
        k_build_rhs<T><<<blocks_for(ncell_, 256), 256, 0, cur_>>>(nx_, ny_, nz_, dx_[0], dx_[1], dx_[2], liquid_phi_,
                                                                  lw_[0], lw_[1], lw_[2], v_[0], v_[1], v_[2], rhs_);
    }
    LHI_LAUNCH_CHECK();
}

// CGSolver<3>::BuildLHS (PressureSolver.cpp:544-664) for every level, then
// the levels' active-tile lists.
template <class T, class TX> void LiquidImpl<T, TX>::build_lhs(double rho, double dt) {
    auto ps_ = scope(LHI_KERNEL_LHS);
    for (int l = 0; l < nlev_; ++l) {
        LevelDev<T>& L = lv_[l];
        if (L.n == 0) continue;
        LevelGeom g{L.nx, L.ny, L.nz, nx_, ny_, nz_, l};
        LHI_CUDA(cudaMemsetAsync(L.tile_flag, 0, size_t(L.ntiles), cur_));
        if (l > 0 && sp_.coarse_operator == LHI_COARSE_GALERKIN) {
            k_level_galerkin<T><<<blocks_for(L.n, 256), 256, 0, cur_>>>(lk(lv_[l - 1]), L.nx, L.ny, L.nz, L.diag,
                                                                        L.cf[0], L.cf[1], L.cf[2], L.type,
                                                                        L.tile_flag, L.tdim[1], L.tdim[2]);
            LHI_LAUNCH_CHECK();
            continue;
        }
        if (l > 0) {  // the finest level's classes, tile flags and mask come with its matrix
            k_level_phi<T><<<blocks_for(L.n, 256), 256, 0, cur_>>>(g, liquid_phi_, L.phi, L.type, L.tile_flag,
                                                                  L.tdim[1], L.tdim[2]);
            LHI_LAUNCH_CHECK();
        }
        const T* phi = (l == 0) ? liquid_phi_ : L.phi;
        bool done = false;
        if constexpr (kHiResidual) {
            if (l == 0) {  // with the FP64 matrix of the outer residual
                k_level_matrix_mixed<T><<<blocks_for(L.n, 256), 256, 0, cur_>>>(
                    g, phi, lw_[0], lw_[1], lw_[2], L.h[0], L.h[1], L.h[2], T(dt), T(rho), L.diag, L.cf[0], L.cf[1],
                    L.cf[2], L.type, L.tile_flag, L.tdim[1], L.tdim[2], L.fused ? L.mask : nullptr, L.mpitch, dxd_[0],
                    dxd_[1], dxd_[2], dt, rho, diag_hi_, cf_hi_[0], cf_hi_[1], cf_hi_[2]);
                LHI_LAUNCH_CHECK();
                done = true;
            }
        }
        if (!done) {
            k_level_matrix<T><<<blocks_for(L.n, 256), 256, 0, cur_>>>(
                g, phi, lw_[0], lw_[1], lw_[2], L.h[0], L.h[1], L.h[2], T(dt), T(rho), L.diag, L.cf[0], L.cf[1],
                L.cf[2], l == 0 ? L.type : nullptr, L.tile_flag, L.tdim[1], L.tdim[2],
                (l == 0 && L.fused) ? L.mask : nullptr, L.mpitch);
            LHI_LAUNCH_CHECK();
        }
    }
    build_tiles();
    build_masks();
    net_type_fresh_ = false;
}

template <class T, class TX> void LiquidImpl<T, TX>::build_masks() {
    for (int l = 1; l < nlev_; ++l) {  // level 0's mask comes with its matrix (k_level_matrix)
        LevelDev<T>& L = lv_[l];
        if (!L.fused) continue;
        k_level_mask<T><<<blocks_for(L.n, 256), 256, 0, cur_>>>(lk(L), L.mask, L.mpitch);
        LHI_LAUNCH_CHECK();
    }
    if (coarse_level_ < nlev_) {
        CoarseLists cl{};
        for (int l = coarse_level_; l < nlev_; ++l) cl.list[l] = coarse_list_ + coarse_list_off_[l];
        cl.counts = coarse_counts_;
        k_coarse_lists<T><<<1, 1024, 0, cur_>>>(
            coarse_levels_of(lv_, nlev_, coarse_level_, coarse_list_, coarse_list_off_, coarse_counts_), cl);
        LHI_LAUNCH_CHECK();
    }
}


// Levels that the fused sweep can take: FP32, z extent a multiple of 4 (TMA
// strides are multiples of 16 bytes), at least 12 cells in x and y and one
// tile (32 cells) in z.  Boxes may reach past the level in z; TMA fills that
// part with zeros, which reads as diag 0 and an empty mask.
template <class T, class TX> void LiquidImpl<T, TX>::setup_fused() {
    if constexpr (std::is_same<T, float>::value) {
        LHI_CUDA(cudaFuncSetAttribute(k_rb_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, rb::kSmem));
        LHI_CUDA(cudaFuncSetAttribute(k_restrict_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, rs::kSmem));
        for (int l = 0; l < nlev_; ++l) {
            LevelDev<T>& L = lv_[l];
            if (L.n == 0 || L.nz % 4 != 0 || L.nx < 12 || L.ny < 12 || L.nz < kTileZ) continue;
            L.mpitch = (L.nz + 15) / 16 * 16;
            const size_t mb = size_t(L.nx) * L.ny * L.mpitch;
            LHI_CUDA(cudaMalloc(&L.zb, sizeof(T) * L.n));
            LHI_CUDA(cudaMalloc(&L.mask, mb));
            LHI_CUDA(cudaMemsetAsync(L.zb, 0, sizeof(T) * L.n, stream_));
            LHI_CUDA(cudaMemsetAsync(L.mask, 0, mb, stream_));
            const auto F32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
            L.tm_z = make_box_map(L.z, F32, 4, L.nx, L.ny, L.nz, L.nz, 12, 12, rb::kZW);
            L.tm_zb = make_box_map(L.zb, F32, 4, L.nx, L.ny, L.nz, L.nz, 12, 12, rb::kZW);
            L.tm_r = make_box_map(L.r, F32, 4, L.nx, L.ny, L.nz, L.nz, 10, 10, rb::kZW);
            L.tm_d = make_box_map(L.diag, F32, 4, L.nx, L.ny, L.nz, L.nz, 10, 10, rb::kZW);
            L.tm_cz = make_box_map(L.cf[2], F32, 4, L.nx, L.ny, L.nz, L.nz, 10, 10, rb::kZW);
            L.tm_cx = make_box_map(L.cf[0], F32, 4, L.nx, L.ny, L.nz, L.nz, 11, 10, rb::kZW);
            L.tm_cy = make_box_map(L.cf[1], F32, 4, L.nx, L.ny, L.nz, L.nz, 10, 11, rb::kZW);
            L.tm_m = make_box_map(L.mask, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, L.nx, L.ny, L.nz, L.mpitch, 10, 10,
                                  rb::kMW);
            L.ts_z = make_box_map(L.z, F32, 4, L.nx, L.ny, L.nz, L.nz, 10, 10, 40);
            L.ts_zb = make_box_map(L.zb, F32, 4, L.nx, L.ny, L.nz, L.nz, 10, 10, 40);
            L.ts_r = make_box_map(L.r, F32, 4, L.nx, L.ny, L.nz, L.nz, 8, 8, 32);
            L.ts_d = make_box_map(L.diag, F32, 4, L.nx, L.ny, L.nz, L.nz, 8, 8, 32);
            L.ts_cx = make_box_map(L.cf[0], F32, 4, L.nx, L.ny, L.nz, L.nz, 9, 8, 32);
            L.ts_cy = make_box_map(L.cf[1], F32, 4, L.nx, L.ny, L.nz, L.nz, 8, 9, 32);
            L.ts_cz = make_box_map(L.cf[2], F32, 4, L.nx, L.ny, L.nz, L.nz, 8, 8, 36);
            L.ts_m = make_box_map(L.mask, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, L.nx, L.ny, L.nz, L.mpitch, 8, 8, 32);
            L.fused = true;
        }
    }
}

// Tensor maps of the finest level's TMA SpMV (on the CG direction p).
template <class T, class TX> void LiquidImpl<T, TX>::setup_spmv() {
    if constexpr (std::is_same<T, float>::value) {
        LevelDev<T>& L = lv_[0];
        if (!L.fused) return;
        LHI_CUDA(cudaFuncSetAttribute(k_spmv_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, sp::kSmem));
        const auto F32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
        tm_sp_[0] = make_box_map(p_, F32, 4, L.nx, L.ny, L.nz, L.nz, 10, 10, 40);
        tm_sp_[1] = make_box_map(L.diag, F32, 4, L.nx, L.ny, L.nz, L.nz, 8, 8, 32);
        tm_sp_[2] = make_box_map(L.cf[0], F32, 4, L.nx, L.ny, L.nz, L.nz, 9, 8, 32);
        tm_sp_[3] = make_box_map(L.cf[1], F32, 4, L.nx, L.ny, L.nz, L.nz, 8, 9, 32);
        tm_sp_[4] = make_box_map(L.cf[2], F32, 4, L.nx, L.ny, L.nz, L.nz, 8, 8, 36);
        tm_sp_[5] = make_box_map(L.mask, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, L.nx, L.ny, L.nz, L.mpitch, 8, 8, 32);
        spmv_tma_ = true;
    }
}

template <class T, class TX> void LiquidImpl<T, TX>::build_tiles() {
    TileLevels tl{};
    tl.nlev = 0;
    for (int l = 0; l < nlev_ && lv_[l].n > 0; ++l) {
        for (int a = 0; a < 3; ++a) tl.tdim[l][a] = lv_[l].tdim[a];
        tl.flag[l] = lv_[l].tile_flag;
        tl.ids[l] = lv_[l].tiles;
        tl.nlev = l + 1;
    }
    if (tl.nlev == 0) return;
    k_tiles_finalize<<<1, 1024, 0, cur_>>>(tl, sc_->tile_count);
    LHI_LAUNCH_CHECK();
}

template <class T, class TX> bool LiquidImpl<T, TX>::smooth(int level, int sweeps, bool final_dot) {
    LevelDev<T>& L = lv_[level];
    const unsigned G = tile_blocks(L, tile_grid_, 4);
    if (L.n == 0 || sweeps <= 0 || G == 0) return false;
    const T w = T(sp_.smoothing_factor);
    const int cat = (level == 0) ? LHI_KERNEL_SMOOTH_FINE : LHI_KERNEL_SMOOTH_COARSE;
    if (L.fused && sp_.sweep_kernel == LHI_SWEEP_FUSED) {
        const unsigned GF = unsigned(std::min(L.ntiles, kSMs));
        for (int s = 0; s < sweeps; ++s) {
            auto ps_ = scope(cat);
            const int fd = (final_dot && s + 1 == sweeps) ? 1 : 0;
            k_rb_fused<<<GF, rb::kThreads, rb::kSmem, cur_>>>(
                L.tm_z, L.tm_r, L.tm_d, L.tm_cx, L.tm_cy, L.tm_cz, L.tm_m, L.nx, L.ny, L.nz, L.tiles,
                &sc_->tile_count[level], L.tdim[1], L.tdim[2], reinterpret_cast<float*>(L.zb), float(w),
                sp_.smoother, sc_, reinterpret_cast<const float*>(ap_), partials_, counter_, fd, sp_.update_region,
                sp_.cg_variant == LHI_CG_FLEXIBLE ? 1 : 0);
            LHI_LAUNCH_CHECK();
            std::swap(L.z, L.zb);
            std::swap(L.tm_z, L.tm_zb);
            std::swap(L.ts_z, L.ts_zb);
        }
        return final_dot;
    }
    const TileK tk = tile_k(L, &sc_->tile_count[level], tile_grid_, 4);
    for (int s = 0; s < sweeps; ++s)
        for (int phase = 0; phase < 2; ++phase) {
            auto ps_ = scope(cat);
            k_sweep<T><<<G, kTileThreads, 0, cur_>>>(lk(L), tk, L.r, L.z, w, sp_.smoother, phase, &sc_->stop);
            LHI_LAUNCH_CHECK();
        }
    return false;
}

template <class T, class TX> void LiquidImpl<T, TX>::restrict_to(int level) {
    LevelDev<T>& C = lv_[level];
    LevelDev<T>& F = lv_[level - 1];
    if (C.n == 0) return;
    auto ps_ = scope(LHI_KERNEL_RESTRICT);
    if (F.fused && sp_.sweep_kernel == LHI_SWEEP_FUSED) {
        const unsigned GR = unsigned(std::min(F.ntiles, 3 * kSMs));
        k_restrict_tma<<<GR, kTileThreads, rs::kSmem, cur_>>>(
            F.ts_z, F.ts_r, F.ts_d, F.ts_cx, F.ts_cy, F.ts_cz, F.ts_m, F.nx, F.ny, F.nz, F.tiles,
            &sc_->tile_count[level - 1], F.tdim[1], F.tdim[2], C.nx, C.ny, C.nz, reinterpret_cast<float*>(C.r),
            reinterpret_cast<float*>(C.z), sc_);
    } else if (level >= coarse_level_) {
        k_restrict_dense<T><<<blocks_for(C.n, 256), 256, 0, cur_>>>(lk(F), F.r, F.z, C.nx, C.ny, C.nz, C.r, C.z,
                                                                     &sc_->stop);
    } else {
        const unsigned G = tile_blocks(C, tile_grid_);
        k_restrict_t<T><<<G, kTileThreads, 0, cur_>>>(lk(F), F.r, F.z, C.nx, C.ny, C.nz,
                                                      tile_k(C, &sc_->tile_count[level], tile_grid_), C.r, C.z,
                                                      &sc_->stop);
    }
    LHI_LAUNCH_CHECK();
}

template <class T, class TX> void LiquidImpl<T, TX>::prolong_to(int level) {
    LevelDev<T>& C = lv_[level + 1];
    LevelDev<T>& F = lv_[level];
    const unsigned G = tile_blocks(F, tile_grid_);
    if (C.n == 0 || F.n == 0 || G == 0) return;
    auto ps_ = scope(LHI_KERNEL_PROLONG);
    k_prolong_t<T><<<G, kTileThreads, 0, cur_>>>(F.nx, F.ny, F.nz, tile_k(F, &sc_->tile_count[level], tile_grid_),
                                                 C.z, C.nx, C.ny, C.nz, F.z, &sc_->stop);
    LHI_LAUNCH_CHECK();
}

// Bytes of shared memory the coarse kernel needs for levels [first, nlev).
template <class T> static size_t coarse_bytes(const LevelDev<T>* lv, int first, int nlev) {
    size_t b = 0;
    for (int l = first; l < nlev; ++l)
        b += size_t(6) * lv[l].n * sizeof(T) + ((size_t(lv[l].n) + 15) & ~size_t(15)) + size_t(4) * lv[l].n;
    return b;
}

// Picks the first level (below the finest) whose cell count is at most
// coarse_cells and whose coarse V-cycle fits in one CTA's shared memory.
template <class T, class TX> void LiquidImpl<T, TX>::setup_coarse() {
    const long long cc = sp_.coarse_cells > 0 ? sp_.coarse_cells : kDefaultCoarseCells;
    coarse_level_ = nlev_;
    coarse_smem_ = 0;
    for (int l = 1; l < nlev_; ++l) {
        const size_t b = coarse_bytes(lv_, l, nlev_);
        if (lv_[l].n <= cc && b <= kCoarseSmemBytes) {
            coarse_level_ = l;
            coarse_smem_ = b;
            break;
        }
    }
    LHI_CUDA(cudaFuncSetAttribute(k_coarse_cycle<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(kCoarseSmemBytes)));
    long long nl = 0;
    for (int l = coarse_level_; l < nlev_; ++l) {
        coarse_list_off_[l] = nl;
        nl += lv_[l].n;
    }
    if (coarse_level_ < nlev_) {
        LHI_CUDA(cudaMalloc(&coarse_list_, sizeof(uint32_t) * size_t(std::max(nl, 1LL))));
        LHI_CUDA(cudaMalloc(&coarse_counts_, sizeof(int) * 2 * kMaxLevels));
        LHI_CUDA(cudaMemsetAsync(coarse_counts_, 0, sizeof(int) * 2 * kMaxLevels, stream_));
    }
}

// CGSolver<3>::ApplyPreconditioner multigrid branch (PressureSolver.cpp:730-771)
template <class T, class TX> void LiquidImpl<T, TX>::enqueue_vcycle() {
    T* z_at_start[kMaxLevels];
    for (int l = 0; l < nlev_; ++l) z_at_start[l] = lv_[l].z;
    enqueue_vcycle_levels();
    // an odd number of fused sweeps on a level leaves its result in the other
    // buffer: copy it back so every V-cycle starts and ends on the same one
    for (int l = 0; l < nlev_; ++l) {
        LevelDev<T>& L = lv_[l];
        if (L.z == z_at_start[l]) continue;
        LHI_CUDA(cudaMemcpyAsync(L.zb, L.z, sizeof(T) * L.n, cudaMemcpyDeviceToDevice, cur_));
        std::swap(L.z, L.zb);
        std::swap(L.tm_z, L.tm_zb);
        std::swap(L.ts_z, L.ts_zb);
    }
}

template <class T, class TX> void LiquidImpl<T, TX>::enqueue_vcycle_levels() {
    const int last = nlev_ - 1;
    const int Lc = coarse_level_;
    if (Lc <= last) {
        for (int l = 0; l < Lc; ++l) {
            smooth(l, sp_.num_pre_smooth);
            restrict_to(l + 1);
        }
        const CoarseLevels<T> c =
            coarse_levels_of(lv_, nlev_, coarse_level_, coarse_list_, coarse_list_off_, coarse_counts_);
        {
            auto ps_ = scope(LHI_KERNEL_SMOOTH_COARSE);
            k_coarse_cycle<T><<<1, kCoarseThreads, coarse_smem_, cur_>>>(c, T(sp_.smoothing_factor), sp_.smoother,
                                                                sp_.num_pre_smooth, sp_.num_post_smooth,
                                                                sp_.num_final_smooth, &sc_->stop);
            LHI_LAUNCH_CHECK();
        }
        for (int l = Lc - 1; l >= 0; --l) {
            prolong_to(l);
            dot_fused_ |= smooth(l, sp_.num_post_smooth, l == 0 && fuse_dot_);
        }
    } else {
        for (int l = 0; l < last; ++l) {
            smooth(l, sp_.num_pre_smooth);
            restrict_to(l + 1);
        }
        smooth(last, sp_.num_final_smooth);
        for (int l = last - 1; l >= 0; --l) {
            prolong_to(l);
            dot_fused_ |= smooth(l, sp_.num_post_smooth, l == 0 && fuse_dot_);
        }
    }
}

template <class T, class TX> void LiquidImpl<T, TX>::vcycle() { enqueue_vcycle(); }

template <class T, class TX> void LiquidImpl<T, TX>::enqueue_precond() {
    LevelDev<T>& L0 = lv_[0];
    const unsigned G = tile_blocks(L0, tile_grid_);
    switch (sp_.preconditioner) {
        case LHI_PRECOND_NONE:
            if (G == 0) break;
            k_precond_none_t<T><<<G, kTileThreads, 0, cur_>>>(lk(L0), tile_k(L0, &sc_->tile_count[0], tile_grid_),
                                                              L0.r, L0.z, &sc_->stop);
            LHI_LAUNCH_CHECK();
            break;
        case LHI_PRECOND_JACOBI:
            if (G == 0) break;
            k_precond_jacobi_t<T><<<G, kTileThreads, 0, cur_>>>(lk(L0), tile_k(L0, &sc_->tile_count[0], tile_grid_),
                                                                L0.r, L0.z, &sc_->stop);
            LHI_LAUNCH_CHECK();
            break;
        case LHI_PRECOND_LEARNED:
            if (net_ && !use_fallback_) {
                ensure_solid_cells();
                ensure_net_type();
                const int dims[3] = {nx_, ny_, nz_};
                if (net_->sparse_enabled_ && (net_plan_stale_ || net_->plan_type_ != net_type_)) {
                    net_->plan_sparse(dims, net_type_, cur_);
                    net_plan_stale_ = false;
                }
                net_->forward(dims, reinterpret_cast<const float*>(L0.r), net_type_, solid_cell_,
                              reinterpret_cast<float*>(L0.z), 0.0, cur_, true);
                break;
            }
            enqueue_vcycle();
            break;
        default: enqueue_vcycle();
    }
}

// CGSolver<3>::ApplyPreconditioner (PressureSolver.cpp:719-772) as a stage
template <class T, class TX> void LiquidImpl<T, TX>::apply_preconditioner() {
    LHI_CUDA(cudaMemsetAsync(&sc_->stop, 0, sizeof(int), cur_));
    enqueue_precond();
}

static CgConf make_conf(const lhi_solver_params& sp, unsigned long long cond, int use_cond) {
    CgConf c;
    c.region = sp.update_region;
    c.maxit = sp.max_iterations;
    c.every = sp.true_residual_every;
    c.flexible = sp.cg_variant == LHI_CG_FLEXIBLE ? 1 : 0;
    c.rel = sp.tolerance_mode == LHI_TOL_RELATIVE ? 1 : 0;
    c.tol = sp.tolerance;
    c.cond = cond;
    c.use_cond = use_cond;
    c.warm = sp.initial_guess == LHI_GUESS_PREVIOUS ? 1 : 0;
    return c;
}

// r = b; z = M r; p = z; rz; ||r0||; threshold (PressureSolver.cpp:845-871)
template <class T, class TX> void LiquidImpl<T, TX>::enqueue_init(unsigned long long cond, int use_cond) {
    LevelDev<T>& L0 = lv_[0];
    const TileK tk = tile_k(L0, &sc_->tile_count[0], tile_grid_);
    const unsigned G = std::max(1u, tile_blocks(L0, tile_grid_));
    const CgConf cf = make_conf(sp_, cond, use_cond);
    {
        auto ps_ = scope(LHI_KERNEL_CG_VECTOR);
        if (sp_.initial_guess == LHI_GUESS_PREVIOUS) {
            k_x_fluid_only<TX><<<blocks_for(ncell_, 256), 256, 0, cur_>>>(ncell_, L0.type, x_);
            LHI_LAUNCH_CHECK();
            k_cg_init_warm<T, TX><<<G, kTileThreads, 0, cur_>>>(lk(L0), tk, rhs_, x_, L0.r, partials_, counter_, sc_);
        } else {
            k_cg_init_r<T><<<G, kTileThreads, 0, cur_>>>(lk(L0), tk, rhs_, L0.r);
        }
        LHI_LAUNCH_CHECK();
    }
    record_snapshot();
    enqueue_precond();
    {
        auto ps_ = scope(LHI_KERNEL_CG_VECTOR);
        k_cg_init_p<T><<<G, kTileThreads, 0, cur_>>>(lk(L0), tk, L0.r, L0.z, p_, partials_, counter_, sc_, cf);
        LHI_LAUNCH_CHECK();
    }
}

// One PCG iteration (PressureSolver.cpp:870-922).
template <class T, class TX> void LiquidImpl<T, TX>::enqueue_body(unsigned long long cond, int use_cond) {
    LevelDev<T>& L0 = lv_[0];
    const TileK tk = tile_k(L0, &sc_->tile_count[0], tile_grid_);
    const unsigned G = std::max(1u, tile_blocks(L0, tile_grid_));
    const CgConf cf = make_conf(sp_, cond, use_cond);
    {
        auto ps_ = scope(LHI_KERNEL_SPMV);
        if (spmv_tma_ && sp_.sweep_kernel == LHI_SWEEP_FUSED)
            k_spmv_tma<<<std::min(G, unsigned(2 * kSMs)), kTileThreads, sp::kSmem, cur_>>>(
                tm_sp_[0], tm_sp_[1], tm_sp_[2], tm_sp_[3], tm_sp_[4], tm_sp_[5], L0.nx, L0.ny, L0.nz, L0.tiles,
                &sc_->tile_count[0], L0.tdim[1], L0.tdim[2], reinterpret_cast<float*>(ap_), partials_, counter_, sc_,
                cf);
        else
            k_cg_spmv<T><<<G, kTileThreads, 0, cur_>>>(lk(L0), tk, p_, ap_, partials_, counter_, sc_, cf);
        LHI_LAUNCH_CHECK();
    }
    {
        auto ps_ = scope(LHI_KERNEL_CG_VECTOR);
        k_cg_update_xr<T, TX><<<G, kTileThreads, 0, cur_>>>(lk(L0), tk, p_, ap_, x_, L0.r, partials_, counter_, sc_,
                                                            cf);
        LHI_LAUNCH_CHECK();
        if (sp_.true_residual_every > 0) {
            if constexpr (kHiResidual)
                k_cg_true_residual<double, TX, T><<<G, kTileThreads, 0, cur_>>>(lk_hi(*this), tk, rhs_hi_, x_, L0.r,
                                                                                partials_, counter_, sc_, cf);
            else
                k_cg_true_residual<T, TX><<<G, kTileThreads, 0, cur_>>>(lk(L0), tk, rhs_, x_, L0.r, partials_,
                                                                        counter_, sc_, cf);
            LHI_LAUNCH_CHECK();
        }
    }
    record_snapshot();
    // with the multigrid preconditioner the last level-0 sweep of the V-cycle
    // also forms r.z and Ap.z (and beta), which saves k_cg_dot_rz's pass
    fuse_dot_ = sp_.preconditioner == LHI_PRECOND_MULTIGRID;
    dot_fused_ = false;
    enqueue_precond();
    fuse_dot_ = false;
    {
        auto ps_ = scope(LHI_KERNEL_CG_VECTOR);
        if (!dot_fused_) {
            k_cg_dot_rz<T><<<G, kTileThreads, 0, cur_>>>(lk(L0), tk, L0.r, L0.z, ap_, partials_, counter_, sc_, cf);
            LHI_LAUNCH_CHECK();
        }
        k_cg_update_p<T><<<G, kTileThreads, 0, cur_>>>(lk(L0), tk, L0.z, p_, sc_);
        LHI_LAUNCH_CHECK();
    }
}

// grid.pressure = x (PressureSolver.cpp:933) and the final true residual
template <class T, class TX> void LiquidImpl<T, TX>::enqueue_final() {
    LevelDev<T>& L0 = lv_[0];
    const unsigned G = std::max(1u, tile_blocks(L0, tile_grid_));
    auto ps_ = scope(LHI_KERNEL_CG_VECTOR);
    k_x_to_pressure<T, TX><<<blocks_for(ncell_, 256), 256, 0, cur_>>>(ncell_, x_, pressure_);
    LHI_LAUNCH_CHECK();
    if constexpr (kHiResidual)
        k_true_residual_final<double, TX><<<G, kTileThreads, 0, cur_>>>(
            lk_hi(*this), tile_k(L0, &sc_->tile_count[0], tile_grid_), sp_.update_region, rhs_hi_, x_, partials_, counter_,
            &sc_->true2);
    else
        k_true_residual_final<T, TX><<<G, kTileThreads, 0, cur_>>>(lk(L0), tile_k(L0, &sc_->tile_count[0], tile_grid_),
                                                                   sp_.update_region, rhs_, x_, partials_, counter_,
                                                                   &sc_->true2);
    LHI_LAUNCH_CHECK();
}

// The solve after BuildLHS as one graph: init; while (!stop) { iteration };
// final.  Pointers and parameters are fixed for the handle's lifetime, so
// the graph is built on the first solve and replayed after.
// with_init: the whole solve (init, the loop, the final pass).  Without it:
// the loop from the current iterate on and the final pass (the tail of a
// solve whose first iterations ran host-driven); its loop condition starts
// at 1 at every launch, and a solve that has already stopped leaves the
// loop in its first body's first kernel.
template <class T, class TX> void LiquidImpl<T, TX>::build_solve_graph(bool with_init) {
    cudaGraph_t g = nullptr;
    LHI_CUDA(cudaStreamSynchronize(stream_));  // surfaces any earlier asynchronous error before capturing
    LHI_CUDA(cudaGetLastError());
    LHI_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    try {
        cudaStreamCaptureStatus st;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        cudaGraph_t cg = nullptr;
        LHI_CUDA(cudaStreamGetCaptureInfo(stream_, &st, nullptr, &cg, nullptr, nullptr));
        cudaGraphConditionalHandle h;
        if (with_init)
            LHI_CUDA(cudaGraphConditionalHandleCreate(&h, cg, 0, 0));
        else
            LHI_CUDA(cudaGraphConditionalHandleCreate(&h, cg, 1, cudaGraphCondAssignDefault));
        const long long c0 = g_kernel_launches.load();
        if (with_init) enqueue_init(h, 1);
        const long long c1 = g_kernel_launches.load();
        LHI_CUDA(cudaStreamGetCaptureInfo(stream_, &st, nullptr, &cg, &deps, &nd));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        LHI_CUDA(cudaGraphAddNode(&node, cg, deps, nd, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        LHI_CUDA(cudaStreamUpdateCaptureDependencies(stream_, &node, 1, cudaStreamSetCaptureDependencies));
        LHI_CUDA(cudaStreamBeginCaptureToGraph(side_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        cur_ = side_;
        long long c2 = 0;
        try {
            enqueue_body(h, 1);
            c2 = g_kernel_launches.load();
        } catch (...) {
            cur_ = stream_;
            cudaGraph_t b2 = nullptr;
            cudaStreamEndCapture(side_, &b2);
            throw;
        }
        cur_ = stream_;
        cudaGraph_t body_out = nullptr;
        LHI_CUDA(cudaStreamEndCapture(side_, &body_out));
        enqueue_final();
        const long long c3 = g_kernel_launches.load();
        LHI_CUDA(cudaStreamEndCapture(stream_, &g));
        if (with_init) graph_init_kernels_ = c1 - c0;
        graph_body_kernels_ = c2 - c1;
        graph_final_kernels_ = c3 - c2;
        // captured launches did not run: the replays below count what runs
        g_kernel_launches.fetch_sub(c3 - c0);
    } catch (...) {
        cur_ = stream_;
        cudaGraph_t g2 = nullptr;
        cudaStreamEndCapture(stream_, &g2);
        if (g2) cudaGraphDestroy(g2);
        throw;
    }
    cudaGraphExec_t exec = nullptr;
    cudaGraphInstantiateParams ip = {};
    cudaError_t e = cudaGraphInstantiateWithParams(&exec, g, &ip);
    std::string why;
    if (e != cudaSuccess) {
        cudaGraphNodeType nt = cudaGraphNodeTypeEmpty;
        if (ip.errNode_out) cudaGraphNodeGetType(ip.errNode_out, &nt);
        why = std::string("solve graph instantiation failed: ") + cudaGetErrorString(e) + " (result " +
              std::to_string(int(ip.result_out)) + ", node type " + std::to_string(int(nt)) + ")";
        cudaGetLastError();
    }
    cudaGraphDestroy(g);
    if (e != cudaSuccess) throw CudaError(e, why);
    (with_init ? solve_exec_ : tail_exec_) = exec;
}

// CGSolver<3>::Solve (PressureSolver.cpp:839-934)
template <class T, class TX> int LiquidImpl<T, TX>::solve(double rho, double dt) {
    if (stats_pending_) finish_stats();
    LHI_CUDA(cudaEventRecord(ev0_, stream_));
    solver_init();
    build_rhs();
    build_lhs(rho, dt);
    bool graph_replayed = false;
    const bool learned = sp_.preconditioner == LHI_PRECOND_LEARNED;
    if (learned && !net_) throw std::invalid_argument("LHI_PRECOND_LEARNED without a network (lhi_solver_set_network)");
    use_fallback_ = false;
    learned_iters_ = 0;
    fallback_at_ = -1;
    // The first solve of a handle runs host-driven: it launches (and so
    // loads) every kernel of the loop once, which must not happen for the
    // first time inside a stream capture; later solves replay the graph.
    const bool graph_ok = solved_once_;
    solved_once_ = true;
    if (!sp_.eager && !prof_.on && !learned && snap_cap_ == 0 && graph_ok && graph_error_.empty() && !solve_exec_) {
        try {
            build_solve_graph(true);
        } catch (const CudaError& err) {
            graph_error_ = err.what();  // keep solving, host-driven (lhi_solver_graph_error)
            cudaGetLastError();         // the failed capture's error is not this solve's
        }
    }
    if (!sp_.eager && !prof_.on && !learned && snap_cap_ == 0 && graph_ok && solve_exec_) {
        LHI_CUDA(cudaGraphLaunch(solve_exec_, stream_));
        graph_replayed = true;
    } else {
        // host-driven loop; with the learned preconditioner the host also
        // applies the fallback rule between iterations
        const bool no_fallback = fallback_iters_ < 0;
        const int cap = fallback_iters_ > 0 ? fallback_iters_ : sp_.max_iterations;
        enqueue_init(0, 0);
        if (learned) {
            learned_iters_ = 1;
            read_scalars();
            if (!no_fallback && !(sc_host_->rz_old > 0.0) && !sc_host_->stop) {
                // r.M(r) <= 0: the network gives no descent direction; start over with the V-cycle
                use_fallback_ = true;
                fallback_at_ = 0;
                learned_iters_ = 0;
                enqueue_init(0, 0);
            }
        }
        double prev = -1.0;
        // after the fallback (and once one V-cycle body has run here, so no
        // kernel loads for the first time inside a capture) the rest of the
        // solve is one replay of the tail graph
        const bool tail_ok = learned && !sp_.eager && !prof_.on && snap_cap_ == 0;
        bool tail = false;
        for (;;) {
            read_scalars();
            if (sc_host_->stop) break;
            if (learned && !use_fallback_ && !no_fallback) {
                const double res = sc_host_->residual;
                const bool slow = prev > 0 && res > 0.95 * prev;
                if (slow || sc_host_->iter >= cap) {
                    use_fallback_ = true;
                    fallback_at_ = sc_host_->iter;
                }
                prev = res;
            }
            if (learned && !use_fallback_) ++learned_iters_;
            if (tail_ok && use_fallback_ && fallback_body_ran_ && tail_error_.empty()) {
                if (!tail_exec_) {
                    try {
                        build_solve_graph(false);
                    } catch (const CudaError& err) {
                        tail_error_ = err.what();  // keep the loop host-driven
                        cudaGetLastError();
                    }
                }
                if (tail_exec_) {
                    tail_from_iter_ = sc_host_->iter;
                    LHI_CUDA(cudaGraphLaunch(tail_exec_, stream_));
                    tail = true;
                    break;
                }
            }
            enqueue_body(0, 0);
            if (use_fallback_) fallback_body_ran_ = true;
        }
        if (!tail) enqueue_final();
    }
    LHI_CUDA(cudaEventRecord(ev1_, stream_));
    last_solve_graph_ = graph_replayed;
    stats_pending_ = true;
    if (async_ && graph_replayed) return LHI_OK;  // read by stats() later
    finish_stats();
    // a network application whose pipeline wait ran out left no usable direction
    if (learned && net_ && net_->check_status(stream_) != LHI_OK) stats_.status = LHI_E_TIMEOUT;
    return stats_.status;
}

// Statistics of the last solve from the device scalars (synchronises).
template <class T, class TX> void LiquidImpl<T, TX>::finish_stats() {
    read_scalars();
    float ms = 0.f;
    LHI_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    if (last_solve_graph_)  // kernels the replay ran: init, one body per loop trip, final
        g_kernel_launches.fetch_add(graph_init_kernels_ + graph_final_kernels_ +
                                    graph_body_kernels_ * (long long)std::max(sc_host_->iter, 0));
    if (tail_from_iter_ >= 0)  // the tail graph: one body per loop trip from where it started (at least one), final
        g_kernel_launches.fetch_add(graph_final_kernels_ +
                                    graph_body_kernels_ * (long long)std::max(sc_host_->iter - tail_from_iter_, 1));
    tail_from_iter_ = -1;
    stats_.iterations = sc_host_->iter;
    stats_.initial_residual = sc_host_->residual0;
    stats_.final_residual = sc_host_->residual;
    stats_.true_residual = std::sqrt(sc_host_->true2);
    stats_.solve_ms = ms;
    stats_.status = sc_host_->timeout ? LHI_E_TIMEOUT : sc_host_->status;
    stats_pending_ = false;
}

template <class T, class TX> void LiquidImpl<T, TX>::spmv(int level, const T* x, T* y) {
    LevelDev<T>& L = lv_[level];
    if (L.n == 0) return;
    k_get_ax<T><<<blocks_for(L.n, 256), 256, 0, cur_>>>(lk(L), x, y);
    LHI_LAUNCH_CHECK();
}

// One SpMV of the PCG body on the handle's p, through the same launch as
// enqueue_body's (so the same kernel and tile order); p.Ap comes back from
// the device scalars.
template <class T, class TX> double LiquidImpl<T, TX>::spmv_p(int* tma) {
    LevelDev<T>& L0 = lv_[0];
    if (L0.n == 0) return 0.0;
    cur_ = stream_;
    LHI_CUDA(cudaMemsetAsync(&sc_->stop, 0, sizeof(int), stream_));  // a finished solve leaves stop set
    const TileK tk = tile_k(L0, &sc_->tile_count[0], tile_grid_);
    const unsigned G = std::max(1u, tile_blocks(L0, tile_grid_));
    const CgConf cf = make_conf(sp_, 0, 0);
    const bool use_tma = spmv_tma_ && sp_.sweep_kernel == LHI_SWEEP_FUSED;
    {
        auto ps_ = scope(LHI_KERNEL_SPMV);
        if (use_tma)
            k_spmv_tma<<<std::min(G, unsigned(2 * kSMs)), kTileThreads, sp::kSmem, cur_>>>(
                tm_sp_[0], tm_sp_[1], tm_sp_[2], tm_sp_[3], tm_sp_[4], tm_sp_[5], L0.nx, L0.ny, L0.nz, L0.tiles,
                &sc_->tile_count[0], L0.tdim[1], L0.tdim[2], reinterpret_cast<float*>(ap_), partials_, counter_, sc_,
                cf);
        else
            k_cg_spmv<T><<<G, kTileThreads, 0, cur_>>>(lk(L0), tk, p_, ap_, partials_, counter_, sc_, cf);
        LHI_LAUNCH_CHECK();
    }
    read_scalars();
    if (sc_host_->timeout) throw std::runtime_error("SpMV: a bounded wait on a staging copy timed out");
    if (tma) *tma = use_tma ? 1 : 0;
    return sc_host_->denom;
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

template <class T, class TX>
void LiquidImpl<T, TX>::active_tiles(int level, int32_t* active, int32_t* total, int32_t* coarse) {
    if (level < 0 || level >= nlev_) throw std::invalid_argument("bad level");
    read_scalars();
    *active = sc_host_->tile_count[level];
    *total = lv_[level].ntiles;
    *coarse = (level >= coarse_level_) ? 1 : 0;
}

template <class T, class TX> void LiquidImpl<T, TX>::set_network(LearnedNet* net, int fallback_iterations) {
    if (sp_.preconditioner != LHI_PRECOND_LEARNED)
        throw std::invalid_argument("lhi_solver_set_network needs a handle created with LHI_PRECOND_LEARNED");
    if (fallback_iterations < -1) throw std::invalid_argument("fallback_iterations must be >= -1");
    net_ = net;
    fallback_iters_ = fallback_iterations;
}

template <class T, class TX> void LiquidImpl<T, TX>::ensure_solid_cells() {
    if (!solid_cell_) LHI_CUDA(cudaMalloc(&solid_cell_, size_t(ncell_)));
    if (solid_cell_fresh_) return;
    k_solid_cells<T><<<blocks_for(ncell_, 256), 256, 0, cur_>>>(solid_phi_, nx_, ny_, nz_, solid_cell_);
    LHI_LAUNCH_CHECK();
    solid_cell_fresh_ = true;
}

template <class T, class TX> void LiquidImpl<T, TX>::ensure_net_type() {
    if (!net_type_) LHI_CUDA(cudaMalloc(&net_type_, size_t(ncell_)));
    if (net_type_fresh_) return;
    k_net_type<T><<<blocks_for(ncell_, 256), 256, 0, cur_>>>(lv_[0].type, lv_[0].diag, ncell_, net_type_);
    LHI_LAUNCH_CHECK();
    net_type_fresh_ = true;
    net_plan_stale_ = true;
}

template <class T, class TX> void LiquidImpl<T, TX>::record_residuals(int max_snapshots) {
    if (max_snapshots < 0 || max_snapshots > 100000) throw std::invalid_argument("max_snapshots out of range");
    if (snaps_) cudaFree(snaps_);
    snaps_ = nullptr;
    snap_cap_ = max_snapshots;
    snap_count_ = snap_next_ = 0;
    if (max_snapshots > 0) LHI_CUDA(cudaMalloc(&snaps_, sizeof(float) * size_t(ncell_) * size_t(max_snapshots)));
}

// Copy of level-0 r (as FP32) into the next snapshot slot (ring buffer).
template <class T, class TX> void LiquidImpl<T, TX>::record_snapshot() {
    if (snap_cap_ == 0) return;
    float* dst = snaps_ + size_t(snap_next_) * size_t(ncell_);
    if (sizeof(T) == sizeof(float)) {
        LHI_CUDA(cudaMemcpyAsync(dst, lv_[0].r, sizeof(float) * ncell_, cudaMemcpyDeviceToDevice, cur_));
    } else {
        throw std::invalid_argument("residual recording needs an FP32 or MIXED handle");
    }
    snap_next_ = (snap_next_ + 1) % snap_cap_;
    snap_count_ = std::min(snap_count_ + 1, snap_cap_);
}

template <class T, class TX>
void LiquidImpl<T, TX>::train(LearnedNet* net, int steps, int batch, double lr, uint64_t seed, double* first,
                              double* last) {
    if (sizeof(T) != sizeof(float)) throw std::invalid_argument("training needs an FP32 or MIXED handle");
    if (snap_count_ == 0) throw std::invalid_argument("no recorded residuals (lhi_solver_record_residuals + solve)");
    if (steps < 1 || batch < 1) throw std::invalid_argument("steps and batch must be >= 1");
    if (!train_z_) {
        LHI_CUDA(cudaMalloc(&train_z_, sizeof(float) * ncell_));
        LHI_CUDA(cudaMalloc(&train_dz_, sizeof(float) * ncell_));
        LHI_CUDA(cudaMalloc(&train_e_, sizeof(float) * ncell_));
        LHI_CUDA(cudaMalloc(&train_red_, sizeof(double) * 4));
    }
    ensure_solid_cells();
    ensure_net_type();
    LevelDev<T>& L0 = lv_[0];
    const int dims[3] = {nx_, ny_, nz_};
    const unsigned nbk = std::min<unsigned>(blocks_for(ncell_, 256), unsigned(sum_blocks_));
    std::mt19937_64 rng(seed);
    double first_loss = 0.0, last_loss = 0.0;
    for (int st = 0; st < steps; ++st) {
        net->zero_grad(cur_);
        LHI_CUDA(cudaMemsetAsync(train_red_ + 2, 0, sizeof(double), cur_));
        for (int b = 0; b < batch; ++b) {
            const int k = int(rng() % uint64_t(snap_count_));
            const float* r = snaps_ + size_t(k) * size_t(ncell_);
            net->forward(dims, r, net_type_, solid_cell_, train_z_, 0.0, cur_);
            k_loss_residual<T><<<nbk, 256, 0, cur_>>>(lk(L0), train_z_, reinterpret_cast<const T*>(r), train_e_,
                                                      partials_, counter_, train_red_);
            LHI_LAUNCH_CHECK();
            k_loss_grad<T><<<nbk, 256, 0, cur_>>>(lk(L0), train_e_, batch, train_dz_, train_red_);
            LHI_LAUNCH_CHECK();
            net->backward(train_dz_, cur_);
        }
        net->adam_step(lr, 0.9, 0.999, 1e-8, cur_);
        if (st == 0 || st == steps - 1) {
            double loss = 0.0;
            LHI_CUDA(cudaMemcpyAsync(&loss, train_red_ + 2, sizeof(double), cudaMemcpyDeviceToHost, cur_));
            LHI_CUDA(cudaStreamSynchronize(cur_));
            if (st == 0) first_loss = loss;
            last_loss = loss;
        }
    }
    if (net->check_status(cur_) != LHI_OK) throw CudaError(cudaErrorLaunchTimeout, "tensor-core pipeline wait timed out");
    *first = first_loss;
    *last = last_loss;
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

void set_stage_wait_limit_ns(unsigned long long ns) {
    LHI_CUDA(cudaMemcpyToSymbol(g_stage_wait_ns, &ns, sizeof(ns)));
}

template class LiquidImpl<float, float>;
template class LiquidImpl<float, double>;
template class LiquidImpl<double, double>;

}  // namespace lhi
