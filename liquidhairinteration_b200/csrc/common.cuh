// common.cuh -- shared device helpers of the B200 liquid step.
//
// Exact-rounding arithmetic: the kernels that must agree bit-for-bit with the
// reference's CPU path (cell keys, liquid SDF, face fractions, matrix
// assembly, G2P, advection) use the round-to-nearest intrinsics below so the
// compiler cannot fuse a multiply and an add into one FMA.  The solver's
// stencil arithmetic is allowed to use FMA (its parity bar is a tolerance).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace lhi {

extern std::atomic<long long> g_kernel_launches;

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const std::string& what) : std::runtime_error(what), code(c) {}
};

#define LHI_CUDA(call)                                                                                     \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess)                                                                             \
            throw ::lhi::CudaError(e_, std::string(#call " failed: ") + cudaGetErrorString(e_) + " at " + \
                                           __FILE__ + ":" + std::to_string(__LINE__));                     \
    } while (0)

// Every kernel launch of the library is followed by this check, which also
// counts it (lhi_kernel_launch_count).
#define LHI_LAUNCH_CHECK()                                                          \
    do {                                                                            \
        ::lhi::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);           \
        LHI_CUDA(cudaGetLastError());                                               \
    } while (0)

constexpr int kSMs = 148;

// (x, y, z) of entry i of an [..][ny][nz] array (z fastest), in 32-bit
// arithmetic: every grid and face array has fewer than 2^32 entries.
__device__ __forceinline__ void idx3(long long i, int ny, int nz, int& x, int& y, int& z) {
    const unsigned u = unsigned(i), t = u / unsigned(nz);
    z = int(u - t * unsigned(nz));
    y = int(t % unsigned(ny));
    x = int(t / unsigned(ny));
}

inline unsigned blocks_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    return unsigned(b);
}

// ----------------------------------------------------------- exact arithmetic
template <class T> struct X;
template <> struct X<float> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
};
template <> struct X<double> {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double sqrt(double a) { return __dsqrt_rn(a); }
};

template <class T> __device__ __forceinline__ T eps8() { return T(1e-8); }  // EPSILON (Definition.h:88)

// windows.h macros (Definition.h:22) and Eigen's maxi
template <class T> __device__ __forceinline__ T mac_min(T a, T b) { return (a < b) ? a : b; }
template <class T> __device__ __forceinline__ T mac_max(T a, T b) { return (a > b) ? a : b; }
template <class T> __device__ __forceinline__ T eig_maxi(T a, T b) { return (a < b) ? b : a; }

// MathUtils::IsSmall (MathUtils.h:8)
template <class T> __device__ __forceinline__ bool is_small(T v) { return fabs(v) < eps8<T>(); }
// MathUtils::Clamp (MathUtils.h:10)
template <class T> __device__ __forceinline__ T clampS(T v, T lo, T hi) { return mac_min(hi, mac_max(lo, v)); }

// MathUtils::Lerp / Bilerp / Trilerp (MathUtils.h:12-33)
template <class T> __device__ __forceinline__ T lerp(T v0, T v1, T f) {
    return X<T>::add(v0, X<T>::mul(clampS(f, T(0), T(1)), X<T>::sub(v1, v0)));
}
template <class T> __device__ __forceinline__ T bilerp(T v00, T v10, T v01, T v11, T f1, T f2) {
    T a = lerp(v00, v10, f1);
    T b = lerp(v01, v11, f1);
    return lerp(a, b, clampS(f2, T(0), T(1)));
}
template <class T>
__device__ __forceinline__ T trilerp(T v000, T v100, T v010, T v110, T v001, T v101, T v011, T v111, T f1, T f2,
                                     T f3) {
    T a = bilerp(v000, v100, v010, v110, f1, f2);
    T b = bilerp(v001, v101, v011, v111, f1, f2);
    return lerp(a, b, clampS(f3, T(0), T(1)));
}

// MathUtils::FractionInRegion(left, right) (MathUtils.cpp:29-35)
template <class T> __device__ __forceinline__ T fraction_in_region(T l, T r) {
    T ans = T(0);
    if (l < T(0) && r < T(0)) ans = T(1);
    else if (l < T(0) && T(0) < r) ans = X<T>::div(l, X<T>::sub(l, r));
    else if (l > T(0) && T(0) > r) ans = X<T>::div(r, X<T>::sub(r, l));
    return ans;
}
// max(0.1, f) through the windows.h macro: compared and selected in double
template <class T> __device__ __forceinline__ T frac_floor(T f) {
    double v = (0.1 > double(f)) ? 0.1 : double(f);
    return T(v);
}
// Clamp(1.0 - FractionInRegion(a, b), 0.0, 1.0): argument evaluated in double
template <class T> __device__ __forceinline__ T open_fraction(T a, T b) {
    T val = T(__dsub_rn(1.0, double(fraction_in_region(a, b))));
    return clampS(val, T(0), T(1));
}

// MathUtils::GetBarycentricCoord (MathUtils.cpp:75-88)
template <class T> __device__ __forceinline__ void barycentric(T x, int minI, int maxI, int& index, T& frac) {
    index = int(floor(x));
    frac = X<T>::sub(x, T(index));
    if (index < minI) {
        index = minI;
        frac = T(0);
    } else if (index > maxI - 2) {
        index = maxI - 2;
        frac = T(1);
    }
}

// BSplineKernel::QuadraticWeight / GradQuadraticWeight (Kernel.h:12-31)
template <class T> __device__ __forceinline__ T qweight(T d) {
    d = fabs(d);
    if (d < T(0.5f)) return X<T>::sub(T(0.75f), X<T>::mul(d, d));
    if (d < T(1.5f)) {
        T e = X<T>::sub(T(1.5f), d);
        return X<T>::mul(X<T>::mul(T(0.5f), e), e);
    }
    return T(0);
}
template <class T> __device__ __forceinline__ T gqweight(T d) {
    d = fabs(d);
    if (d < T(0.5f)) return X<T>::mul(T(-2.f), d);
    if (d < T(1.5f)) return X<T>::sub(d, T(1.5f));
    return T(0);
}

// Eigen fixed-size 3-vector reductions: a0 + (a1 + a2)
template <class T> __device__ __forceinline__ T sqnorm3(T a, T b, T c) {
    return X<T>::add(X<T>::mul(a, a), X<T>::add(X<T>::mul(b, b), X<T>::mul(c, c)));
}
template <class T> __device__ __forceinline__ T dot3(T a0, T a1, T a2, T b0, T b1, T b2) {
    return X<T>::add(X<T>::mul(a0, b0), X<T>::add(X<T>::mul(a1, b1), X<T>::mul(a2, b2)));
}

// ------------------------------------------------------------ reductions
template <class T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <class T> __device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum; result valid in thread 0.  Needs blockDim.x % 32 == 0.
template <class T> __device__ __forceinline__ T block_sum(T v) {
    __shared__ T s[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) s[w] = v;
    __syncthreads();
    int nw = blockDim.x >> 5;
    v = (threadIdx.x < nw) ? s[lane] : T(0);
    if (w == 0) v = warp_sum(v);
    return v;
}
template <class T> __device__ __forceinline__ T block_max(T v) {
    __shared__ T s[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) s[w] = v;
    __syncthreads();
    int nw = blockDim.x >> 5;
    v = (threadIdx.x < nw) ? s[lane] : T(-INFINITY);
    if (w == 0) v = warp_max(v);
    return v;
}

// Deterministic grid-wide sum of K doubles: every block writes its partials,
// the last block to finish adds them in block order and writes out[k].
// partials: gridDim.x * K doubles; counter: one zero-initialised uint that
// the last block resets.  Call from all threads of every block.
template <int K>
__device__ __forceinline__ void grid_sum_finish(double (&v)[K], double* partials, unsigned* counter, double* out) {
    __shared__ bool last;
    double tot[K];
#pragma unroll
    for (int k = 0; k < K; ++k) tot[k] = block_sum(v[k]);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) partials[size_t(blockIdx.x) * K + k] = tot[k];
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    // fixed order: thread t sums blocks t, t+blockDim, ...; then block_sum
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] += ((volatile double*)partials)[size_t(b) * K + k];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = block_sum(acc[k]);
        if (threadIdx.x == 0) out[k] = s;
    }
    if (threadIdx.x == 0) *counter = 0u;
}

// grid_sum_finish, but the totals go to thread 0 of the last block to
// finish (the call returns true there, false everywhere else) instead of
// being stored, so that block can act on them (scalar updates, decisions).
template <int K>
__device__ __forceinline__ bool grid_sum_last(double (&v)[K], double* partials, unsigned* counter, double (&tot)[K]) {
    __shared__ bool last;
    double part[K];
#pragma unroll
    for (int k = 0; k < K; ++k) part[k] = block_sum(v[k]);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) partials[size_t(blockIdx.x) * K + k] = part[k];
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] += ((volatile double*)partials)[size_t(b) * K + k];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = block_sum(acc[k]);
        if (threadIdx.x == 0) tot[k] = s;
    }
    if (threadIdx.x == 0) {
        *counter = 0u;
        return true;
    }
    return false;
}

}  // namespace lhi
