// noalloc.cu -- lhi_divergence_noalloc: the divergence diagnostic of
// LiquidModel<3>::ComputeDivergence for callers that cannot allocate device
// memory.
//
// Who needs it: a host that owns every byte of device memory itself (an
// engine with a fixed memory budget and its own pool), or a frame loop that
// must not stall (cudaMalloc / cudaFree may synchronise the whole device).
// Such a caller passes device pointers to fields it already holds and gets
// the same mean and max-norm as lhi_liquid_compute_divergence, without a
// handle and without any allocation.  The call synchronises the stream it is
// given, to return the two values.
//
// Scratch lives in one file-scope __device__ array (below): every GPU that
// loads the library holds it until the process exits.  In host code the
// array's name is only a host-side stand-in, so its device address is looked
// up once per device with cudaGetSymbolAddress and passed to the kernel.
// The stream must belong to the current device, whose copy of the array the
// kernel is given.
#include <mutex>
#include <vector>

#include "common.cuh"
#include "lhi.h"

namespace lhi {

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaCellsPerThread = 8;
constexpr int kNaCellsPerBlock = kNaThreads * kNaCellsPerThread;  // 2048
constexpr int kNaMaxBlocks = LHI_NOALLOC_MAX_CELLS / kNaCellsPerBlock;  // 8192
static_assert(LHI_NOALLOC_MAX_CELLS % kNaCellsPerBlock == 0, "cell limit must be whole blocks");

// Layout (doubles): [3 * kNaMaxBlocks] per-block partials (sum, count, max),
// then one slot holding the unsigned block counter, then the 3 results.
constexpr int kNaCounterSlot = 3 * kNaMaxBlocks;
constexpr int kNaResultSlot = kNaCounterSlot + 1;
constexpr int kNaScratchDoubles = kNaResultSlot + 3;

static __device__ __align__(256) double g_noalloc_scratch[kNaScratchDoubles];

std::mutex g_na_mutex;
std::vector<double*> g_na_ptr;  // per device ordinal, sized by the device count on first use

// Device address of the scratch array on the current device; looked up on
// the first call per device.
double* scratch_on_current_device() {
    int dev = 0, count = 0;
    LHI_CUDA(cudaGetDevice(&dev));
    LHI_CUDA(cudaGetDeviceCount(&count));
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (int(g_na_ptr.size()) < count) g_na_ptr.resize(size_t(count), nullptr);
    if (dev < 0 || dev >= int(g_na_ptr.size())) throw std::invalid_argument("current device ordinal out of range");
    if (!g_na_ptr[dev]) {
        void* p = nullptr;
        LHI_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_na_ptr[dev] = static_cast<double*>(p);
    }
    return g_na_ptr[dev];
}

// Per fluid cell divergence exactly as k_divergence (LiquidModel.cpp:1066-1083):
// same Scalar expression per cell; the sums are taken in double in a fixed
// block order, so results match the handle's call to double rounding.
template <class T>
__global__ void __launch_bounds__(kNaThreads)
    k_divergence_noalloc(int nx, int ny, int nz, T h, const T* __restrict__ phi, const T* __restrict__ lwx,
                         const T* __restrict__ lwy, const T* __restrict__ lwz, const T* __restrict__ vx,
                         const T* __restrict__ vy, const T* __restrict__ vz, double* __restrict__ scratch) {
    const long long n = (long long)nx * ny * nz;
    const long long base = (long long)blockIdx.x * kNaCellsPerBlock;
    double s = 0.0, cnt = 0.0, mx = 0.0;
#pragma unroll 1
    for (int k = 0; k < kNaCellsPerThread; ++k) {
        const long long c = base + (long long)k * kNaThreads + threadIdx.x;
        if (c >= n || phi[c] > T(0)) continue;
        const int z = int(c % nz), y = int((c / nz) % ny), x = int(c / ((long long)ny * nz));
        const long long fxi = ((long long)x * ny + y) * nz + z, fxs = (long long)ny * nz;
        const long long fyi = ((long long)x * (ny + 1) + y) * nz + z, fys = nz;
        const long long fzi = ((long long)x * ny + y) * (nz + 1) + z;
        T d = X<T>::sub(X<T>::mul(lwx[fxi + fxs], vx[fxi + fxs]), X<T>::mul(lwx[fxi], vx[fxi]));
        d = X<T>::add(d, X<T>::sub(X<T>::mul(lwy[fyi + fys], vy[fyi + fys]), X<T>::mul(lwy[fyi], vy[fyi])));
        d = X<T>::add(d, X<T>::sub(X<T>::mul(lwz[fzi + 1], vz[fzi + 1]), X<T>::mul(lwz[fzi], vz[fzi])));
        d = X<T>::div(d, h);
        s += double(d);
        cnt += 1.0;
        // max-norm over the cells whose six faces the velocity update touches
        if (x >= 1 && x <= nx - 3 && y >= 1 && y <= ny - 3 && z >= 1 && z <= nz - 3) mx = fmax(mx, fabs(double(d)));
    }
    const double bs = block_sum(s);
    const double bc = block_sum(cnt);
    const double bm = block_max(mx);
    __shared__ bool last;
    unsigned* counter = reinterpret_cast<unsigned*>(scratch + kNaCounterSlot);
    if (threadIdx.x == 0) {
        scratch[3 * blockIdx.x + 0] = bs;
        scratch[3 * blockIdx.x + 1] = bc;
        scratch[3 * blockIdx.x + 2] = bm;
        __threadfence();
        last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const volatile double* part = scratch;
    double a = 0.0, b = 0.0, m = 0.0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
        a += part[3 * k + 0];
        b += part[3 * k + 1];
        m = fmax(m, part[3 * k + 2]);
    }
    a = block_sum(a);
    b = block_sum(b);
    m = block_max(m);
    if (threadIdx.x == 0) {
        scratch[kNaResultSlot + 0] = a;
        scratch[kNaResultSlot + 1] = b;
        scratch[kNaResultSlot + 2] = m;
        *counter = 0u;
    }
}

template <class T>
void launch_noalloc(const int32_t dim[3], double dx, const void* phi, const void* lwx, const void* lwy,
                    const void* lwz, const void* vx, const void* vy, const void* vz, cudaStream_t s,
                    double* scratch) {
    const long long n = (long long)dim[0] * dim[1] * dim[2];
    const unsigned blocks = unsigned((n + kNaCellsPerBlock - 1) / kNaCellsPerBlock);
    k_divergence_noalloc<T><<<blocks, kNaThreads, 0, s>>>(
        dim[0], dim[1], dim[2], T(dx), static_cast<const T*>(phi), static_cast<const T*>(lwx),
        static_cast<const T*>(lwy), static_cast<const T*>(lwz), static_cast<const T*>(vx),
        static_cast<const T*>(vy), static_cast<const T*>(vz), scratch);
    LHI_LAUNCH_CHECK();
}

}  // namespace

// Entry point body; argument checks are in api.cu's C wrapper style.
int divergence_noalloc(const int32_t dim[3], double dx, int32_t precision, const void* liquid_phi,
                       const void* liquid_wx, const void* liquid_wy, const void* liquid_wz, const void* vx,
                       const void* vy, const void* vz, void* stream, double* mean, double* max_abs) {
    if (!dim || !liquid_phi || !liquid_wx || !liquid_wy || !liquid_wz || !vx || !vy || !vz)
        throw std::invalid_argument("null argument");
    if (dim[0] < 1 || dim[1] < 1 || dim[2] < 1) throw std::invalid_argument("grid dimensions must be >= 1");
    const long long n = (long long)dim[0] * dim[1] * dim[2];
    if (n > LHI_NOALLOC_MAX_CELLS)
        throw std::invalid_argument("lhi_divergence_noalloc: " + std::to_string(n) +
                                    " cells exceed the fixed scratch limit of " +
                                    std::to_string(LHI_NOALLOC_MAX_CELLS) + " cells (256^3)");
    if (!(dx > 0.0)) throw std::invalid_argument("dx must be > 0");
    if (precision != LHI_PRECISION_FP32 && precision != LHI_PRECISION_MIXED && precision != LHI_PRECISION_FP64)
        throw std::invalid_argument("unknown precision");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* scratch = scratch_on_current_device();
    // the block counter must start at zero even if an earlier launch was cut short
    LHI_CUDA(cudaMemsetAsync(scratch + kNaCounterSlot, 0, sizeof(double), s));
    if (precision == LHI_PRECISION_FP64)
        launch_noalloc<double>(dim, dx, liquid_phi, liquid_wx, liquid_wy, liquid_wz, vx, vy, vz, s, scratch);
    else
        launch_noalloc<float>(dim, dx, liquid_phi, liquid_wx, liquid_wy, liquid_wz, vx, vy, vz, s, scratch);
    double res[3];
    LHI_CUDA(cudaMemcpyAsync(res, scratch + kNaResultSlot, sizeof(res), cudaMemcpyDeviceToHost, s));
    LHI_CUDA(cudaStreamSynchronize(s));
    if (mean) *mean = (res[1] > 0) ? res[0] / res[1] : std::nan("");
    if (max_abs) *max_abs = res[2];
    return LHI_OK;
}

}  // namespace lhi
