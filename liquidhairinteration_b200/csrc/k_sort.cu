// k_sort.cu -- device-wide exclusive scan (the per-cell particle ranges of
// the counting sort by cell key, k_particles.cu).
#include "impl.cuh"

namespace lhi {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;


__global__ void k_scan_reduce(const int32_t* __restrict__ in, long long n, int32_t* __restrict__ sums) {
    long long base = (long long)blockIdx.x * kScanTile;
    int s = 0;
    for (int i = threadIdx.x; i < kScanTile; i += kScanThreads) {
        long long k = base + i;
        if (k < n) s += in[k];
    }
    s = block_sum(s);
    if (threadIdx.x == 0) sums[blockIdx.x] = s;
}

// Exclusive scan of one tile plus the tile's offset.  In-place safe: each
// thread reads its 16 items before writing them and tiles are disjoint.
__global__ void k_scan_down(const int32_t* in, int32_t* out, long long n, const int32_t* __restrict__ offs) {
    __shared__ int ws[kScanThreads / 32];
    long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int v[kScanItems];
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) v[i] = (base + i < n) ? in[base + i] : 0;
    int t = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        int x = v[i];
        v[i] = t;
        t += x;
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) ws[w] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int k = 0; k < kScanThreads / 32; ++k) {
            int c = ws[k];
            ws[k] = run;
            run += c;
        }
    }
    __syncthreads();
    int excl = incl - t + ws[w] + (offs ? offs[blockIdx.x] : 0);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
        if (base + i < n) out[base + i] = excl + v[i];
}

long long align_up(long long x, long long a) { return (x + a - 1) / a * a; }

void scan_rec(const int32_t* in, int32_t* out, long long n, int32_t* tmp, cudaStream_t s) {
    long long nb = (n + kScanTile - 1) / kScanTile;
    if (nb <= 1) {
        k_scan_down<<<1, kScanThreads, 0, s>>>(in, out, n, nullptr);
        LHI_LAUNCH_CHECK();
        return;
    }
    int32_t* sums = tmp;
    tmp += align_up(nb, 64);
    k_scan_reduce<<<unsigned(nb), kScanThreads, 0, s>>>(in, n, sums);
    LHI_LAUNCH_CHECK();
    scan_rec(sums, sums, nb, tmp, s);
    k_scan_down<<<unsigned(nb), kScanThreads, 0, s>>>(in, out, n, sums);
    LHI_LAUNCH_CHECK();
}

}  // namespace

long long scan_tmp_bytes(long long n) {
    long long total = 0;
    while (true) {
        long long nb = (n + kScanTile - 1) / kScanTile;
        if (nb <= 1) break;
        total += align_up(nb, 64);
        n = nb;
    }
    return (total + 64) * 4;
}

void device_exclusive_scan_i32(const int32_t* in, int32_t* out, long long n, void* tmp, long long tmp_bytes,
                               cudaStream_t s) {
    if (n <= 0) return;
    if (tmp_bytes < scan_tmp_bytes(n)) throw std::runtime_error("scan scratch too small");
    scan_rec(in, out, n, static_cast<int32_t*>(tmp), s);
}

}  // namespace lhi
