// k_sort.cu -- device-wide exclusive scan and the stable LSD radix sort that
// orders particles by cell key (the first half of the sorted P2G).
//
// Radix sort: 8-bit digits, one histogram pass and one scatter pass per digit.
// A tile is 4096 keys handled by 8 warps; each warp owns 512 consecutive keys
// and walks them 32 at a time, so the in-tile order is (warp, round, lane),
// i.e. the input order.  Ranks inside a round come from __match_any_sync, so
// equal digits keep their input order: the sort is stable.  The scatter
// stages its tile in shared memory in digit order and writes every digit's
// run of keys to consecutive global positions.
#include "impl.cuh"

namespace lhi {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;  // 4096 keys
constexpr int kRadix = 256;

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

__global__ void k_radix_hist(const uint32_t* __restrict__ keys, long long n, int shift, uint32_t* __restrict__ hist,
                             long long ntiles) {
    __shared__ uint32_t cnt[kRadix];
    for (int i = threadIdx.x; i < kRadix; i += kSortThreads) cnt[i] = 0;
    __syncthreads();
    long long base = (long long)blockIdx.x * kSortTile;
    for (int i = threadIdx.x; i < kSortTile; i += kSortThreads) {
        long long k = base + i;
        if (k < n) atomicAdd(&cnt[(keys[k] >> shift) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kSortThreads) hist[(long long)d * ntiles + blockIdx.x] = cnt[d];
}

__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const uint32_t* __restrict__ kin, const int32_t* __restrict__ vin,
                                               uint32_t* __restrict__ kout, int32_t* __restrict__ vout, long long n,
                                               int shift, const int32_t* __restrict__ offs, long long ntiles) {
    __shared__ uint32_t wcnt[kSortWarps][kRadix];
    for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    const long long wbase = (long long)blockIdx.x * kSortTile + (long long)w * (kSortRounds * 32);
    uint32_t key[kSortRounds];
    int32_t val[kSortRounds];
    uint32_t rank[kSortRounds];
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        long long idx = wbase + r * 32 + lane;
        bool valid = idx < n;
        key[r] = valid ? kin[idx] : 0u;
        val[r] = valid ? vin[idx] : 0;
        unsigned d = (key[r] >> shift) & (kRadix - 1);
        unsigned tag = valid ? d : (kRadix + lane);  // invalid lanes never match
        unsigned peers = __match_any_sync(0xffffffffu, tag);
        unsigned before = valid ? wcnt[w][d] : 0u;
        rank[r] = before + __popc(peers & lt_mask);
        __syncwarp();
        if (valid && (peers & lt_mask) == 0u) wcnt[w][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // exclusive prefix over warps, digit by digit, then over digits: the
    // tile-local start of every digit
    __shared__ uint32_t dstart[kRadix];
    __shared__ uint32_t dsum[kSortWarps];
    static_assert(kSortThreads == kRadix, "one thread per digit");
    {
        const int d = threadIdx.x;
        uint32_t run = 0;
        for (int k = 0; k < kSortWarps; ++k) {
            uint32_t c = wcnt[k][d];
            wcnt[k][d] = run;
            run += c;
        }
        uint32_t incl = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) dsum[w] = incl;
        __syncthreads();
        uint32_t wofs = 0;
        for (int k = 0; k < w; ++k) wofs += dsum[k];
        dstart[d] = wofs + incl - run;
    }
    __syncthreads();
    // stage the tile in digit order (input order inside a digit) ...
    __shared__ uint32_t skey[kSortTile];
    __shared__ int32_t sval[kSortTile];
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        long long idx = wbase + r * 32 + lane;
        if (idx < n) {
            unsigned d = (key[r] >> shift) & (kRadix - 1);
            const uint32_t lp = dstart[d] + wcnt[w][d] + rank[r];
            skey[lp] = key[r];
            sval[lp] = val[r];
        }
    }
    __syncthreads();
    // ... and write each digit's run to consecutive global positions
    const long long tbase = (long long)blockIdx.x * kSortTile;
    const int tn = int(min((long long)kSortTile, n - tbase));
    for (int i = threadIdx.x; i < tn; i += kSortThreads) {
        const uint32_t k = skey[i];
        const unsigned d = (k >> shift) & (kRadix - 1);
        const long long pos = (long long)offs[(long long)d * ntiles + blockIdx.x] + (i - int(dstart[d]));
        kout[pos] = k;
        vout[pos] = sval[i];
    }
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

long long radix_hist_entries(long long n) {
    long long ntiles = (n + kSortTile - 1) / kSortTile;
    return (long long)kRadix * (ntiles < 1 ? 1 : ntiles);
}

void radix_sort_pairs(uint32_t* keys[2], int32_t* vals[2], int& cur, long long n, int key_bits, uint32_t* hist,
                      void* tmp, long long tmp_bytes, cudaStream_t s) {
    if (n <= 1) return;
    long long ntiles = (n + kSortTile - 1) / kSortTile;
    long long nh = (long long)kRadix * ntiles;
    for (int shift = 0; shift < key_bits; shift += 8) {
        k_radix_hist<<<unsigned(ntiles), kSortThreads, 0, s>>>(keys[cur], n, shift, hist, ntiles);
        LHI_LAUNCH_CHECK();
        device_exclusive_scan_i32(reinterpret_cast<int32_t*>(hist), reinterpret_cast<int32_t*>(hist), nh, tmp,
                                  tmp_bytes, s);
        k_radix_scatter<<<unsigned(ntiles), kSortThreads, 0, s>>>(keys[cur], vals[cur], keys[cur ^ 1],
                                                                   vals[cur ^ 1], n, shift,
                                                                   reinterpret_cast<int32_t*>(hist), ntiles);
        LHI_LAUNCH_CHECK();
        cur ^= 1;
    }
}

}  // namespace lhi
