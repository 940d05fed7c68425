// k_learned.cu -- the learned preconditioner's kernels on sm_100a.
//
// Convolutions are implicit GEMMs on the 5th-generation tensor cores:
//   forward / input gradient: D[voxel][cout] += A[voxel][cin] * B[cout][cin]
//     per tap; M = 128 voxels per CTA, N = cout (16/32/64), K = 27 taps x cin.
//     A rows are gathered (zero padding at the grid edge) from channels-last
//     BF16 activations into shared memory in the UMMA K-major core-matrix
//     layout; B is the tap's pre-formatted weight tile.
//   weight gradient: D[cout][cin] += A[cout][voxel] * B[cin][voxel] per tap
//     with K = voxels; both operands are MN-major, which is what
//     channels-last activations already are, so each voxel's channels are
//     one 16-byte shared-memory store.
// One thread issues tcgen05.mma into a TMEM accumulator; tcgen05.commit
// arrives on an mbarrier; the epilogue reads TMEM with tcgen05.ld.  The
// gathering kernel (k_conv) stages two taps at a time; the brick kernel
// (k_conv_brick, every layer of this network) stages each output tile's
// input brick once by TMA and runs its tiles as a warp-specialised pipeline
// over two accumulators.  The solver's forward passes run tile-sparse: a
// plan (plan_sparse) lists, per stage, the tiles the cells with type != 0
// depend on.
// Every mbarrier wait is bounded: on timeout the kernel records it in
// NetStatus, waits (bounded) for its own copies and MMAs in flight, frees
// TMEM and returns.
#include <algorithm>
#include <cmath>
#include <random>

#include "net.cuh"
#include "lhi.h"
#include "tma.cuh"

namespace lhi {

namespace {

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for the completion of the barrier phase with this parity:
// non-blocking test_wait polled against a 200 ms deadline.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    const uint32_t addr = smem_u32(bar);
    const uint64_t deadline = global_ns() + 200000000ull;
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if (global_ns() > deadline) return false;
    }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// warp-wide
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// UMMA shared-memory descriptor, no swizzle (canonical INTERLEAVE layout):
// start address, leading (K-direction) and stride (M/N-direction) byte
// offsets between 8 x 16-byte core matrices, version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3FFFu);
    d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
    d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
    d |= uint64_t(1) << 46;
    return d;
}

// Instruction descriptor of kind::f16: BF16 x BF16 -> F32, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(a_mn) << 15) | (uint32_t(b_mn) << 16) |
           (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(d_tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// warp-collective: callers reconverge the warp first (__syncwarp)
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void tap_offset(int tap, int& dx, int& dy, int& dz) {
    dx = tap / 9 - 1;
    dy = (tap / 3) % 3 - 1;
    dz = tap % 3 - 1;
}

// ------------------------------------------------------------ convolution
constexpr int kConvM = 128;  // voxels per CTA

struct ConvParams {
    const uint16_t* in;   // channels-last BF16, cin channels
    int cin;              // padded: 16, 32 or 64
    const uint16_t* w;    // 27 formatted B tiles [cout][cin]
    int cout;             // padded: 16, 32 or 64
    const float* bias;    // cout_real entries or null
    int cout_real;
    int nx, ny, nz;
    long long nvox;
    int mode;             // 0: BF16 out (+bias +skip, relu); 1: FP32 out, all channels; 2: FP32 channel 0 + bias
    const uint16_t* skip; // BF16, cout channels (mode 0), or null
    int relu;
    uint16_t* out_b;
    float* out_f;
    NetStatus* status;
    const int32_t* tiles;  // brick kernel: the output tiles to evaluate (indices as the dense loop's), or null: all
    const int* ntiles;     // their count (device)
};

// Epilogue of one output row (TMEM lane = this thread's row; warp-collective
// loads, so every lane calls it and only valid rows store): mode 0 BF16 with
// bias, skip and activation; mode 1 FP32, all channels; mode 2 FP32 channel 0.
__device__ __forceinline__ void conv_store(const ConvParams& P, uint32_t trow, bool valid, long long v) {
    if (P.mode == 2) {
        float a[8];
        tmem_ld8(trow, a);
        if (valid) P.out_f[v] = a[0] + (P.bias ? P.bias[0] : 0.f);
        return;
    }
    for (int c0 = 0; c0 < P.cout; c0 += 8) {
        float a[8];
        tmem_ld8(trow + c0, a);
        if (!valid) continue;
        if (P.mode == 1) {
            float4* o = reinterpret_cast<float4*>(P.out_f + v * P.cout + c0);
            o[0] = make_float4(a[0], a[1], a[2], a[3]);
            o[1] = make_float4(a[4], a[5], a[6], a[7]);
        } else {
            uint16_t sk[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            if (P.skip) *reinterpret_cast<uint4*>(sk) = *reinterpret_cast<const uint4*>(P.skip + v * P.cout + c0);
            uint16_t o[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int c = c0 + k;
                float val = a[k];
                if (P.bias && c < P.cout_real) val += P.bias[c];
                if (P.skip) val += bf16_float(sk[k]);
                if (P.relu) val = fmaxf(val, 0.f);
                o[k] = (c < P.cout_real) ? bf16_bits(val) : uint16_t(0);
            }
            *reinterpret_cast<uint4*>(P.out_b + v * P.cout + c0) = *reinterpret_cast<uint4*>(o);
        }
    }
}

// out[v][n] = sum_tap sum_k in[v + off(tap)][k] * w[tap][n][k]
__global__ void __launch_bounds__(kConvM) k_conv(ConvParams P) {
    extern __shared__ __align__(1024) uint8_t sm[];
    const int abytes = kConvM * P.cin * 2;
    const int bbytes = P.cout * P.cin * 2;
    uint8_t* A[2] = {sm, sm + abytes};
    uint8_t* B[2] = {sm + 2 * abytes, sm + 2 * abytes + bbytes};
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + 2 * abytes + 2 * bbytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2);
    __shared__ int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t ncols = P.cout < 32 ? 32u : uint32_t(P.cout);
    if (tid == 0) {
        abort_flag = 0;
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) tmem_alloc(tslot, ncols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    const long long v = (long long)blockIdx.x * kConvM + tid;
    const bool valid = v < P.nvox;
    int x = 0, y = 0, z = 0;
    if (valid) {
        z = int(v % P.nz);
        const long long t = v / P.nz;
        y = int(t % P.ny);
        x = int(t / P.ny);
    }
    const int kc = P.cin / 8;             // 16-byte chunks per A/B row
    const uint32_t sbo = uint32_t(kc) * 128;
    const uint32_t idesc = idesc_bf16(kConvM, P.cout, 0, 0);
    int last_tap = -1;
    for (int tap = 0; tap < kNetTaps; ++tap) {
        const int s = tap & 1;
        if (tap >= 2 && !mbar_wait(&bar[s], unsigned((tap - 2) >> 1) & 1u)) abort_flag = 1;
        int dx, dy, dz;
        tap_offset(tap, dx, dy, dz);
        const int xx = x + dx, yy = y + dy, zz = z + dz;
        const bool in = valid && xx >= 0 && xx < P.nx && yy >= 0 && yy < P.ny && zz >= 0 && zz < P.nz;
        const uint4* src = reinterpret_cast<const uint4*>(P.in + (((long long)xx * P.ny + yy) * P.nz + zz) * P.cin);
        uint8_t* arow = A[s] + (tid >> 3) * sbo + (tid & 7) * 16;
        for (int c = 0; c < kc; ++c) {
            const uint4 val = in ? src[c] : make_uint4(0u, 0u, 0u, 0u);
            *reinterpret_cast<uint4*>(arow + c * 128) = val;
        }
        const uint4* wsrc = reinterpret_cast<const uint4*>(P.w + (long long)tap * P.cout * P.cin);
        for (int i = tid; i < bbytes / 16; i += kConvM) reinterpret_cast<uint4*>(B[s])[i] = wsrc[i];
        fence_async_smem();
        __syncthreads();
        if (abort_flag) break;
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(A[s]), b0 = smem_u32(B[s]);
            for (int k = 0; k < P.cin / 16; ++k)
                umma_bf16(tmem, sdesc(a0 + k * 256, 128, sbo), sdesc(b0 + k * 256, 128, sbo), idesc,
                          (tap > 0 || k > 0) ? 1u : 0u);
            umma_commit(&bar[s]);
        }
        last_tap = tap;
    }
    bool ok = !abort_flag;
    if (last_tap >= 0 && !mbar_wait(&bar[last_tap & 1], unsigned(last_tap >> 1) & 1u)) ok = false;
    tc_fence_after();
    __syncwarp();
    // tcgen05.ld is warp-collective: every lane loads, only valid rows store
    if (ok) {
        conv_store(P, tmem + (uint32_t(warp * 32) << 16), valid, v);
    } else if (!ok && valid) {
        // keep the tensor well defined after a timeout
        if (P.mode == 2) P.out_f[v] = 0.f;
    }
    if (!ok && tid == 0 && atomicExch(&P.status->timeout, 1) == 0) {
        P.status->pad[0] = 1;  // kernel: convolution
        P.status->pad[1] = last_tap;
        P.status->pad[2] = int(blockIdx.x);
    }
    tc_fence_before();
    __syncthreads();
    __syncwarp();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ------------------------------------------------------ brick convolution
// The same convolution with the 27 taps reading one staged input brick
// instead of 27 gathers (every layer whose weights and brick fit in shared
// memory).
// An output tile is 128 voxels: one x plane, 16 y rows, 8 z (TMEM lane /
// A row r = (y - y0) * 8 + (z - z0)).  Its input brick, grown by one voxel
// (3 x 18 x 10), sits in shared memory as one plane per 8-channel chunk with
// z fastest, so for any tap the 8 z of a y row are one contiguous 8 x 16-byte
// core matrix: the tap's A operand is the brick at offset (dx, dy, dz), with
// M-direction stride one brick row (160 bytes) and K-direction stride one
// plane.  Each plane is one TMA box {8 channels, 10 z, 18 y, 3 x} of the
// channels-last activations (a 4D tensor map, channels innermost), which
// reads zeros outside the grid: the convolution's zero padding.
//
// CTAs are persistent, keep all 27 weight tiles resident and run their tiles
// as a warp-specialised pipeline over two TMEM accumulators: warp 4 (one
// lane) loads the bricks and issues each tile's MMAs (compile-time
// descriptor offsets from two bases); warps 0-3 drain the accumulators, each
// its 32 TMEM lanes.  They hand over through mbarriers only: a brick has
// landed, a tile's MMAs are done, an accumulator is drained.  Where shared
// memory holds two bricks, tile i + 1's brick loads while tile i's MMAs run.
constexpr int kBrX = 3, kBrY = 18, kBrZ = 10;
constexpr int kBrVox = kBrX * kBrY * kBrZ;  // 540
constexpr int kBrBox = kBrVox * 16;         // bytes of one 8-channel plane (one TMA box)
constexpr int kBrPlane = 68 * 128;          // plane stride: the box rounded up to 128 bytes
constexpr size_t kBrickSmemMax = 227 * 1024;
constexpr int kBrBars = 64;                 // six mbarriers, the TMEM address slot and the abort flag
constexpr int kBrThreads = 160;             // warps 0-3 drain, warp 4 produces

// Shared-memory bytes of the brick kernel for one layer with `stages` bricks.
__host__ __device__ constexpr size_t brick_smem_bytes(int cin, int cout, int stages) {
    return size_t(27) * cout * cin * 2 + size_t(stages) * (cin / 8) * kBrPlane + kBrBars;
}

__device__ __forceinline__ void brick_tile(const ConvParams& P, long long t, int tyn, int tzn, int& x0, int& y0,
                                           int& z0) {
    const long long tt = P.tiles ? (long long)P.tiles[t] : t;
    const int tzi = int(tt % tzn);
    const long long rest = tt / tzn;
    y0 = int(rest % tyn) * 16;
    x0 = int(rest / tyn);
    z0 = tzi * 8;
}

// one thread: the kc planes of tile t's brick into buf
__device__ __forceinline__ void brick_issue(const CUtensorMap* tin, const ConvParams& P, long long t, int tyn, int tzn,
                                            int kc, uint8_t* buf, uint64_t* bar) {
    int x0, y0, z0;
    brick_tile(P, t, tyn, tzn, x0, y0, z0);
    bar_expect_tx(bar, uint32_t(kc * kBrBox));
    for (int c = 0; c < kc; ++c) tma_load_box4(buf + c * kBrPlane, tin, c * 8, z0 - 1, y0 - 1, x0 - 1, bar);
}

// one thread: the 27 x CIN/16 MMAs of one tile, accumulating into acc
template <int CIN, int COUT>
__device__ __forceinline__ void brick_mmas(uint32_t acc, uint32_t a_stage, uint32_t b0) {
    constexpr int KC = CIN / 8;
    constexpr uint32_t idesc = idesc_bf16(kConvM, COUT, 0, 0);
    const uint64_t ad0 = sdesc(a_stage, kBrPlane, kBrZ * 16);
    const uint64_t bd0 = sdesc(b0, 128, uint32_t(KC) * 128);
#pragma unroll
    for (int tap = 0; tap < kNetTaps; ++tap) {
        const int dx = tap / 9, dy = (tap / 3) % 3, dz = tap % 3;  // offsets + 1
        const uint64_t aoff = uint64_t(((dx * kBrY + dy) * kBrZ + dz) * 16) >> 4;
#pragma unroll
        for (int k = 0; k < CIN / 16; ++k)
            umma_bf16(acc, ad0 + aoff + (uint64_t(2 * k * kBrPlane) >> 4),
                      bd0 + (uint64_t(tap * COUT * CIN * 2 + k * 256) >> 4), idesc, (tap > 0 || k > 0) ? 1u : 0u);
    }
}

// Epilogue of one output row (TMEM lane = this thread's row; the loads are
// warp-collective, so every lane calls it and only valid rows store), the
// arithmetic of conv_store: mode 0 BF16 with bias, skip (sk, loaded ahead)
// and activation; mode 1 FP32, all channels; mode 2 FP32 channel 0.
template <int COUT>
__device__ __forceinline__ void brick_store(const ConvParams& P, uint32_t trow, bool valid, long long v,
                                            const uint4 (&sk)[COUT / 8]) {
    if (P.mode == 2) {
        float a[8];
        tmem_ld8(trow, a);
        if (valid) P.out_f[v] = a[0] + (P.bias ? P.bias[0] : 0.f);
        return;
    }
#pragma unroll
    for (int q = 0; q < COUT / 8; ++q) {
        const int c0 = q * 8;
        float a[8];
        tmem_ld8(trow + c0, a);
        if (!valid) continue;
        if (P.mode == 1) {
            float4* o = reinterpret_cast<float4*>(P.out_f + v * COUT + c0);
            o[0] = make_float4(a[0], a[1], a[2], a[3]);
            o[1] = make_float4(a[4], a[5], a[6], a[7]);
        } else {
            uint16_t s8[8];
            *reinterpret_cast<uint4*>(s8) = sk[q];
            uint16_t o[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int c = c0 + k;
                float val = a[k];
                if (P.bias && c < P.cout_real) val += P.bias[c];
                if (P.skip) val += bf16_float(s8[k]);
                if (P.relu) val = fmaxf(val, 0.f);
                o[k] = (c < P.cout_real) ? bf16_bits(val) : uint16_t(0);
            }
            *reinterpret_cast<uint4*>(P.out_b + v * COUT + c0) = *reinterpret_cast<uint4*>(o);
        }
    }
}

// Limit of the brick convolution's pipeline waits (200 ms;
// lhi_debug_set_stage_wait_limit lowers it to test the timeout path, 0
// gives up at once).  The waits for a CTA's own copies and MMAs in flight
// before it leaves keep the fixed 200 ms.
__device__ unsigned long long g_net_wait_ns = 200000000ull;

// Bounded wait on a pipeline barrier that also gives up once another warp of
// the CTA has set the abort flag (a wait of its own that timed out).
__device__ __forceinline__ bool brick_wait(uint64_t* bar, unsigned parity, volatile int* abort_flag) {
    const unsigned long long limit = g_net_wait_ns;
    if (limit == 0) return false;
    const uint32_t addr = smem_u32(bar);
    const uint64_t deadline = global_ns() + limit;
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        if (ok) return true;
        if (*abort_flag || global_ns() > deadline) return false;
    }
}

// Barriers: full[2] (a brick stage has landed), done[2] (an accumulator's
// MMAs completed), empty[2] (an accumulator has been drained: one arrival
// per draining warp).  Tile i of this CTA uses accumulator i & 1 and, with
// two bricks, brick i & 1.
template <int CIN, int COUT>
__global__ void __launch_bounds__(kBrThreads) k_conv_brick(const __grid_constant__ CUtensorMap tin, ConvParams P,
                                                           int stages) {
    extern __shared__ __align__(1024) uint8_t sm[];
    constexpr int KC = CIN / 8;
    constexpr int WBYTES = COUT * CIN * 2;  // one tap's B tile
    constexpr uint32_t NCOLS = COUT < 32 ? 32u : uint32_t(COUT);
    uint8_t* Bs = sm;
    uint8_t* Ab = sm + 27 * WBYTES;  // brick s at Ab + s * KC * kBrPlane
    uint64_t* full = reinterpret_cast<uint64_t*>(Ab + stages * KC * kBrPlane);
    uint64_t* done = full + 2;
    uint64_t* empty = full + 4;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(full + 6);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) {
            mbar_init(&full[b], 1);
            mbar_init(&done[b], 1);
            mbar_init(&empty[b], 4);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) tmem_alloc(tslot, 2 * NCOLS);
    for (int i = tid; i < 27 * WBYTES / 16; i += kBrThreads)
        reinterpret_cast<uint4*>(Bs)[i] = reinterpret_cast<const uint4*>(P.w)[i];
    fence_async_smem();  // the weight tiles (generic stores) before the tensor cores read them
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const int tyn = (P.ny + 15) / 16, tzn = (P.nz + 7) / 8;
    const long long ntiles = P.tiles ? (long long)*P.ntiles : (long long)P.nx * tyn * tzn;
    const long long G = gridDim.x;
    const int nmine = (long long)blockIdx.x < ntiles ? int((ntiles - 1 - blockIdx.x) / G) + 1 : 0;
    if (warp == 4) {
        // ---- producer (one lane)
        if (lane == 0 && nmine > 0) {
            bool pending[2] = {false, false};  // a brick load in flight, not yet waited for
            unsigned use[2] = {0u, 0u};        // completed waits per brick barrier: its next phase's parity
            int last_commit = -1;
            bool ok = true;
            auto brick_buf = [&](int s) { return Ab + s * KC * kBrPlane; };
            brick_issue(&tin, P, blockIdx.x, tyn, tzn, KC, brick_buf(0), &full[0]);
            pending[0] = true;
            for (int i = 0; i < nmine; ++i) {
                const long long t = blockIdx.x + (long long)i * G;
                const int s = stages == 2 ? (i & 1) : 0, b = i & 1;
                if (stages == 1 && i > 0) {
                    // the one brick was read by tile i - 1's MMAs
                    if (!(ok = brick_wait(&done[(i - 1) & 1], unsigned((i - 1) >> 1) & 1u, abort_flag))) break;
                    brick_issue(&tin, P, t, tyn, tzn, KC, brick_buf(0), &full[0]);
                    pending[0] = true;
                }
                if (!(ok = brick_wait(&full[s], use[s] & 1u, abort_flag))) break;
                pending[s] = false;
                ++use[s];
                // accumulator b was last drained after tile i - 2
                if (i >= 2 && !(ok = brick_wait(&empty[b], unsigned((i >> 1) + 1) & 1u, abort_flag))) break;
                tc_fence_after();
                brick_mmas<CIN, COUT>(tmem + uint32_t(b) * NCOLS, smem_u32(brick_buf(s)), smem_u32(Bs));
                umma_commit(&done[b]);
                last_commit = i;
                if (stages == 2 && i + 1 < nmine) {
                    // the other brick was read by tile i - 1's MMAs
                    if (i >= 1 && !(ok = brick_wait(&done[(i - 1) & 1], unsigned((i - 1) >> 1) & 1u, abort_flag)))
                        break;
                    brick_issue(&tin, P, t + G, tyn, tzn, KC, brick_buf(s ^ 1), &full[s ^ 1]);
                    pending[s ^ 1] = true;
                }
            }
            if (!ok) {
                *abort_flag = 1;
                if (atomicExch(&P.status->timeout, 1) == 0) {
                    P.status->pad[0] = 3;  // kernel: brick convolution
                    P.status->pad[2] = int(blockIdx.x);
                }
                // no brick load or MMA of this CTA may still be in flight when it exits
                for (int s2 = 0; s2 < 2; ++s2)
                    if (pending[s2]) mbar_wait(&full[s2], use[s2] & 1u);
                if (last_commit >= 0) mbar_wait(&done[last_commit & 1], unsigned(last_commit >> 1) & 1u);
            }
        }
        __syncwarp();
    } else {
        // ---- drain: warp w reads TMEM lanes 32w .. 32w + 31
        for (int i = 0; i < nmine; ++i) {
            const long long t = blockIdx.x + (long long)i * G;
            const int b = i & 1;
            int x0, y0, z0;
            brick_tile(P, t, tyn, tzn, x0, y0, z0);
            const int y = y0 + (tid >> 3), z = z0 + (tid & 7);
            const bool valid = y < P.ny && z < P.nz;
            const long long v = ((long long)x0 * P.ny + y) * P.nz + z;
            uint4 sk[COUT / 8];
#pragma unroll
            for (int q = 0; q < COUT / 8; ++q) sk[q] = make_uint4(0u, 0u, 0u, 0u);
            if (valid && P.mode == 0 && P.skip) {  // loaded while the MMAs run
                const uint4* src = reinterpret_cast<const uint4*>(P.skip + v * COUT);
#pragma unroll
                for (int q = 0; q < COUT / 8; ++q) sk[q] = src[q];
            }
            // one decision per warp: the TMEM loads are warp-collective
            if (!__all_sync(0xffffffffu, brick_wait(&done[b], unsigned(i >> 1) & 1u, abort_flag))) {
                if (lane == 0) *abort_flag = 1;
                break;
            }
            tc_fence_after();
            brick_store<COUT>(P, tmem + uint32_t(b) * NCOLS + (uint32_t(warp * 32) << 16), valid, v, sk);
            tc_fence_before();
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&empty[b])) : "memory");
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, 2 * NCOLS);
}

// ------------------------------------------------------- weight gradient
constexpr int kWgChunk = 128;        // voxels per MMA batch (K)
constexpr int kWgChunksPerCta = 16;

struct WgradParams {
    const uint16_t* g;   // BF16 gradient at the layer output, cout channels (padded)
    int cout;            // padded
    int cout_real;
    const uint16_t* in;  // BF16 layer input, cin channels (padded)
    int cin;             // padded
    int cin_real;
    int nx, ny, nz;
    long long nvox;
    float* grad_w;       // packed W[27][cout_real][cin_real] of the layer
    NetStatus* status;
};

// D[co][ci] = sum_v g[v][co] * in[v + off(tap)][ci] for tap = blockIdx.y over
// kWgChunksPerCta chunks of 128 voxels; A rows co >= cout stay zero.
__global__ void __launch_bounds__(128) k_wgrad(WgradParams P) {
    extern __shared__ __align__(1024) uint8_t sm[];
    constexpr int abytes = 128 * kWgChunk * 2;  // M = 128 rows (cout padded to 128 with zeros)
    const int bbytes = P.cin * kWgChunk * 2;
    uint8_t* A[2] = {sm, sm + abytes};
    uint8_t* B[2] = {sm + 2 * abytes, sm + 2 * abytes + bbytes};
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + 2 * abytes + 2 * bbytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2);
    __shared__ int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t ncols = P.cin < 32 ? 32u : uint32_t(P.cin);
    // zero both A stages once (rows >= cout are never written again)
    for (int i = tid; i < 2 * abytes / 16; i += 128) reinterpret_cast<uint4*>(sm)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (tid == 0) {
        abort_flag = 0;
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) tmem_alloc(tslot, ncols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const int tap = blockIdx.y;
    int dx, dy, dz;
    tap_offset(tap, dx, dy, dz);
    // MN-major layout: element (m, k) at (m / 8) * SBO + (k / 8) * 128 + (k % 8) * 16 + (m % 8) * 2
    constexpr uint32_t sbo = (kWgChunk / 8) * 128;
    const uint32_t idesc = idesc_bf16(128, P.cin, 1, 1);
    int issued = 0;
    const long long vbase = (long long)blockIdx.x * kWgChunksPerCta * kWgChunk;
    for (int ch = 0; ch < kWgChunksPerCta; ++ch) {
        const long long v0 = vbase + (long long)ch * kWgChunk;
        if (v0 >= P.nvox) break;
        const int s = ch & 1;
        if (ch >= 2 && !mbar_wait(&bar[s], unsigned((ch - 2) >> 1) & 1u)) abort_flag = 1;
        const long long v = v0 + tid;  // voxel k = tid of this chunk
        bool vin = v < P.nvox, src_in = false;
        long long src = 0;
        if (vin) {
            const int z = int(v % P.nz);
            const long long t = v / P.nz;
            const int y = int(t % P.ny), x = int(t / P.ny);
            const int xx = x + dx, yy = y + dy, zz = z + dz;
            src_in = xx >= 0 && xx < P.nx && yy >= 0 && yy < P.ny && zz >= 0 && zz < P.nz;
            src = ((long long)xx * P.ny + yy) * P.nz + zz;
        }
        const uint32_t koff = (tid >> 3) * 128 + (tid & 7) * 16;
        for (int c = 0; c < P.cout / 8; ++c) {
            const uint4 val = vin ? reinterpret_cast<const uint4*>(P.g + v * P.cout)[c] : make_uint4(0u, 0u, 0u, 0u);
            *reinterpret_cast<uint4*>(A[s] + c * sbo + koff) = val;
        }
        for (int c = 0; c < P.cin / 8; ++c) {
            const uint4 val = src_in ? reinterpret_cast<const uint4*>(P.in + src * P.cin)[c] : make_uint4(0u, 0u, 0u, 0u);
            *reinterpret_cast<uint4*>(B[s] + c * sbo + koff) = val;
        }
        fence_async_smem();
        __syncthreads();
        if (abort_flag) break;
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(A[s]), b0 = smem_u32(B[s]);
            for (int k = 0; k < kWgChunk / 16; ++k)
                umma_bf16(tmem, sdesc(a0 + k * 256, 128, sbo), sdesc(b0 + k * 256, 128, sbo), idesc,
                          (issued > 0 || k > 0) ? 1u : 0u);
            umma_commit(&bar[s]);
        }
        issued = ch + 1;
    }
    bool ok = !abort_flag;
    if (issued > 0 && !mbar_wait(&bar[(issued - 1) & 1], unsigned((issued - 1) >> 1) & 1u)) ok = false;
    tc_fence_after();
    __syncwarp();
    if (ok && issued > 0) {
        const uint32_t trow = tmem + (uint32_t(warp * 32) << 16);
        const int co = tid;  // TMEM lane = row of D
        for (int c0 = 0; c0 < P.cin; c0 += 8) {
            float a[8];
            tmem_ld8(trow + c0, a);
            if (co < P.cout_real)
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    if (c0 + k < P.cin_real)
                        atomicAdd(&P.grad_w[((long long)tap * P.cout_real + co) * P.cin_real + c0 + k], a[k]);
        }
    }
    if (!ok && tid == 0 && atomicExch(&P.status->timeout, 1) == 0) {
        P.status->pad[0] = 2;  // kernel: weight gradient
        P.status->pad[1] = issued;
        P.status->pad[2] = int(blockIdx.x);
    }
    tc_fence_before();
    __syncthreads();
    __syncwarp();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

// One CTA, one 128 x N x K bf16 GEMM through the same descriptors and
// pipeline pieces as the convolutions: D[m][n] = sum_k A[m][k] B[n][k], A and
// B given row-major in global memory (K-major).  Records in status how far
// it got: pad[3] = 1 after TMEM allocation, 2 after the MMAs were issued, 3
// after their commit arrived, 4 after the TMEM read.
__global__ void __launch_bounds__(128) k_umma_selftest(const uint16_t* __restrict__ a, const uint16_t* __restrict__ b,
                                                       int N, int K, float* __restrict__ d, NetStatus* status) {
    __shared__ __align__(1024) uint8_t As[128 * 64 * 2];
    __shared__ __align__(1024) uint8_t Bs[64 * 64 * 2];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int kc = K / 8;
    const uint32_t sbo = uint32_t(kc) * 128;
    for (int c = 0; c < kc; ++c)
        *reinterpret_cast<uint4*>(As + (tid >> 3) * sbo + (tid & 7) * 16 + c * 128) =
            reinterpret_cast<const uint4*>(a + (long long)tid * K)[c];
    if (tid < N)
        for (int c = 0; c < kc; ++c)
            *reinterpret_cast<uint4*>(Bs + (tid >> 3) * sbo + (tid & 7) * 16 + c * 128) =
                reinterpret_cast<const uint4*>(b + (long long)tid * K)[c];
    if (tid == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tmem_alloc(&tslot, 64);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;
    if (tid == 0) {
        status->pad[3] = 1;
        const uint32_t idesc = idesc_bf16(128, N, 0, 0);
        for (int k = 0; k < K / 16; ++k)
            umma_bf16(tmem, sdesc(smem_u32(As) + k * 256, 128, sbo), sdesc(smem_u32(Bs) + k * 256, 128, sbo), idesc,
                      k > 0 ? 1u : 0u);
        umma_commit(&bar);
        status->pad[3] = 2;
    }
    const bool ok = mbar_wait(&bar, 0);
    if (tid == 0 && ok) status->pad[3] = 3;
    tc_fence_after();
    __syncwarp();
    if (ok) {
        for (int c0 = 0; c0 < N; c0 += 8) {
            float v[8];
            tmem_ld8(tmem + (uint32_t(warp * 32) << 16) + c0, v);
            for (int k = 0; k < 8; ++k) d[(long long)tid * N + c0 + k] = v[k];
        }
        if (tid == 0) status->pad[3] = 4;
    } else if (tid == 0) {
        atomicExch(&status->timeout, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 64);
}

// ------------------------------------------------------------ elementwise
__device__ __forceinline__ void dec3(long long v, int ny, int nz, int& x, int& y, int& z) {
    z = int(v % nz);
    const long long t = v / nz;
    y = int(t % ny);
    x = int(t / ny);
}

// sum r^2 and count over fluid cells -> s = sqrt(sum / count) (1 if empty)
__global__ void k_net_scale(const float* __restrict__ r, const uint8_t* __restrict__ type, long long n,
                            double* __restrict__ partials, unsigned* __restrict__ counter, float* __restrict__ scale) {
    double v[2] = {0.0, 0.0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (type[i] != 0) {
            v[0] += double(r[i]) * double(r[i]);
            v[1] += 1.0;
        }
    double tot[2];
    if (!grid_sum_last<2>(v, partials, counter, tot)) return;
    const double s = (tot[1] > 0 && tot[0] > 0) ? sqrt(tot[0] / tot[1]) : 1.0;
    *scale = float(s);
}

// Input channels, all linear in r so that M(a r) = a M(r) for a > 0 and
// M(0) = 0: [r/s, r/s on cells next to air, r/s on cells next to a solid
// (or the domain edge), 0], on cells with type != 0.
__device__ __forceinline__ void net_input_voxel(const float* __restrict__ r, const uint8_t* __restrict__ type,
                                                const uint8_t* __restrict__ solid, int nx, int ny, int nz,
                                                const float* __restrict__ scale, uint16_t* __restrict__ a0,
                                                long long v) {
    const bool fl = type[v] != 0;
    bool air = false, sol = false;
    if (fl) {
        int x, y, z;
        z = int(v % nz);
        const long long t = v / nz;
        y = int(t % ny);
        x = int(t / ny);
        const int dx[6] = {1, -1, 0, 0, 0, 0}, dy[6] = {0, 0, 1, -1, 0, 0}, dz[6] = {0, 0, 0, 0, 1, -1};
        for (int k = 0; k < 6; ++k) {
            const int xx = x + dx[k], yy = y + dy[k], zz = z + dz[k];
            if (xx < 0 || xx >= nx || yy < 0 || yy >= ny || zz < 0 || zz >= nz) {
                sol = true;
                continue;
            }
            const long long u = ((long long)xx * ny + yy) * nz + zz;
            if (solid && solid[u]) sol = true;
            else if (type[u] == 0) air = true;
        }
    }
    const float rh = fl ? r[v] / *scale : 0.f;
    uint16_t o[16] = {};
    o[0] = bf16_bits(rh);
    o[1] = bf16_bits(air ? rh : 0.f);
    o[2] = bf16_bits(sol ? rh : 0.f);
    uint4* dst = reinterpret_cast<uint4*>(a0 + v * 16);
    dst[0] = reinterpret_cast<uint4*>(o)[0];
    dst[1] = reinterpret_cast<uint4*>(o)[1];
}

__global__ void k_net_input(const float* __restrict__ r, const uint8_t* __restrict__ type,
                            const uint8_t* __restrict__ solid, int nx, int ny, int nz, const float* __restrict__ scale,
                            uint16_t* __restrict__ a0) {
    const long long n = (long long)nx * ny * nz;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    net_input_voxel(r, type, solid, nx, ny, nz, scale, a0, v);
}

// The voxel of this thread in tile u of a brick-tile list (one x plane,
// 16 y, 8 z; thread = (y - y0) * 8 + (z - z0), as the convolution's rows);
// false past the grid's edge.
__device__ __forceinline__ bool list_voxel(const int32_t* __restrict__ list, int u, int ny, int nz, int& x, int& y,
                                           int& z) {
    const int tyn = (ny + 15) / 16, tzn = (nz + 7) / 8;
    const long long tt = list[u];
    const int tzi = int(tt % tzn);
    const long long rest = tt / tzn;
    x = int(rest / tyn);
    y = int(rest % tyn) * 16 + (threadIdx.x >> 3);
    z = tzi * 8 + (threadIdx.x & 7);
    return y < ny && z < nz;
}

// k_net_input on the voxels of the listed tiles (128 threads per block)
__global__ void __launch_bounds__(128) k_net_input_tiles(const float* __restrict__ r, const uint8_t* __restrict__ type,
                                                         const uint8_t* __restrict__ solid, int nx, int ny, int nz,
                                                         const float* __restrict__ scale, uint16_t* __restrict__ a0,
                                                         const int32_t* __restrict__ list, const int* __restrict__ count) {
    const int n = *count;
    for (int u = blockIdx.x; u < n; u += gridDim.x) {
        int x, y, z;
        if (list_voxel(list, u, ny, nz, x, y, z)) net_input_voxel(r, type, solid, nx, ny, nz, scale, a0, ((long long)x * ny + y) * nz + z);
    }
}

// k_pool on the coarse voxels of the listed tiles: the same per-channel sums
// (children in order, FP32) for the voxel's C channels
__global__ void __launch_bounds__(128) k_pool_tiles(const uint16_t* __restrict__ fine, int fny, int fnz,
                                                    uint16_t* __restrict__ coarse, int cny, int cnz, int C,
                                                    const int32_t* __restrict__ list, const int* __restrict__ count) {
    const int n = *count;
    for (int u = blockIdx.x; u < n; u += gridDim.x) {
        int x, y, z;
        if (!list_voxel(list, u, cny, cnz, x, y, z)) continue;
        const long long v = ((long long)x * cny + y) * cnz + z;
        for (int q = 0; q < C / 8; ++q) {
            float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const long long f = ((long long)(2 * x + (k >> 2)) * fny + (2 * y + ((k >> 1) & 1))) * fnz + (2 * z + (k & 1));
                uint16_t c8[8];
                *reinterpret_cast<uint4*>(c8) = reinterpret_cast<const uint4*>(fine + f * C)[q];
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[j] += bf16_float(c8[j]);
            }
            uint16_t o[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) o[j] = bf16_bits(acc[j] * 0.125f);
            reinterpret_cast<uint4*>(coarse + v * C)[q] = *reinterpret_cast<uint4*>(o);
        }
    }
}

// k_upsample on the fine voxels of the listed tiles
__global__ void __launch_bounds__(128) k_upsample_tiles(const uint16_t* __restrict__ coarse, int cnx, int cny, int cnz,
                                                        uint16_t* __restrict__ fine, int fny, int fnz, int C,
                                                        const int32_t* __restrict__ list, const int* __restrict__ count) {
    const int n = *count;
    for (int u = blockIdx.x; u < n; u += gridDim.x) {
        int x, y, z;
        if (!list_voxel(list, u, fny, fnz, x, y, z)) continue;
        const int px = x >> 1, py = y >> 1, pz = z >> 1;
        const bool in = px < cnx && py < cny && pz < cnz;
        const uint4* src = reinterpret_cast<const uint4*>(coarse + (((long long)px * cny + py) * cnz + pz) * C);
        uint4* dst = reinterpret_cast<uint4*>(fine + (((long long)x * fny + y) * fnz + z) * C);
        for (int q = 0; q < C / 8; ++q) dst[q] = in ? src[q] : make_uint4(0u, 0u, 0u, 0u);
    }
}

// coarse[v][c] = bf16(0.125 * sum of the 8 children), children in (x, y, z) order
__global__ void k_pool(const uint16_t* __restrict__ fine, int fny, int fnz, uint16_t* __restrict__ coarse, int cnx,
                       int cny, int cnz, int C) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)cnx * cny * cnz * C;
    if (i >= n) return;
    const int c = int(i % C);
    const long long v = i / C;
    int x, y, z;
    dec3(v, cny, cnz, x, y, z);
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const long long f = ((long long)(2 * x + (k >> 2)) * fny + (2 * y + ((k >> 1) & 1))) * fnz + (2 * z + (k & 1));
        acc += bf16_float(fine[f * C + c]);
    }
    coarse[i] = bf16_bits(acc * 0.125f);
}

// fine[v][c] = coarse[parent(v)][c] (0 beyond 2 * coarse extent)
// fine voxel (x, y, z) = coarse voxel (x/2, y/2, z/2), 0 past the coarse
// grid.  One thread per fine voxel and 8-channel (16-byte) chunk; C is a
// multiple of 8 and every voxel's channels start on a 16-byte boundary.
__global__ void k_upsample(const uint16_t* __restrict__ coarse, int cnx, int cny, int cnz, uint16_t* __restrict__ fine,
                           int fnx, int fny, int fnz, int C) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned q = unsigned(C) / 8;
    if (i >= unsigned(fnx) * unsigned(fny) * unsigned(fnz) * q) return;
    const unsigned v = i / q, ch = i - v * q;
    int x, y, z;
    idx3(v, fny, fnz, x, y, z);
    const int px = x >> 1, py = y >> 1, pz = z >> 1;
    uint4 val = make_uint4(0u, 0u, 0u, 0u);
    if (px < cnx && py < cny && pz < cnz)
        val = reinterpret_cast<const uint4*>(coarse)[((unsigned(px) * cny + py) * cnz + pz) * q + ch];
    reinterpret_cast<uint4*>(fine)[i] = val;
}

// dcoarse[v][c] = sum of the 8 children's dfine (FP32, children in order)
__global__ void k_sum_children(const float* __restrict__ fine, int fny, int fnz, float* __restrict__ coarse, int cnx,
                               int cny, int cnz, int C) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)cnx * cny * cnz * C;
    if (i >= n) return;
    const int c = int(i % C);
    const long long v = i / C;
    int x, y, z;
    dec3(v, cny, cnz, x, y, z);
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const long long f = ((long long)(2 * x + (k >> 2)) * fny + (2 * y + ((k >> 1) & 1))) * fnz + (2 * z + (k & 1));
        acc += fine[f * C + c];
    }
    coarse[i] = acc;
}

// g = bf16(d * relu'(u)), or bf16(d) for the linear network
__global__ void k_relu_grad(const float* __restrict__ d, const uint16_t* __restrict__ u, long long n, int relu,
                            uint16_t* __restrict__ g) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    g[i] = bf16_bits((!relu || bf16_float(u[i]) > 0.f) ? d[i] : 0.f);
}

// g = bf16((skip + 0.125 * dcoarse[parent]) * relu'(u)) at a fine level
__global__ void k_relu_grad_unpool(const uint16_t* __restrict__ skip, const float* __restrict__ dcoarse, int cnx, int cny,
                                   int cnz, const uint16_t* __restrict__ u, int fnx, int fny, int fnz, int C,
                                   int relu, uint16_t* __restrict__ g) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)fnx * fny * fnz * C;
    if (i >= n) return;
    const int c = int(i % C);
    const long long v = i / C;
    int x, y, z;
    dec3(v, fny, fnz, x, y, z);
    const int px = x >> 1, py = y >> 1, pz = z >> 1;
    float d = bf16_float(skip[i]);
    if (px < cnx && py < cny && pz < cnz) d += 0.125f * dcoarse[(((long long)px * cny + py) * cnz + pz) * C + c];
    g[i] = bf16_bits((!relu || bf16_float(u[i]) > 0.f) ? d : 0.f);
}

// z = s * y on fluid cells
__global__ void k_net_output(const float* __restrict__ y, const uint8_t* __restrict__ type, long long n,
                             const float* __restrict__ scale, float* __restrict__ z) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    z[v] = (type[v] != 0) ? y[v] * *scale : 0.f;
}

// g5[v] = [bf16(s * dz * fluid), 0, ..., 0]
__global__ void k_net_dy(const float* __restrict__ dz, const uint8_t* __restrict__ type, long long n,
                         const float* __restrict__ scale, uint16_t* __restrict__ g5) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    uint16_t o[16] = {};
    o[0] = bf16_bits(type[v] != 0 ? dz[v] * *scale : 0.f);
    uint4* dst = reinterpret_cast<uint4*>(g5 + v * 16);
    dst[0] = reinterpret_cast<uint4*>(o)[0];
    dst[1] = reinterpret_cast<uint4*>(o)[1];
}

// B tiles of one layer: forward [tap][n = cout_pad][k = cin_pad] holding
// W[tap][n][k]; backward [tap][n = cin_pad][k = cout_pad] holding
// W[26 - tap][k][n].  K-major core-matrix layout, zero padding.
__global__ void k_format_weights(const float* __restrict__ w, int cout, int cin, uint16_t* __restrict__ fwd,
                                 uint16_t* __restrict__ bwd) {
    const int cop = pad16(cout), cip = pad16(cin);
    const long long per_tap = (long long)cop * cip;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= per_tap * kNetTaps) return;
    const int tap = int(i / per_tap);
    const int rem = int(i % per_tap);
    {  // forward element (n, k)
        const int n = rem / cip, k = rem % cip;
        const float val = (n < cout && k < cin) ? w[((long long)tap * cout + n) * cin + k] : 0.f;
        const long long off = (long long)(n / 8) * (cip / 8) * 64 + (k / 8) * 64 + (n % 8) * 8 + (k % 8);
        fwd[tap * per_tap + off] = bf16_bits(val);
    }
    if (bwd) {  // backward element (n = ci, k = co)
        const int n = rem / cop, k = rem % cop;
        const float val = (n < cin && k < cout) ? w[((long long)(kNetTaps - 1 - tap) * cout + k) * cin + n] : 0.f;
        const long long off = (long long)(n / 8) * (cop / 8) * 64 + (k / 8) * 64 + (n % 8) * 8 + (k % 8);
        bwd[tap * per_tap + off] = bf16_bits(val);
    }
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

unsigned nb(long long n, int t = 256) { return unsigned(std::max<long long>(1, (n + t - 1) / t)); }


// ------------------------------------------------- sparse evaluation plan
// Byte masks of the voxels each convolution's output must be right on, and
// from them the output tiles (the brick kernel's 128-voxel tiles) to
// evaluate.  Voxels outside these sets may hold stale values: every value a
// needed voxel reads (its 27 neighbours, its pooled children, its upsampled
// parent, its skip input) is itself needed, and the tensor-core product of
// a tile row reads that row's inputs only.
__global__ void k_mask_type(const uint8_t* __restrict__ type, long long n, uint8_t* __restrict__ m) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) m[v] = type[v] != 0;
}

// out = in dilated by one voxel along z (axis 0) or along x and y (axis 1)
__global__ void k_mask_dilate(const uint8_t* __restrict__ in, int nx, int ny, int nz, int axis,
                              uint8_t* __restrict__ out) {
    const long long n = (long long)nx * ny * nz;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    int x, y, z;
    dec3(v, ny, nz, x, y, z);
    uint8_t o = 0;
    if (axis == 0) {
        o = in[v];
        if (z > 0) o |= in[v - 1];
        if (z + 1 < nz) o |= in[v + 1];
    } else {
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy) {
                const int xx = x + dx, yy = y + dy;
                if (xx >= 0 && xx < nx && yy >= 0 && yy < ny) o |= in[((long long)xx * ny + yy) * nz + z];
            }
    }
    out[v] = o;
}

// k_mask_dilate over 4-voxel words along z (nz a multiple of 4, so a word
// never spans two z rows): axis 0 along z, axis 1 along x and y
__global__ void k_mask_dilate4(const uint32_t* __restrict__ in, int nx, int ny, int nzw, int axis,
                               uint32_t* __restrict__ out) {
    const long long n = (long long)nx * ny * nzw;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    int x, y, zw;
    dec3(v, ny, nzw, x, y, zw);
    uint32_t o;
    if (axis == 0) {
        const uint32_t w = in[v];
        o = w | (w << 8) | (w >> 8);
        if (zw > 0) o |= in[v - 1] >> 24;       // z - 1 of the first voxel
        if (zw + 1 < nzw) o |= in[v + 1] << 24;  // z + 1 of the last voxel
    } else {
        o = 0u;
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy) {
                const int xx = x + dx, yy = y + dy;
                if (xx >= 0 && xx < nx && yy >= 0 && yy < ny) o |= in[((long long)xx * ny + yy) * nzw + zw];
            }
    }
    out[v] = o;
}

// k_mask_tile_flags over 4-voxel words (nz a multiple of 4: a word lies in
// one tile's 8 z)
__global__ void k_mask_tile_flags4(const uint32_t* __restrict__ m, int nx, int ny, int nzw, int nz,
                                   uint8_t* __restrict__ flag) {
    const long long n = (long long)nx * ny * nzw;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n || !m[v]) return;
    int x, y, zw;
    dec3(v, ny, nzw, x, y, zw);
    const int tyn = (ny + 15) / 16, tzn = (nz + 7) / 8;
    flag[((long long)x * tyn + (y >> 4)) * tzn + (zw >> 1)] = 1;
}

// coarse voxel set if any of its 8 children is (the voxels whose upsampled
// value a needed fine voxel reads)
__global__ void k_mask_up(const uint8_t* __restrict__ fine, int fny, int fnz, int cnx, int cny, int cnz,
                          uint8_t* __restrict__ coarse) {
    const long long n = (long long)cnx * cny * cnz;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    int x, y, z;
    dec3(v, cny, cnz, x, y, z);
    uint8_t o = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k)
        o |= fine[((long long)(2 * x + (k >> 2)) * fny + (2 * y + ((k >> 1) & 1))) * fnz + (2 * z + (k & 1))];
    coarse[v] = o;
}

// out = other | (fine voxels whose parent is set: the children a needed
// pooled voxel averages)
__global__ void k_mask_down_or(const uint8_t* __restrict__ coarse, int cnx, int cny, int cnz,
                               const uint8_t* __restrict__ other, int fnx, int fny, int fnz, uint8_t* __restrict__ out) {
    const long long n = (long long)fnx * fny * fnz;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    int x, y, z;
    dec3(v, fny, fnz, x, y, z);
    const int px = x >> 1, py = y >> 1, pz = z >> 1;
    uint8_t o = other[v];
    if (px < cnx && py < cny && pz < cnz) o |= coarse[((long long)px * cny + py) * cnz + pz];
    out[v] = o;
}

// flag[t] = 1 for the brick tiles (x, y / 16, z / 8) holding a set voxel
__global__ void k_mask_tile_flags(const uint8_t* __restrict__ m, int nx, int ny, int nz, uint8_t* __restrict__ flag) {
    const long long n = (long long)nx * ny * nz;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n || !m[v]) return;
    int x, y, z;
    dec3(v, ny, nz, x, y, z);
    const int tyn = (ny + 15) / 16, tzn = (nz + 7) / 8;
    flag[((long long)x * tyn + (y >> 4)) * tzn + (z >> 3)] = 1;
}

// list of the flagged tiles (in any order) and their count
__global__ void k_mask_tile_list(const uint8_t* __restrict__ flag, long long ntiles, int32_t* __restrict__ list,
                                 int* __restrict__ count) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles || !flag[t]) return;
    list[atomicAdd(count, 1)] = int32_t(t);
}

}  // namespace

// ------------------------------------------------------------- host side
LearnedNet::LearnedNet(uint64_t seed) {
    const long long np = net_param_count();
    std::vector<float> w(size_t(np), 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < kNetLayers; ++l) {
        const long long off = net_param_offset(l);
        const int fan_in = kNetTaps * kNetCin[l];
        const double sd = std::sqrt(2.0 / fan_in) * (l == kNetLayers - 1 ? 0.5 : 1.0);
        std::normal_distribution<double> nd(0.0, sd);
        const long long nw = (long long)kNetTaps * kNetCout[l] * kNetCin[l];
        for (long long i = 0; i < nw; ++i) w[size_t(off + i)] = float(nd(rng));
    }
    LHI_CUDA(cudaMalloc(&w32_, sizeof(float) * np));
    LHI_CUDA(cudaMalloc(&grad_, sizeof(float) * np));
    LHI_CUDA(cudaMalloc(&adam_m_, sizeof(float) * np));
    LHI_CUDA(cudaMalloc(&adam_v_, sizeof(float) * np));
    LHI_CUDA(cudaMemcpy(w32_, w.data(), sizeof(float) * np, cudaMemcpyHostToDevice));
    LHI_CUDA(cudaMemset(grad_, 0, sizeof(float) * np));
    LHI_CUDA(cudaMemset(adam_m_, 0, sizeof(float) * np));
    LHI_CUDA(cudaMemset(adam_v_, 0, sizeof(float) * np));
    long long f = 0;
    for (int l = 0; l < kNetLayers; ++l) {
        wfwd_off_[l] = f;
        wbwd_off_[l] = f;
        f += (long long)kNetTaps * pad16(kNetCout[l]) * pad16(kNetCin[l]);
    }
    LHI_CUDA(cudaMalloc(&wfwd_, sizeof(uint16_t) * f));
    LHI_CUDA(cudaMalloc(&wbwd_, sizeof(uint16_t) * f));
    LHI_CUDA(cudaMalloc(&status_, sizeof(NetStatus)));
    LHI_CUDA(cudaMemset(status_, 0, sizeof(NetStatus)));
    LHI_CUDA(cudaMalloc(&scale_, sizeof(float)));
    LHI_CUDA(cudaMalloc(&red_, sizeof(double) * 2 * 1024));
    LHI_CUDA(cudaMalloc(&counter_, sizeof(unsigned) * 4));
    LHI_CUDA(cudaMemset(counter_, 0, sizeof(unsigned) * 4));
    LHI_CUDA(cudaFuncSetAttribute(k_conv, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    LHI_CUDA(cudaFuncSetAttribute(k_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, 120 * 1024));
}

static void free_buffers(NetBuffers& b) {
    auto F = [](void* p) {
        if (p) cudaFree(p);
    };
    F(b.a0), F(b.h0), F(b.p0), F(b.h1), F(b.p1), F(b.h2), F(b.q1), F(b.u1), F(b.q0), F(b.u0), F(b.y), F(b.dx), F(b.acc);
    for (int l = 0; l < kNetLayers; ++l) F(b.g[l]);
    b = NetBuffers();
}

LearnedNet::~LearnedNet() {
    free_buffers(b_);
    free_plan();
    auto F = [](void* p) {
        if (p) cudaFree(p);
    };
    F(w32_), F(grad_), F(adam_m_), F(adam_v_), F(wfwd_), F(wbwd_), F(status_), F(scale_), F(red_), F(counter_);
}

void LearnedNet::set_params(const float* host) {
    LHI_CUDA(cudaMemcpy(w32_, host, sizeof(float) * net_param_count(), cudaMemcpyHostToDevice));
    wfmt_stale_ = true;
}
void LearnedNet::get_params(float* host) {
    LHI_CUDA(cudaMemcpy(host, w32_, sizeof(float) * net_param_count(), cudaMemcpyDeviceToHost));
}
void LearnedNet::get_grads(float* host, cudaStream_t s) {
    LHI_CUDA(cudaMemcpyAsync(host, grad_, sizeof(float) * net_param_count(), cudaMemcpyDeviceToHost, s));
    LHI_CUDA(cudaStreamSynchronize(s));
}
void LearnedNet::zero_grad(cudaStream_t s) {
    LHI_CUDA(cudaMemsetAsync(grad_, 0, sizeof(float) * net_param_count(), s));
}
int LearnedNet::check_status(cudaStream_t s) {
    NetStatus h{};
    LHI_CUDA(cudaMemcpyAsync(&h, status_, sizeof(h), cudaMemcpyDeviceToHost, s));
    LHI_CUDA(cudaStreamSynchronize(s));
    if (h.timeout) {
        last_timeout_[0] = h.pad[0];
        last_timeout_[1] = h.pad[1];
        last_timeout_[2] = h.pad[2];
        // reported once: the next call starts from a clear status
        LHI_CUDA(cudaMemsetAsync(status_, 0, sizeof(NetStatus), s));
        LHI_CUDA(cudaStreamSynchronize(s));
    }
    return h.timeout ? LHI_E_TIMEOUT : LHI_OK;
}

void set_net_wait_limit_ns(unsigned long long ns) {
    LHI_CUDA(cudaMemcpyToSymbol(g_net_wait_ns, &ns, sizeof(ns)));
}

void LearnedNet::ensure(const int dims[3]) {
    int d1[3], d2[3];
    for (int a = 0; a < 3; ++a) {
        d1[a] = dims[a] / 2;
        d2[a] = d1[a] / 2;
        if (dims[a] < 4) throw std::invalid_argument("learned preconditioner: grid below 4 cells on an axis");
    }
    const long long v0 = (long long)dims[0] * dims[1] * dims[2];
    bool same = true;
    for (int a = 0; a < 3; ++a) same = same && b_.dims[0][a] == dims[a];
    if (same && b_.cap_vox0 == v0) return;
    free_buffers(b_);
    for (int a = 0; a < 3; ++a) {
        b_.dims[0][a] = dims[a];
        b_.dims[1][a] = d1[a];
        b_.dims[2][a] = d2[a];
    }
    b_.vox[0] = v0;
    b_.vox[1] = (long long)d1[0] * d1[1] * d1[2];
    b_.vox[2] = (long long)d2[0] * d2[1] * d2[2];
    b_.cap_vox0 = v0;
    const long long V0 = b_.vox[0], V1 = std::max(1LL, b_.vox[1]), V2 = std::max(1LL, b_.vox[2]);
    auto A16 = [](uint16_t** p, long long n) { LHI_CUDA(cudaMalloc(p, sizeof(uint16_t) * size_t(n))); };
    A16(&b_.a0, V0 * 16);
    A16(&b_.h0, V0 * 16);
    A16(&b_.p0, V1 * 16);
    A16(&b_.h1, V1 * 32);
    A16(&b_.p1, V2 * 32);
    A16(&b_.h2, V2 * 64);
    A16(&b_.q1, V1 * 64);
    A16(&b_.u1, V1 * 32);
    A16(&b_.q0, V0 * 32);
    A16(&b_.u0, V0 * 16);
    LHI_CUDA(cudaMalloc(&b_.y, sizeof(float) * V0));
    const long long gsz[kNetLayers] = {V0 * 16, V1 * 32, V2 * 64, V1 * 32, V0 * 16, V0 * 16};
    for (int l = 0; l < kNetLayers; ++l) A16(&b_.g[l], gsz[l]);
    LHI_CUDA(cudaMalloc(&b_.dx, sizeof(float) * std::max(V0 * 32, V1 * 64)));
    LHI_CUDA(cudaMalloc(&b_.acc, sizeof(float) * std::max(V1 * 32, V2 * 64)));
}

void LearnedNet::format_weights(cudaStream_t s) {
    for (int l = 0; l < kNetLayers; ++l) {
        const long long n = (long long)kNetTaps * pad16(kNetCout[l]) * pad16(kNetCin[l]);
        k_format_weights<<<nb(n), 256, 0, s>>>(w32_ + net_param_offset(l), kNetCout[l], kNetCin[l], wfwd_ + wfwd_off_[l],
                                               l == 0 ? nullptr : wbwd_ + wbwd_off_[l]);
        LHI_LAUNCH_CHECK();
    }
    wfmt_stale_ = false;
}

namespace {
template <int CIN, int COUT>
void launch_brick_t(const CUtensorMap& tin, const ConvParams& P, int stages, unsigned grid, size_t smem, cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        LHI_CUDA(cudaFuncSetAttribute(k_conv_brick<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(kBrickSmemMax)));
        attr = true;
    }
    k_conv_brick<CIN, COUT><<<grid, kBrThreads, smem, s>>>(tin, P, stages);
    LHI_LAUNCH_CHECK();
}

// The brick kernel's instances: the (input, output) channel counts of the
// network's forward and input-gradient convolutions.
bool launch_brick(const CUtensorMap& tin, const ConvParams& P, int stages, unsigned grid, size_t smem, cudaStream_t s) {
    if (P.cin == 16 && P.cout == 16) launch_brick_t<16, 16>(tin, P, stages, grid, smem, s);
    else if (P.cin == 16 && P.cout == 32) launch_brick_t<16, 32>(tin, P, stages, grid, smem, s);
    else if (P.cin == 32 && P.cout == 16) launch_brick_t<32, 16>(tin, P, stages, grid, smem, s);
    else if (P.cin == 32 && P.cout == 64) launch_brick_t<32, 64>(tin, P, stages, grid, smem, s);
    else if (P.cin == 64 && P.cout == 32) launch_brick_t<64, 32>(tin, P, stages, grid, smem, s);
    else return false;
    return true;
}

void launch_conv(const uint16_t* in, int cin, const uint16_t* w, int cout, const float* bias, int cout_real,
                 const int* d, int mode, const uint16_t* skip, int relu, uint16_t* out_b, float* out_f, NetStatus* st,
                 cudaStream_t s, const int32_t* tiles = nullptr, const int* ntiles_dev = nullptr) {
    ConvParams P;
    P.tiles = nullptr;  // the gathering kernel evaluates every voxel
    P.ntiles = nullptr;
    P.in = in;
    P.cin = cin;
    P.w = w;
    P.cout = cout;
    P.bias = bias;
    P.cout_real = cout_real;
    P.nx = d[0];
    P.ny = d[1];
    P.nz = d[2];
    P.nvox = (long long)d[0] * d[1] * d[2];
    P.mode = mode;
    P.skip = skip;
    P.relu = relu;
    P.out_b = out_b;
    P.out_f = out_f;
    P.status = st;
    if (P.nvox == 0) return;
    // the brick kernel keeps all 27 weight tiles and the brick in shared
    // memory: every layer but the 64 -> 64 input gradient fits
    if (brick_smem_bytes(cin, cout, 1) <= kBrickSmemMax) {
        const int stages = brick_smem_bytes(cin, cout, 2) <= kBrickSmemMax ? 2 : 1;
        const size_t smem = brick_smem_bytes(cin, cout, stages);
        // the input as a 4D tensor (channel, z, y, x), boxes of one 8-channel
        // plane of a brick; zeros outside the grid
        CUtensorMap tin;
        const cuuint64_t dims[4] = {cuuint64_t(cin), cuuint64_t(d[2]), cuuint64_t(d[1]), cuuint64_t(d[0])};
        const cuuint64_t strides[3] = {cuuint64_t(cin) * 2, cuuint64_t(cin) * 2 * d[2],
                                       cuuint64_t(cin) * 2 * d[2] * d[1]};
        const cuuint32_t box[4] = {8, cuuint32_t(kBrZ), cuuint32_t(kBrY), cuuint32_t(kBrX)};
        const cuuint32_t estr[4] = {1, 1, 1, 1};
        const CUresult r = tensor_map_encoder()(&tin, CU_TENSOR_MAP_DATA_TYPE_UINT16, 4, const_cast<uint16_t*>(in),
                                                dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
            throw CudaError(cudaErrorInvalidValue, "brick tensor map: cuTensorMapEncodeTiled failed with CUresult " +
                                                       std::to_string(int(r)));
        const long long ntiles = (long long)d[0] * ((d[1] + 15) / 16) * ((d[2] + 7) / 8);
        const long long per_sm = std::max<long long>(1, (228LL * 1024) / (long long)(smem + 1024));
        const unsigned grid = unsigned(std::min<long long>(ntiles, kSMs * per_sm));
        P.tiles = tiles;
        P.ntiles = tiles ? ntiles_dev : nullptr;
        if (launch_brick(tin, P, stages, grid, smem, s)) return;
        P.tiles = nullptr;  // no instance for these channel counts: the gathering kernel
        P.ntiles = nullptr;
    }
    const size_t smem = size_t(2) * kConvM * cin * 2 + size_t(2) * cout * cin * 2 + 32;
    k_conv<<<unsigned((P.nvox + kConvM - 1) / kConvM), kConvM, smem, s>>>(P);
    LHI_LAUNCH_CHECK();
}

void launch_wgrad(const uint16_t* g, int cout, int cout_real, const uint16_t* in, int cin, int cin_real, const int* d,
                  float* grad_w, NetStatus* st, cudaStream_t s) {
    WgradParams P;
    P.g = g;
    P.cout = cout;
    P.cout_real = cout_real;
    P.in = in;
    P.cin = cin;
    P.cin_real = cin_real;
    P.nx = d[0];
    P.ny = d[1];
    P.nz = d[2];
    P.nvox = (long long)d[0] * d[1] * d[2];
    P.grad_w = grad_w;
    P.status = st;
    if (P.nvox == 0) return;
    const size_t smem = size_t(2) * 128 * kWgChunk * 2 + size_t(2) * cin * kWgChunk * 2 + 32;
    dim3 grid(unsigned((P.nvox + kWgChunk * kWgChunksPerCta - 1) / (kWgChunk * kWgChunksPerCta)), kNetTaps);
    k_wgrad<<<grid, 128, smem, s>>>(P);
    LHI_LAUNCH_CHECK();
}
}  // namespace

static long long brick_tiles(const int d[3]) { return (long long)d[0] * ((d[1] + 15) / 16) * ((d[2] + 7) / 8); }

void LearnedNet::free_plan() {
    for (auto& p : mask_) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    for (auto& p : tflag_) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    for (auto& p : tlist_) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    if (tcount_) cudaFree(tcount_);
    tcount_ = nullptr;
    plan_type_ = nullptr;
    plan_cap_vox0_ = 0;
    for (int& d : plan_dims_) d = 0;
}

// Needed voxel sets, from the output back to the input (F = type != 0;
// dil = one-voxel dilation; up = coarse voxels with a needed child;
// down = fine voxels with a needed parent):
//   conv5 out F                      (T5)   u0 needed on D = dil(F)
//   conv4 out D (skip h0 on D)       (T4)   q0 needed on dil(D)
//   u1 needed on U1 = up(dil(D))
//   conv3 out U1 (skip h1 on U1)     (T3)   q1 needed on dil(U1)
//   h2 needed on U2 = up(dil(U1))
//   conv2 out U2                     (T2)   p1 needed on dil(U2)
//   h1 needed on H1 = U1 | down(dil(U2))
//   conv1 out H1                     (T1)   p0 needed on dil(H1)
//   h0 needed on H0 = D | down(dil(H1))
//   conv0 out H0                     (T0)   a0 needed on dil(H0): computed everywhere
// Masks: level 0 A, B; level 1 P, Q; level 2 U, W.
void LearnedNet::plan_sparse(const int dims[3], const uint8_t* type, cudaStream_t s) {
    ensure(dims);
    const int* d0 = b_.dims[0];
    const int* d1 = b_.dims[1];
    const int* d2 = b_.dims[2];
    const long long V0 = b_.vox[0], V1 = b_.vox[1], V2 = b_.vox[2];
    if (plan_cap_vox0_ != V0) {
        free_plan();
        const long long vl[7] = {V0, V0, V1, V1, V2, V2, V0};
        for (int i = 0; i < 7; ++i) LHI_CUDA(cudaMalloc(&mask_[i], size_t(std::max(1LL, vl[i]))));
        const int* dl[3] = {d0, d1, d2};
        for (int l = 0; l < 3; ++l) LHI_CUDA(cudaMalloc(&tflag_[l], size_t(std::max(1LL, brick_tiles(dl[l])))));
        // list levels: the six convolutions' outputs, then the input
        // channels (0), pool to 1, pool to 2, upsample to 1, upsample to 0
        const int lvl[kPlanLists] = {0, 1, 2, 1, 0, 0, 0, 1, 2, 1, 0};
        for (int l = 0; l < kPlanLists; ++l)
            LHI_CUDA(cudaMalloc(&tlist_[l], sizeof(int32_t) * size_t(std::max(1LL, brick_tiles(dl[lvl[l]])))));
        LHI_CUDA(cudaMalloc(&tcount_, sizeof(int) * kPlanLists));
        plan_cap_vox0_ = V0;
    }
    uint8_t *A = mask_[0], *B = mask_[1], *P = mask_[2], *Q = mask_[3], *U = mask_[4], *W = mask_[5];
    uint8_t* S = mask_[6];  // the dilations' intermediate (sized for level 0, used at every level)
    LHI_CUDA(cudaMemsetAsync(tcount_, 0, sizeof(int) * kPlanLists, s));
    auto dil = [&](const uint8_t* in, const int* d, uint8_t* out) {
        const long long n = (long long)d[0] * d[1] * d[2];
        if (n == 0) return;
        if (d[2] % 4 == 0) {  // 4-voxel words (the mask buffers are 256-byte aligned)
            const long long nw = n / 4;
            k_mask_dilate4<<<nb(nw), 256, 0, s>>>(reinterpret_cast<const uint32_t*>(in), d[0], d[1], d[2] / 4, 0,
                                                  reinterpret_cast<uint32_t*>(S));
            LHI_LAUNCH_CHECK();
            k_mask_dilate4<<<nb(nw), 256, 0, s>>>(reinterpret_cast<const uint32_t*>(S), d[0], d[1], d[2] / 4, 1,
                                                  reinterpret_cast<uint32_t*>(out));
            LHI_LAUNCH_CHECK();
            return;
        }
        k_mask_dilate<<<nb(n), 256, 0, s>>>(in, d[0], d[1], d[2], 0, S);
        LHI_LAUNCH_CHECK();
        k_mask_dilate<<<nb(n), 256, 0, s>>>(S, d[0], d[1], d[2], 1, out);
        LHI_LAUNCH_CHECK();
    };
    auto up = [&](const uint8_t* fine, const int* fd, const int* cd, uint8_t* coarse) {
        const long long n = (long long)cd[0] * cd[1] * cd[2];
        if (n == 0) return;
        k_mask_up<<<nb(n), 256, 0, s>>>(fine, fd[1], fd[2], cd[0], cd[1], cd[2], coarse);
        LHI_LAUNCH_CHECK();
    };
    auto down_or = [&](const uint8_t* coarse, const int* cd, const uint8_t* other, const int* fd, uint8_t* out) {
        const long long n = (long long)fd[0] * fd[1] * fd[2];
        if (n == 0) return;
        k_mask_down_or<<<nb(n), 256, 0, s>>>(coarse, cd[0], cd[1], cd[2], other, fd[0], fd[1], fd[2], out);
        LHI_LAUNCH_CHECK();
    };
    auto tiles = [&](const uint8_t* m, const int* d, int level, int layer) {
        const long long n = (long long)d[0] * d[1] * d[2], nt = brick_tiles(d);
        if (n == 0) return;
        LHI_CUDA(cudaMemsetAsync(tflag_[level], 0, size_t(nt), s));
        if (d[2] % 4 == 0)
            k_mask_tile_flags4<<<nb(n / 4), 256, 0, s>>>(reinterpret_cast<const uint32_t*>(m), d[0], d[1], d[2] / 4,
                                                         d[2], tflag_[level]);
        else
            k_mask_tile_flags<<<nb(n), 256, 0, s>>>(m, d[0], d[1], d[2], tflag_[level]);
        LHI_LAUNCH_CHECK();
        k_mask_tile_list<<<nb(nt), 256, 0, s>>>(tflag_[level], nt, tlist_[layer], tcount_ + layer);
        LHI_LAUNCH_CHECK();
    };
    k_mask_type<<<nb(V0), 256, 0, s>>>(type, V0, A);  // A = F
    LHI_LAUNCH_CHECK();
    tiles(A, d0, 0, 5);
    dil(A, d0, B);  // B = D
    tiles(B, d0, 0, 4);
    dil(B, d0, A);  // A = dil(D): q0 needed
    tiles(A, d0, 0, kPlanUp0);
    up(A, d0, d1, P);  // P = U1
    tiles(P, d1, 1, 3);
    dil(P, d1, Q);  // q1 needed
    tiles(Q, d1, 1, kPlanUp1);
    up(Q, d1, d2, U);  // U = U2
    tiles(U, d2, 2, 2);
    dil(U, d2, W);  // p1 needed
    tiles(W, d2, 2, kPlanPool1);
    down_or(W, d2, P, d1, Q);  // Q = H1
    tiles(Q, d1, 1, 1);
    dil(Q, d1, P);  // p0 needed
    tiles(P, d1, 1, kPlanPool0);
    down_or(P, d1, B, d0, A);  // A = H0
    tiles(A, d0, 0, 0);
    dil(A, d0, B);  // a0 needed
    tiles(B, d0, 0, kPlanInput);
    plan_type_ = type;
    for (int a = 0; a < 3; ++a) plan_dims_[a] = dims[a];
}

void LearnedNet::forward(const int dims[3], const float* r, const uint8_t* type, const uint8_t* solid, float* z,
                         double scale_fixed, cudaStream_t s, bool sparse) {
    ensure(dims);
    sparse = sparse && sparse_enabled_ && plan_type_ == type && plan_cap_vox0_ == b_.vox[0] &&
             plan_dims_[0] == dims[0] && plan_dims_[1] == dims[1] && plan_dims_[2] == dims[2];
    auto TL = [&](int l) -> const int32_t* { return sparse ? tlist_[l] : nullptr; };
    auto TC = [&](int l) -> const int* { return sparse ? tcount_ + l : nullptr; };
    if (wfmt_stale_) format_weights(s);
    last_type_ = type;
    const int* d0 = b_.dims[0];
    const int* d1 = b_.dims[1];
    const int* d2 = b_.dims[2];
    const long long V0 = b_.vox[0];
    if (scale_fixed > 0) {
        const float sf = float(scale_fixed);
        LHI_CUDA(cudaMemcpyAsync(scale_, &sf, sizeof(float), cudaMemcpyHostToDevice, s));
    } else {
        k_net_scale<<<std::min<unsigned>(nb(V0), 1024), 256, 0, s>>>(r, type, V0, red_, counter_, scale_);
        LHI_LAUNCH_CHECK();
    }
    // the elementwise stages on their plan's tiles: a persistent grid
    const auto tgrid = [](const int* d) {
        return unsigned(std::max(1LL, std::min<long long>(brick_tiles(d), (long long)kSMs * 16)));
    };
    if (sparse)
        k_net_input_tiles<<<tgrid(d0), 128, 0, s>>>(r, type, solid, d0[0], d0[1], d0[2], scale_, b_.a0,
                                                    tlist_[kPlanInput], tcount_ + kPlanInput);
    else
        k_net_input<<<nb(V0), 256, 0, s>>>(r, type, solid, d0[0], d0[1], d0[2], scale_, b_.a0);
    LHI_LAUNCH_CHECK();
    auto W = [&](int l) { return wfwd_ + wfwd_off_[l]; };
    // bias-free: M(0) = 0 (the packed bias entries are kept and ignored)
    auto Bv = [&](int l) -> const float* {
        (void)l;
        return nullptr;
    };
    const int act = relu_ ? 1 : 0;
    launch_conv(b_.a0, 16, W(0), 16, Bv(0), 16, d0, 0, nullptr, act, b_.h0, nullptr, status_, s, TL(0), TC(0));
    if (sparse)
        k_pool_tiles<<<tgrid(d1), 128, 0, s>>>(b_.h0, d0[1], d0[2], b_.p0, d1[1], d1[2], 16, tlist_[kPlanPool0],
                                               tcount_ + kPlanPool0);
    else
        k_pool<<<nb(b_.vox[1] * 16), 256, 0, s>>>(b_.h0, d0[1], d0[2], b_.p0, d1[0], d1[1], d1[2], 16);
    LHI_LAUNCH_CHECK();
    launch_conv(b_.p0, 16, W(1), 32, Bv(1), 32, d1, 0, nullptr, act, b_.h1, nullptr, status_, s, TL(1), TC(1));
    if (sparse)
        k_pool_tiles<<<tgrid(d2), 128, 0, s>>>(b_.h1, d1[1], d1[2], b_.p1, d2[1], d2[2], 32, tlist_[kPlanPool1],
                                               tcount_ + kPlanPool1);
    else
        k_pool<<<nb(b_.vox[2] * 32), 256, 0, s>>>(b_.h1, d1[1], d1[2], b_.p1, d2[0], d2[1], d2[2], 32);
    LHI_LAUNCH_CHECK();
    launch_conv(b_.p1, 32, W(2), 64, Bv(2), 64, d2, 0, nullptr, act, b_.h2, nullptr, status_, s, TL(2), TC(2));
    if (sparse)
        k_upsample_tiles<<<tgrid(d1), 128, 0, s>>>(b_.h2, d2[0], d2[1], d2[2], b_.q1, d1[1], d1[2], 64,
                                                   tlist_[kPlanUp1], tcount_ + kPlanUp1);
    else
        k_upsample<<<nb(b_.vox[1] * 64 / 8), 256, 0, s>>>(b_.h2, d2[0], d2[1], d2[2], b_.q1, d1[0], d1[1], d1[2], 64);
    LHI_LAUNCH_CHECK();
    launch_conv(b_.q1, 64, W(3), 32, Bv(3), 32, d1, 0, b_.h1, act, b_.u1, nullptr, status_, s, TL(3), TC(3));
    if (sparse)
        k_upsample_tiles<<<tgrid(d0), 128, 0, s>>>(b_.u1, d1[0], d1[1], d1[2], b_.q0, d0[1], d0[2], 32,
                                                   tlist_[kPlanUp0], tcount_ + kPlanUp0);
    else
        k_upsample<<<nb(V0 * 32 / 8), 256, 0, s>>>(b_.u1, d1[0], d1[1], d1[2], b_.q0, d0[0], d0[1], d0[2], 32);
    LHI_LAUNCH_CHECK();
    launch_conv(b_.q0, 32, W(4), 16, Bv(4), 16, d0, 0, b_.h0, act, b_.u0, nullptr, status_, s, TL(4), TC(4));
    launch_conv(b_.u0, 16, W(5), 16, Bv(5), 1, d0, 2, nullptr, 0, nullptr, b_.y, status_, s, TL(5), TC(5));
    k_net_output<<<nb(V0), 256, 0, s>>>(b_.y, type, V0, scale_, z);
    LHI_LAUNCH_CHECK();
}

void LearnedNet::backward(const float* dz, cudaStream_t s) {
    const int* d0 = b_.dims[0];
    const int* d1 = b_.dims[1];
    const int* d2 = b_.dims[2];
    const long long V0 = b_.vox[0], V1 = b_.vox[1], V2 = b_.vox[2];
    auto WB = [&](int l) { return wbwd_ + wbwd_off_[l]; };
    auto GW = [&](int l) { return grad_ + net_param_offset(l); };
    // the network is bias-free: the packed bias entries keep zero gradient
    // layer 5
    k_net_dy<<<nb(V0), 256, 0, s>>>(dz, last_type_, V0, scale_, b_.g[5]);
    LHI_LAUNCH_CHECK();
    launch_wgrad(b_.g[5], 16, 1, b_.u0, 16, 16, d0, GW(5), status_, s);
    launch_conv(b_.g[5], 16, WB(5), 16, nullptr, 16, d0, 1, nullptr, 0, nullptr, b_.dx, status_, s);
    // layer 4
    k_relu_grad<<<nb(V0 * 16), 256, 0, s>>>(b_.dx, b_.u0, V0 * 16, relu_ ? 1 : 0, b_.g[4]);
    LHI_LAUNCH_CHECK();
    launch_wgrad(b_.g[4], 16, 16, b_.q0, 32, 32, d0, GW(4), status_, s);
    launch_conv(b_.g[4], 16, WB(4), 32, nullptr, 32, d0, 1, nullptr, 0, nullptr, b_.dx, status_, s);
    k_sum_children<<<nb(V1 * 32), 256, 0, s>>>(b_.dx, d0[1], d0[2], b_.acc, d1[0], d1[1], d1[2], 32);
    LHI_LAUNCH_CHECK();
    // layer 3
    k_relu_grad<<<nb(V1 * 32), 256, 0, s>>>(b_.acc, b_.u1, V1 * 32, relu_ ? 1 : 0, b_.g[3]);
    LHI_LAUNCH_CHECK();
    launch_wgrad(b_.g[3], 32, 32, b_.q1, 64, 64, d1, GW(3), status_, s);
    launch_conv(b_.g[3], 32, WB(3), 64, nullptr, 64, d1, 1, nullptr, 0, nullptr, b_.dx, status_, s);
    k_sum_children<<<nb(V2 * 64), 256, 0, s>>>(b_.dx, d1[1], d1[2], b_.acc, d2[0], d2[1], d2[2], 64);
    LHI_LAUNCH_CHECK();
    // layer 2
    k_relu_grad<<<nb(V2 * 64), 256, 0, s>>>(b_.acc, b_.h2, V2 * 64, relu_ ? 1 : 0, b_.g[2]);
    LHI_LAUNCH_CHECK();
    launch_wgrad(b_.g[2], 64, 64, b_.p1, 32, 32, d2, GW(2), status_, s);
    launch_conv(b_.g[2], 64, WB(2), 32, nullptr, 32, d2, 1, nullptr, 0, nullptr, b_.dx, status_, s);
    // layer 1: dh1 = g3 (skip) + unpool(dp1) / 8
    k_relu_grad_unpool<<<nb(V1 * 32), 256, 0, s>>>(b_.g[3], b_.dx, d2[0], d2[1], d2[2], b_.h1, d1[0], d1[1], d1[2], 32,
                                                    relu_ ? 1 : 0, b_.g[1]);
    LHI_LAUNCH_CHECK();
    launch_wgrad(b_.g[1], 32, 32, b_.p0, 16, 16, d1, GW(1), status_, s);
    launch_conv(b_.g[1], 32, WB(1), 16, nullptr, 16, d1, 1, nullptr, 0, nullptr, b_.dx, status_, s);
    // layer 0: dh0 = g4 (skip) + unpool(dp0) / 8
    k_relu_grad_unpool<<<nb(V0 * 16), 256, 0, s>>>(b_.g[4], b_.dx, d1[0], d1[1], d1[2], b_.h0, d0[0], d0[1], d0[2], 16,
                                                    relu_ ? 1 : 0, b_.g[0]);
    LHI_LAUNCH_CHECK();
    launch_wgrad(b_.g[0], 16, 16, b_.a0, 16, 4, d0, GW(0), status_, s);
}

int umma_selftest(const uint16_t* a_host, const uint16_t* b_host, int N, int K, float* d_host, int* stage) {
    if (N < 16 || N > 64 || N % 16 || K < 16 || K > 64 || K % 16) throw std::invalid_argument("selftest: N, K in {16, 32, 48, 64}");
    uint16_t *a = nullptr, *b = nullptr;
    float* d = nullptr;
    NetStatus* st = nullptr;
    LHI_CUDA(cudaMalloc(&a, 2 * 128 * K));
    LHI_CUDA(cudaMalloc(&b, 2 * N * K));
    LHI_CUDA(cudaMalloc(&d, 4 * 128 * N));
    LHI_CUDA(cudaMalloc(&st, sizeof(NetStatus)));
    LHI_CUDA(cudaMemset(st, 0, sizeof(NetStatus)));
    LHI_CUDA(cudaMemset(d, 0, 4 * 128 * N));
    LHI_CUDA(cudaMemcpy(a, a_host, 2 * 128 * K, cudaMemcpyHostToDevice));
    LHI_CUDA(cudaMemcpy(b, b_host, 2 * N * K, cudaMemcpyHostToDevice));
    k_umma_selftest<<<1, 128>>>(a, b, N, K, d, st);
    LHI_LAUNCH_CHECK();
    LHI_CUDA(cudaDeviceSynchronize());
    NetStatus h{};
    LHI_CUDA(cudaMemcpy(&h, st, sizeof(h), cudaMemcpyDeviceToHost));
    LHI_CUDA(cudaMemcpy(d_host, d, 4 * 128 * N, cudaMemcpyDeviceToHost));
    cudaFree(a);
    cudaFree(b);
    cudaFree(d);
    cudaFree(st);
    *stage = h.pad[3];
    return h.timeout ? LHI_E_TIMEOUT : LHI_OK;
}

void LearnedNet::adam_step(double lr, double beta1, double beta2, double eps, cudaStream_t s) {
    ++adam_t_;
    const double c1 = 1.0 - std::pow(beta1, double(adam_t_));
    const double c2 = 1.0 - std::pow(beta2, double(adam_t_));
    const long long n = net_param_count();
    k_adam<<<nb(n), 256, 0, s>>>(w32_, grad_, adam_m_, adam_v_, n, float(lr), float(beta1), float(beta2), float(eps),
                                 float(c1), float(c2));
    LHI_LAUNCH_CHECK();
    wfmt_stale_ = true;
}

}  // namespace lhi
