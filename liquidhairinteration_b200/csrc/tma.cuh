// tma.cuh -- tensor-memory-accelerator staging of 3D grid boxes into shared
// memory: tensor-map encoding on the host, bulk tensor loads completing on an
// mbarrier, and a bounded wait on the device.
//
// Grid arrays are [nx][ny][pitch] with z fastest (pitch = nz for the Scalar
// fields, a multiple of 16 for byte fields), so a map's dimensions are
// (z, y, x) innermost first.  Boxes start on a z coordinate that is a
// multiple of 16 bytes, may start at negative x / y / z, and read zeros
// outside the grid.  No multicast: every CTA loads its own boxes.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "common.cuh"

namespace lhi {

// Host: a 3D tiled map over base[nx][ny][pitch] of esz-byte elements whose
// valid z extent is nz, copying boxes of (bz, by, bx) elements.
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        LHI_CUDA(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn)
            throw CudaError(cudaErrorNotSupported, "cuTensorMapEncodeTiled is not available from the driver");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    return encode;
}

inline CUtensorMap make_box_map(const void* base, CUtensorMapDataType dt, int esz, int nx, int ny, int nz,
                                int pitch, int bx, int by, int bz) {
    const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    CUtensorMap m;
    const cuuint64_t dims[3] = {cuuint64_t(nz), cuuint64_t(ny), cuuint64_t(nx)};
    const cuuint64_t strides[2] = {cuuint64_t(pitch) * esz, cuuint64_t(pitch) * ny * esz};
    const cuuint32_t box[3] = {cuuint32_t(bz), cuuint32_t(by), cuuint32_t(bx)};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encode(&m, dt, 3, const_cast<void*>(base), dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        throw CudaError(cudaErrorInvalidValue, "cuTensorMapEncodeTiled failed with CUresult " + std::to_string(int(r)));
    return m;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void bar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void bar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) writes to the same shared memory.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Box load at element coordinates (z, y, x) into dst; completes on bar.
__device__ __forceinline__ void tma_load_box(void* dst, const CUtensorMap* map, int z, int y, int x, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(z), "r"(y), "r"(x), "r"(smem_addr(bar))
        : "memory");
}

// 4D box load at element coordinates (c0 innermost .. c3) into dst.
__device__ __forceinline__ void tma_load_box4(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                              uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
            smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ uint64_t timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr uint64_t kWaitLimitNs = 200000000ull;  // 200 ms

// Waits for the barrier phase of this parity; gives up after limit_ns
// (200 ms unless the caller passes another limit).  A limit of 0 gives up
// at once, without looking at the barrier: the timeout path on demand.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, unsigned parity, uint64_t limit_ns = kWaitLimitNs) {
    if (limit_ns == 0) return false;
    const uint32_t addr = smem_addr(bar);
    uint64_t deadline = 0;
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        const uint64_t now = timer_ns();
        if (deadline == 0) deadline = now + limit_ns;
        else if (now > deadline) return false;
    }
}

}  // namespace lhi
