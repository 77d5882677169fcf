// tma.cuh — tensor-memory-accelerator (TMA) tile loads and mbarrier pipelines for the persistent step passes.
//
// A persistent pass keeps one block per SM. Its producer warp streams wave tiles from HBM into a ring of
// shared-memory stages with cp.async.bulk.tensor (one elected thread; the copy engine moves the tile while
// the consumer warps transform the previous one), and two mbarriers per stage hand each stage over:
//   full[s]  : the producer arms it with the tile's byte count; the copy engine completes it
//   empty[s] : each consumer warp arrives once it has read the stage for the last time (or, in the passes that
//              store through TMA, once it has written its results into the stage)
// All loads are plain (no cluster multicast) and read this GPU's own wave buffer; stores write only it.
//
// Every wait is bounded: a wait that does not complete within kWaitSpins polls records an error code in a
// device word the host reads after the launch and reports, and the kernel winds down instead of hanging.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace ms {

// error codes a persistent pass records in its error word (0 = none)
enum StepError : int { STEP_OK = 0, STEP_WAIT_FULL = 1, STEP_WAIT_EMPTY = 2, STEP_WAIT_DRAIN = 3 };

// polls of try_wait before a wait is abandoned: each poll suspends for up to the hardware's time limit, so
// this bound is seconds, far beyond any healthy wait (microseconds)
constexpr unsigned kWaitSpins = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// make the initialised barriers visible to the async proxy (the copy engine) and to the other threads
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// wait for the phase of `parity` to complete; false (with *err set to code) if it did not within the bound
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int *err, int code) {
    for (unsigned i = 0; i < kWaitSpins; i++)
        if (mbar_try_wait(bar, parity)) return true;
    atomicCAS(err, 0, code);
    return false;
}

// order this thread's generic-proxy shared-memory accesses before later async-proxy (copy engine) accesses
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap *m) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(m)) : "memory");
}
// 2-D tiled load of the box at element coordinates (x, y) of tensor map `m` into shared memory at dst;
// completion is signalled on `bar` as transferred bytes. x times the element size must be a multiple of 16.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *m, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(m)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// 2-D tiled store of the box at element coordinates (x, y) of tensor map `m` from shared memory at src, in
// this thread's current bulk async-group; same alignment rule as the load. The source must have been written
// before a fence.proxy.async by its writers and a barrier that orders them before this thread.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *m, int x, int y, const void *src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<uint64_t>(m)),
                 "r"(x), "r"(y), "r"(smem_u32(src))
                 : "memory");
}
// 1-D bulk copy of `bytes` from global memory at src into shared memory at dst (both 16-byte aligned, bytes a
// multiple of 16); completion is signalled on `bar` as transferred bytes
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// wait until this thread's bulk groups have finished reading their shared-memory sources (the stage may be
// overwritten), or have completed entirely (their global writes are done)
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// wait until at most PENDING of this thread's most recent bulk groups are still reading their sources
template <int PENDING> __device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(PENDING) : "memory");
}

// named barrier over `count` threads (a multiple of 32) of the block
struct NamedBar {
    int id, count;
    __device__ __forceinline__ void operator()() const { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory"); }
};

// Host: a 2-D tensor map over `rows` rows of `row_floats` FP32 values (row stride row_floats * 4 bytes) at
// `base`, with boxes of box_floats x box_rows, no interleave, and the shared-memory swizzle of swizzle_bytes
// (0: none; 32, 64 or 128: 16-byte chunks XORed with the row's position in a 256 / 512 / 1024-byte atom, which
// needs a box row of at most that many bytes and stage addresses aligned to 1024 bytes). cuTensorMapEncodeTiled checks the
// base (16-byte aligned), the stride and the box's inner extent (multiples of 16 bytes); the kernels keep
// every box's x coordinate a multiple of box_floats, so each copy starts on a 16-byte boundary.
inline CUtensorMap wave_tensor_map(const void *base, unsigned long long row_floats, unsigned long long rows,
                                   unsigned box_floats, unsigned box_rows, int swizzle_bytes = 0) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        cudaError_t e = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
            throw std::runtime_error("cuTensorMapEncodeTiled is not available from the driver");
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    if ((box_floats * 4) % 16 != 0 || box_floats > 256 || box_rows > 256 || box_rows == 0 ||
        (reinterpret_cast<uintptr_t>(base) & 15) != 0 || (row_floats * 4) % 16 != 0)
        throw std::runtime_error("tensor map: misaligned base, stride or box");
    CUtensorMapSwizzle sw = CU_TENSOR_MAP_SWIZZLE_NONE;
    if (swizzle_bytes == 32) sw = CU_TENSOR_MAP_SWIZZLE_32B;
    else if (swizzle_bytes == 64) sw = CU_TENSOR_MAP_SWIZZLE_64B;
    else if (swizzle_bytes == 128) sw = CU_TENSOR_MAP_SWIZZLE_128B;
    else if (swizzle_bytes != 0) throw std::runtime_error("tensor map: swizzle must be 0, 32, 64 or 128 bytes");
    if (swizzle_bytes && box_floats * 4 > (unsigned)swizzle_bytes)
        throw std::runtime_error("tensor map: box row wider than the swizzle span");
    CUtensorMap m;
    const cuuint64_t dims[2] = {row_floats, rows};
    const cuuint64_t strides[1] = {row_floats * 4};
    const cuuint32_t box[2] = {box_floats, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = encode(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return m;
}

}  // namespace ms
