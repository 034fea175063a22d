// async_copy.cuh — bulk global->shared copies (TMA, 1-D, no multicast) completed
// on a CTA-local mbarrier, with bounded waits.
//
// A copy must start and end on 16-byte boundaries (source, destination and
// size).  Waits spin at most kMbarSpinLimit polls; a wait that runs out returns
// false and the caller records LLG_ERR_TIMEOUT in the film's state instead of
// hanging the GPU.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace llg {

constexpr int kErrAsyncTimeout = -3;   // LLG_ERR_TIMEOUT
constexpr long long kMbarSpinLimit = 1LL << 26;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Make barrier initialisation visible to the async proxy (then __syncthreads()).
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Order this thread's earlier generic-proxy shared-memory accesses before later
// async-proxy writes (a bulk copy into a buffer the block has just read).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity to complete; false after the spin limit.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (long long i = 0; i < kMbarSpinLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 16-byte asynchronous global->shared copy (per thread), completed by cp_async_wait_all().
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// 16-byte vector of reals (float4 / double2 shaped) for vectorised plane access.
template <typename R>
struct alignas(16) Vec16 {
    static constexpr int W = 16 / (int)sizeof(R);
    R v[W];
};
// W consecutive reals loaded / stored as one vector (W * sizeof(R) bytes, aligned).
template <typename R, int W>
struct alignas(sizeof(R) * W) VecW {
    R v[W];
};
template <typename R, int W>
__device__ __forceinline__ VecW<R, W> ldw(const R* p) {
    return *reinterpret_cast<const VecW<R, W>*>(p);
}
template <typename R, int W>
__device__ __forceinline__ void stw(R* p, const VecW<R, W>& x) {
    *reinterpret_cast<VecW<R, W>*>(p) = x;
}
template <typename R>
__device__ __forceinline__ Vec16<R> ldv(const R* p) {
    return *reinterpret_cast<const Vec16<R>*>(p);
}
template <typename R>
__device__ __forceinline__ void stv(R* p, const Vec16<R>& x) {
    *reinterpret_cast<Vec16<R>*>(p) = x;
}

}  // namespace llg
