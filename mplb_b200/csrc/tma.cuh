// Inline-PTX wrappers for mbarriers and TMA tiled loads (sm_100a) and the
// driver's tensor-map encoder, for the warm-start network's kernels.
//
// Every wait here is bounded: a wait that runs out of polls returns false
// and the caller records an error word and winds the kernel down.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

namespace mplb {
namespace tma {

// Polls before a barrier wait gives up (each try_wait suspends the thread for
// a hardware-chosen interval, so this is seconds, far beyond any real wait).
constexpr long long kWaitLimit = 1ll << 24;

__device__ __forceinline__ uint32_t SmemAddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void BarInit(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)),
                 "r"(count));
}

__device__ __forceinline__ void FenceBarrierInit() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void FenceProxyAsync() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void BarArriveExpectTx(uint64_t* bar,
                                                  uint32_t bytes) {
    asm volatile(
        "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
            SmemAddr(bar)),
        "r"(bytes)
        : "memory");
}

__device__ __forceinline__ bool BarTryWait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(SmemAddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete; false on timeout or
// when another thread of the CTA has already flagged an error (cta_err, may
// be null).
__device__ __forceinline__ bool BarWait(uint64_t* bar, uint32_t parity,
                                        volatile int* cta_err) {
    for (long long i = 0; i < kWaitLimit; i++) {
        if (BarTryWait(bar, parity)) return true;
        if ((i & 1023) == 1023 && cta_err != nullptr && *cta_err) return false;
    }
    return false;
}

// Bounded wait that ignores any error word (used to drain copies still in
// flight before a CTA exits after an error).
__device__ __forceinline__ bool BarWaitDrain(uint64_t* bar, uint32_t parity) {
    for (long long i = 0; i < kWaitLimit; i++)
        if (BarTryWait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void PrefetchTmap(const CUtensorMap* m) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(m))
                 : "memory");
}

// Tiled TMA loads into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void TmaLoad2D(void* dst, const CUtensorMap* m,
                                          uint64_t* bar, int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::"
        "bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(SmemAddr(dst)),
        "l"(reinterpret_cast<uint64_t>(m)), "r"(SmemAddr(bar)), "r"(c0),
        "r"(c1)
        : "memory");
}

__device__ __forceinline__ void TmaLoad4D(void* dst, const CUtensorMap* m,
                                          uint64_t* bar, int c0, int c1,
                                          int c2, int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::"
        "bytes [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(SmemAddr(dst)),
        "l"(reinterpret_cast<uint64_t>(m)), "r"(SmemAddr(bar)), "r"(c0),
        "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}

// cuTensorMapEncodeTiled from the driver (no link against libcuda), or null.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType,
                                  cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);
inline EncodeTiledFn Encoder() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p,
                                             12000, cudaEnableDefault,
                                             &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

}  // namespace tma
}  // namespace mplb
