// Thin inline-PTX wrappers for the sm_100a tensor-core path of the warm-start
// network (the mbarrier and TMA wrappers are tma.cuh's): tcgen05 (TMEM allocation, MMA with
// shared-memory operand descriptors, commit, TMEM loads) and the UMMA
// descriptor encodings.
//
// Descriptor formats (PTX ISA "tcgen05 matrix descriptors"; the bit layout is
// the one CUTLASS 4.5 spells out in cute/arch/mma_sm100_desc.hpp):
//   shared-memory descriptor (64 bit): start address >> 4 in [0,14), leading
//   byte offset >> 4 in [16,30), stride byte offset >> 4 in [32,46), version
//   1 in [46,48), base offset in [49,52), swizzle mode in [61,64) (2 = 128 B,
//   4 = 64 B).
//   instruction descriptor for kind::f16 (32 bit): D format in [4,6) (1 =
//   F32), A format [7,10) and B format [10,13) (1 = BF16), A major bit 15,
//   B major bit 16 (0 = K-major, 1 = MN-major), N >> 3 in [17,23), M >> 4 in
//   [24,29).
//
// Every wait here is bounded: a wait that runs out of polls returns false
// and the caller records an error word and winds the kernel down.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_bf16.h>

#include "../tma.cuh"

namespace mplb {
namespace umma {

using tma::BarArriveExpectTx;
using tma::BarInit;
using tma::BarTryWait;
using tma::BarWait;
using tma::BarWaitDrain;
using tma::FenceBarrierInit;
using tma::FenceProxyAsync;
using tma::kWaitLimit;
using tma::PrefetchTmap;
using tma::SmemAddr;
using tma::TmaLoad2D;
using tma::TmaLoad4D;

// ---- tensor memory ---------------------------------------------------------

// Whole warp: allocates `ncols` TMEM columns (power of two >= 32) and writes
// the base address to *dst (shared memory).
__device__ __forceinline__ void TmemAlloc(uint32_t* dst, uint32_t ncols) {
    asm volatile(
        "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::
            "r"(SmemAddr(dst)),
        "r"(ncols)
        : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::
                     : "memory");
}

__device__ __forceinline__ void TmemFree(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(
                     taddr),
                 "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void FenceBeforeSync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void FenceAfterSync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, one elected thread.
__device__ __forceinline__ void Mma(uint32_t d_tmem, uint64_t a_desc,
                                   uint64_t b_desc, uint32_t idesc,
                                   uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(
            d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrives once on `bar` when every tcgen05 operation this thread issued so
// far has completed.
__device__ __forceinline__ void Commit(uint64_t* bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
        "[%0];" ::"r"(SmemAddr(bar))
        : "memory");
}

// Warp: 32 TMEM lanes (this warp's quarter) x 16 consecutive 32-bit columns.
__device__ __forceinline__ void TmemLoad16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]),
          "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
          "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// ---- descriptors -----------------------------------------------------------

// swizzle_bytes: 128 or 64.  K-major: rows of `swizzle_bytes` along K, 8-row
// groups `sbo` bytes apart (= 8 * swizzle_bytes for a dense tile).  MN-major:
// rows of swizzle_bytes along MN (one K index per row), 8-row K groups `sbo`
// apart, MN atoms `lbo` apart.
__device__ __forceinline__ uint64_t SmemDesc(uint32_t saddr, uint32_t lbo,
                                             uint32_t sbo,
                                             int swizzle_bytes) {
    const uint64_t mode = swizzle_bytes == 128 ? 2ull : 4ull;
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= 1ull << 46;
    d |= mode << 61;
    return d;
}

__host__ __device__ constexpr uint32_t InstrDescBf16(int m, int n, bool a_mn,
                                                     bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) |
           ((b_mn ? 1u : 0u) << 16) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

}  // namespace umma
}  // namespace mplb
