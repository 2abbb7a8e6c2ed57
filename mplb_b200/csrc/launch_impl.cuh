// Definitions of the launchers declared in launch.h (included by the
// translation units that instantiate them).
#pragma once

#include "launch.h"
#include "swap.cuh"

namespace mplb {

static_assert(kSplitCta == kStepThreads, "SplitStepKernel CTA size");
static_assert(StageSmemBytes<3, __half>() <= 48 * 1024,
              "staged interior within the default shared memory");

// CTAs of SplitStepKernel (STAGED: with the staged interior of
// StagedStep<T>()) or SplitSwapKernel (never staged) for block b (0: too
// many).
template <int D, typename T, bool STAGED = StagedStep<T>()>
long long SplitBlocks(const BlockDev& b) {
    const long long nbx = (b.n[0] + kStepThreads - 1) / kStepThreads;
    const long long ny = b.n[1] - 2;
    const long long nz = D == 3 ? b.n[2] : 1;
    const long long rows = ny * (D == 3 ? b.n[2] - 2 : 1);
    const long long nsr = nbx * (2 * nz + (D == 3 ? 2 * ny : 0));
    const long long chunks = (rows + kSplitRows - 1) / kSplitRows;
    const long long blocks =
        nsr + chunks * SplitChunkCtas<SplitGroup<T>(), STAGED>(b.n[0]);
    return blocks > 0x7fffffffLL ? 0 : blocks;
}

// Shell-row CTAs of SplitStepKernel for block b (its first CTAs).
template <int D>
long long SplitShellBlocks(const BlockDev& b) {
    const long long nbx = (b.n[0] + kStepThreads - 1) / kStepThreads;
    const long long ny = b.n[1] - 2;
    const long long nz = D == 3 ? b.n[2] : 1;
    return nbx * (2 * nz + (D == 3 ? 2 * ny : 0));
}

template <int D, typename T>
cudaError_t Launch<D, T>::StepPart(int part, cudaStream_t s, const BlockDev& b,
                                   const PhysConst& pc, const T* src, T* dst) {
    if (!b.split || (part != 1 && part != 2)) return cudaErrorInvalidValue;
    const long long blocks = SplitBlocks<D, T>(b);
    if (blocks == 0) return cudaErrorInvalidConfiguration;
    const long long shell = SplitShellBlocks<D>(b);
    // part 1: x faces and interior rows (CTAs shell .. blocks - 1);
    // part 2: the shell rows (CTAs 0 .. shell - 1)
    const unsigned grid = (unsigned)(part == 1 ? blocks - shell : shell);
    const unsigned blk0 = part == 1 ? (unsigned)shell : 0u;
    if (grid == 0) return cudaSuccess;
    const int smem = StagedStep<T>() ? StageSmemBytes<D, T>() : 0;
    if (b.off32)
        SplitStepKernel<D, T, true><<<grid, kStepThreads, smem, s>>>(
            b, pc, src, dst, blk0, 0u);
    else
        SplitStepKernel<D, T, false><<<grid, kStepThreads, smem, s>>>(
            b, pc, src, dst, blk0, 0u);
    return cudaGetLastError();
}

template <int D, typename T>
cudaError_t Launch<D, T>::Step(int mode, dim3 grid, cudaStream_t s,
                               const BlockDev& b, const PhysConst& pc,
                               const T* src, T* dst, double* o0, double* o1,
                               double* o2, double* o3) {
    if (mode == kModeStep && b.split) {
        if (SplitBlocks<D, T>(b) == 0) return cudaErrorInvalidConfiguration;
        // the shell rows interleaved with the chunks: spc of them after
        // each chunk's CTAs
        const long long nsr = SplitShellBlocks<D>(b);
        const long long rows =
            (long long)(b.n[1] - 2) * (D == 3 ? b.n[2] - 2 : 1);
        const long long chunks = (rows + kSplitRows - 1) / kSplitRows;
        const long long per_chunk =
            SplitChunkCtas<SplitGroup<T>(), StagedStep<T>()>(b.n[0]);
        const long long spc = (nsr + chunks - 1) / chunks;
        const long long blocks = chunks * (per_chunk + spc);
        if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
        const int smem = StagedStep<T>() ? StageSmemBytes<D, T>() : 0;
        if (b.off32)
            SplitStepKernel<D, T, true><<<(unsigned)blocks, kStepThreads, smem,
                                          s>>>(b, pc, src, dst, 0u,
                                               (unsigned)spc);
        else
            SplitStepKernel<D, T, false><<<(unsigned)blocks, kStepThreads,
                                           smem, s>>>(b, pc, src, dst, 0u,
                                                      (unsigned)spc);
    } else if (mode == kModeStep && b.off32)
        StepKernel<D, T, kModeStep, true><<<grid, kStepThreads, 0, s>>>(
            b, pc, src, dst, o0, o1, o2, o3);
    else if (mode == kModeStep)
        StepKernel<D, T, kModeStep><<<grid, kStepThreads, 0, s>>>(
            b, pc, src, dst, o0, o1, o2, o3);
    else if (mode == kModeMacro)
        StepKernel<D, T, kModeMacro><<<grid, kStepThreads, 0, s>>>(
            b, pc, src, dst, o0, o1, o2, o3);
    else
        StepKernel<D, T, kModeF><<<grid, kStepThreads, 0, s>>>(
            b, pc, src, dst, o0, o1, o2, o3);
    return cudaGetLastError();
}

template <int D, typename T>
cudaError_t Launch<D, T>::DeferredFused(unsigned grid, cudaStream_t s,
                                        const BlockDev& b, const PhysConst& pc,
                                        const T* src, T* dst) {
    DeferredFusedKernel<D, T><<<grid, kStepThreads, 0, s>>>(b, pc, src, dst);
    return cudaGetLastError();
}

template <int D, typename T>
cudaError_t Launch<D, T>::DeferredStream(unsigned grid, cudaStream_t s,
                                         const BlockDev& b,
                                         const PhysConst& pc, const T* src) {
    DeferredStreamKernel<D, T><<<grid, kStepThreads, 0, s>>>(b, pc, src);
    return cudaGetLastError();
}

template <int D, typename T>
cudaError_t Launch<D, T>::DeferredOp(unsigned grid, cudaStream_t s,
                                     const BlockDev& b, const PhysConst& pc,
                                     const T* src, const DeferredSeg* segs,
                                     int nseg, long long total) {
    DeferredOpKernel<D, T><<<grid, kStepThreads, 0, s>>>(b, pc, src, segs,
                                                         nseg, total);
    return cudaGetLastError();
}

template <int D, typename T>
cudaError_t Launch<D, T>::DeferredFinish(int mode, unsigned grid,
                                         cudaStream_t s, const BlockDev& b,
                                         const PhysConst& pc, T* dst,
                                         double* o0, double* o1, double* o2,
                                         double* o3) {
    if (mode == kModeStep)
        DeferredFinishKernel<D, T, kModeStep><<<grid, kStepThreads, 0, s>>>(
            b, pc, dst, o0, o1, o2, o3);
    else if (mode == kModeMacro)
        DeferredFinishKernel<D, T, kModeMacro><<<grid, kStepThreads, 0, s>>>(
            b, pc, dst, o0, o1, o2, o3);
    else
        DeferredFinishKernel<D, T, kModeF><<<grid, kStepThreads, 0, s>>>(
            b, pc, dst, o0, o1, o2, o3);
    return cudaGetLastError();
}

template <int D, typename T>
cudaError_t Launch<D, T>::FillZero(cudaStream_t s, T* p, long long popstride,
                                   int Q, const PhysConst& pc) {
    FillZeroFKernel<T><<<1024, 256, 0, s>>>(p, popstride, Q, pc);
    return cudaGetLastError();
}

template <int D, typename T>
cudaError_t Launch<D, T>::Init(dim3 grid, cudaStream_t s, const BlockDev& b,
                               const PhysConst& pc, const double* rho,
                               const double* u, const double* v,
                               const double* w, const double* fin, T* fdirect,
                               T* g) {
    InitKernel<D, T><<<grid, kStepThreads, 0, s>>>(b, pc, rho, u, v, w, fin,
                                                   fdirect, g);
    return cudaGetLastError();
}

template <int D, typename T>
cudaError_t Launch<D, T>::DirectObserve(int mode, dim3 grid, cudaStream_t s,
                                        const BlockDev& b,
                                        const PhysConst& pc, const T* fdirect,
                                        double* o0, double* o1, double* o2,
                                        double* o3) {
    if (mode == kModeMacro)
        DirectObserveKernel<D, T, kModeMacro><<<grid, kStepThreads, 0, s>>>(
            b, pc, fdirect, o0, o1, o2, o3);
    else
        DirectObserveKernel<D, T, kModeF><<<grid, kStepThreads, 0, s>>>(
            b, pc, fdirect, o0, o1, o2, o3);
    return cudaGetLastError();
}

template <int D, typename T>
cudaError_t Launch<D, T>::Face(bool exp, unsigned grid, cudaStream_t s,
                               const BlockDev& b, const FaceDev& fd, T* f,
                               T* buf) {
    if (exp)
        FaceKernel<D, T, true><<<grid, 256, 0, s>>>(b, fd, f, buf);
    else
        FaceKernel<D, T, false><<<grid, 256, 0, s>>>(b, fd, f, buf);
    return cudaGetLastError();
}

template <int D, typename T>
cudaError_t Launch<D, T>::HaloFused(cudaStream_t s, const HaloFusedDev& h,
                                    int cur, unsigned ctas) {
    HaloFusedKernel<D, T><<<ctas, kHaloThreads, 0, s>>>(h, cur);
    return cudaGetLastError();
}

template <typename T, bool GATHER, bool BC, bool O32>
cudaError_t LaunchSplitSwap(cudaStream_t s, const BlockDev& b,
                            const PhysConst& pc, T* f) {
    const long long blocks = SplitBlocks<3, T, false>(b);
    if (blocks == 0) return cudaErrorInvalidConfiguration;
    SplitSwapKernel<T, GATHER, BC, O32><<<(unsigned)blocks, kStepThreads, 0,
                                          s>>>(b, pc, f);
    return cudaGetLastError();
}

template <typename T, int MODE, bool O32>
cudaError_t LaunchSwap(bool gather, bool bc, dim3 grid, cudaStream_t s,
                       const BlockDev& b, const PhysConst& pc, T* f,
                       double* o0, double* o1, double* o2, double* o3) {
    if (MODE == kModeStep && b.split) {
        if (gather && !bc) return cudaErrorInvalidValue;
        if (gather) return LaunchSplitSwap<T, true, true, O32>(s, b, pc, f);
        if (bc) return LaunchSplitSwap<T, false, true, O32>(s, b, pc, f);
        return LaunchSplitSwap<T, false, false, O32>(s, b, pc, f);
    }
    if (gather && bc)
        SwapKernel<T, MODE, true, true, O32><<<grid, kStepThreads, 0, s>>>(
            b, pc, f, o0, o1, o2, o3);
    else if (gather)
        return cudaErrorInvalidValue;   // a gathered state always has one
    else if (bc)
        SwapKernel<T, MODE, false, true, O32><<<grid, kStepThreads, 0, s>>>(
            b, pc, f, o0, o1, o2, o3);
    else
        SwapKernel<T, MODE, false, false, O32><<<grid, kStepThreads, 0, s>>>(
            b, pc, f, o0, o1, o2, o3);
    return cudaGetLastError();
}

template <int D, typename T>
cudaError_t Launch<D, T>::Swap(int mode, bool gather, bool bc, dim3 grid,
                               cudaStream_t s, const BlockDev& b,
                               const PhysConst& pc, T* f, double* o0,
                               double* o1, double* o2, double* o3) {
    if constexpr (D != 3) {
        return cudaErrorInvalidValue;
    } else {
        if (mode == kModeStep)
            return b.off32 ? LaunchSwap<T, kModeStep, true>(
                                 gather, bc, grid, s, b, pc, f, o0, o1, o2, o3)
                           : LaunchSwap<T, kModeStep, false>(
                                 gather, bc, grid, s, b, pc, f, o0, o1, o2, o3);
        if (mode == kModeMacro)
            return LaunchSwap<T, kModeMacro, false>(gather, bc, grid, s, b, pc,
                                                    f, o0, o1, o2, o3);
        return LaunchSwap<T, kModeF, false>(gather, bc, grid, s, b, pc, f, o0,
                                            o1, o2, o3);
    }
}

}  // namespace mplb
