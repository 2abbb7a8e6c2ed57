// Definitions of the launchers declared in launch.h (included by the
// translation units that instantiate them).
#pragma once

#include <algorithm>

#include "launch.h"
#include "swap.cuh"

namespace mplb {

static_assert(kSplitCta == kStepThreads, "SplitStepKernel CTA size");

// CTAs of SplitStepKernel / SplitSwapKernel for block b (0: too many).
template <int D, typename T>
long long SplitBlocks(const BlockDev& b) {
    const long long nbx = (b.n[0] + kStepThreads - 1) / kStepThreads;
    const long long ny = b.n[1] - 2;
    const long long nz = D == 3 ? b.n[2] : 1;
    const long long rows = ny * (D == 3 ? b.n[2] - 2 : 1);
    const long long nsr = nbx * (2 * nz + (D == 3 ? 2 * ny : 0));
    const long long chunks = (rows + kSplitRows - 1) / kSplitRows;
    const long long blocks =
        nsr + chunks * SplitChunkCtas<SplitGroup<T>()>(b.n[0]);
    return blocks > 0x7fffffffLL ? 0 : blocks;
}

// Task geometry of PipeStepKernel for block b.
template <int D, typename T>
PipeGeom PipeGeometry(const BlockDev& b) {
    constexpr int S = SectorNodes<T>();
    constexpr int G = SplitGroup<T>();
    PipeGeom g;
    g.xs = S;
    g.xe = b.n[0] - S;
    g.tpr = (g.xe - g.xs + 32 * G - 1) / (32 * G);
    g.ny = b.n[1] - 2;
    g.rows = (long long)g.ny * (D == 3 ? b.n[2] - 2 : 1);
    g.tasks = (long long)g.tpr * g.rows;
    return g;
}

// Persistent grid of PipeStepKernel: the CTAs that fit on the device at
// once (looked up once per instantiation).
template <int D, typename T, bool O32>
unsigned PipeCtas() {
    static const unsigned ctas = [] {
        int dev = 0, sms = 0, per = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount,
                                   dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per, PipeStepKernel<D, T, O32>, kStepThreads, 0) !=
                cudaSuccess)
            return 0u;
        return (unsigned)(sms * (per > 0 ? per : 1));
    }();
    return ctas;
}

// parts: bit 0 the edge launch (shell rows and row edges), bit 1 the
// pipelined interior; the edge launch goes first when both are asked for.
template <int D, typename T, bool O32>
cudaError_t LaunchPipe(cudaStream_t s, const BlockDev& b, const PhysConst& pc,
                       const T* src, T* dst, int parts) {
    constexpr int S = SectorNodes<T>();
    const PipeGeom g = PipeGeometry<D, T>(b);
    const long long nbx = (b.n[0] + kStepThreads - 1) / kStepThreads;
    const long long nz = D == 3 ? b.n[2] : 1;
    const long long nsr = nbx * (2 * nz + (D == 3 ? 2 * (long long)g.ny : 0));
    const long long edge =
        nsr + (g.rows * 2 * S + kStepThreads - 1) / kStepThreads;
    const unsigned ctas = PipeCtas<D, T, O32>();
    if (edge > 0x7fffffffLL || ctas == 0) return cudaErrorInvalidConfiguration;
    if (parts & 1) {
        EdgeStepKernel<D, T, O32><<<(unsigned)edge, kStepThreads, 0, s>>>(
            b, pc, src, dst, g);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if ((parts & 2) && g.tasks > 0) {
        const unsigned grid = (unsigned)std::min<long long>(ctas, g.tasks);
        PipeStepKernel<D, T, O32><<<grid, kStepThreads, 0, s>>>(b, pc, src,
                                                                dst, g);
    }
    return cudaGetLastError();
}

template <int D, typename T>
cudaError_t Launch<D, T>::StepPart(int part, cudaStream_t s, const BlockDev& b,
                                   const PhysConst& pc, const T* src, T* dst) {
    if (!(b.split && b.pipe) || (part != 1 && part != 2))
        return cudaErrorInvalidValue;
    const int parts = part == 1 ? 2 : 1;
    return b.off32 ? LaunchPipe<D, T, true>(s, b, pc, src, dst, parts)
                   : LaunchPipe<D, T, false>(s, b, pc, src, dst, parts);
}

template <int D, typename T>
cudaError_t Launch<D, T>::Step(int mode, dim3 grid, cudaStream_t s,
                               const BlockDev& b, const PhysConst& pc,
                               const T* src, T* dst, double* o0, double* o1,
                               double* o2, double* o3) {
    if (mode == kModeStep && b.split && b.pipe) {
        return b.off32 ? LaunchPipe<D, T, true>(s, b, pc, src, dst, 3)
                       : LaunchPipe<D, T, false>(s, b, pc, src, dst, 3);
    }
    if (mode == kModeStep && b.split) {
        const long long blocks = SplitBlocks<D, T>(b);
        if (blocks == 0) return cudaErrorInvalidConfiguration;
        if (b.off32)
            SplitStepKernel<D, T, true><<<(unsigned)blocks, kStepThreads, 0, s>>>(
                b, pc, src, dst);
        else
            SplitStepKernel<D, T, false><<<(unsigned)blocks, kStepThreads, 0, s>>>(
                b, pc, src, dst);
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
cudaError_t Launch<D, T>::Halo(unsigned grid, cudaStream_t s, const HaloDev& h,
                               const BlockDev& fb, const BlockDev& tb,
                               const T* cur_from, const T* prev_from,
                               T* cur_to) {
    HaloKernel<D, T><<<grid, 256, 0, s>>>(h, fb, tb, cur_from, prev_from,
                                          cur_to);
    return cudaGetLastError();
}

template <typename T, bool GATHER, bool BC, bool O32>
cudaError_t LaunchSplitSwap(cudaStream_t s, const BlockDev& b,
                            const PhysConst& pc, T* f) {
    const long long blocks = SplitBlocks<3, T>(b);
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
