// Host-side launchers of the step kernels, one instantiation per lattice
// dimension and storage form.  The FP64 form is compiled in
// kernels_f64.cu with -fmad=false (bitwise reference arithmetic), the
// shifted FP32/FP16 forms in kernels_lp.cu with fused multiply-adds.
#pragma once

#include <cuda_runtime.h>

#include "kernels.cuh"

namespace mplb {

template <int D, typename T>
struct Launch {
    static cudaError_t Step(int mode, dim3 grid, cudaStream_t s,
                            const BlockDev& b, const PhysConst& pc,
                            const T* src, T* dst, double* o0, double* o1,
                            double* o2, double* o3);
    // the two parts of a split step (b.split): 1 = the x faces and the
    // interior rows (no node of theirs reads a halo layer beyond a y or z
    // face), 2 = the shell rows
    static cudaError_t StepPart(int part, cudaStream_t s, const BlockDev& b,
                                const PhysConst& pc, const T* src, T* dst);
    static cudaError_t DeferredFused(unsigned grid, cudaStream_t s,
                                     const BlockDev& b, const PhysConst& pc,
                                     const T* src, T* dst);
    static cudaError_t DeferredStream(unsigned grid, cudaStream_t s,
                                      const BlockDev& b, const PhysConst& pc,
                                      const T* src);
    static cudaError_t DeferredOp(unsigned grid, cudaStream_t s,
                                  const BlockDev& b, const PhysConst& pc,
                                  const T* src, const DeferredSeg* segs,
                                  int nseg, long long total);
    static cudaError_t DeferredFinish(int mode, unsigned grid, cudaStream_t s,
                                      const BlockDev& b, const PhysConst& pc,
                                      T* dst, double* o0, double* o1,
                                      double* o2, double* o3);
    // a population array (Q x popstride elements) set to f = 0
    static cudaError_t FillZero(cudaStream_t s, T* p, long long popstride,
                                int Q, const PhysConst& pc);
    static cudaError_t Init(dim3 grid, cudaStream_t s, const BlockDev& b,
                            const PhysConst& pc, const double* rho,
                            const double* u, const double* v, const double* w,
                            const double* fin, T* fdirect, T* g);
    static cudaError_t DirectObserve(int mode, dim3 grid, cudaStream_t s,
                                     const BlockDev& b, const PhysConst& pc,
                                     const T* fdirect, double* o0, double* o1,
                                     double* o2, double* o3);
    // every halo copy of a step in one launch (pop[cur] is current)
    static cudaError_t HaloFused(cudaStream_t s, const HaloFusedDev& h,
                                 int cur, unsigned ctas);
    // face exchange of a decomposed block: export (block -> buf) or import
    static cudaError_t Face(bool exp, unsigned grid, cudaStream_t s,
                            const BlockDev& b, const FaceDev& fd, T* f,
                            T* buf);
    // swap scheme (3D only): one step (kModeStep) or an observation of the
    // current f, from the array in place; gather: slots at their streamed
    // places; bc: boundary programme pending
    static cudaError_t Swap(int mode, bool gather, bool bc, dim3 grid,
                            cudaStream_t s, const BlockDev& b,
                            const PhysConst& pc, T* f, double* o0, double* o1,
                            double* o2, double* o3);
};

constexpr int kStepThreads = 128;

}  // namespace mplb
