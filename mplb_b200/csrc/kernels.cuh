// CUDA kernels of the fused stream-collision step (sm_100a).
//
// State: g = post-collision populations (the reference's fStage after
// collision and halo transfer), structure of arrays per block with a one
// node halo: element (i, x, y, z) at
//     i * popstride + (z + 1) * plane + (y + 1) * pitch + (x + xoff)
// (no z halo in 2D).  One step reads g^n from `src` and writes g^{n+1} to
// `dst`: each node pulls its populations from the upstream nodes
// (KerStream3D), applies its boundary programme (ImplementBoundary3D),
// takes moments (UpdateMacroVars3D) and collides (KerCollideBGKIsothermal3D)
// - 2 Q values of memory traffic per node.
//
// FP64 arithmetic follows the reference's operation order exactly; the
// translation unit is compiled with -fmad=false so no product is fused into
// an add, and terms the reference multiplies by a zero lattice component
// are skipped (adding a signed zero never changes a non-zero sum).
#pragma once

#include <cstdint>

#include "lattice.h"
#include "plan.h"

namespace mplb {

struct PhysConst {
    double cs;
    double omc;        // 1 - omega
    double tw;         // tau * omega
    int force;         // BodyForce_1st
    int force_vel;     // Variable_U_Force family
    double hdta[3];    // dt * a / 2
    double cf[kMaxQ];  // CS c_i . a
    double w[kMaxQ];
};

struct BlockDev {
    int n[3];
    int xoff;
    long long pitch, plane, popstride;
    const RegionInfo* regions;
    const RegionOp* ops;
    double* stale;       // LOCAL regions' stale populations, node-major
    double* fdef;        // DEFERRED f store, population-major (Q x ndef)
    long long ndef;
    const int4* dregions;  // deferred regions: (region, base, count, -)
    int ndregions;
};

enum StepMode : int { kModeStep = 0, kModeMacro = 1, kModeF = 2 };

__device__ __forceinline__ int RegionOf(int x, int y, int z, const int n[3],
                                        int D) {
    const int rx = x == 0 ? 0 : (x == n[0] - 1 ? 2 : 1);
    const int ry = y == 0 ? 0 : (y == n[1] - 1 ? 2 : 1);
    const int rz = D == 2 ? 1 : (z == 0 ? 0 : (z == n[2] - 1 ? 2 : 1));
    return rx + 3 * ry + 9 * rz;
}

template <int D>
__device__ __forceinline__ long long NodeIndex(const BlockDev& b, int x, int y,
                                               int z) {
    return (long long)(D == 3 ? z + 1 : 0) * b.plane +
           (long long)(y + 1) * b.pitch + (long long)(x + b.xoff);
}

template <typename L>
__device__ __forceinline__ long long UpOffset(const BlockDev& b, int i) {
    // offset of the upstream node x - c_i
    return -((long long)L::cx(i) + (long long)L::cy(i) * b.pitch +
             (long long)L::cz(i) * b.plane);
}

__device__ __forceinline__ long long LocalIndex(const RegionInfo& R, int x,
                                                int y, int z) {
    return ((long long)(z - R.org[2]) * R.ext[1] + (y - R.org[1])) * R.ext[0] +
           (x - R.org[0]);
}

// Moments of f (KerCalcDensity3D, KerCalcU3D/V3D/W3D and the _Force
// variants, Src/model_kernel.inc:570-759).
template <typename L>
__device__ __forceinline__ void Moments(const double* f, const PhysConst& pc,
                                        bool fluidlike, double& rho,
                                        double u[3]) {
    constexpr int Q = L::Q;
    rho = 0.0;
#pragma unroll
    for (int i = 0; i < Q; i++) rho = rho + f[i];
#pragma unroll
    for (int a = 0; a < L::D; a++) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < Q; i++) {
            const int c = comp<L>(i, a);
            if (c > 0) s = s + pc.cs * f[i];
            if (c < 0) s = s - pc.cs * f[i];
        }
        s = s / rho;
        if (pc.force_vel && fluidlike) s = s + pc.hdta[a];
        u[a] = s;
    }
    if (L::D == 2) u[2] = 0.0;
}

// BGK collision (KerCollideBGKIsothermal3D with CalcBGKFeq and
// CalcBodyForce, Src/model_kernel.inc:410-455, model_host_device.h:25-82).
template <typename L>
__device__ __forceinline__ void Collide(double* f, const PhysConst& pc,
                                        bool fluidlike, double rho,
                                        const double u[3]) {
    constexpr int Q = L::Q;
    const double cu0 = pc.cs * u[0], cu1 = pc.cs * u[1], cu2 = pc.cs * u[2];
    const double u2 = L::D == 3 ? (u[0] * u[0] + u[1] * u[1]) + u[2] * u[2]
                                : u[0] * u[0] + u[1] * u[1];
    const bool force = pc.force && fluidlike;
#pragma unroll
    for (int i = 0; i < Q; i++) {
        double cu = 0.0;
        bool first = true;
        const int c0 = L::cx(i), c1 = L::cy(i), c2 = L::cz(i);
        if (c0 != 0) { cu = c0 > 0 ? cu0 : -cu0; first = false; }
        if (c1 != 0) {
            const double t = c1 > 0 ? cu1 : -cu1;
            cu = first ? t : cu + t;
            first = false;
        }
        if (c2 != 0) {
            const double t = c2 > 0 ? cu2 : -cu2;
            cu = first ? t : cu + t;
        }
        const double res = (1.0 + cu) + 0.5 * (cu * cu - u2);
        const double wr = pc.w[i] * rho;
        const double feq = wr * res;
        double g = feq + pc.omc * (f[i] - feq);
        if (force) g = g + pc.tw * (wr * pc.cf[i]);
        f[i] = g;
    }
}

// EQMDiffuseRefl (KerCutCellEQMDiffuseRefl3D, Src/boundary_kernel.inc:
// 1184-1276) with the wall constants precomputed per region.
template <typename L>
__device__ __forceinline__ void ApplyEqm(double* f, const RegionOp& op,
                                         const PhysConst& pc) {
    constexpr int Q = L::Q;
    double rhoIn = 0.0;
#pragma unroll
    for (int i = 0; i < Q; i++)
        if (op.in_mask >> i & 1u) rhoIn = rhoIn + f[i];
    const double rhoWall = (2.0 * rhoIn) / op.denom;
#pragma unroll
    for (int i = 0; i < Q; i++)
        if (op.par_mask >> i & 1u) f[i] = (pc.w[i] * rhoWall) * op.a[i];
#pragma unroll
    for (int i = 0; i < Q; i++)
        if (op.out_mask >> i & 1u)
            f[i] = f[L::opp(i)] + ((2.0 * rhoWall) * pc.w[i]) * op.b[i];
}

// Fused step over one block.  kModeStep writes g^{n+1}; kModeMacro and
// kModeF recompute the current f = post-boundary populations from the
// previous g and write moments or f instead (no collision).
template <int D, int MODE>
__global__ void __launch_bounds__(128)
    StepKernel(BlockDev b, PhysConst pc, const double* __restrict__ src,
               double* __restrict__ dst, double* __restrict__ out0,
               double* __restrict__ out1, double* __restrict__ out2,
               double* __restrict__ out3) {
    using L = Lattice<D>;
    constexpr int Q = L::Q;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = D == 3 ? (int)blockIdx.z : 0;
    if (x >= b.n[0]) return;
    const int r = RegionOf(x, y, z, b.n, D);
    const RegionInfo& R = b.regions[r];
    const int cls = R.cls;
    if (cls == kDeferred) return;
    const long long node = NodeIndex<D>(b, x, y, z);
    double f[Q];
    if (cls == kPure) {
#pragma unroll
        for (int i = 0; i < Q; i++)
            f[i] = src[i * b.popstride + node + UpOffset<L>(b, i)];
    } else {
        const uint32_t pull = R.pull;
        const uint32_t stale = R.stale;
        const double* st = b.stale + (R.side_base >= 0
                                          ? (R.side_base + LocalIndex(R, x, y, z)) * Q
                                          : 0);
#pragma unroll
        for (int i = 0; i < Q; i++) {
            if (pull >> i & 1u)
                f[i] = src[i * b.popstride + node + UpOffset<L>(b, i)];
            else if (stale >> i & 1u)
                f[i] = st[i];
            else
                f[i] = 0.0;
        }
        for (int k = 0; k < R.nops; k++) {
            const RegionOp& op = b.ops[R.op[k]];
            if (op.kind == kOpEqm) {
                ApplyEqm<L>(f, op, pc);
            } else if (op.kind == kOpHbb) {
#pragma unroll
                for (int i = 0; i < Q; i++)
                    if (op.out_mask >> i & 1u)
                        f[i] = src[L::opp(i) * b.popstride + node] + op.b[i];
            }
        }
    }
    const bool fl = R.fluidlike != 0;
    if (MODE == kModeF) {
        const long long dn =
            ((long long)z * b.n[1] + y) * (long long)b.n[0] + x;
#pragma unroll
        for (int i = 0; i < Q; i++) out0[dn * Q + i] = f[i];
        return;
    }
    double rho, u[3];
    Moments<L>(f, pc, fl, rho, u);
    if (MODE == kModeMacro) {
        const long long dn =
            ((long long)z * b.n[1] + y) * (long long)b.n[0] + x;
        out0[dn] = rho;
        out1[dn] = u[0];
        out2[dn] = u[1];
        if (D == 3) out3[dn] = u[2];
        return;
    }
    Collide<L>(f, pc, fl, rho, u);
#pragma unroll
    for (int i = 0; i < Q; i++) dst[i * b.popstride + node] = f[i];
}

// Deferred nodes: thread t -> (region, node).
__device__ __forceinline__ bool DeferredNode(const BlockDev& b, long long t,
                                             int& region, int& x, int& y,
                                             int& z, long long& k) {
    for (int s = 0; s < b.ndregions; s++) {
        const int4 d = b.dregions[s];
        if (t >= d.y && t < (long long)d.y + d.z) {
            const RegionInfo& R = b.regions[d.x];
            const long long loc = t - d.y;
            x = R.org[0] + (int)(loc % R.ext[0]);
            y = R.org[1] + (int)((loc / R.ext[0]) % R.ext[1]);
            z = R.org[2] + (int)(loc / ((long long)R.ext[0] * R.ext[1]));
            region = d.x;
            k = t;
            return true;
        }
    }
    return false;
}

// Deferred nodes, part 1: streaming into the explicit f store (populations
// not pulled keep their previous value, as in KerStream3D).
template <int D>
__global__ void DeferredStreamKernel(BlockDev b, const double* __restrict__ src) {
    using L = Lattice<D>;
    constexpr int Q = L::Q;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= b.ndef) return;
    int r, x, y, z;
    long long k;
    if (!DeferredNode(b, t, r, x, y, z, k)) return;
    const RegionInfo& R = b.regions[r];
    const long long node = NodeIndex<D>(b, x, y, z);
#pragma unroll
    for (int i = 0; i < Q; i++)
        if (R.pull >> i & 1u)
            b.fdef[i * b.ndef + k] =
                src[i * b.popstride + node + UpOffset<L>(b, i)];
}

struct DeferredSeg {
    int region;
    int op;
    long long start;   // first thread of this segment
    long long count;
};

// Deferred nodes, part 2: one boundary of the definition order
// (EQMDiffuseRefl, ExtrapolPressure1ST or halfway bounce-back).  The
// extrapolation reads the inner neighbour's current f: from the store when
// it is deferred, otherwise (a pure node) straight from its upstream g.
template <int D>
__global__ void DeferredOpKernel(BlockDev b, PhysConst pc,
                                 const double* __restrict__ src,
                                 const DeferredSeg* __restrict__ segs,
                                 int nseg, long long total) {
    using L = Lattice<D>;
    constexpr int Q = L::Q;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    int s = 0;
    while (s < nseg - 1 && t >= segs[s + 1].start) s++;
    const DeferredSeg sg = segs[s];
    const RegionInfo& R = b.regions[sg.region];
    const long long loc = t - sg.start;
    const int x = R.org[0] + (int)(loc % R.ext[0]);
    const int y = R.org[1] + (int)((loc / R.ext[0]) % R.ext[1]);
    const int z = R.org[2] + (int)(loc / ((long long)R.ext[0] * R.ext[1]));
    const long long k = R.side_base + loc;
    const RegionOp& op = b.ops[sg.op];
    double f[Q];
#pragma unroll
    for (int i = 0; i < Q; i++) f[i] = b.fdef[i * b.ndef + k];
    if (op.kind == kOpEqm) {
        ApplyEqm<L>(f, op, pc);
    } else if (op.kind == kOpHbb) {
        const long long node = NodeIndex<D>(b, x, y, z);
#pragma unroll
        for (int i = 0; i < Q; i++)
            if (op.out_mask >> i & 1u)
                f[i] = src[L::opp(i) * b.popstride + node] + op.b[i];
    } else if (op.kind == kOpExtrapol) {
        int q[3] = {x, y, z};
        if (op.nb_axis >= 0) q[op.nb_axis] += op.nb_sign;
        const int nr = RegionOf(q[0], q[1], q[2], b.n, D);
        const RegionInfo& N = b.regions[nr];
        const bool nbdef = N.cls == kDeferred;
        const long long nk = nbdef ? N.side_base + LocalIndex(N, q[0], q[1], q[2])
                                   : 0;
        const long long nnode = NodeIndex<D>(b, q[0], q[1], q[2]);
        double rho = 0.0;
#pragma unroll
        for (int i = 0; i < Q; i++) {
            if (op.in_mask >> i & 1u) {
                f[i] = nbdef ? b.fdef[i * b.ndef + nk]
                             : src[i * b.popstride + nnode + UpOffset<L>(b, i)];
            }
            rho = rho + f[i];
        }
        const double ratio = op.rho_given / rho;
#pragma unroll
        for (int i = 0; i < Q - 1; i++) f[i] = f[i] * ratio;
    }
#pragma unroll
    for (int i = 0; i < Q; i++) b.fdef[i * b.ndef + k] = f[i];
}

// Deferred nodes, part 3: moments and collision (or observation).
template <int D, int MODE>
__global__ void DeferredFinishKernel(BlockDev b, PhysConst pc,
                                     double* __restrict__ dst,
                                     double* __restrict__ out0,
                                     double* __restrict__ out1,
                                     double* __restrict__ out2,
                                     double* __restrict__ out3) {
    using L = Lattice<D>;
    constexpr int Q = L::Q;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= b.ndef) return;
    int r, x, y, z;
    long long k;
    if (!DeferredNode(b, t, r, x, y, z, k)) return;
    const RegionInfo& R = b.regions[r];
    double f[Q];
#pragma unroll
    for (int i = 0; i < Q; i++) f[i] = b.fdef[i * b.ndef + k];
    const long long dn = ((long long)z * b.n[1] + y) * (long long)b.n[0] + x;
    if (MODE == kModeF) {
#pragma unroll
        for (int i = 0; i < Q; i++) out0[dn * Q + i] = f[i];
        return;
    }
    double rho, u[3];
    Moments<L>(f, pc, R.fluidlike != 0, rho, u);
    if (MODE == kModeMacro) {
        out0[dn] = rho;
        out1[dn] = u[0];
        out2[dn] = u[1];
        if (D == 3) out3[dn] = u[2];
        return;
    }
    Collide<L>(f, pc, R.fluidlike != 0, rho, u);
    const long long node = NodeIndex<D>(b, x, y, z);
#pragma unroll
    for (int i = 0; i < Q; i++) dst[i * b.popstride + node] = f[i];
}

// Initial state of one block from per-node macroscopic values
// (KerInitialiseBGK2nd3D: f = feq(rho, u), Src/model_kernel.inc:352-380) or
// from uploaded f (fin != nullptr, point-major).  Writes f^0 to `fdirect`
// (same layout as g), the stale and deferred stores, and g^0 = collision of
// f^0 with its own moments to `g`.
template <int D>
__global__ void __launch_bounds__(128)
    InitKernel(BlockDev b, PhysConst pc, const double* __restrict__ rho0,
               const double* __restrict__ u0, const double* __restrict__ v0,
               const double* __restrict__ w0, const double* __restrict__ fin,
               double* __restrict__ fdirect, double* __restrict__ g) {
    using L = Lattice<D>;
    constexpr int Q = L::Q;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = D == 3 ? (int)blockIdx.z : 0;
    if (x >= b.n[0]) return;
    const long long dn = ((long long)z * b.n[1] + y) * (long long)b.n[0] + x;
    double f[Q];
    if (fin != nullptr) {
#pragma unroll
        for (int i = 0; i < Q; i++) f[i] = fin[dn * Q + i];
    } else {
        // CalcBGKFeq(l, rho, u, v, w, 1, 2), Src/model_host_device.h:58-82
        const double rho = rho0[dn];
        const double u[3] = {u0[dn], v0[dn], D == 3 ? w0[dn] : 0.0};
        const double cu0 = pc.cs * u[0], cu1 = pc.cs * u[1], cu2 = pc.cs * u[2];
        const double u2 = D == 3 ? (u[0] * u[0] + u[1] * u[1]) + u[2] * u[2]
                                 : u[0] * u[0] + u[1] * u[1];
#pragma unroll
        for (int i = 0; i < Q; i++) {
            double cu = 0.0;
            bool first = true;
            const int c0 = L::cx(i), c1 = L::cy(i), c2 = L::cz(i);
            if (c0 != 0) { cu = c0 > 0 ? cu0 : -cu0; first = false; }
            if (c1 != 0) {
                const double t = c1 > 0 ? cu1 : -cu1;
                cu = first ? t : cu + t;
                first = false;
            }
            if (c2 != 0) {
                const double t = c2 > 0 ? cu2 : -cu2;
                cu = first ? t : cu + t;
            }
            const double res = (1.0 + cu) + 0.5 * (cu * cu - u2);
            f[i] = (pc.w[i] * rho) * res;
        }
    }
    const int r = RegionOf(x, y, z, b.n, D);
    const RegionInfo& R = b.regions[r];
    const long long node = NodeIndex<D>(b, x, y, z);
#pragma unroll
    for (int i = 0; i < Q; i++) fdirect[i * b.popstride + node] = f[i];
    if (R.side_base >= 0) {
        const long long k = R.side_base + LocalIndex(R, x, y, z);
        if (R.cls == kLocal) {
#pragma unroll
            for (int i = 0; i < Q; i++) b.stale[k * Q + i] = f[i];
        } else if (R.cls == kDeferred) {
#pragma unroll
            for (int i = 0; i < Q; i++) b.fdef[i * b.ndef + k] = f[i];
        }
    }
    double rho, u[3];
    Moments<L>(f, pc, R.fluidlike != 0, rho, u);
    Collide<L>(f, pc, R.fluidlike != 0, rho, u);
#pragma unroll
    for (int i = 0; i < Q; i++) g[i * b.popstride + node] = f[i];
}

// Observation straight from f^0 stored by InitKernel (before any step).
template <int D, int MODE>
__global__ void DirectObserveKernel(BlockDev b, PhysConst pc,
                                    const double* __restrict__ fdirect,
                                    double* __restrict__ out0,
                                    double* __restrict__ out1,
                                    double* __restrict__ out2,
                                    double* __restrict__ out3) {
    using L = Lattice<D>;
    constexpr int Q = L::Q;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = D == 3 ? (int)blockIdx.z : 0;
    if (x >= b.n[0]) return;
    const long long dn = ((long long)z * b.n[1] + y) * (long long)b.n[0] + x;
    const long long node = NodeIndex<D>(b, x, y, z);
    double f[Q];
#pragma unroll
    for (int i = 0; i < Q; i++) f[i] = fdirect[i * b.popstride + node];
    if (MODE == kModeF) {
#pragma unroll
        for (int i = 0; i < Q; i++) out0[dn * Q + i] = f[i];
        return;
    }
    const RegionInfo& R = b.regions[RegionOf(x, y, z, b.n, D)];
    double rho, u[3];
    Moments<L>(f, pc, R.fluidlike != 0, rho, u);
    out0[dn] = rho;
    out1[dn] = u[0];
    out2[dn] = u[1];
    if (D == 3) out3[dn] = u[2];
}

struct HaloDev {
    int iter[3];
    int fbase[3];
    int tbase[3];
    uint32_t pops;
    const uint8_t* prev;   // nullptr: every source cell is current
};

// One connection's halo copy (Field::TransferHalos / ops_halo_transfer):
// the face layer of the source block into the destination block's halo,
// only the populations that point into the destination.
template <int D>
__global__ void HaloKernel(HaloDev h, BlockDev fb, BlockDev tb,
                           const double* __restrict__ cur_from,
                           const double* __restrict__ prev_from,
                           double* __restrict__ cur_to) {
    using L = Lattice<D>;
    constexpr int Q = L::Q;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long cells = (long long)h.iter[0] * h.iter[1] * h.iter[2];
    if (t >= cells) return;
    const int i = (int)(t % h.iter[0]);
    const int j = (int)((t / h.iter[0]) % h.iter[1]);
    const int k = (int)(t / ((long long)h.iter[0] * h.iter[1]));
    const long long s = NodeIndex<D>(fb, h.fbase[0] + i, h.fbase[1] + j,
                                     h.fbase[2] + k);
    const long long d = NodeIndex<D>(tb, h.tbase[0] + i, h.tbase[1] + j,
                                     h.tbase[2] + k);
    const double* from = (h.prev != nullptr && h.prev[t]) ? prev_from : cur_from;
#pragma unroll
    for (int q = 0; q < Q; q++)
        if (h.pops >> q & 1u)
            cur_to[q * tb.popstride + d] = from[q * fb.popstride + s];
}

// Residual sums of one macroscopic variable over one block, per CTA:
// sum (q - q_old)^2 and sum q^2 (KerCalcMacroVarSquareofDifference /
// KerCalcMacroVarSquare, Src/flowfield_kernel.inc:131-153); q_old <- q.
__global__ void ResidualPartialKernel(const double* __restrict__ q,
                                      double* __restrict__ qold, long long n,
                                      double* __restrict__ part) {
    __shared__ double sd[256];
    __shared__ double ss[256];
    double d = 0.0, s = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const double v = q[t];
        const double dv = v - qold[t];
        d = d + dv * dv;
        s = s + v * v;
        qold[t] = v;
    }
    sd[threadIdx.x] = d;
    ss[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sd[threadIdx.x] = sd[threadIdx.x] + sd[threadIdx.x + w];
            ss[threadIdx.x] = ss[threadIdx.x] + ss[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sd[0];
        part[2 * blockIdx.x + 1] = ss[0];
    }
}

// Sum of a field over n values, per CTA (mass), and a count of
// non-finite or non-positive values (health word).
__global__ void SumPartialKernel(const double* __restrict__ q, long long n,
                                 double* __restrict__ part,
                                 unsigned long long* __restrict__ bad) {
    __shared__ double ss[256];
    double s = 0.0;
    unsigned long long nb = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const double v = q[t];
        s = s + v;
        if (!(v > 0.0) || !isfinite(v)) nb++;
    }
    ss[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) ss[threadIdx.x] = ss[threadIdx.x] + ss[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = ss[0];
    if (nb) atomicAdd(bad, nb);
}

}  // namespace mplb
