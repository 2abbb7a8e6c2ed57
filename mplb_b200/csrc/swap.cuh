// One-array swap scheme of the reference (SwapStreamCollision,
// Src/evolution.cpp:195-252) on the B200.
//
// The reference collides in place (KerSwapCollideBGKIsothermal3D,
// Src/model_kernel.inc:385-408; the _Swap body force is added after the
// collision, KerSwapCalcBodyForce1ST3D, :543-568), applies a local swap at
// every node (KerLocalSwap3D, Src/scheme_kernel.inc:959-1194) and then
// exchanges population l + Q/2 of x with population l of x + c_l
// (KerSwapStream3D, :1196-1398) before the boundary conditions.  Every
// exchange pairs two fixed slots and no slot is in two pairs, so the whole
// stream is a fixed involution pi on the slots of the array.
//
// Here two kernels alternate on the one array (the "AA" access pattern):
//   own   (GATHER = false): node x reads its own slots, collides, applies
//          its local swap and writes its own slots back;
//   gather (GATHER = true): node x reads slot k from pi(x, k) - slot opp(k)
//          of x - c_k where the region's exchange mask says so, else its own
//          slot - which is the streamed population, applies the boundary
//          programme, collides, applies the local swap and writes each slot
//          back to the place it was read from, which is where the next
//          stream would have put it.
// After an own step the array holds the locally swapped state; after a
// gather step it holds the streamed state, whose boundary programme the next
// step applies first (BC = true).  Each slot is read and written by exactly
// one thread, so both kernels run in place without races, and a step moves
// 2 Q values per node as the two-array step does.
#pragma once

#include "kernels.cuh"

namespace mplb {

// Element index of slot k of the node at `node`: own slot, or slot opp(k)
// of the upstream node.
template <bool O32>
__device__ __forceinline__ long long SwapSlot(const BlockDev& b,
                                              long long node, int k,
                                              bool exch) {
    if constexpr (O32)
        return node + (long long)(exch ? b.swap_off32[k] : b.pop_off32[k]);
    else
        return node + (exch ? b.swap_off[k] : b.pop_off[k]);
}

// One node, any region.
template <typename T, int MODE, bool GATHER, bool BC, bool O32>
__device__ __forceinline__ void SwapNode(const BlockDev& b,
                                         const PhysConst& pc, T* f,
                                         double* __restrict__ out0,
                                         double* __restrict__ out1,
                                         double* __restrict__ out2,
                                         double* __restrict__ out3, int x,
                                         int y, int z) {
    using L = Lattice<3>;
    using P = Prec<T>;
    using C = typename P::C;
    constexpr int Q = L::Q;
    const int r = RegionOf(x, y, z, b.n, 3);
    const bool interior = r == 13;
    const long long node = NodeIndexT<3, O32>(b, x, y, z);
    // the interior exchanges every moving population, its local swap is the
    // opposite map, and it has no boundary programme
    const uint32_t exch = GATHER ? (interior ? ~1u : b.swap_exch[r]) : 0u;
    C v[Q];
#pragma unroll
    for (int k = 0; k < Q; k++)
        v[k] = P::Load(f, SwapSlot<O32>(b, node, k, exch >> k & 1u), k, pc);
    if (BC && !interior) {
        const RegionInfo& R = b.regions[r];
        for (int i = 0; i < R.nops; i++)
            ApplyEqm<L, T>(v, b.ops[R.op[i]], pc, x, y, z);
    }
    const bool fl = (b.rflags[r] & 4) != 0;
    if (MODE == kModeF) {
        const long long dn =
            ((long long)z * b.n[1] + y) * (long long)b.n[0] + x;
#pragma unroll
        for (int i = 0; i < Q; i++) out0[dn * Q + i] = ToF<T>(v[i], i, pc);
        return;
    }
    if (MODE == kModeMacro) {
        double rho, u[3];
        MomentsT<L, T>(v, pc, fl, rho, u);
        const long long dn =
            ((long long)z * b.n[1] + y) * (long long)b.n[0] + x;
        out0[dn] = rho;
        out1[dn] = u[0];
        out2[dn] = u[1];
        out3[dn] = u[2];
        return;
    }
    MomentsCollideT<L, T>(v, pc, fl);
    Rng rng = SeedRng(pc.seed, node);
    if (interior) {
#pragma unroll
        for (int k = 0; k < Q; k++)
            P::Store(f, SwapSlot<O32>(b, node, k, GATHER && k != 0), k,
                     v[L::opp(k)], pc, rng);
    } else {
        // slot k takes collided population sigma[k] (k or opp(k)); selected
        // without indexing the register array
        const uint8_t* sg = b.swap_sigma[r];
#pragma unroll
        for (int k = 0; k < Q; k++) {
            const int s = sg[k];
            const C w = s == k ? v[k] : v[L::opp(k)];
            P::Store(f, SwapSlot<O32>(b, node, k, exch >> k & 1u), k, w, pc,
                     rng);
        }
    }
}

// One node per thread over the whole block (observations, and steps of
// blocks too thin for SplitSwapKernel).
template <typename T, int MODE, bool GATHER, bool BC, bool O32>
__global__ void __launch_bounds__(128, std::is_same<T, double>::value
                                           ? MPLB_F64_MIN_BLOCKS
                                           : MPLB_LP_MIN_BLOCKS)
    SwapKernel(BlockDev b, PhysConst pc, T* f, double* __restrict__ out0,
               double* __restrict__ out1, double* __restrict__ out2,
               double* __restrict__ out3) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= b.n[0]) return;
    SwapNode<T, MODE, GATHER, BC, O32>(b, pc, f, out0, out1, out2, out3, x,
                                       blockIdx.y, blockIdx.z);
}

// The G interior nodes x0 + 32 j of one row (the layout of
// PureNodeGroup): no boundary programme, opposite local swap, every moving
// slot exchanged when gathering.
template <typename T, bool GATHER, bool O32, int G>
__device__ __forceinline__ void SwapInteriorGroup(const BlockDev& b,
                                                  const PhysConst& pc, T* f,
                                                  int x0, int y, int z) {
    using L = Lattice<3>;
    using P = Prec<T>;
    using C = typename P::C;
    constexpr int Q = L::Q;
    bool valid[G];
    int first = -1;
#pragma unroll
    for (int j = 0; j < G; j++) {
        const int x = x0 + 32 * j;
        valid[j] = x >= 1 && x <= b.n[0] - 2;
        if (valid[j] && first < 0) first = j;
    }
    if (first < 0) return;
    T* p[G];
    long long node[G];
#pragma unroll
    for (int j = 0; j < G; j++) {
        node[j] = NodeIndexT<3, O32>(b, x0 + 32 * (valid[j] ? j : first), y, z);
        p[j] = f + node[j];
    }
    // element offset of slot k from the node (compile-time choice per k)
    auto off = [&](int k) -> long long {
        const bool e = GATHER && k != 0;
        if constexpr (O32) return e ? b.swap_off32[k] : b.pop_off32[k];
        else return e ? b.swap_off[k] : b.pop_off[k];
    };
    C v[G][Q];
#pragma unroll
    for (int k = 0; k < Q; k++) {
#pragma unroll
        for (int j = 0; j < G; j++) v[j][k] = P::Load(p[j], off(k), k, pc);
    }
    const bool fl = b.center_fluid != 0;
    constexpr bool kPair = P::kShifted && G == 2;
    if constexpr (kPair) MomentsCollidePair<L>(v[0], v[1], pc, fl, pc.omcf);
#pragma unroll
    for (int j = 0; j < G; j++) {
        if (!valid[j]) continue;
        if constexpr (!kPair) MomentsCollideT<L, T>(v[j], pc, fl);
        Rng rg = SeedRng(pc.seed, node[j]);
#pragma unroll
        for (int k = 0; k < Q; k++)
            P::Store(p[j], off(k), k, v[j][L::opp(k)], pc, rg);
    }
}

// CTAs per SM of the FP64 swap step: 4 (128 registers); at 5 the in-place
// step spills.
#ifndef MPLB_SWAP_F64_MIN_BLOCKS
#define MPLB_SWAP_F64_MIN_BLOCKS 4
#endif

// A step with no warp mixing interior and boundary nodes, in the CTA layout
// of SplitStepKernel: shell rows (y or z on the block boundary), then per
// chunk of kSplitRows interior rows one CTA for their x faces followed by
// the CTAs of the rows' interior nodes (the x-face CTA runs next to its
// rows, so the sectors they share meet in L2; as separate launches FP32 lost
// 11 %).
template <typename T, bool GATHER, bool BC, bool O32>
__global__ void __launch_bounds__(128, std::is_same<T, double>::value
                                           ? MPLB_SWAP_F64_MIN_BLOCKS
                                           : MPLB_LP_MIN_BLOCKS)
    SplitSwapKernel(BlockDev b, PhysConst pc, T* f) {
    const int nbx = (b.n[0] + (int)blockDim.x - 1) / (int)blockDim.x;
    const int ny = b.n[1] - 2;
    const int nz = b.n[2];
    const unsigned nsr = (unsigned)nbx * (2 * nz + 2 * ny);
    unsigned blk = blockIdx.x;
    if (blk < nsr) {
        const int row = (int)(blk / nbx);
        const int x = (int)(blk % nbx) * blockDim.x + threadIdx.x;
        if (x >= b.n[0]) return;
        int y, z;
        if (row < 2 * nz) {
            y = (row & 1) ? b.n[1] - 1 : 0;
            z = row >> 1;
        } else {
            const int r2 = row - 2 * nz;
            z = (r2 & 1) ? b.n[2] - 1 : 0;
            y = 1 + (r2 >> 1);
        }
        SwapNode<T, kModeStep, GATHER, BC, O32>(b, pc, f, nullptr, nullptr,
                                                nullptr, nullptr, x, y, z);
        return;
    }
    blk -= nsr;
    const int rows = ny * (b.n[2] - 2);
    constexpr int G = SplitGroup<T>();
    const unsigned per_chunk = (unsigned)SplitChunkCtas<G>(b.n[0]);
    const int chunk = (int)(blk / per_chunk);
    const int w = (int)(blk % per_chunk);
    if (w == 0) {
        const int r = chunk * kSplitRows + (int)(threadIdx.x >> 1);
        if (threadIdx.x >= 2 * kSplitRows || r >= rows) return;
        const int x = (threadIdx.x & 1) ? b.n[0] - 1 : 0;
        SwapNode<T, kModeStep, GATHER, BC, O32>(b, pc, f, nullptr, nullptr,
                                                nullptr, nullptr, x,
                                                1 + r % ny, 1 + r / ny);
        return;
    }
    const SplitTask k = InteriorTask<G>(b, chunk, w);
    if (k.r < 0 || k.r >= rows) return;
    SwapInteriorGroup<T, GATHER, O32, G>(b, pc, f, k.x0, 1 + k.r % ny,
                                         1 + k.r / ny);
}

}  // namespace mplb
