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

template <typename T, int MODE, bool GATHER, bool BC, bool O32>
__global__ void __launch_bounds__(128, std::is_same<T, double>::value
                                           ? MPLB_F64_MIN_BLOCKS
                                           : MPLB_LP_MIN_BLOCKS)
    SwapKernel(BlockDev b, PhysConst pc, T* f, double* __restrict__ out0,
               double* __restrict__ out1, double* __restrict__ out2,
               double* __restrict__ out3) {
    using L = Lattice<3>;
    using P = Prec<T>;
    using C = typename P::C;
    constexpr int Q = L::Q;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= b.n[0]) return;
    const int r = RegionOf(x, y, z, b.n, 3);
    const bool interior = r == 13;
    const long long node = NodeIndex<3>(b, x, y, z);
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
            ApplyEqm<L, T>(v, b.ops[R.op[i]], pc);
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

}  // namespace mplb
