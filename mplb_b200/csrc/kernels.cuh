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
// Storage forms (template parameter T):
//   double : the reference's arithmetic.  Every FP64 expression follows the
//            reference's operation order; the translation unit is compiled
//            with -fmad=false so no product is fused into an add, and terms
//            the reference multiplies by a zero lattice component are skipped
//            (adding a signed zero never changes a non-zero sum).  Results
//            are bit-identical to the reference.
//   float  : the shifted deviation h_i = f_i - w_i in FP32 with FP32
//            arithmetic (rho = 1 + sum h, feq - w computed directly).
//   __half : the same deviation scaled by its weight, 256 h_i / w_i, in
//            FP16 storage (stochastic rounding); arithmetic in FP32, the
//            interior pairs' on the stored values themselves.
// Moments, residuals and the side stores are FP64 in every form.
#pragma once

#include <cuda_fp16.h>

#include <cstdint>
#include <type_traits>

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
    // single-precision copies for the shifted forms
    float csf, omcf, twf;
    float hdtaf[3];
    float hdta_csf[3];   // dt a / (2 CS): momentum the equilibrium's
                         // half-step velocity shift adds, per unit density
    float cff[kMaxQ];
    float wcff[kMaxQ];   // w_i CS c_i . a (body force per unit density)
    float tw_omf;        // tau omega / omega: the force term relative to
                         // the relaxation rate
    float wf[kMaxQ];
    float cf256f[kMaxQ]; // kHalfScale CS c_i . a (FP16 pairs' force term)
    float winvf[kMaxQ];  // FP16 store scale kHalfScale / w_i
    float wlf[kMaxQ];    // FP16 load scale w_i / kHalfScale
    uint32_t seed;       // per launch (FP16 stochastic rounding)
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
    // per population: element offset of the upstream value (i * popstride -
    // c_i . strides) and of the own value (i * popstride)
    long long pull_off[kMaxQ];
    long long pop_off[kMaxQ];
    // the same offsets in 32 bits, valid when off32 (every offset and the
    // whole population array fit in an int): one IMAD per access instead of
    // 64-bit index arithmetic
    int pull_off32[kMaxQ];
    int pop_off32[kMaxQ];
    int off32;
    int plane32, pitch32;   // strides in 32 bits (valid when off32)
    // the step runs as SplitStepKernel (every extent >= 3 and the interior
    // region PURE); center_fluid: the interior is fluid-like
    int split;
    int center_fluid;
    // deferred nodes in one kernel (no deferred node reads another):
    // per region, the first entry of its operation list in dops_flat (each
    // list in definition order, ended by -1)
    int deferred_fused;
    int dops_first[kNumRegions];
    const int* dops_flat;
    // per region: class (bits 0-1) and fluid-like flag (bit 2); the pulled
    // and the stale populations (copies of RegionInfo::pull / ::stale)
    uint8_t rflags[kNumRegions];
    uint32_t rpull[kNumRegions];
    uint32_t rstale[kNumRegions];
    // swap scheme (swap.cuh): per region the slots that live at slot opp(k)
    // of the upstream node and the local-swap map; per population the
    // element offset of that upstream slot (opp(k) * popstride - c_k .
    // strides), 64- and 32-bit
    uint32_t swap_exch[kNumRegions];
    uint8_t swap_sigma[kNumRegions][kMaxQ];
    long long swap_off[kMaxQ];
    int swap_off32[kMaxQ];
};

enum StepMode : int { kModeStep = 0, kModeMacro = 1, kModeF = 2 };

// ---------------------------------------------------------------------------
// storage forms
struct Rng;
template <typename T>
struct Prec;

// Store/load cache policy of the population arrays (every value is written
// once and read once per step, so neither wants to stay in the caches).
#ifndef MPLB_STORE_HINT
#define MPLB_STORE_HINT 0
#endif
template <typename V>
__device__ __forceinline__ void PopStore(V* p, V v) {
#if MPLB_STORE_HINT == 1
    __stcs(p, v);
#else
    *p = v;
#endif
}

template <>
struct Prec<double> {
    using C = double;
    static constexpr bool kShifted = false;
    __device__ static __forceinline__ C Load(const double* p, long long k, int,
                                             const PhysConst&) {
        return p[k];
    }
    __device__ static __forceinline__ void Store(double* p, long long k, int,
                                                 C v, const PhysConst&, Rng&) {
        PopStore(p + k, v);
    }
};

template <>
struct Prec<float> {
    using C = float;
    static constexpr bool kShifted = true;
    __device__ static __forceinline__ C Load(const float* p, long long k, int,
                                             const PhysConst&) {
        return p[k];
    }
    __device__ static __forceinline__ void Store(float* p, long long k, int,
                                                 C v, const PhysConst&, Rng&) {
        PopStore(p + k, v);
    }
};

// FP16 stores round stochastically, so increments far below one FP16 unit -
// a small body force per step - survive in expectation instead of being
// rounded away every step.  The rounding is the hardware's
// (cvt.rs.f16x2.f32, sm_100a): two values per instruction, random bits from
// a 32-bit word.  The stored value is kHalfScale h_i / w_i:
// h_i / w_i = f_i / w_i - 1 lies in [-1, 255) for any population within 256
// times its weight (a lattice Boltzmann state stays within a few times it),
// so the scaled value stays in FP16's range.  Draws: one 32-bit hash of
// (node, step) per node (or node pair), times an odd constant per
// population (a bijection of the hash, so each draw is uniform).
constexpr float kHalfScale = 256.0f;

struct Rng {
    uint32_t s;
};

__device__ __forceinline__ Rng SeedRng(uint32_t seed, long long node) {
    uint32_t k = (uint32_t)node * 0x9e3779b9u ^ (uint32_t)(node >> 32) ^
                 seed * 0x85ebca6bu;
    k ^= k >> 16;
    k *= 0x7feb352du;
    k ^= k >> 15;
    k *= 0x846ca68bu;
    k ^= k >> 16;
    return Rng{k};
}

// 32 random bits for population i.
__device__ __forceinline__ uint32_t SrDraw32(const Rng& g, int i) {
    return g.s * (0x9e3779b1u * (uint32_t)(2 * i + 1) | 1u);
}

// lo and hi to FP16 with the hardware's stochastic rounding, random bits
// from r; lo in the low half of the result.
__device__ __forceinline__ uint32_t StochasticHalf2(float lo, float hi,
                                                    uint32_t r) {
    uint32_t d;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo),
        "r"(r));
    return d;
}

__device__ __forceinline__ __half StochasticHalf(float v, uint32_t r) {
    return __ushort_as_half(
        (unsigned short)(StochasticHalf2(v, 0.0f, r) & 0xffffu));
}

template <>
struct Prec<__half> {
    using C = float;
    static constexpr bool kShifted = true;
    __device__ static __forceinline__ C Load(const __half* p, long long k,
                                             int i, const PhysConst& pc) {
        return __half2float(p[k]) * pc.wlf[i];
    }
    __device__ static __forceinline__ void Store(__half* p, long long k, int i,
                                                 C v, const PhysConst& pc,
                                                 Rng& rng) {
        PopStore(p + k, StochasticHalf(v * pc.winvf[i], SrDraw32(rng, i)));
    }
};

// Value of the reference's f_i from a value of form T (for FP64 outputs).
template <typename T>
__device__ __forceinline__ double ToF(typename Prec<T>::C v, int i,
                                      const PhysConst& pc) {
    if constexpr (Prec<T>::kShifted) return (double)v + pc.w[i];
    else return v;
}
template <typename T>
__device__ __forceinline__ typename Prec<T>::C FromF(double f, int i,
                                                     const PhysConst& pc) {
    if constexpr (Prec<T>::kShifted)
        return (typename Prec<T>::C)(f - pc.w[i]);
    else return f;
}

// ---------------------------------------------------------------------------
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

// The same in 32-bit arithmetic when the population array fits (off32).
template <int D, bool O32>
__device__ __forceinline__ long long NodeIndexT(const BlockDev& b, int x, int y,
                                                int z) {
    if constexpr (O32)
        return (D == 3 ? z + 1 : 0) * b.plane32 + (y + 1) * b.pitch32 +
               (x + b.xoff);
    else
        return NodeIndex<D>(b, x, y, z);
}

template <typename L>
__device__ __forceinline__ long long UpOffset(const BlockDev& b, int i) {
    // offset of the upstream node x - c_i
    return -((long long)L::cx(i) + (long long)L::cy(i) * b.pitch +
             (long long)L::cz(i) * b.plane);
}

// Element index of population i at the upstream node / at the node itself:
// mode 1 adds per-population offsets precomputed on the host (fewer integer
// instructions per node), mode 0 computes them from the strides.
#ifndef MPLB_ADDR_MODE
#define MPLB_ADDR_MODE 1
#endif
template <typename L>
__device__ __forceinline__ long long PullIndex(const BlockDev& b,
                                               long long node, int i) {
#if MPLB_ADDR_MODE == 1
    return node + b.pull_off[i];
#else
    return i * b.popstride + node + UpOffset<L>(b, i);
#endif
}

__device__ __forceinline__ long long OwnIndex(const BlockDev& b,
                                              long long node, int i) {
#if MPLB_ADDR_MODE == 1
    return node + b.pop_off[i];
#else
    return i * b.popstride + node;
#endif
}

__device__ __forceinline__ long long LocalIndex(const RegionInfo& R, int x,
                                                int y, int z) {
    return ((long long)(z - R.org[2]) * R.ext[1] + (y - R.org[1])) * R.ext[0] +
           (x - R.org[0]);
}

// ---------------------------------------------------------------------------
// FP64 form: moments (KerCalcDensity3D, KerCalcU3D/V3D/W3D and the _Force
// variants, Src/model_kernel.inc:570-759).
template <typename L>
__device__ __forceinline__ void MomentsF64(const double* f, const PhysConst& pc,
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

// FP64 form: BGK collision (KerCollideBGKIsothermal3D with CalcBGKFeq and
// CalcBodyForce, Src/model_kernel.inc:410-455, model_host_device.h:25-82).
template <typename L>
__device__ __forceinline__ void CollideF64(double* f, const PhysConst& pc,
                                           bool fluidlike, double rho,
                                           const double u[3], double omc) {
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
        double g = feq + omc * (f[i] - feq);
        if (force) g = g + pc.tw * (wr * pc.cf[i]);
        f[i] = g;
    }
}

// Shifted forms: h = f - w.  rho = 1 + sum h, j = sum CS c h (sum c w = 0).
//
// The arithmetic is written once over V = float (one node) or V = float2
// (two nodes: sm_100a's paired FP32 instructions, one instruction for both
// nodes), every operation rounded explicitly (no contraction left to the
// compiler), so a node gives the same bits alone or in a pair.
template <typename V>
struct VOps;

template <>
struct VOps<float> {
    __device__ static __forceinline__ float add(float a, float b) {
        return __fadd_rn(a, b);
    }
    __device__ static __forceinline__ float sub(float a, float b) {
        return __fsub_rn(a, b);
    }
    __device__ static __forceinline__ float mul(float a, float b) {
        return __fmul_rn(a, b);
    }
    __device__ static __forceinline__ float fma(float a, float b, float c) {
        return __fmaf_rn(a, b, c);
    }
    __device__ static __forceinline__ float neg(float a) { return -a; }
    __device__ static __forceinline__ float splat(float c) { return c; }
    __device__ static __forceinline__ float rcp(float a) {
        return __frcp_rn(a);
    }
};

template <>
struct VOps<float2> {
    __device__ static __forceinline__ float2 add(float2 a, float2 b) {
        return __fadd2_rn(a, b);
    }
    __device__ static __forceinline__ float2 sub(float2 a, float2 b) {
        return __fadd2_rn(a, neg(b));
    }
    __device__ static __forceinline__ float2 mul(float2 a, float2 b) {
        return __fmul2_rn(a, b);
    }
    __device__ static __forceinline__ float2 fma(float2 a, float2 b,
                                                 float2 c) {
        return __ffma2_rn(a, b, c);
    }
    __device__ static __forceinline__ float2 neg(float2 a) {
        return make_float2(-a.x, -a.y);
    }
    __device__ static __forceinline__ float2 splat(float c) {
        return make_float2(c, c);
    }
    __device__ static __forceinline__ float2 rcp(float2 a) {
        return make_float2(__frcp_rn(a.x), __frcp_rn(a.y));
    }
};

template <typename L, typename V>
__device__ __forceinline__ void MomentsShiftedV(const V* h,
                                                const PhysConst& pc,
                                                bool fluidlike, V& drho,
                                                V u[3]) {
    using O = VOps<V>;
    constexpr int Q = L::Q;
    // Opposite populations are combined first: h_i + h_opp(i) cancels the
    // large odd parts (exactly, by Sterbenz's lemma, when they dominate) and
    // h_i - h_opp(i) the even parts, so the partial sums stay at the size of
    // the result instead of the size of the populations.  Summed in index
    // order, the partial sums of rho - 1 reach the odd parts' size and their
    // rounding breaks mass and momentum conservation coherently from step to
    // step (30x larger velocity error on a forced channel).
    drho = h[0];
#pragma unroll
    for (int i = 1; i < Q; i++)
        if (i < L::opp(i)) drho = O::add(drho, O::add(h[i], h[L::opp(i)]));
    const V rinv = O::rcp(O::add(O::splat(1.0f), drho));
#pragma unroll
    for (int a = 0; a < L::D; a++) {
        V s = O::splat(0.0f);
        bool first = true;
#pragma unroll
        for (int i = 0; i < Q; i++) {
            if (comp<L>(i, a) > 0) {
                const V d = O::sub(h[i], h[L::opp(i)]);
                s = first ? d : O::add(s, d);
                first = false;
            }
        }
        s = O::mul(O::mul(O::splat(pc.csf), s), rinv);
        if (pc.force_vel && fluidlike) s = O::add(s, O::splat(pc.hdtaf[a]));
        u[a] = s;
    }
    if (L::D == 2) u[2] = O::splat(0.0f);
}

// feq_i - w_i = w_i [(rho - 1) + rho (cu + (cu^2 - u^2) / 2)], computed
// directly so that no term is rounded against 1.  (Splitting it into the
// parts even and odd in c_i saves arithmetic but rounds the even part, which
// carries the mass, against the odd part; on a forced channel that was 15x
// less accurate, so the direct form is used.)
//
// The collision relaxes the non-equilibrium part m_i = h_i - heq_i, after
// projecting out of it the mass and momentum that rounding put there:
// m_i -= w_i (M0 + 3 c_i . M), with M0 = sum m_i and M = sum c_i m_i minus
// its exact value (-rho dt a / (2 CS) where the equilibrium velocity carries
// the half-step force shift, else 0).  In FP32 the equilibrium's moments
// miss the computed (rho, u) by ~1e-8 relative (the weights and CS are not
// representable), always with the same sign while u changes slowly; a
// forced flow accumulates that as a spurious force (1e-3 relative velocity
// error after 5e4 steps of a channel spinning up); with the projection BGK
// conserves mass and momentum to the final rounding.  m_i is small, so the
// sums over opposite pairs are accurate to its own ulp.
template <typename L, typename V>
__device__ __forceinline__ void CollideShiftedV(V* h, const PhysConst& pc,
                                                bool fluidlike, V drho,
                                                const V u[3], float omc) {
    using O = VOps<V>;
    constexpr int Q = L::Q;
    const V rho = O::add(O::splat(1.0f), drho);
    const V hr = O::mul(O::splat(0.5f), rho);   // rest: w (drho - rho u^2 / 2)
    const V csf = O::splat(pc.csf);
    const V cu0 = O::mul(csf, u[0]), cu1 = O::mul(csf, u[1]),
            cu2 = O::mul(csf, u[2]);
    const V u2 = O::fma(u[0], u[0], O::fma(u[1], u[1], O::mul(u[2], u[2])));
    const V half = O::splat(0.5f);
    // m_i = h_i - heq_i.  heq is evaluated whole for each direction (the
    // pair i, opp(i) shares cu^2 - u^2 only): splitting it into an even and
    // an odd part rounded separately biases the stress it carries, which a
    // channel spinning up shows as a 10x larger velocity error.
    V m[Q];
    m[0] = O::fma(O::splat(-pc.wf[0]), O::fma(O::neg(hr), u2, drho), h[0]);
    V m0 = m[0], mv0 = O::splat(0.0f), mv1 = O::splat(0.0f),
      mv2 = O::splat(0.0f);
#pragma unroll
    for (int i = 1; i < Q; i++) {
        if (i > L::opp(i)) continue;
        const int j = L::opp(i);
        V cu = O::splat(0.0f);
        bool first = true;
        const V comps[3] = {cu0, cu1, cu2};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const int c = comp<L>(i, a);
            if (c == 0 || a >= L::D) continue;
            const V t = c > 0 ? comps[a] : O::neg(comps[a]);
            cu = first ? t : O::add(cu, t);
            first = false;
        }
        const V y = O::fma(cu, cu, O::neg(u2));
        m[i] = O::fma(O::splat(-pc.wf[i]),
                      O::fma(rho, O::fma(half, y, cu), drho), h[i]);
        m[j] = O::fma(O::splat(-pc.wf[j]),
                      O::fma(rho, O::fma(half, y, O::neg(cu)), drho), h[j]);
        m0 = O::add(m0, O::add(m[i], m[j]));
        const V d = O::sub(m[i], m[j]);
        if (L::cx(i) > 0) mv0 = O::add(mv0, d);
        if (L::cx(i) < 0) mv0 = O::sub(mv0, d);
        if (L::cy(i) > 0) mv1 = O::add(mv1, d);
        if (L::cy(i) < 0) mv1 = O::sub(mv1, d);
        if (L::cz(i) > 0) mv2 = O::add(mv2, d);
        if (L::cz(i) < 0) mv2 = O::sub(mv2, d);
    }
    if (pc.force_vel && fluidlike) {
        mv0 = O::fma(rho, O::splat(pc.hdta_csf[0]), mv0);
        mv1 = O::fma(rho, O::splat(pc.hdta_csf[1]), mv1);
        mv2 = O::fma(rho, O::splat(pc.hdta_csf[2]), mv2);
    }
    const V three = O::splat(3.0f);
    mv0 = O::mul(mv0, three);
    mv1 = O::mul(mv1, three);
    mv2 = O::mul(mv2, three);
    // g_i = h_i + omega (w_i (M0 + 3 c_i . M) - m_i + F_i / omega), with
    // F_i = w_i CS c_i.a tau omega rho: one rounding at the size of h_i.
    const V om = O::splat(1.0f - omc);
    const bool force = pc.force && fluidlike;
    const V fr = O::mul(O::splat(pc.tw_omf), rho);
#pragma unroll
    for (int i = 0; i < Q; i++) {
        V cm = m0;
        if (L::cx(i) > 0) cm = O::add(cm, mv0);
        if (L::cx(i) < 0) cm = O::sub(cm, mv0);
        if (L::cy(i) > 0) cm = O::add(cm, mv1);
        if (L::cy(i) < 0) cm = O::sub(cm, mv1);
        if (L::cz(i) > 0) cm = O::add(cm, mv2);
        if (L::cz(i) < 0) cm = O::sub(cm, mv2);
        V t = O::fma(O::splat(pc.wf[i]), cm, O::neg(m[i]));
        if (force) t = O::fma(fr, O::splat(pc.wcff[i]), t);
        h[i] = O::fma(om, t, h[i]);
    }
}

template <typename L>
__device__ __forceinline__ void MomentsShifted(const float* h,
                                               const PhysConst& pc,
                                               bool fluidlike, float& drho,
                                               float u[3]) {
    MomentsShiftedV<L, float>(h, pc, fluidlike, drho, u);
}

template <typename L>
__device__ __forceinline__ void CollideShifted(float* h, const PhysConst& pc,
                                               bool fluidlike, float drho,
                                               const float u[3], float omc) {
    CollideShiftedV<L, float>(h, pc, fluidlike, drho, u, omc);
}

// Moments and collision of two nodes at once (paired FP32 instructions);
// bit for bit what MomentsCollideT does to each of them alone.
template <typename L>
__device__ __forceinline__ void MomentsCollidePair(float* ha, float* hb,
                                                   const PhysConst& pc,
                                                   bool fluidlike,
                                                   float omcf) {
    constexpr int Q = L::Q;
    float2 h[Q];
#pragma unroll
    for (int i = 0; i < Q; i++) h[i] = make_float2(ha[i], hb[i]);
    float2 drho, u[3];
    MomentsShiftedV<L, float2>(h, pc, fluidlike, drho, u);
    CollideShiftedV<L, float2>(h, pc, fluidlike, drho, u, omcf);
#pragma unroll
    for (int i = 0; i < Q; i++) {
        ha[i] = h[i].x;
        hb[i] = h[i].y;
    }
}

template <typename L, typename T>
__device__ __forceinline__ void MomentsT(const typename Prec<T>::C* f,
                                         const PhysConst& pc, bool fluidlike,
                                         double& rho, double u[3]) {
    if constexpr (Prec<T>::kShifted) {
        float drho, uf[3];
        MomentsShifted<L>(f, pc, fluidlike, drho, uf);
        rho = 1.0 + (double)drho;
        u[0] = uf[0];
        u[1] = uf[1];
        u[2] = uf[2];
    } else {
        MomentsF64<L>(f, pc, fluidlike, rho, u);
    }
}

// Moments then collision with relaxation 1 - omega = omc (per cavity in
// the batched solver); returns the moments in FP64.
template <typename L, typename T>
__device__ __forceinline__ void MomentsCollideT(typename Prec<T>::C* f,
                                                const PhysConst& pc,
                                                bool fluidlike, double omc,
                                                float omcf, double& rho_out,
                                                double u_out[3]) {
    if constexpr (Prec<T>::kShifted) {
        float drho, u[3];
        MomentsShifted<L>(f, pc, fluidlike, drho, u);
        rho_out = 1.0 + (double)drho;
        u_out[0] = u[0];
        u_out[1] = u[1];
        u_out[2] = u[2];
        CollideShifted<L>(f, pc, fluidlike, drho, u, omcf);
    } else {
        double rho, u[3];
        MomentsF64<L>(f, pc, fluidlike, rho, u);
        rho_out = rho;
        u_out[0] = u[0];
        u_out[1] = u[1];
        u_out[2] = u[2];
        CollideF64<L>(f, pc, fluidlike, rho, u, omc);
    }
}

template <typename L, typename T>
__device__ __forceinline__ void MomentsCollideT(typename Prec<T>::C* f,
                                                const PhysConst& pc,
                                                bool fluidlike) {
    double rho, u[3];
    MomentsCollideT<L, T>(f, pc, fluidlike, pc.omc, pc.omcf, rho, u);
}

// The operation that applies at node (x, y, z): the region's own, or with
// a per-node wall velocity that node's entry of the boundary's per-node
// operations (the same masks, its own constants).
__device__ __forceinline__ const RegionOp& NodeOp(const RegionOp& op, int x,
                                                  int y, int z) {
    if (op.node_ops == nullptr) return op;
    const long long k =
        ((long long)(z - op.forg[2]) * op.fext[1] + (y - op.forg[1])) *
            op.fext[0] +
        (x - op.forg[0]);
    return op.node_ops[k];
}

// EQMDiffuseRefl (KerCutCellEQMDiffuseRefl3D, Src/boundary_kernel.inc:
// 1184-1276) with the wall constants precomputed per region.  Shifted
// forms use sum_in f = sum_in h + sum_in w and w_opp(i) = w_i.
template <typename L, typename T>
__device__ __forceinline__ void ApplyEqm(typename Prec<T>::C* f,
                                         const RegionOp& rop,
                                         const PhysConst& pc, int x, int y,
                                         int z) {
    constexpr int Q = L::Q;
    const RegionOp& op = NodeOp(rop, x, y, z);
    if constexpr (Prec<T>::kShifted) {
        // rhoWall - 1 and w_i (rhoWall a_i - 1) without cancellation
        float sin = 0.0f;
#pragma unroll
        for (int i = 0; i < Q; i++)
            if (op.in_mask >> i & 1u) sin += f[i];
        const float drw = (op.c0f + 2.0f * sin) * op.invf;
        const float rhoWall = 1.0f + drw;
#pragma unroll
        for (int i = 0; i < Q; i++)
            if (op.par_mask >> i & 1u)
                f[i] = pc.wf[i] * (op.am1f[i] + drw * op.af[i]);
#pragma unroll
        for (int i = 0; i < Q; i++)
            if (op.out_mask >> i & 1u)
                f[i] = f[L::opp(i)] + 2.0f * rhoWall * pc.wf[i] * op.bf[i];
    } else {
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
}

// FDPeriodic (KerCutCellPeriodic3D, Src/boundary_kernel.inc:1278-1666):
// f = the halo cell's f, which no step writes: f = 0.
template <typename L, typename T>
__device__ __forceinline__ void ApplyZero(typename Prec<T>::C* f,
                                          const PhysConst& pc) {
#pragma unroll
    for (int i = 0; i < L::Q; i++) f[i] = FromF<T>(0.0, i, pc);
}

// Halfway bounce-back: f_i = g_opp(i)(x) + 2 w_i (c_i . u_wall); the same
// for the deviation because w_opp(i) = w_i.
template <typename L, typename T>
__device__ __forceinline__ void ApplyHbb(typename Prec<T>::C* f,
                                         const RegionOp& rop,
                                         const PhysConst& pc,
                                         const T* __restrict__ src,
                                         const BlockDev& b, long long node,
                                         int x, int y, int z) {
    constexpr int Q = L::Q;
    using P = Prec<T>;
    const RegionOp& op = NodeOp(rop, x, y, z);
#pragma unroll
    for (int i = 0; i < Q; i++)
        if (op.out_mask >> i & 1u)
            f[i] = P::Load(src, L::opp(i) * b.popstride + node, L::opp(i), pc) +
                   (P::kShifted ? (typename P::C)op.bf[i]
                                : (typename P::C)op.b[i]);
}

// ---------------------------------------------------------------------------
// Fused step over one block.  kModeStep writes g^{n+1}; kModeMacro and
// kModeF recompute the current f = post-boundary populations from the
// previous g and write moments or f (FP64, dense) instead.
// The shifted forms hold two interior nodes per thread (PureNodeGroup) and
// collide them with paired FP32 instructions: 5 CTAs of 128 threads per SM
// (<= 102 registers) keeps the register pairs with almost no spills (at 6
// CTAs the paired form spilled and lost 17 % in FP32).
#ifndef MPLB_LP_MIN_BLOCKS
#define MPLB_LP_MIN_BLOCKS 5
#endif
// The FP64 form holds 19 doubles per node; 5 CTAs per SM (<= 102 registers)
// keeps it spill-free with 20 warps of loads in flight.
#ifndef MPLB_F64_MIN_BLOCKS
#define MPLB_F64_MIN_BLOCKS 5
#endif
// One node of the step, any region class.
template <int D, typename T, int MODE, bool O32>
__device__ __forceinline__ void StepNode(const BlockDev& b,
                                         const PhysConst& pc,
                                         const T* __restrict__ src,
                                         T* __restrict__ dst,
                                         double* __restrict__ out0,
                                         double* __restrict__ out1,
                                         double* __restrict__ out2,
                                         double* __restrict__ out3, int x,
                                         int y, int z) {
    using L = Lattice<D>;
    using P = Prec<T>;
    using C = typename P::C;
    constexpr int Q = L::Q;
    const int r = RegionOf(x, y, z, b.n, D);
    const int rf = b.rflags[r];
    const int cls = rf & 3;
    if (cls == kDeferred) return;
    const long long node = NodeIndexT<D, O32>(b, x, y, z);
    C f[Q];
    if (cls == kPure) {
        if constexpr (O32) {
            const T* ps = src + node;
#pragma unroll
            for (int i = 0; i < Q; i++)
                f[i] = P::Load(ps, b.pull_off32[i], i, pc);
        } else {
#pragma unroll
            for (int i = 0; i < Q; i++)
                f[i] = P::Load(src, PullIndex<L>(b, node, i), i, pc);
        }
    } else {
        // pull and stale masks from the kernel parameters, so the population
        // loads do not wait for the region record
        const uint32_t pull = b.rpull[r];
        const uint32_t stale = b.rstale[r];
        const T* ps = src + node;
#pragma unroll
        for (int i = 0; i < Q; i++) {
            if (pull >> i & 1u) {
                if constexpr (O32) f[i] = P::Load(ps, b.pull_off32[i], i, pc);
                else f[i] = P::Load(src, PullIndex<L>(b, node, i), i, pc);
            } else {
                f[i] = (C)0;
            }
        }
        const RegionInfo& R = b.regions[r];
        if (stale) {
            const double* st =
                b.stale + (R.side_base >= 0
                               ? (R.side_base + LocalIndex(R, x, y, z)) * Q
                               : 0);
#pragma unroll
            for (int i = 0; i < Q; i++)
                if (stale >> i & 1u) f[i] = (C)st[i];
        }
        for (int k = 0; k < R.nops; k++) {
            const RegionOp& op = b.ops[R.op[k]];
            if (op.kind == kOpEqm) ApplyEqm<L, T>(f, op, pc, x, y, z);
            else if (op.kind == kOpHbb)
                ApplyHbb<L, T>(f, op, pc, src, b, node, x, y, z);
            else if (op.kind == kOpZero) ApplyZero<L, T>(f, pc);
        }
    }
    const bool fl = (rf & 4) != 0;
    if (MODE == kModeF) {
        const long long dn =
            ((long long)z * b.n[1] + y) * (long long)b.n[0] + x;
#pragma unroll
        for (int i = 0; i < Q; i++) out0[dn * Q + i] = ToF<T>(f[i], i, pc);
        return;
    }
    if (MODE == kModeMacro) {
        double rho, u[3];
        MomentsT<L, T>(f, pc, fl, rho, u);
        const long long dn =
            ((long long)z * b.n[1] + y) * (long long)b.n[0] + x;
        out0[dn] = rho;
        out1[dn] = u[0];
        out2[dn] = u[1];
        if (D == 3) out3[dn] = u[2];
        return;
    }
    MomentsCollideT<L, T>(f, pc, fl);
    Rng rng = SeedRng(pc.seed, node);
    if constexpr (O32) {
        T* pd = dst + node;
#pragma unroll
        for (int i = 0; i < Q; i++)
            P::Store(pd, b.pop_off32[i], i, f[i], pc, rng);
    } else {
#pragma unroll
        for (int i = 0; i < Q; i++)
            P::Store(dst, OwnIndex(b, node, i), i, f[i], pc, rng);
    }
}

template <int D, typename T, int MODE, bool O32 = false>
__global__ void __launch_bounds__(128, std::is_same<T, double>::value
                                           ? MPLB_F64_MIN_BLOCKS
                                           : MPLB_LP_MIN_BLOCKS)
    StepKernel(BlockDev b, PhysConst pc, const T* __restrict__ src,
               T* __restrict__ dst, double* __restrict__ out0,
               double* __restrict__ out1, double* __restrict__ out2,
               double* __restrict__ out3) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = D == 3 ? (int)blockIdx.z : 0;
    if (x >= b.n[0]) return;
    StepNode<D, T, MODE, O32>(b, pc, src, dst, out0, out1, out2, out3, x, y,
                              z);
}

// Interior nodes per thread (G, 32 apart along x): all G nodes' loads are
// issued before any is computed, so a warp keeps 19 G loads in flight, and
// for G >= 2 each population access of the warp covers 32 G contiguous
// values (the FP32 and FP16 forms otherwise move 128 or 64 bytes per
// access).  The FP64 form moves enough bytes per load and has no registers
// for a second node.
#ifndef MPLB_LP_GROUP
#define MPLB_LP_GROUP 2
#endif
#ifndef MPLB_F64_GROUP
#define MPLB_F64_GROUP 1
#endif
template <typename T>
__host__ __device__ constexpr int SplitGroup() {
    return sizeof(T) < 8 ? MPLB_LP_GROUP : MPLB_F64_GROUP;
}

// G interior nodes of one row held by one thread: their populations, their
// element indices and which of them are stored.
template <int D, typename T, int G>
struct NodeGroup {
    typename Prec<T>::C f[G][Lattice<D>::Q];
    long long node[G];
    bool valid[G];
    int first;   // first valid node (the one a node group's seed follows)
};

// Loads the pulled populations of every node of the group.
template <int D, typename T, bool O32, int G>
__device__ __forceinline__ void GroupLoad(const BlockDev& b,
                                          const PhysConst& pc,
                                          const T* __restrict__ src,
                                          NodeGroup<D, T, G>& n) {
    using L = Lattice<D>;
    using P = Prec<T>;
    constexpr int Q = L::Q;
#pragma unroll
    for (int i = 0; i < Q; i++) {
#pragma unroll
        for (int j = 0; j < G; j++) {
            if constexpr (O32)
                n.f[j][i] = P::Load(src + n.node[j], b.pull_off32[i], i, pc);
            else
                n.f[j][i] = P::Load(src, PullIndex<L>(b, n.node[j], i), i, pc);
        }
    }
}

// Moments, collision and stores of the valid nodes of a loaded group, one
// node at a time (the shifted forms' pairs are PurePair's).
template <int D, typename T, bool O32, int G>
__device__ __forceinline__ void GroupFinish(const BlockDev& b,
                                            const PhysConst& pc,
                                            T* __restrict__ dst,
                                            NodeGroup<D, T, G>& n) {
    using L = Lattice<D>;
    using P = Prec<T>;
    constexpr int Q = L::Q;
    const bool fl = b.center_fluid != 0;
#pragma unroll
    for (int j = 0; j < G; j++) {
        if (!n.valid[j]) continue;
        MomentsCollideT<L, T>(n.f[j], pc, fl);
        Rng rg = SeedRng(pc.seed, n.node[j]);
        if constexpr (O32) {
            T* pd = dst + n.node[j];
#pragma unroll
            for (int i = 0; i < Q; i++)
                P::Store(pd, b.pop_off32[i], i, n.f[j][i], pc, rg);
        } else {
#pragma unroll
            for (int i = 0; i < Q; i++)
                P::Store(dst, OwnIndex(b, n.node[j], i), i, n.f[j][i], pc, rg);
        }
    }
}

// Moments and collision of an FP16 node pair on the stored values
// themselves, s_i = kHalfScale h_i / w_i (one node per half of each float2):
// the same steps as MomentsShiftedV and CollideShiftedV (opposite pairs
// summed first, heq whole per direction, the mass and momentum
// projection), with each h_i = (w_i / kHalfScale) s_i and m_i taken into
// the sums as multiply-adds by w_i / kHalfScale, and the equilibrium and
// the update written for s directly - there the equilibrium carries no
// weight (s_eq,i = kHalfScale [drho + rho (cu + (cu^2 - u^2) / 2)]), so
// neither the loads nor the stores scale the populations.
template <typename L>
__device__ __forceinline__ void MomentsCollideScaledPair(float2* s,
                                                         const PhysConst& pc,
                                                         bool fluidlike) {
    using O = VOps<float2>;
    constexpr int Q = L::Q;
    auto wl = [&](int i) { return O::splat(pc.wlf[i]); };
    // moments
    float2 drho = O::mul(s[0], wl(0));
#pragma unroll
    for (int i = 1; i < Q; i++)
        if (i < L::opp(i))
            drho = O::fma(O::add(s[i], s[L::opp(i)]), wl(i), drho);
    const float2 rho = O::add(O::splat(1.0f), drho);
    const float2 rinv = O::rcp(rho);
    float2 u[3];
#pragma unroll
    for (int a = 0; a < L::D; a++) {
        float2 j = O::splat(0.0f);
        bool first = true;
#pragma unroll
        for (int i = 0; i < Q; i++) {
            if (comp<L>(i, a) > 0) {
                const float2 d = O::sub(s[i], s[L::opp(i)]);
                j = first ? O::mul(d, wl(i)) : O::fma(d, wl(i), j);
                first = false;
            }
        }
        j = O::mul(O::mul(O::splat(pc.csf), j), rinv);
        if (pc.force_vel && fluidlike) j = O::add(j, O::splat(pc.hdtaf[a]));
        u[a] = j;
    }
    if (L::D == 2) u[2] = O::splat(0.0f);
    // collision: ms_i = s_i - s_eq,i, M0 = sum m_i, M = sum c_i m_i
    const float2 hr = O::mul(O::splat(0.5f), rho);
    const float2 csf = O::splat(pc.csf);
    const float2 cu0 = O::mul(csf, u[0]), cu1 = O::mul(csf, u[1]),
                 cu2 = O::mul(csf, u[2]);
    const float2 u2 =
        O::fma(u[0], u[0], O::fma(u[1], u[1], O::mul(u[2], u[2])));
    const float2 half = O::splat(0.5f);
    const float2 nscale = O::splat(-kHalfScale);
    float2 m[Q];
    m[0] = O::fma(nscale, O::fma(O::neg(hr), u2, drho), s[0]);
    float2 m0 = O::mul(m[0], wl(0)), mv0 = O::splat(0.0f),
           mv1 = O::splat(0.0f), mv2 = O::splat(0.0f);
#pragma unroll
    for (int i = 1; i < Q; i++) {
        if (i > L::opp(i)) continue;
        const int j = L::opp(i);
        float2 cu = O::splat(0.0f);
        bool first = true;
        const float2 comps[3] = {cu0, cu1, cu2};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const int c = comp<L>(i, a);
            if (c == 0 || a >= L::D) continue;
            const float2 t = c > 0 ? comps[a] : O::neg(comps[a]);
            cu = first ? t : O::add(cu, t);
            first = false;
        }
        const float2 y = O::fma(cu, cu, O::neg(u2));
        m[i] = O::fma(nscale, O::fma(rho, O::fma(half, y, cu), drho), s[i]);
        m[j] = O::fma(nscale, O::fma(rho, O::fma(half, y, O::neg(cu)), drho),
                      s[j]);
        m0 = O::fma(O::add(m[i], m[j]), wl(i), m0);
        const float2 d = O::mul(O::sub(m[i], m[j]), wl(i));
        if (L::cx(i) > 0) mv0 = O::add(mv0, d);
        if (L::cx(i) < 0) mv0 = O::sub(mv0, d);
        if (L::cy(i) > 0) mv1 = O::add(mv1, d);
        if (L::cy(i) < 0) mv1 = O::sub(mv1, d);
        if (L::cz(i) > 0) mv2 = O::add(mv2, d);
        if (L::cz(i) < 0) mv2 = O::sub(mv2, d);
    }
    if (pc.force_vel && fluidlike) {
        mv0 = O::fma(rho, O::splat(pc.hdta_csf[0]), mv0);
        mv1 = O::fma(rho, O::splat(pc.hdta_csf[1]), mv1);
        mv2 = O::fma(rho, O::splat(pc.hdta_csf[2]), mv2);
    }
    const float2 three = O::splat(3.0f);
    mv0 = O::mul(mv0, three);
    mv1 = O::mul(mv1, three);
    mv2 = O::mul(mv2, three);
    // s'_i = s_i + omega (kHalfScale (M0 + 3 c_i . M) - ms_i
    //                     + kHalfScale F_i / (omega w_i))
    const float2 om = O::splat(1.0f - pc.omcf);
    const bool force = pc.force && fluidlike;
    const float2 fr = O::mul(O::splat(pc.tw_omf), rho);
    const float2 scale = O::splat(kHalfScale);
#pragma unroll
    for (int i = 0; i < Q; i++) {
        float2 cm = m0;
        if (L::cx(i) > 0) cm = O::add(cm, mv0);
        if (L::cx(i) < 0) cm = O::sub(cm, mv0);
        if (L::cy(i) > 0) cm = O::add(cm, mv1);
        if (L::cy(i) < 0) cm = O::sub(cm, mv1);
        if (L::cz(i) > 0) cm = O::add(cm, mv2);
        if (L::cz(i) < 0) cm = O::sub(cm, mv2);
        float2 t = O::fma(scale, cm, O::neg(m[i]));
        if (force) t = O::fma(fr, O::splat(pc.cf256f[i]), t);
        s[i] = O::fma(om, t, s[i]);
    }
}

// Collision and stores of a shifted-form node pair whose populations are
// loaded, population by population, in float2 registers (node, node + 32).
template <int D, typename T, bool O32>
__device__ __forceinline__ void PairFinish(const BlockDev& b,
                                           const PhysConst& pc,
                                           T* __restrict__ dst, long long node,
                                           bool v0, bool v1, float2* h) {
    using L = Lattice<D>;
    constexpr int Q = L::Q;
    const bool fl = b.center_fluid != 0;
    if constexpr (std::is_same<T, __half>::value) {
        MomentsCollideScaledPair<L>(h, pc, fl);
        // population i of the two converted together by the hardware's
        // stochastic rounding (cvt.rs.f16x2.f32, 32 random bits per pair
        // from the first valid node's draw)
        const Rng rg = SeedRng(pc.seed, v0 ? node : node + 32);
#pragma unroll
        for (int i = 0; i < Q; i++) {
            const uint32_t pair =
                StochasticHalf2(h[i].x, h[i].y, SrDraw32(rg, i));
            const long long k = O32 ? node + b.pop_off32[i]
                                    : OwnIndex(b, node, i);
            if (v0)
                PopStore(dst + k,
                         __ushort_as_half((unsigned short)(pair & 0xffffu)));
            if (v1)
                PopStore(dst + k + 32,
                         __ushort_as_half((unsigned short)(pair >> 16)));
        }
    } else {
        float2 drho, u[3];
        MomentsShiftedV<L, float2>(h, pc, fl, drho, u);
        CollideShiftedV<L, float2>(h, pc, fl, drho, u, pc.omcf);
#pragma unroll
        for (int i = 0; i < Q; i++) {
            const long long k = O32 ? node + b.pop_off32[i]
                                    : OwnIndex(b, node, i);
            if (v0) PopStore(dst + k, (T)h[i].x);
            if (v1) PopStore(dst + k + 32, (T)h[i].y);
        }
    }
}

// The shifted forms' node pair x0, x0 + 32 of one interior row, held
// population by population in float2 registers from the loads through the
// paired collision to the stores (no packing between the two).  A node
// outside [1, n0 - 2] is computed on whatever its place holds (an x face, a
// halo column, the row padding, the next row or the slack after the last
// population, all inside the allocation) and not stored; the pair's element
// indices stay 32 apart, so one address serves both.  Same bits as the
// single-node collision of each (FP32; FP16 pairs collide on their stored
// values, MomentsCollideScaledPair).
template <int D, typename T, bool O32>
__device__ __forceinline__ void PurePair(const BlockDev& b,
                                         const PhysConst& pc,
                                         const T* __restrict__ src,
                                         T* __restrict__ dst, int x0, int y,
                                         int z) {
    using L = Lattice<D>;
    using P = Prec<T>;
    constexpr int Q = L::Q;
    const bool v0 = x0 >= 1 && x0 <= b.n[0] - 2;
    const bool v1 = x0 + 32 >= 1 && x0 + 32 <= b.n[0] - 2;
    if (!v0 && !v1) return;
    const long long node = NodeIndexT<D, O32>(b, x0, y, z);
    float2 h[Q];
#pragma unroll
    for (int i = 0; i < Q; i++) {
        const long long k = O32 ? node + b.pull_off32[i]
                                : PullIndex<L>(b, node, i);
        if constexpr (std::is_same<T, __half>::value) {
            // the stored values themselves (MomentsCollideScaledPair)
            h[i] = make_float2(__half2float(src[k]), __half2float(src[k + 32]));
        } else {
            h[i] = make_float2(P::Load(src, k, i, pc),
                               P::Load(src, k + 32, i, pc));
        }
    }
    PairFinish<D, T, O32>(b, pc, dst, node, v0, v1, h);
}

// The G nodes x0 + 32 j (j < G) of one interior row (the shifted forms'
// pairs: PurePair); nodes outside [1, n0 - 2] are computed on whatever
// their places hold and not stored.
template <int D, typename T, bool O32, int G>
__device__ __forceinline__ void PureNodeGroup(const BlockDev& b,
                                              const PhysConst& pc,
                                              const T* __restrict__ src,
                                              T* __restrict__ dst, int x0,
                                              int y, int z) {
    if constexpr (Prec<T>::kShifted && G == 2) {
        PurePair<D, T, O32>(b, pc, src, dst, x0, y, z);
    } else {
        NodeGroup<D, T, G> n;
        n.first = -1;
#pragma unroll
        for (int j = 0; j < G; j++) {
            const int x = x0 + 32 * j;
            n.valid[j] = x >= 1 && x <= b.n[0] - 2;
            if (n.valid[j] && n.first < 0) n.first = j;
        }
        if (n.first < 0) return;
        n.node[0] = NodeIndexT<D, O32>(b, x0, y, z);
#pragma unroll
        for (int j = 1; j < G; j++) n.node[j] = n.node[0] + 32 * j;
        GroupLoad<D, T, O32, G>(b, pc, src, n);
        GroupFinish<D, T, O32, G>(b, pc, dst, n);
    }
}

// Rows of interior nodes handled per x-face block of SplitStepKernel.
constexpr int kSplitRows = 64;
constexpr int kSplitCta = 128;   // threads per CTA of SplitStepKernel
constexpr int kSplitWarps = kSplitCta / 32;

// Staged interior of the shifted forms.  Each warp takes kStageTasks
// consecutive 64-node row segments and runs them through a pipeline of
// StageDepth<T>() shared-memory stages: while it computes one segment, the
// copies of the next segments' 19 source windows are in flight (16-byte
// cp.async copies into shared memory, which take no registers), so a warp
// keeps several segments' bytes in flight where the per-thread loads keep
// one.  A window is the row segment x - c_x needs, widened to 16-byte
// boundaries: columns [xs - StageLead, xs + 64 + StageLead).
#ifndef MPLB_LP_STAGED
#define MPLB_LP_STAGED 1
#endif
#ifndef MPLB_STAGE_TASKS
#define MPLB_STAGE_TASKS 8
#endif
constexpr int kStageTasks = MPLB_STAGE_TASKS;
template <typename T>
__host__ __device__ constexpr int StageLead() {   // 16 bytes of elements
    return 16 / (int)sizeof(T);
}
template <typename T>
__host__ __device__ constexpr int StageWinElems() {
    return 64 + 2 * StageLead<T>();
}
#ifndef MPLB_STAGE_DEPTH
#define MPLB_STAGE_DEPTH 2
#endif
template <typename T>
__host__ __device__ constexpr int StageDepth() {
    return MPLB_STAGE_DEPTH;
}
template <int D, typename T>
__host__ __device__ constexpr int StageSmemBytes() {
    return kSplitWarps * StageDepth<T>() * Lattice<D>::Q * StageWinElems<T>() *
           (int)sizeof(T);
}
// The FP16 form only: its 2-byte loads keep half the FP32 form's bytes in
// flight per warp, and the staged interior runs it 9-11 % faster at 256^3
// (341-347 us against 382 us; 8 segments per warp in 2 stages, or 4 in 3,
// or 2 in 3: within 2 % of each other); the FP32 form, which needs 2.6 KB
// more per stage, ran 25 % slower staged.
template <typename T>
__host__ __device__ constexpr bool StagedStep() {
    return MPLB_LP_STAGED != 0 && std::is_same<T, __half>::value &&
           SplitGroup<T>() == 2;
}


// Interior "warp tasks": 32 G consecutive nodes of a row per warp; CTA c of
// a chunk's interior takes tasks kSplitWarps c .. + kSplitWarps - 1.
struct SplitTask {
    int r;    // interior row (chunk-relative rows included), or -1
    int x0;   // first node of the lane
};
template <int G>
__device__ __forceinline__ SplitTask InteriorTask(const BlockDev& b,
                                                  int chunk, int w) {
    const int tpr = (b.n[0] + 32 * G - 1) / (32 * G);   // tasks per row
    const int t = (w - 1) * kSplitWarps + (int)(threadIdx.x >> 5);
    const int rl = t / tpr;
    SplitTask k;
    k.r = rl < kSplitRows ? chunk * kSplitRows + rl : -1;
    k.x0 = (t - rl * tpr) * 32 * G + (int)(threadIdx.x & 31);
    return k;
}

// CTAs of one chunk: the x-face CTA and the interior CTAs (a warp takes
// one task, or kStageTasks with the staged interior).
template <int G, bool STAGED = false>
__host__ __device__ constexpr long long SplitChunkCtas(int n0) {
    return 1 + ((long long)kSplitRows * ((n0 + 32 * G - 1) / (32 * G)) +
                kSplitWarps * (STAGED ? kStageTasks : 1) - 1) /
                   (kSplitWarps * (STAGED ? kStageTasks : 1));
}

__device__ __forceinline__ void CpAsync16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void CpAsyncCommit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void CpAsyncWait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The staged interior of one CTA of a chunk (see StagedStep): warp k takes
// the chunk's tasks (w - 1) kSplitWarps kStageTasks + k kStageTasks + t,
// t < kStageTasks (task -> row t / tasks per row, segment t % tasks per
// row).  Lane l computes the pair l, l + 32 of the segment (PairFinish).
template <int D, typename T, bool O32>
__device__ __forceinline__ void StagedInterior(const BlockDev& b,
                                               const PhysConst& pc,
                                               const T* __restrict__ src,
                                               T* __restrict__ dst, int chunk,
                                               int w, int rows, int ny) {
    using L = Lattice<D>;
    constexpr int Q = L::Q;
    constexpr int S = StageDepth<T>();
    constexpr int kWin = StageWinElems<T>();
    constexpr int kLead = StageLead<T>();
    constexpr int kChunks = kWin * (int)sizeof(T) / 16;   // 16-byte copies
    static_assert(kChunks <= 32, "one copy per lane and population");
    extern __shared__ __align__(16) unsigned char stage_raw[];
    const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
    T* stages = reinterpret_cast<T*>(stage_raw) + warp * S * Q * kWin;
    const int tpr = (b.n[0] + 63) / 64;
    const int t0 = ((w - 1) * kSplitWarps + warp) * kStageTasks;
    // task t of this warp: its row (or -1) and first column
    auto task = [&](int t, int& r, int& xs) {
        const int g = t0 + t;
        const int rl = g / tpr;
        r = (t < kStageTasks && rl < kSplitRows &&
             chunk * kSplitRows + rl < rows)
                ? chunk * kSplitRows + rl
                : -1;
        xs = (g - rl * tpr) * 64;
    };
    // copies of task t's windows into stage st (one group, maybe empty)
    constexpr int kE = 16 / (int)sizeof(T);   // elements per copy
    auto issue = [&](int t, int st) {
        int r, xs;
        task(t, r, xs);
        if (r >= 0 && lane < kChunks) {
            const long long node = NodeIndexT<D, O32>(
                b, xs, 1 + r % ny, D == 3 ? 1 + r / ny : 0);
            T* win = stages + st * Q * kWin;
#pragma unroll
            for (int i = 0; i < Q; i++) {
                const long long k0 =
                    (O32 ? node + b.pull_off32[i] : PullIndex<L>(b, node, i)) +
                    L::cx(i) - kLead;
                CpAsync16(win + i * kWin + lane * kE, src + k0 + lane * kE);
            }
        }
        CpAsyncCommit();
    };
#pragma unroll
    for (int t = 0; t < S - 1; t++) issue(t, t);
    for (int t = 0; t < kStageTasks; t++) {
        issue(t + S - 1, (t + S - 1) % S);
        CpAsyncWait<S - 1>();
        __syncwarp();
        int r, xs;
        task(t, r, xs);
        if (r >= 0) {
            const int x0 = xs + lane;
            const bool v0 = x0 >= 1 && x0 <= b.n[0] - 2;
            const bool v1 = x0 + 32 >= 1 && x0 + 32 <= b.n[0] - 2;
            if (v0 || v1) {
                const T* win = stages + (t % S) * Q * kWin + lane + kLead;
                const long long node = NodeIndexT<D, O32>(
                    b, x0, 1 + r % ny, D == 3 ? 1 + r / ny : 0);
                float2 h[Q];
#pragma unroll
                for (int i = 0; i < Q; i++) {
                    const T* p = win + i * kWin - L::cx(i);
                    if constexpr (std::is_same<T, __half>::value)
                        h[i] = make_float2(__half2float(p[0]),
                                           __half2float(p[32]));
                    else
                        h[i] = make_float2((float)p[0], (float)p[32]);
                }
                PairFinish<D, T, O32>(b, pc, dst, node, v0, v1, h);
            }
        }
        __syncwarp();   // every lane is done with stage t % S
    }
}

// The step with no warp mixing interior and boundary nodes (a warp holding
// one boundary node runs that node's boundary programme with the other 31
// lanes idle: at 128^3 a third of the issue slots had no work).  One launch,
// three kinds of CTA by blockIdx.x + blk0 (a step in two parts launches
// kinds 2 and 3, which read no halo layer of a cut z face, apart from
// kind 1):
//   1. shell rows: every row with y or z on the block boundary (coalesced);
//   2. per chunk of 64 interior rows, one CTA for their x = 0 and x = n0 - 1
//      nodes, followed by
//   3. the CTAs of those rows' interior nodes, each warp taking 32 G
//      consecutive nodes of a row (PureNodeGroup).  A row's tasks start on
//      the row's first node so every store begins on the row's 32-byte
//      boundary (the x-face lanes idle); the x-face CTA runs next to them,
//      so the sectors they share meet in L2 instead of costing a
//      read-modify-write in HBM.
template <int D, typename T, bool O32>
__global__ void __launch_bounds__(128, std::is_same<T, double>::value
                                           ? MPLB_F64_MIN_BLOCKS
                                           : MPLB_LP_MIN_BLOCKS)
    SplitStepKernel(BlockDev b, PhysConst pc, const T* __restrict__ src,
                    T* __restrict__ dst, unsigned blk0, unsigned spc) {
    // block and row counts fit in 32 bits (the launcher checks the grid),
    // so the index arithmetic stays 32-bit
    const int nbx = (b.n[0] + (int)blockDim.x - 1) / (int)blockDim.x;
    const int ny = b.n[1] - 2;
    const int nz = D == 3 ? b.n[2] : 1;
    const unsigned nsr = (unsigned)nbx * (2 * nz + (D == 3 ? 2 * ny : 0));
    constexpr int G = SplitGroup<T>();
    constexpr bool kStaged = StagedStep<T>();
    const unsigned per_chunk = (unsigned)SplitChunkCtas<G, kStaged>(b.n[0]);
    // CTA order: spc = 0, the shell rows first, then the chunks (blk0: a
    // launch of the chunks alone starts after the shell rows); spc > 0, each
    // chunk's CTAs followed by spc shell-row CTAs, so the shell rows' long
    // boundary programmes run beside interior CTAs instead of in waves of
    // their own at the start
    unsigned blk;
    if (spc > 0) {
        const unsigned slot = blockIdx.x / (per_chunk + spc);
        const unsigned r = blockIdx.x - slot * (per_chunk + spc);
        if (r >= per_chunk) {
            blk = slot * spc + (r - per_chunk);
            if (blk >= nsr) return;
        } else {
            blk = nsr + slot * per_chunk + r;
        }
    } else {
        blk = blockIdx.x + blk0;
    }
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
        StepNode<D, T, kModeStep, O32>(b, pc, src, dst, nullptr, nullptr,
                                       nullptr, nullptr, x, y, z);
        return;
    }
    blk -= nsr;
    const int rows = ny * (D == 3 ? b.n[2] - 2 : 1);
    const int chunk = (int)(blk / per_chunk);
    const int w = (int)(blk % per_chunk);
    if (w == 0) {
        const int r = chunk * kSplitRows + (int)(threadIdx.x >> 1);
        if (threadIdx.x >= 2 * kSplitRows || r >= rows) return;
        const int x = (threadIdx.x & 1) ? b.n[0] - 1 : 0;
        StepNode<D, T, kModeStep, O32>(b, pc, src, dst, nullptr, nullptr,
                                       nullptr, nullptr, x, 1 + r % ny,
                                       D == 3 ? 1 + r / ny : 0);
        return;
    }
    if constexpr (kStaged) {
        StagedInterior<D, T, O32>(b, pc, src, dst, chunk, w, rows, ny);
    } else {
        const SplitTask k = InteriorTask<G>(b, chunk, w);
        if (k.r < 0 || k.r >= rows) return;
        PureNodeGroup<D, T, O32, G>(b, pc, src, dst, k.x0, 1 + k.r % ny,
                                    D == 3 ? 1 + k.r / ny : 0);
    }
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
// not pulled keep their previous value, as in KerStream3D).  The store holds
// f (FP64 form) or the deviation h (shifted forms) in FP64.
template <int D, typename T>
__global__ void DeferredStreamKernel(BlockDev b, PhysConst pc,
                                     const T* __restrict__ src) {
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
            b.fdef[i * b.ndef + k] = Prec<T>::Load(
                src, i * b.popstride + node + UpOffset<L>(b, i), i, pc);
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
// One boundary operation on a deferred node (x, y, z) holding f
// (EQMDiffuseRefl, halfway bounce-back or ExtrapolPressure1ST).  The
// extrapolation reads the inner neighbour's current f: from the store when
// it is deferred, otherwise from its upstream g (pure), with its earlier
// boundary operations applied (local).
template <int D, typename T>
__device__ __forceinline__ void DeferredApply(const BlockDev& b,
                                              const PhysConst& pc,
                                              const T* __restrict__ src,
                                              const RegionOp& op, int x, int y,
                                              int z,
                                              typename Prec<T>::C* f) {
    using L = Lattice<D>;
    using P = Prec<T>;
    using C = typename P::C;
    constexpr int Q = L::Q;
    if (op.kind == kOpEqm) {
        ApplyEqm<L, T>(f, op, pc, x, y, z);
    } else if (op.kind == kOpHbb) {
        ApplyHbb<L, T>(f, op, pc, src, b, NodeIndex<D>(b, x, y, z), x, y, z);
    } else if (op.kind == kOpZero) {
        ApplyZero<L, T>(f, pc);
    } else if (op.kind == kOpExtrapol) {
        int q[3] = {x, y, z};
        if (op.nb_axis >= 0) q[op.nb_axis] += op.nb_sign;
        const int nr = RegionOf(q[0], q[1], q[2], b.n, D);
        const RegionInfo& N = b.regions[nr];
        const bool nbdef = N.cls == kDeferred;
        const long long nk =
            nbdef ? N.side_base + LocalIndex(N, q[0], q[1], q[2]) : 0;
        const long long nnode = NodeIndex<D>(b, q[0], q[1], q[2]);
        // the neighbour's post-boundary f as the reference has it when this
        // boundary runs: the store (deferred), its pulled values (pure), or
        // its pulled and stale values after its boundary operations that
        // come before this one (local)
        C g[Q];
        if (N.cls == kLocal) {
#pragma unroll
            for (int i = 0; i < Q; i++)
                g[i] = (N.pull >> i & 1u)
                           ? P::Load(src, i * b.popstride + nnode +
                                              UpOffset<L>(b, i), i, pc)
                           : (C)0;
            if (N.stale) {
                const double* st =
                    b.stale + (N.side_base + LocalIndex(N, q[0], q[1], q[2])) * Q;
#pragma unroll
                for (int i = 0; i < Q; i++)
                    if (N.stale >> i & 1u) g[i] = (C)st[i];
            }
            for (int j = 0; j < N.nops; j++) {
                const RegionOp& nop = b.ops[N.op[j]];
                if (nop.bc >= op.bc) break;
                if (nop.kind == kOpEqm)
                    ApplyEqm<L, T>(g, nop, pc, q[0], q[1], q[2]);
                else if (nop.kind == kOpHbb)
                    ApplyHbb<L, T>(g, nop, pc, src, b, nnode, q[0], q[1],
                                   q[2]);
                else if (nop.kind == kOpZero)
                    ApplyZero<L, T>(g, pc);
            }
        }
        if constexpr (P::kShifted) {
            // f_i = (h_i + w_i) rho_given / rho for all but the last
            float drho = 0.0f;
#pragma unroll
            for (int i = 0; i < Q; i++) {
                if (op.in_mask >> i & 1u)
                    f[i] = nbdef ? (C)b.fdef[i * b.ndef + nk]
                           : N.cls == kLocal
                               ? g[i]
                               : P::Load(src, i * b.popstride + nnode +
                                                  UpOffset<L>(b, i), i, pc);
                drho += f[i];
            }
            const float rm1 = ((float)(op.rho_given - 1.0) - drho) / (1.0f + drho);
#pragma unroll
            for (int i = 0; i < Q - 1; i++) f[i] += (f[i] + pc.wf[i]) * rm1;
        } else {
            double rho = 0.0;
#pragma unroll
            for (int i = 0; i < Q; i++) {
                if (op.in_mask >> i & 1u)
                    f[i] = nbdef ? b.fdef[i * b.ndef + nk]
                           : N.cls == kLocal
                               ? g[i]
                               : P::Load(src, i * b.popstride + nnode +
                                                  UpOffset<L>(b, i), i, pc);
                rho = rho + f[i];
            }
            const double ratio = op.rho_given / rho;
#pragma unroll
            for (int i = 0; i < Q - 1; i++) f[i] = f[i] * ratio;
        }
    }
}

template <int D, typename T>
__global__ void DeferredOpKernel(BlockDev b, PhysConst pc,
                                 const T* __restrict__ src,
                                 const DeferredSeg* __restrict__ segs,
                                 int nseg, long long total) {
    using L = Lattice<D>;
    using P = Prec<T>;
    using C = typename P::C;
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
    C f[Q];
#pragma unroll
    for (int i = 0; i < Q; i++) f[i] = (C)b.fdef[i * b.ndef + k];
    DeferredApply<D, T>(b, pc, src, b.ops[sg.op], x, y, z, f);
#pragma unroll
    for (int i = 0; i < Q; i++) b.fdef[i * b.ndef + k] = (double)f[i];
}

// The whole deferred programme of a node in one thread, where no deferred
// node reads another's value (the usual case: an outlet reads the interior
// next to it): streaming (non-pulled populations keep the stored value),
// every boundary operation of its region in definition order, the store
// for the next step and observations, moments, collision.
template <int D, typename T>
__global__ void DeferredFusedKernel(BlockDev b, PhysConst pc,
                                    const T* __restrict__ src,
                                    T* __restrict__ dst) {
    using L = Lattice<D>;
    using P = Prec<T>;
    using C = typename P::C;
    constexpr int Q = L::Q;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= b.ndef) return;
    int r, x, y, z;
    long long k;
    if (!DeferredNode(b, t, r, x, y, z, k)) return;
    const RegionInfo& R = b.regions[r];
    const long long node = NodeIndex<D>(b, x, y, z);
    C f[Q];
#pragma unroll
    for (int i = 0; i < Q; i++)
        f[i] = (R.pull >> i & 1u)
                   ? P::Load(src, i * b.popstride + node + UpOffset<L>(b, i),
                             i, pc)
                   : (C)b.fdef[i * b.ndef + k];
    for (const int* o = b.dops_flat + b.dops_first[r]; *o >= 0; o++)
        DeferredApply<D, T>(b, pc, src, b.ops[*o], x, y, z, f);
#pragma unroll
    for (int i = 0; i < Q; i++) b.fdef[i * b.ndef + k] = (double)f[i];
    MomentsCollideT<L, T>(f, pc, R.fluidlike != 0);
    Rng rng = SeedRng(pc.seed, node);
#pragma unroll
    for (int i = 0; i < Q; i++)
        P::Store(dst, i * b.popstride + node, i, f[i], pc, rng);
}

// Deferred nodes, part 3: moments and collision (or observation).
template <int D, typename T, int MODE>
__global__ void DeferredFinishKernel(BlockDev b, PhysConst pc,
                                     T* __restrict__ dst,
                                     double* __restrict__ out0,
                                     double* __restrict__ out1,
                                     double* __restrict__ out2,
                                     double* __restrict__ out3) {
    using L = Lattice<D>;
    using P = Prec<T>;
    using C = typename P::C;
    constexpr int Q = L::Q;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= b.ndef) return;
    int r, x, y, z;
    long long k;
    if (!DeferredNode(b, t, r, x, y, z, k)) return;
    const RegionInfo& R = b.regions[r];
    C f[Q];
#pragma unroll
    for (int i = 0; i < Q; i++) f[i] = (C)b.fdef[i * b.ndef + k];
    const long long dn = ((long long)z * b.n[1] + y) * (long long)b.n[0] + x;
    if (MODE == kModeF) {
#pragma unroll
        for (int i = 0; i < Q; i++) out0[dn * Q + i] = ToF<T>(f[i], i, pc);
        return;
    }
    if (MODE == kModeMacro) {
        double rho, u[3];
        MomentsT<L, T>(f, pc, R.fluidlike != 0, rho, u);
        out0[dn] = rho;
        out1[dn] = u[0];
        out2[dn] = u[1];
        if (D == 3) out3[dn] = u[2];
        return;
    }
    MomentsCollideT<L, T>(f, pc, R.fluidlike != 0);
    const long long node = NodeIndex<D>(b, x, y, z);
    Rng rng = SeedRng(pc.seed, node);
#pragma unroll
    for (int i = 0; i < Q; i++)
        P::Store(dst, i * b.popstride + node, i, f[i], pc, rng);
}

// Initial state of one block from per-node macroscopic values
// (KerInitialiseBGK2nd3D: f = feq(rho, u), Src/model_kernel.inc:352-380) or
// from uploaded f (fin != nullptr, point-major, FP64).  Writes f^0 to
// `fdirect` (form T, same layout as g), the stale and deferred stores, and
// g^0 = collision of f^0 with its own moments to `g`.
template <int D, typename T>
__global__ void __launch_bounds__(128)
    InitKernel(BlockDev b, PhysConst pc, const double* __restrict__ rho0,
               const double* __restrict__ u0, const double* __restrict__ v0,
               const double* __restrict__ w0, const double* __restrict__ fin,
               T* __restrict__ fdirect, T* __restrict__ g) {
    using L = Lattice<D>;
    using P = Prec<T>;
    using C = typename P::C;
    constexpr int Q = L::Q;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = D == 3 ? (int)blockIdx.z : 0;
    if (x >= b.n[0]) return;
    const long long dn = ((long long)z * b.n[1] + y) * (long long)b.n[0] + x;
    C f[Q];
    if (fin != nullptr) {
#pragma unroll
        for (int i = 0; i < Q; i++) f[i] = FromF<T>(fin[dn * Q + i], i, pc);
    } else if constexpr (P::kShifted) {
        const float drho = (float)(rho0[dn] - 1.0);
        const float rho = 1.0f + drho;
        const float u[3] = {(float)u0[dn], (float)v0[dn],
                            D == 3 ? (float)w0[dn] : 0.0f};
        const float u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
#pragma unroll
        for (int i = 0; i < Q; i++) {
            const float cu = pc.csf * ((float)L::cx(i) * u[0] +
                                       (float)L::cy(i) * u[1] +
                                       (float)L::cz(i) * u[2]);
            f[i] = pc.wf[i] * (drho + rho * (cu + 0.5f * (cu * cu - u2)));
        }
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
    Rng rng = SeedRng(pc.seed, node);
#pragma unroll
    for (int i = 0; i < Q; i++)
        P::Store(fdirect, i * b.popstride + node, i, f[i], pc, rng);
    if (R.side_base >= 0) {
        const long long k = R.side_base + LocalIndex(R, x, y, z);
        if (R.cls == kLocal) {
#pragma unroll
            for (int i = 0; i < Q; i++) b.stale[k * Q + i] = (double)f[i];
        } else if (R.cls == kDeferred) {
#pragma unroll
            for (int i = 0; i < Q; i++) b.fdef[i * b.ndef + k] = (double)f[i];
        }
    }
    if (g == nullptr) return;   // one-array scheme: f^0 only
    MomentsCollideT<L, T>(f, pc, R.fluidlike != 0);
#pragma unroll
    for (int i = 0; i < Q; i++)
        P::Store(g, i * b.popstride + node, i, f[i], pc, rng);
}

// Every element of a population array, halo layers and row padding
// included, set to the storage form's encoding of f = 0.  The reference's
// dats start at zero and a halo cell that no transfer writes keeps f = 0
// (a stale value a boundary node can pull); the shifted forms store
// h = f - w, so their zero is h = -w (FP16: -kHalfScale), not 0.
template <typename T>
__global__ void FillZeroFKernel(T* __restrict__ p, long long popstride,
                                int Q, PhysConst pc) {
    const long long total = popstride * Q;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
         e < total; e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e / popstride);
        if constexpr (std::is_same<T, __half>::value)
            p[e] = __float2half(-kHalfScale);
        else if constexpr (std::is_same<T, float>::value)
            p[e] = -pc.wf[i];
        else
            p[e] = 0.0;
    }
}

// Observation straight from f^0 stored by InitKernel (before any step).
template <int D, typename T, int MODE>
__global__ void DirectObserveKernel(BlockDev b, PhysConst pc,
                                    const T* __restrict__ fdirect,
                                    double* __restrict__ out0,
                                    double* __restrict__ out1,
                                    double* __restrict__ out2,
                                    double* __restrict__ out3) {
    using L = Lattice<D>;
    using P = Prec<T>;
    using C = typename P::C;
    constexpr int Q = L::Q;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = D == 3 ? (int)blockIdx.z : 0;
    if (x >= b.n[0]) return;
    const long long dn = ((long long)z * b.n[1] + y) * (long long)b.n[0] + x;
    const long long node = NodeIndex<D>(b, x, y, z);
    const RegionInfo& R = b.regions[RegionOf(x, y, z, b.n, D)];
    C f[Q];
    if (R.cls == kDeferred && R.side_base >= 0) {
        const long long k = R.side_base + LocalIndex(R, x, y, z);
#pragma unroll
        for (int i = 0; i < Q; i++) f[i] = (C)b.fdef[i * b.ndef + k];
    } else {
#pragma unroll
        for (int i = 0; i < Q; i++)
            f[i] = P::Load(fdirect, i * b.popstride + node, i, pc);
    }
    if (MODE == kModeF) {
#pragma unroll
        for (int i = 0; i < Q; i++) out0[dn * Q + i] = ToF<T>(f[i], i, pc);
        return;
    }
    double rho, u[3];
    MomentsT<L, T>(f, pc, R.fluidlike != 0, rho, u);
    out0[dn] = rho;
    out1[dn] = u[0];
    out2[dn] = u[1];
    if (D == 3) out3[dn] = u[2];
}

// All halo copies of a step in one launch.  Copies run in definition order
// in the reference; here every cell whose value one copy gives directly (its
// source not written earlier in the step, its destination written by that
// copy alone) is copied by its copy's box, a range of one copy per CTA, and
// every other halo element is copied from its origin resolved on the host
// (HaloElem), a range of those per CTA: no element is written twice and no
// source is written in the launch, so the CTAs run in any order.
struct HaloBlockDev {          // what a copy needs of a block
    long long pitch, plane, popstride;
    int xoff;
    void* pop[2];
};

struct HaloCopyDev {
    int iter[3];
    int fbase[3];
    int tbase[3];
    uint32_t pops;
    int from, to;              // block indices
    long long cells;
    const uint8_t* prev;       // per cell: read the previous array (or null)
    const uint8_t* ordered;    // per cell: copied as resolved elements
};

// A resolved element copy with its element offsets (population included).
struct HaloElemDev {
    long long s, d;
    int from2;                 // 2 * origin block + (previous array ? 1 : 0)
    int to;
};

constexpr int kHaloThreads = 512;
constexpr int kHaloCellsPerCta = 4 * kHaloThreads;
constexpr int kHaloMaxBlocks = 64;   // blocks whose descriptors go to smem

struct HaloFusedDev {
    const HaloCopyDev* copies;
    const HaloBlockDev* blocks;
    int nblocks;
    const int2* ctas;          // per CTA: (copy, first cell) or (-1, first
                               // resolved element)
    const HaloElemDev* elems;
    int nelems;
};

template <int D>
__device__ __forceinline__ long long HaloNodeIndex(const HaloBlockDev& b,
                                                  int x, int y, int z) {
    return (long long)(D == 3 ? z + 1 : 0) * b.plane +
           (long long)(y + 1) * b.pitch + (long long)(x + b.xoff);
}

template <int D, typename T>
__global__ void __launch_bounds__(kHaloThreads)
    HaloFusedKernel(HaloFusedDev h, int cur) {
    using L = Lattice<D>;
    constexpr int Q = L::Q;
    const int2 a = h.ctas[blockIdx.x];
    if (a.x < 0) {
        // resolved elements a.y .. a.y + kHaloCellsPerCta - 1
        __shared__ const void* pops[2 * kHaloMaxBlocks];
        const bool in_smem = h.nblocks <= kHaloMaxBlocks;
        if (in_smem)
            for (int b = threadIdx.x; b < h.nblocks; b += blockDim.x) {
                pops[2 * b] = h.blocks[b].pop[cur];
                pops[2 * b + 1] = h.blocks[b].pop[1 - cur];
            }
        __syncthreads();
        const int end = min(a.y + kHaloCellsPerCta, h.nelems);
        for (int m = a.y + threadIdx.x; m < end; m += blockDim.x) {
            const HaloElemDev e = h.elems[m];
            const int fb = e.from2 >> 1;
            const T* from = static_cast<const T*>(
                in_smem ? pops[e.from2]
                        : h.blocks[fb].pop[(e.from2 & 1) ? 1 - cur : cur]);
            T* to = static_cast<T*>(const_cast<void*>(
                in_smem ? pops[2 * e.to] : h.blocks[e.to].pop[cur]));
            to[e.d] = from[e.s];
        }
        return;
    }
    __shared__ HaloCopyDev sc;
    __shared__ HaloBlockDev sb[2];
    if (threadIdx.x == 0) {
        sc = h.copies[a.x];
        sb[0] = h.blocks[sc.from];
        sb[1] = h.blocks[sc.to];
    }
    __syncthreads();
    const int cells = (int)sc.cells;
    const int end = min(a.y + kHaloCellsPerCta, cells);
    const T* cur_from = static_cast<const T*>(sb[0].pop[cur]);
    const T* prev_from = static_cast<const T*>(sb[0].pop[1 - cur]);
    T* to = static_cast<T*>(sb[1].pop[cur]);
    for (int t = a.y + threadIdx.x; t < end; t += blockDim.x) {
        if (sc.ordered[t]) continue;
        const int i = t % sc.iter[0];
        const int j = (t / sc.iter[0]) % sc.iter[1];
        const int k = t / (sc.iter[0] * sc.iter[1]);
        const long long s = HaloNodeIndex<D>(sb[0], sc.fbase[0] + i,
                                             sc.fbase[1] + j, sc.fbase[2] + k);
        const long long d = HaloNodeIndex<D>(sb[1], sc.tbase[0] + i,
                                             sc.tbase[1] + j, sc.tbase[2] + k);
        const T* from =
            (sc.prev != nullptr && sc.prev[t]) ? prev_from : cur_from;
        // every load of the cell before its stores: they overlap
        T v[Q];
#pragma unroll
        for (int q = 0; q < Q; q++)
            if (sc.pops >> q & 1u) v[q] = from[q * sb[0].popstride + s];
#pragma unroll
        for (int q = 0; q < Q; q++)
            if (sc.pops >> q & 1u) to[q * sb[1].popstride + d] = v[q];
    }
}

struct FaceDev {
    int axis, layer;
    int ua, va;          // in-plane axes (va = -1 in 2D)
    int nu, nv;
    int npop;
    int pop[kMaxQ];
};

template <int D, typename T, bool EXPORT>
__global__ void __launch_bounds__(256)
    FaceKernel(BlockDev b, FaceDev fd, T* __restrict__ f,
               T* __restrict__ buf) {
    const long long total = (long long)fd.npop * fd.nu * fd.nv;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
         t < total; t += (long long)gridDim.x * blockDim.x) {
        const int u = (int)(t % fd.nu);
        const long long r = t / fd.nu;
        const int v = (int)(r % fd.nv);
        const int p = (int)(r / fd.nv);
        int c[3] = {0, 0, 0};
        c[fd.axis] = fd.layer;
        c[fd.ua] = u;
        if (fd.va >= 0) c[fd.va] = v;
        const long long e = (long long)fd.pop[p] * b.popstride +
                            NodeIndex<D>(b, c[0], c[1], c[2]);
        if (EXPORT) buf[t] = f[e];
        else f[e] = buf[t];
    }
}

__global__ void ResidualPartialKernel(const double* __restrict__ q,
                                      double* __restrict__ qold, long long n,
                                      double* __restrict__ part);

// Sum of a field over n values, per CTA (mass), and a count of
// non-finite or non-positive values (health word).
__global__ void SumPartialKernel(const double* __restrict__ q, long long n,
                                 double* __restrict__ part,
                                 unsigned long long* __restrict__ bad);

}  // namespace mplb
