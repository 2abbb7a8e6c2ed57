// Batched lid-driven cavities: many independent square D2Q9 blocks of
// different sizes advanced together.
//
// Every cavity is the single-block case of the fused step (kernels.cuh)
// with halfway bounce-back on its four walls, the top one moving: a
// population whose upstream node lies beyond a wall takes the node's own
// post-collision opposite population plus 2 w_i (c_i . u_wall) (the top
// wall wins at the two top corners, as when the top boundary is defined
// after the side walls).  Cavities are cut into tiles of consecutive nodes;
// a CTA advances one tile per iteration of a grid-stride loop over the
// active tiles (tiles of converged cavities are dropped between check
// periods).  Population p of node k (= y n + x) of a cavity sits at
// base + p n^2 + k, structure of arrays per cavity, no halo.
#pragma once

#include "kernels.cuh"

namespace mplb {

struct BatchCav {
    long long base;    // element offset of the cavity in a population array
    long long mbase;   // offset of its nodes in the macro arrays
    int n;             // nodes per side
    int pad;
    double omc;        // 1 - omega of this cavity
    double dt;         // MPLB time step (residual normalisation)
    float omcf;
    float ninv;        // 1 / n (row of node k: (k + 1/2) / n rounded down)
    double lidb[9];    // 2 w_i (c_i . u_lid) for populations bounced at the lid
    float lidbf[9];
};

struct BatchDev {
    const BatchCav* cavs;
    // active tiles: (cavity, first node, nodes per side, element offset of
    // the cavity in 128-byte units), so a tile's population addresses wait
    // on the tile's own load alone and the cavity's constants load beside
    // the populations
    const int4* tiles;
    const int* ntiles;      // number of active tiles (device word)
    int tile_nodes;         // nodes per tile
    double* macro[3];       // rho, u, v of every cavity, packed
    double* macro_old[3];
};

struct GridSync {           // bounded grid-wide barrier state
    unsigned* count;
    unsigned* gen;
    int* err;               // set to 1 when a wait gives up
    long long limit;        // polls before giving up
};

// Every population value is read once and written once per step, so the
// batch's loads and stores take the streaming (evict-first) cache hint and
// leave L2 to the tile entries and cavity constants that every step reads
// again (measured faster than plain accesses and than an L2 evict-last
// policy on the tile loads, which cost registers).
template <typename T>
__device__ __forceinline__ typename Prec<T>::C BatchLoad(
    const T* __restrict__ s, long long k, int i, const PhysConst& pc) {
    if constexpr (std::is_same<T, float>::value ||
                  std::is_same<T, double>::value)
        return __ldcs(s + k);
    else
        return Prec<T>::Load(s, k, i, pc);
}
template <typename T>
__device__ __forceinline__ void BatchStore(T* __restrict__ d, long long k,
                                           int i, typename Prec<T>::C v,
                                           const PhysConst& pc, Rng& rng) {
    if constexpr (std::is_same<T, float>::value ||
                  std::is_same<T, double>::value)
        __stcs(d + k, v);
    else
        Prec<T>::Store(d, k, i, v, pc, rng);
}

// Population i of node (x, y) = k of a cavity: pulled from x - c_i, or, when
// that lies beyond a wall, the node's own opposite population plus the
// lid's 2 w_i (c_i . u_lid) (the top wall).  Only the axes population i
// moves along are checked (one unsigned compare each).
template <typename T, int i>
__device__ __forceinline__ typename Prec<T>::C BatchPull(
    const BatchCav& cv, const T* __restrict__ s, int n, int nn, int x, int y,
    int k, const PhysConst& pc) {
    using L = Lattice<2>;
    using P = Prec<T>;
    using C = typename P::C;
    constexpr int cx = L::cx(i), cy = L::cy(i);
    const int sx = x - cx, sy = y - cy;
    bool in = true;
    if constexpr (cx != 0) in = in && (unsigned)sx < (unsigned)n;
    if constexpr (cy != 0) in = in && (unsigned)sy < (unsigned)n;
    if (in) return BatchLoad<T>(s, (long long)i * nn + (long long)sy * n + sx, i, pc);
    C b = (C)0;
    if constexpr (cy < 0) {
        if (sy > n - 1) {
            if constexpr (P::kShifted) b = cv.lidbf[i];
            else b = cv.lidb[i];
        }
    }
    return BatchLoad<T>(s, (long long)L::opp(i) * nn + k, L::opp(i), pc) + b;
}

template <typename T, int I>
struct BatchPullAll {
    __device__ static __forceinline__ void run(typename Prec<T>::C* f,
                                               const BatchCav& cv,
                                               const T* __restrict__ s, int n,
                                               int nn, int x, int y, int k,
                                               const PhysConst& pc) {
        f[I] = BatchPull<T, I>(cv, s, n, nn, x, y, k, pc);
        BatchPullAll<T, I + 1>::run(f, cv, s, n, nn, x, y, k, pc);
    }
};
template <typename T>
struct BatchPullAll<T, 9> {
    __device__ static __forceinline__ void run(typename Prec<T>::C*,
                                               const BatchCav&, const T*, int,
                                               int, int, int, int,
                                               const PhysConst&) {}
};

// One node of one cavity: pull with bounce-back, moments, collision.
template <typename T, bool MACRO>
__device__ __forceinline__ void BatchNode(const BatchDev& bd,
                                          const PhysConst& pc,
                                          const BatchCav& cv, int n,
                                          long long base, float ninv, int k,
                                          const T* __restrict__ src,
                                          T* __restrict__ dst) {
    using L = Lattice<2>;
    using P = Prec<T>;
    using C = typename P::C;
    constexpr int Q = 9;
    const long long nn = (long long)n * n;
    // k / n without an integer division: (k + 1/2) / n is at least 1/(2n)
    // from an integer and the float product is off by less than
    // (k + 1/2) / n * 2^-22, so truncating it is exact while n <= 1024
    const int y = n <= 1024 ? (int)(((float)k + 0.5f) * ninv) : k / n;
    const int x = k - y * n;
    const T* s = src + base;
    T* d = dst + base;
    C f[Q];
    BatchPullAll<T, 0>::run(f, cv, s, n, (int)nn, x, y, k, pc);
    double rho, u[3];
    MomentsCollideT<L, T>(f, pc, false, cv.omc, cv.omcf, rho, u);
    Rng rng = SeedRng(pc.seed, base + k);
#pragma unroll
    for (int i = 0; i < Q; i++) BatchStore<T>(d, i * nn + k, i, f[i], pc, rng);
    if (MACRO) {
        bd.macro[0][cv.mbase + k] = rho;
        bd.macro[1][cv.mbase + k] = u[0];
        bd.macro[2][cv.mbase + k] = u[1];
    }
}

// G nodes of one cavity per thread, 32 apart (the FP32 form): all of their
// loads are issued before any node is computed, and each warp access covers
// 32 G contiguous values.  Nodes beyond the cavity are skipped (their loads
// repeat node ka's).
template <typename T, bool MACRO, int G>
__device__ __forceinline__ void BatchNodeGroup(const BatchDev& bd,
                                               const PhysConst& pc,
                                               const BatchCav& cv, int n,
                                               long long base, float ninv,
                                               int ka,
                                               const T* __restrict__ src,
                                               T* __restrict__ dst) {
    using L = Lattice<2>;
    using P = Prec<T>;
    using C = typename P::C;
    constexpr int Q = 9;
    const int nn = n * n;   // a cavity's populations fit in 32-bit offsets
    int kk[G];
#pragma unroll
    for (int j = 0; j < G; j++) kk[j] = ka + 32 * j < nn ? ka + 32 * j : ka;
    const T* s = src + base;
    T* d = dst + base;
    C f[G][Q];
#pragma unroll
    for (int j = 0; j < G; j++) {
        const int k = kk[j];
        const int y = n <= 1024 ? (int)(((float)k + 0.5f) * ninv) : k / n;
        const int x = k - y * n;
        BatchPullAll<T, 0>::run(f[j], cv, s, n, nn, x, y, k, pc);
    }
#pragma unroll
    for (int j = 0; j < G; j++) {
        if (j > 0 && ka + 32 * j >= nn) break;
        const int k = kk[j];
        double rho, u[3];
        MomentsCollideT<L, T>(f[j], pc, false, cv.omc, cv.omcf, rho, u);
        Rng rng = SeedRng(pc.seed, base + k);
#pragma unroll
        for (int i = 0; i < Q; i++) BatchStore<T>(d, i * nn + k, i, f[j][i], pc, rng);
        if (MACRO) {
            bd.macro[0][cv.mbase + k] = rho;
            bd.macro[1][cv.mbase + k] = u[0];
            bd.macro[2][cv.mbase + k] = u[1];
        }
    }
}

#ifndef MPLB_BATCH_GROUP
#define MPLB_BATCH_GROUP 2
#endif

// Nodes per thread of the step kernels (threads per CTA = tile nodes / this):
// MPLB_BATCH_GROUP in the FP32 form, one in FP64.
template <typename T>
__host__ __device__ constexpr int BatchNodesPerThread() {
    return sizeof(T) < 8 ? MPLB_BATCH_GROUP : 1;
}


template <typename T, bool MACRO>
__device__ __forceinline__ void BatchSweep(const BatchDev& bd,
                                           const PhysConst& pc, int nt,
                                           const T* __restrict__ src,
                                           T* __restrict__ dst) {
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int4 tile = bd.tiles[t];
        const BatchCav& cv = bd.cavs[tile.x];
        const int n = tile.z;
        const int nn = n * n;
        const long long base = (long long)tile.w * (long long)(128 / sizeof(T));
        // the correctly rounded 1 / n, as the host computes it
        const float ninv = __frcp_rn((float)n);
        constexpr int G = BatchNodesPerThread<T>();
        if constexpr (G > 1) {
            // warp w has nodes [32 G w, 32 G (w + 1)) of the tile, lane l
            // the nodes 32 G w + l + 32 j
            const int ka = tile.y + (int)(threadIdx.x >> 5) * (32 * G) +
                           (int)(threadIdx.x & 31);
            if (ka < nn)
                BatchNodeGroup<T, MACRO, G>(bd, pc, cv, n, base, ninv, ka,
                                            src, dst);
        } else {
            const int k = tile.y + threadIdx.x;
            if (k < nn)
                BatchNode<T, MACRO>(bd, pc, cv, n, base, ninv, k, src, dst);
        }
    }
}

// One step over every active tile (a CUDA graph replays a chunk of these).
// `nt` is the active tile count when the launch was made (one-step graphs
// are captured again when it changes), so the tile loads need not wait for
// the device word.
template <typename T, bool MACRO>
__global__ void __launch_bounds__(256)
    BatchStepKernel(BatchDev bd, PhysConst pc, int nt,
                    const T* __restrict__ src, T* __restrict__ dst) {
    BatchSweep<T, MACRO>(bd, pc, nt, src, dst);
}

// Grid-wide barrier with a bounded wait: thread 0 of each CTA arrives and
// polls the generation word; after `limit` polls it records an error and
// the kernel returns instead of waiting on.
__device__ __forceinline__ bool GridBarrier(const GridSync& g,
                                            unsigned& my_gen) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const unsigned target = my_gen + 1;
        __threadfence();
        if (atomicAdd(g.count, 1u) == gridDim.x - 1) {
            atomicExch(g.count, 0u);
            __threadfence();
            atomicExch(g.gen, target);
        } else {
            long long polls = 0;
            while (atomicAdd(g.gen, 0u) != target) {
                if (++polls > g.limit || atomicAdd(g.err, 0) != 0) {
                    atomicExch(g.err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        my_gen = target;
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// `nsteps` steps in one launch (all CTAs co-resident, cooperative launch),
// ping-ponging between a and b; moments are written on the last step when
// `macro_last` is set.
template <typename T>
__global__ void __launch_bounds__(256)
    BatchPersistentKernel(BatchDev bd, PhysConst pc, T* a, T* b, int nsteps,
                          int macro_last, GridSync gs) {
    unsigned my_gen = 0;
    if (threadIdx.x == 0) my_gen = atomicAdd(gs.gen, 0u);
    const int nt = *bd.ntiles;
    for (int s = 0; s < nsteps; s++) {
        const T* src = (s & 1) ? b : a;
        T* dst = (s & 1) ? a : b;
        if (macro_last && s == nsteps - 1)
            BatchSweep<T, true>(bd, pc, nt, src, dst);
        else
            BatchSweep<T, false>(bd, pc, nt, src, dst);
        if (s + 1 < nsteps && !GridBarrier(gs, my_gen)) return;
        pc.seed += 1;
    }
}

// Per active tile: sum (q - q_old)^2 and sum q^2 of rho, u, v; q_old <- q.
__global__ void BatchResidualPartialKernel(BatchDev bd,
                                           double* __restrict__ part);

// Per active cavity c (CTA c): sums its tiles' partials in order and writes
// max_q [sum (q - q_old)^2 / sum q^2] / (check_period dt) (the reference's
// CalcResidualError + GetMaximumResidual on one cavity).
__global__ void BatchResidualFinalKernel(BatchDev bd,
                                         const double* __restrict__ part,
                                         const int4* __restrict__ ranges,
                                         int ncav, int check_period,
                                         double* __restrict__ res);

// Initial state: f^0 = feq(rho, u, v) from the packed macro fields
// (KerInitialiseBGK2nd), then g^0 = collision of f^0 with its own moments,
// as the first StreamCollision would do, into `a`.
template <typename T>
__global__ void BatchInitKernel(BatchDev bd, PhysConst pc,
                                const int4* __restrict__ alltiles, int ntiles,
                                T* __restrict__ a) {
    using L = Lattice<2>;
    using P = Prec<T>;
    using C = typename P::C;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int4 tile = alltiles[t];
        const BatchCav& cv = bd.cavs[tile.x];
        const int k = tile.y + threadIdx.x;
        if (k >= cv.n * cv.n) continue;
        const long long nn = (long long)cv.n * cv.n;
        const double rho = bd.macro[0][cv.mbase + k];
        const double ux = bd.macro[1][cv.mbase + k];
        const double uy = bd.macro[2][cv.mbase + k];
        const double u2 = ux * ux + uy * uy;
        C f[9];
#pragma unroll
        for (int i = 0; i < 9; i++) {
            double cu = 0.0;
            bool first = true;
            const int c0 = L::cx(i), c1 = L::cy(i);
            if (c0 != 0) {
                cu = c0 > 0 ? pc.cs * ux : -(pc.cs * ux);
                first = false;
            }
            if (c1 != 0) {
                const double t1 = c1 > 0 ? pc.cs * uy : -(pc.cs * uy);
                cu = first ? t1 : cu + t1;
            }
            if constexpr (P::kShifted)
                f[i] = (C)(pc.w[i] *
                           ((rho - 1.0) + rho * (cu + 0.5 * (cu * cu - u2))));
            else
                f[i] = (pc.w[i] * rho) * ((1.0 + cu) + 0.5 * (cu * cu - u2));
        }
        double r, u[3];
        MomentsCollideT<L, T>(f, pc, false, cv.omc, cv.omcf, r, u);
        Rng rng = SeedRng(0x5eedu, cv.base + k);
#pragma unroll
        for (int i = 0; i < 9; i++) P::Store(a + cv.base, i * nn + k, i, f[i], pc, rng);
    }
}

}  // namespace mplb

namespace mplb {

// Host launchers, instantiated with the FP64 and the FP32 forms.
template <typename T>
struct BatchLaunch {
    static cudaError_t Step(bool macro, int grid, int threads, cudaStream_t s,
                            const BatchDev& bd, const PhysConst& pc, int nt,
                            const T* src, T* dst) {
        if (macro)
            BatchStepKernel<T, true><<<grid, threads, 0, s>>>(bd, pc, nt, src,
                                                              dst);
        else
            BatchStepKernel<T, false><<<grid, threads, 0, s>>>(bd, pc, nt, src,
                                                               dst);
        return cudaGetLastError();
    }
    static cudaError_t Persistent(int grid, int threads, cudaStream_t s,
                                  const BatchDev& bd, const PhysConst& pc,
                                  T* a, T* b, int nsteps, int macro_last,
                                  const GridSync& gs) {
        BatchDev bdv = bd;
        PhysConst pcv = pc;
        GridSync gsv = gs;
        void* args[] = {&bdv, &pcv, &a, &b, &nsteps, &macro_last, &gsv};
        return cudaLaunchCooperativeKernel(
            (const void*)BatchPersistentKernel<T>, dim3(grid), dim3(threads),
            args, 0, s);
    }
    static cudaError_t MaxCoResident(int threads, int* per_sm) {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            per_sm, (const void*)BatchPersistentKernel<T>, threads, 0);
    }
    static cudaError_t Init(int grid, int threads, cudaStream_t s,
                            const BatchDev& bd, const PhysConst& pc,
                            const int4* alltiles, int ntiles, T* a) {
        BatchInitKernel<T><<<grid, threads, 0, s>>>(bd, pc, alltiles, ntiles,
                                                    a);
        return cudaGetLastError();
    }
};

}  // namespace mplb
