// FP64 (reference arithmetic) instantiations and the FP64 reductions.
// Compiled with -fmad=false: see kernels.cuh.
#include "launch_impl.cuh"

namespace mplb {

template struct Launch<2, double>;
template struct Launch<3, double>;

// Sum of v over the CTA (blockDim.x a multiple of 32): shuffles within each
// warp, then over the warps' sums; the total is valid in thread 0.  `ws`
// is 32 doubles of shared memory, reusable when this returns.
__device__ __forceinline__ double BlockSum(double v, double* ws) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) ws[w] = v;
    __syncthreads();
    if (w == 0) {
        v = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;
}

__global__ void ResidualPartialKernel(const double* __restrict__ q,
                                      double* __restrict__ qold, long long n,
                                      double* __restrict__ part) {
    __shared__ double ws[32];
    double d = 0.0, s = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const double v = q[t];
        const double dv = v - qold[t];
        d = d + dv * dv;
        s = s + v * v;
        qold[t] = v;
    }
    d = BlockSum(d, ws);
    s = BlockSum(s, ws);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = d;
        part[2 * blockIdx.x + 1] = s;
    }
}

__global__ void SumPartialKernel(const double* __restrict__ q, long long n,
                                 double* __restrict__ part,
                                 unsigned long long* __restrict__ bad) {
    __shared__ double ws[32];
    double s = 0.0;
    unsigned long long nb = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const double v = q[t];
        s = s + v;
        if (!(v > 0.0) || !isfinite(v)) nb++;
    }
    s = BlockSum(s, ws);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
    if (nb) atomicAdd(bad, nb);
}

}  // namespace mplb

#include "batch_kernels.cuh"

namespace mplb {

template struct BatchLaunch<double>;

__global__ void BatchResidualPartialKernel(BatchDev bd,
                                           double* __restrict__ part) {
    __shared__ double ws[32];
    const int nt = *bd.ntiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int4 tile = bd.tiles[t];
        const BatchCav& cv = bd.cavs[tile.x];
        const int k = tile.y + threadIdx.x;
        double v[6] = {0, 0, 0, 0, 0, 0};
        if (k < cv.n * cv.n) {
            for (int m = 0; m < 3; m++) {
                const double q = bd.macro[m][cv.mbase + k];
                const double dq = q - bd.macro_old[m][cv.mbase + k];
                v[2 * m] = dq * dq;
                v[2 * m + 1] = q * q;
                bd.macro_old[m][cv.mbase + k] = q;
            }
        }
        for (int j = 0; j < 6; j++) {
            const double sum = BlockSum(v[j], ws);
            if (threadIdx.x == 0) part[(long long)t * 6 + j] = sum;
        }
    }
}

__global__ void BatchResidualFinalKernel(BatchDev bd,
                                         const double* __restrict__ part,
                                         const int4* __restrict__ ranges,
                                         int ncav, int check_period,
                                         double* __restrict__ res) {
    // ranges[c] = (cavity, first active tile, tile count, -)
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncav) return;
    const int4 r = ranges[c];
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int t = r.y; t < r.y + r.z; t++)
        for (int j = 0; j < 6; j++) s[j] = s[j] + part[(long long)t * 6 + j];
    const BatchCav& cv = bd.cavs[r.x];
    double mx = 0.0;
    for (int m = 0; m < 3; m++) {
        const double rel = (s[2 * m] / s[2 * m + 1]) / (check_period * cv.dt);
        // A NaN ratio (a diverged cavity) is kept, not skipped: the host
        // reports the cavity as diverged instead of converged.
        if (isnan(rel)) {
            mx = rel;
            break;
        }
        if (mx <= rel) mx = rel;
    }
    res[c] = mx;
}

}  // namespace mplb
