// FP64 (reference arithmetic) instantiations and the FP64 reductions.
// Compiled with -fmad=false: see kernels.cuh.
#include "launch_impl.cuh"

namespace mplb {

template struct Launch<2, double>;
template struct Launch<3, double>;

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
