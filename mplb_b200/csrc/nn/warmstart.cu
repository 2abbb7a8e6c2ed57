// The warm-start network (include/mplbnn.h): a 4-level convolutional
// encoder-decoder on the tensor-core convolutions of conv.cu, its
// element-wise kernels (input planes, pooling, upsampling and their
// gradients, loss, bias gradients, Adam, weight flips), and the resampling
// of cavity fields to and from the network grid.
//
// Levels l = 0..3: side 128 >> l, channels 32 << l.  Encoder level l: two
// 3x3 convolutions with ReLU, then 2x2 average pooling; the second
// convolution writes straight into the upper channels of the decoder's
// concatenation buffer of that level.  Bottleneck (16 x 16, 256 channels):
// two convolutions.  Decoder level l: nearest 2x upsampling of the level
// below into the lower channels of the concatenation buffer, two 3x3
// convolutions with ReLU.  Output: 1x1 convolution to 16 fp32 channels of
// which the first three are the normalised (rho, u, v).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../../include/mplbnn.h"
#include "conv_host.h"

namespace mplb {
namespace nn {

namespace {

constexpr int kOK = 0, kInvalid = 1, kCuda = 3, kTimeout = 5;
constexpr int kGrid = 128;
constexpr int kInCh = 32;    // input planes, padded
constexpr int kOutCh = 16;   // output channels, first 3 used
constexpr int kEw = 256;     // threads of the element-wise kernels

struct LayerSpec {
    int cin, cout, taps, relu;
};

// e0a e0 | e1a e1 | e2a e2 | ba bb | d2a d2 | d1a d1 | d0a d0 | out
constexpr LayerSpec kLayers[15] = {
    {32, 32, 9, 1},   {32, 32, 9, 1},   {32, 64, 9, 1},   {64, 64, 9, 1},
    {64, 128, 9, 1},  {128, 128, 9, 1}, {128, 256, 9, 1}, {256, 256, 9, 1},
    {384, 128, 9, 1}, {128, 128, 9, 1}, {192, 64, 9, 1},  {64, 64, 9, 1},
    {96, 32, 9, 1},   {32, 32, 9, 1},   {32, kOutCh, 1, 0}};
constexpr int kNumLayers = 15;

void LayerOffsets(long long* w_off, long long* b_off, long long* total) {
    long long o = 0;
    for (int l = 0; l < kNumLayers; l++) {
        const LayerSpec& s = kLayers[l];
        w_off[l] = o;
        o += (long long)s.cout * s.taps * s.cin;
        b_off[l] = o;
        o += s.cout;
    }
    *total = o;
}

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ void Unpack8(const uint4& q, float* f) {
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        f[2 * i] = __uint_as_float(w[i] << 16);
        f[2 * i + 1] = __uint_as_float(w[i] & 0xFFFF0000u);
    }
}

__device__ __forceinline__ uint32_t Pack2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

__device__ __forceinline__ uint4 Pack8(const float* f) {
    return make_uint4(Pack2(f[0], f[1]), Pack2(f[2], f[3]), Pack2(f[4], f[5]),
                      Pack2(f[6], f[7]));
}

__device__ __forceinline__ uint4 Ld8(const bf16* base, long long pix,
                                     long long ps, int c) {
    return *reinterpret_cast<const uint4*>(base + pix * ps + c);
}

__device__ __forceinline__ void St8(bf16* base, long long pix, long long ps,
                                    int c, const uint4& v) {
    *reinterpret_cast<uint4*>(base + pix * ps + c) = v;
}

// Input planes of one pixel: cond0..2, x, y (node centres), zeros.
__global__ void InputKernel(const float* __restrict__ cond, int n,
                            bf16* __restrict__ xin) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)n * kGrid * kGrid) return;
    const int img = (int)(p / (kGrid * kGrid));
    const int r = (int)(p - (long long)img * kGrid * kGrid);
    const int y = r / kGrid, x = r % kGrid;
    float f[8] = {cond[3 * img], cond[3 * img + 1], cond[3 * img + 2],
                  (x + 0.5f) / kGrid, (y + 0.5f) / kGrid, 0.f, 0.f, 0.f};
    uint4* o = reinterpret_cast<uint4*>(xin + p * kInCh);
    o[0] = Pack8(f);
    const uint4 z = make_uint4(0, 0, 0, 0);
    o[1] = z;
    o[2] = z;
    o[3] = z;
}

// 2x2 average pooling: dst (h, w) from src (2h, 2w); one thread per
// (destination pixel, 8 channels).
__global__ void PoolKernel(const bf16* __restrict__ src, long long sps,
                           bf16* __restrict__ dst, long long dps, int n, int h,
                           int w, int c) {
    const int groups = c / 8;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * h * w * groups) return;
    const int g = (int)(t % groups);
    const long long q = t / groups;
    const int img = (int)(q / ((long long)h * w));
    const int r = (int)(q - (long long)img * h * w);
    const int y = r / w, x = r % w;
    const long long s0 = ((long long)img * 2 * h + 2 * y) * (2 * w) + 2 * x;
    float acc[8] = {}, f[8];
    const long long kids[4] = {s0, s0 + 1, s0 + 2 * w, s0 + 2 * w + 1};
    for (int k = 0; k < 4; k++) {
        Unpack8(Ld8(src, kids[k], sps, 8 * g), f);
#pragma unroll
        for (int i = 0; i < 8; i++) acc[i] += f[i];
    }
#pragma unroll
    for (int i = 0; i < 8; i++) acc[i] *= 0.25f;
    St8(dst, q, dps, 8 * g, Pack8(acc));
}

// Nearest 2x upsampling: dst (2h, 2w) from src (h, w).
__global__ void UpsampleKernel(const bf16* __restrict__ src, long long sps,
                               bf16* __restrict__ dst, long long dps, int n,
                               int h, int w, int c) {
    const int groups = c / 8;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int H = 2 * h, W = 2 * w;
    if (t >= (long long)n * H * W * groups) return;
    const int g = (int)(t % groups);
    const long long p = t / groups;
    const int img = (int)(p / ((long long)H * W));
    const int r = (int)(p - (long long)img * H * W);
    const int y = r / W, x = r % W;
    const long long q = ((long long)img * h + y / 2) * w + x / 2;
    St8(dst, p, dps, 8 * g, Ld8(src, q, sps, 8 * g));
}

__device__ __forceinline__ void MaskPositive(const uint4& a, float* v) {
    float f[8];
    Unpack8(a, f);
#pragma unroll
    for (int i = 0; i < 8; i++)
        if (!(f[i] > 0.0f)) v[i] = 0.0f;
}

// Gradient of the upsampling, times the ReLU mask of its source:
// gdst(h, w) = sum of the four gsrc children * (act > 0).
__global__ void UpBwdKernel(const bf16* __restrict__ gsrc, long long gps,
                            const bf16* __restrict__ act, long long aps,
                            bf16* __restrict__ gdst, long long dps, int n,
                            int h, int w, int c) {
    const int groups = c / 8;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * h * w * groups) return;
    const int g = (int)(t % groups);
    const long long q = t / groups;
    const int img = (int)(q / ((long long)h * w));
    const int r = (int)(q - (long long)img * h * w);
    const int y = r / w, x = r % w;
    const long long s0 = ((long long)img * 2 * h + 2 * y) * (2 * w) + 2 * x;
    float acc[8] = {}, f[8];
    const long long kids[4] = {s0, s0 + 1, s0 + 2 * w, s0 + 2 * w + 1};
    for (int k = 0; k < 4; k++) {
        Unpack8(Ld8(gsrc, kids[k], gps, 8 * g), f);
#pragma unroll
        for (int i = 0; i < 8; i++) acc[i] += f[i];
    }
    MaskPositive(Ld8(act, q, aps, 8 * g), acc);
    St8(gdst, q, dps, 8 * g, Pack8(acc));
}

// Gradient reaching an encoder output through the skip connection and the
// pooling: gdst(H, W) = (gskip + gpool(parent) / 4) * (act > 0).
__global__ void SkipBwdKernel(const bf16* __restrict__ gskip, long long sps,
                              const bf16* __restrict__ gpool, long long pps,
                              const bf16* __restrict__ act, long long aps,
                              bf16* __restrict__ gdst, long long dps, int n,
                              int H, int W, int c) {
    const int groups = c / 8;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * H * W * groups) return;
    const int g = (int)(t % groups);
    const long long p = t / groups;
    const int img = (int)(p / ((long long)H * W));
    const int r = (int)(p - (long long)img * H * W);
    const int y = r / W, x = r % W;
    const long long q = ((long long)img * (H / 2) + y / 2) * (W / 2) + x / 2;
    float a[8], b[8];
    Unpack8(Ld8(gskip, p, sps, 8 * g), a);
    Unpack8(Ld8(gpool, q, pps, 8 * g), b);
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] += 0.25f * b[i];
    MaskPositive(Ld8(act, p, aps, 8 * g), a);
    St8(gdst, p, dps, 8 * g, Pack8(a));
}

// Mean squared error over the 3 used output channels; dpred = dL/dpred.
__global__ void LossKernel(const float* __restrict__ pred,
                           const float* __restrict__ target, long long npix,
                           float scale, bf16* __restrict__ dpred,
                           double* __restrict__ loss) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double s = 0.0;
    if (p < npix) {
        float d[kOutCh] = {};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            d[c] = pred[p * kOutCh + c] - target[p * 3 + c];
            s += (double)d[c] * d[c];
        }
        uint4* o = reinterpret_cast<uint4*>(dpred + p * kOutCh);
        float g[8];
#pragma unroll
        for (int h = 0; h < 2; h++) {
#pragma unroll
            for (int i = 0; i < 8; i++) g[i] = scale * d[8 * h + i];
            o[h] = Pack8(g);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(~0u, s, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, s);
}

// db[c] += sum over pixels of dz[p][c].
__global__ void BiasGradKernel(const bf16* __restrict__ dz, long long ps,
                               long long npix, int c, float* __restrict__ db) {
    __shared__ float part[kEw];
    const int lanes = kEw / c;              // c divides 256
    const int ch = threadIdx.x % c, lane = threadIdx.x / c;
    float s = 0.0f;
    for (long long p = (long long)blockIdx.x * lanes + lane; p < npix;
         p += (long long)gridDim.x * lanes)
        s += __bfloat162float(dz[p * ps + ch]);
    part[threadIdx.x] = s;
    __syncthreads();
    if (lane == 0) {
        for (int l = 1; l < lanes; l++) s += part[l * c + ch];
        atomicAdd(db + ch, s);
    }
}

__global__ void AdamKernel(float* __restrict__ w, const float* __restrict__ g,
                           float* __restrict__ m, float* __restrict__ v,
                           bf16* __restrict__ wbf, long long n, float lr_t,
                           float b1, float b2, float eps) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr_t * mi / (sqrtf(vi) + eps);
    w[i] = wi;
    wbf[i] = __float2bfloat16_rn(wi);
}

__global__ void ToBf16Kernel(const float* __restrict__ w, bf16* __restrict__ o,
                             long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = __float2bfloat16_rn(w[i]);
}

// wd[c][taps - 1 - t][k] = w[k][t][c] (weights of the data gradient).
__global__ void FlipKernel(const float* __restrict__ w, bf16* __restrict__ wd,
                           int cout, int taps, int cin) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)cout * taps * cin) return;
    const int c = (int)(i % cin);
    const int t = (int)((i / cin) % taps);
    const int k = (int)(i / ((long long)cin * taps));
    wd[((long long)c * taps + (taps - 1 - t)) * cout + k] =
        __float2bfloat16_rn(w[i]);
}

__global__ void CompactKernel(const float* __restrict__ pred, long long npix,
                              float* __restrict__ out) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    for (int c = 0; c < 3; c++) out[p * 3 + c] = pred[p * kOutCh + c];
}

struct CavMeta {
    int n;
    long long off;
    double rho_scale, u_scale;
};

// Catmull-Rom (bicubic) sample of a cell-centred n x n field on the unit
// square (node i at i, walls at -1/2 and n - 1/2) at (xs, ys) in node units.
// The stencil reaches beyond the walls through ghost nodes mirrored across
// them (node -1-k <-> k): with `walls`, as 2 w - f for the velocity (the
// moving lid at y = n - 1/2 has `top`, the other walls 0); without, as f
// (the density, which has no wall value).  On converged cavities the
// 128 <-> N round trip of u is 0.4-0.8 % this way, against 1.1-2.9 % for
// bilinear with the same ghosts and 1.5-3.5 % for bilinear held at the edge
// node.
template <typename Get>
__device__ __forceinline__ double SampleCavity(Get get, int n, double xs,
                                               double ys, bool walls,
                                               double top) {
    xs = fmin(fmax(xs, -0.5), n - 0.5);
    ys = fmin(fmax(ys, -0.5), n - 0.5);
    const int i0 = (int)floor(xs), j0 = (int)floor(ys);
    const double fx = xs - i0, fy = ys - j0;
    auto mirror = [n](int i) {
        int m = i < 0 ? -1 - i : (i > n - 1 ? 2 * n - 1 - i : i);
        return min(max(m, 0), n - 1);
    };
    auto val = [&](int i, int j) {
        double v = get((long long)mirror(j) * n + mirror(i));
        if (walls) {
            if (i < 0 || i > n - 1) v = -v;
            if (j < 0) v = -v;
            if (j > n - 1) v = 2.0 * top - v;
        }
        return v;
    };
    auto weights = [](double t, double* w) {
        const double t2 = t * t, t3 = t2 * t;
        w[0] = 0.5 * (-t3 + 2.0 * t2 - t);
        w[1] = 0.5 * (3.0 * t3 - 5.0 * t2 + 2.0);
        w[2] = 0.5 * (-3.0 * t3 + 4.0 * t2 + t);
        w[3] = 0.5 * (t3 - t2);
    };
    double wx[4], wy[4];
    weights(fx, wx);
    weights(fy, wy);
    double out = 0.0;
#pragma unroll
    for (int a = 0; a < 4; a++) {
        double row = 0.0;
#pragma unroll
        for (int c = 0; c < 4; c++) row += wx[c] * val(i0 - 1 + c, j0 - 1 + a);
        out += wy[a] * row;
    }
    return out;
}

__global__ void FieldsToGridKernel(const double* __restrict__ rho,
                                   const double* __restrict__ u,
                                   const double* __restrict__ v,
                                   const CavMeta* __restrict__ meta, int ncav,
                                   float* __restrict__ grid) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ncav * kGrid * kGrid) return;
    const int k = (int)(t / (kGrid * kGrid));
    const int r = (int)(t - (long long)k * kGrid * kGrid);
    const int gy = r / kGrid, gx = r % kGrid;
    const CavMeta m = meta[k];
    const double xs = (gx + 0.5) / kGrid * m.n - 0.5;
    const double ys = (gy + 0.5) / kGrid * m.n - 0.5;
    const double* fr = rho + m.off;
    const double* fu = u + m.off;
    const double* fv = v + m.off;
    grid[t * 3] = (float)((SampleCavity([&](long long q) { return fr[q]; },
                                        m.n, xs, ys, false, 0.0) - 1.0) /
                          m.rho_scale);
    grid[t * 3 + 1] = (float)(SampleCavity([&](long long q) { return fu[q]; },
                                           m.n, xs, ys, true, m.u_scale) /
                              m.u_scale);
    grid[t * 3 + 2] = (float)(SampleCavity([&](long long q) { return fv[q]; },
                                           m.n, xs, ys, true, 0.0) /
                              m.u_scale);
}

// One thread per cavity node; cavity found by binary search of offsets.
// The grid holds normalised fields: the lid's u is 1 there.
__global__ void GridToFieldsKernel(const float* __restrict__ grid,
                                   const CavMeta* __restrict__ meta, int ncav,
                                   long long total, double* __restrict__ rho,
                                   double* __restrict__ u,
                                   double* __restrict__ v) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    int lo = 0, hi = ncav - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (meta[mid].off <= t) lo = mid;
        else hi = mid - 1;
    }
    const CavMeta m = meta[lo];
    const int r = (int)(t - m.off);
    const int y = r / m.n, x = r % m.n;
    const double xs = (x + 0.5) / m.n * kGrid - 0.5;
    const double ys = (y + 0.5) / m.n * kGrid - 0.5;
    const float* g = grid + (long long)lo * kGrid * kGrid * 3;
    rho[t] = 1.0 + m.rho_scale *
                       SampleCavity([&](long long q) { return (double)g[q * 3]; },
                                    kGrid, xs, ys, false, 0.0);
    u[t] = m.u_scale *
           SampleCavity([&](long long q) { return (double)g[q * 3 + 1]; }, kGrid,
                        xs, ys, true, 1.0);
    v[t] = m.u_scale *
           SampleCavity([&](long long q) { return (double)g[q * 3 + 2]; }, kGrid,
                        xs, ys, true, 0.0);
}

unsigned Blocks(long long n) { return (unsigned)((n + kEw - 1) / kEw); }

}  // namespace
}  // namespace nn
}  // namespace mplb

using namespace mplb::nn;

struct mplbnn_net {
    int batch = 0;
    cudaStream_t stream = nullptr;
    int* err_dev = nullptr;
    int sm_count = 148;
    std::string error;
    long long w_off[kNumLayers], b_off[kNumLayers], np = 0;
    float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
    bf16 *wf = nullptr, *wd = nullptr;
    long long step = 0;
    double* loss_dev = nullptr;
    std::vector<void*> allocs;
    // activations
    bf16 *xin, *e0a, *cat0, *p0, *e1a, *cat1, *p1, *e2a, *cat2, *p2, *ba, *bb,
        *d2a, *d2, *d1a, *d1, *d0a, *d0;
    float* pred;
    // gradients of activations
    bf16 *dpred, *g_d0, *g_d0a, *g_cat0, *g_d1, *g_d1a, *g_cat1, *g_d2, *g_d2a,
        *g_cat2, *g_bb, *g_ba, *g_p2, *g_e2, *g_e2a, *g_p1, *g_e1, *g_e1a,
        *g_p0, *g_e0, *g_e0a;
    float *cond_buf = nullptr, *target_buf = nullptr;   // gathered samples
    CavMeta* meta = nullptr;
    int meta_cap = 0;
};

namespace {

thread_local std::string g_prim_error;

int Fail(mplbnn_net* net, int code, const std::string& msg) {
    if (net) net->error = msg;
    return code;
}

#define NCK(call)                                                           \
    do {                                                                    \
        cudaError_t e_ = (call);                                            \
        if (e_ != cudaSuccess)                                              \
            return Fail(net, kCuda, std::string(#call) + ": " +             \
                                        cudaGetErrorString(e_));            \
    } while (0)

template <typename T>
int Alloc(mplbnn_net* net, T** p, long long count) {
    void* q = nullptr;
    NCK(cudaMalloc(&q, (size_t)count * sizeof(T)));
    NCK(cudaMemsetAsync(q, 0, (size_t)count * sizeof(T), net->stream));
    net->allocs.push_back(q);
    *p = static_cast<T*>(q);
    return kOK;
}

View V(void* p, int n, int s, int c, long long ps = 0) {
    return View{p, n, s, s, c, ps ? ps : c};
}

int Sync(mplbnn_net* net) {
    NCK(cudaStreamSynchronize(net->stream));
    int err = 0;
    NCK(cudaMemcpy(&err, net->err_dev, sizeof(int), cudaMemcpyDeviceToHost));
    if (err != 0)
        return Fail(net, kTimeout,
                    "a tensor-core kernel gave up waiting on a barrier");
    return kOK;
}

// Convolution of layer l (forward), or its data gradient.
int Conv(mplbnn_net* net, int l, const View& x, const View& y, bool y_f32) {
    const LayerSpec& s = kLayers[l];
    std::string err;
    if (!LaunchConv(x, net->wf + net->w_off[l], s.taps,
                    net->params + net->b_off[l], s.relu, y, y_f32, nullptr,
                    net->stream, net->err_dev, err))
        return Fail(net, kInvalid, "layer " + std::to_string(l) + ": " + err);
    return kOK;
}

int Dgrad(mplbnn_net* net, int l, const View& dz, const View& dx,
          const View* mask) {
    const LayerSpec& s = kLayers[l];
    std::string err;
    if (!LaunchConv(dz, net->wd + net->w_off[l], s.taps, nullptr, 0, dx, false,
                    mask, net->stream, net->err_dev, err))
        return Fail(net, kInvalid,
                    "data gradient of layer " + std::to_string(l) + ": " + err);
    return kOK;
}

int Wgrad(mplbnn_net* net, int l, const View& dz, const View& x) {
    const LayerSpec& s = kLayers[l];
    std::string err;
    if (!LaunchWgrad(dz, x, s.taps, net->grads + net->w_off[l], net->sm_count,
                     net->stream, net->err_dev, err))
        return Fail(net, kInvalid, "weight gradient of layer " +
                                       std::to_string(l) + ": " + err);
    const long long npix = (long long)dz.nimg * dz.h * dz.w;
    const int c = dz.c;
    int blocks = (int)((npix + 63) / 64);
    if (blocks > 4 * net->sm_count) blocks = 4 * net->sm_count;
    BiasGradKernel<<<blocks, kEw, 0, net->stream>>>(
        static_cast<const bf16*>(dz.ptr), dz.ps, npix, c,
        net->grads + net->b_off[l]);
    NCK(cudaGetLastError());
    return kOK;
}

int RefreshWeights(mplbnn_net* net) {
    ToBf16Kernel<<<Blocks(net->np), kEw, 0, net->stream>>>(net->params,
                                                           net->wf, net->np);
    NCK(cudaGetLastError());
    for (int l = 0; l < kNumLayers; l++) {
        const LayerSpec& s = kLayers[l];
        const long long n = (long long)s.cout * s.taps * s.cin;
        FlipKernel<<<Blocks(n), kEw, 0, net->stream>>>(
            net->params + net->w_off[l], net->wd + net->w_off[l], s.cout,
            s.taps, s.cin);
        NCK(cudaGetLastError());
    }
    return kOK;
}

#define RET(x)                     \
    do {                           \
        int r_ = (x);              \
        if (r_ != kOK) return r_;  \
    } while (0)

int Forward(mplbnn_net* net, const float* cond, int n) {
    const int S0 = 128, S1 = 64, S2 = 32, S3 = 16;
    cudaStream_t st = net->stream;
    InputKernel<<<Blocks((long long)n * S0 * S0), kEw, 0, st>>>(cond, n,
                                                                 net->xin);
    NCK(cudaGetLastError());
    // encoder
    RET(Conv(net, 0, V(net->xin, n, S0, 32), V(net->e0a, n, S0, 32), false));
    RET(Conv(net, 1, V(net->e0a, n, S0, 32), V(net->cat0 + 64, n, S0, 32, 96),
             false));
    PoolKernel<<<Blocks((long long)n * S1 * S1 * 4), kEw, 0, st>>>(
        net->cat0 + 64, 96, net->p0, 32, n, S1, S1, 32);
    RET(Conv(net, 2, V(net->p0, n, S1, 32), V(net->e1a, n, S1, 64), false));
    RET(Conv(net, 3, V(net->e1a, n, S1, 64),
             V(net->cat1 + 128, n, S1, 64, 192), false));
    PoolKernel<<<Blocks((long long)n * S2 * S2 * 8), kEw, 0, st>>>(
        net->cat1 + 128, 192, net->p1, 64, n, S2, S2, 64);
    RET(Conv(net, 4, V(net->p1, n, S2, 64), V(net->e2a, n, S2, 128), false));
    RET(Conv(net, 5, V(net->e2a, n, S2, 128),
             V(net->cat2 + 256, n, S2, 128, 384), false));
    PoolKernel<<<Blocks((long long)n * S3 * S3 * 16), kEw, 0, st>>>(
        net->cat2 + 256, 384, net->p2, 128, n, S3, S3, 128);
    // bottleneck
    RET(Conv(net, 6, V(net->p2, n, S3, 128), V(net->ba, n, S3, 256), false));
    RET(Conv(net, 7, V(net->ba, n, S3, 256), V(net->bb, n, S3, 256), false));
    // decoder
    UpsampleKernel<<<Blocks((long long)n * S2 * S2 * 32), kEw, 0, st>>>(
        net->bb, 256, net->cat2, 384, n, S3, S3, 256);
    RET(Conv(net, 8, V(net->cat2, n, S2, 384), V(net->d2a, n, S2, 128), false));
    RET(Conv(net, 9, V(net->d2a, n, S2, 128), V(net->d2, n, S2, 128), false));
    UpsampleKernel<<<Blocks((long long)n * S1 * S1 * 16), kEw, 0, st>>>(
        net->d2, 128, net->cat1, 192, n, S2, S2, 128);
    RET(Conv(net, 10, V(net->cat1, n, S1, 192), V(net->d1a, n, S1, 64), false));
    RET(Conv(net, 11, V(net->d1a, n, S1, 64), V(net->d1, n, S1, 64), false));
    UpsampleKernel<<<Blocks((long long)n * S0 * S0 * 8), kEw, 0, st>>>(
        net->d1, 64, net->cat0, 96, n, S1, S1, 64);
    RET(Conv(net, 12, V(net->cat0, n, S0, 96), V(net->d0a, n, S0, 32), false));
    RET(Conv(net, 13, V(net->d0a, n, S0, 32), V(net->d0, n, S0, 32), false));
    RET(Conv(net, 14, V(net->d0, n, S0, 32), V(net->pred, n, S0, kOutCh),
             true));
    NCK(cudaGetLastError());
    return kOK;
}

int Backward(mplbnn_net* net, const float* target, int n) {
    const int S0 = 128, S1 = 64, S2 = 32, S3 = 16;
    cudaStream_t st = net->stream;
    const long long npix = (long long)n * S0 * S0;
    NCK(cudaMemsetAsync(net->grads, 0, net->np * sizeof(float), st));
    NCK(cudaMemsetAsync(net->loss_dev, 0, sizeof(double), st));
    LossKernel<<<Blocks(npix), kEw, 0, st>>>(
        net->pred, target, npix, (float)(2.0 / (3.0 * (double)npix)),
        net->dpred, net->loss_dev);
    NCK(cudaGetLastError());
    // decoder, level 0
    const View dpred = V(net->dpred, n, S0, kOutCh);
    RET(Wgrad(net, 14, dpred, V(net->d0, n, S0, 32)));
    View mk = V(net->d0, n, S0, 32);
    RET(Dgrad(net, 14, dpred, V(net->g_d0, n, S0, 32), &mk));
    RET(Wgrad(net, 13, V(net->g_d0, n, S0, 32), V(net->d0a, n, S0, 32)));
    mk = V(net->d0a, n, S0, 32);
    RET(Dgrad(net, 13, V(net->g_d0, n, S0, 32), V(net->g_d0a, n, S0, 32), &mk));
    RET(Wgrad(net, 12, V(net->g_d0a, n, S0, 32), V(net->cat0, n, S0, 96)));
    RET(Dgrad(net, 12, V(net->g_d0a, n, S0, 32), V(net->g_cat0, n, S0, 96),
              nullptr));
    UpBwdKernel<<<Blocks((long long)n * S1 * S1 * 8), kEw, 0, st>>>(
        net->g_cat0, 96, net->d1, 64, net->g_d1, 64, n, S1, S1, 64);
    // level 1
    RET(Wgrad(net, 11, V(net->g_d1, n, S1, 64), V(net->d1a, n, S1, 64)));
    mk = V(net->d1a, n, S1, 64);
    RET(Dgrad(net, 11, V(net->g_d1, n, S1, 64), V(net->g_d1a, n, S1, 64), &mk));
    RET(Wgrad(net, 10, V(net->g_d1a, n, S1, 64), V(net->cat1, n, S1, 192)));
    RET(Dgrad(net, 10, V(net->g_d1a, n, S1, 64), V(net->g_cat1, n, S1, 192),
              nullptr));
    UpBwdKernel<<<Blocks((long long)n * S2 * S2 * 16), kEw, 0, st>>>(
        net->g_cat1, 192, net->d2, 128, net->g_d2, 128, n, S2, S2, 128);
    // level 2
    RET(Wgrad(net, 9, V(net->g_d2, n, S2, 128), V(net->d2a, n, S2, 128)));
    mk = V(net->d2a, n, S2, 128);
    RET(Dgrad(net, 9, V(net->g_d2, n, S2, 128), V(net->g_d2a, n, S2, 128),
              &mk));
    RET(Wgrad(net, 8, V(net->g_d2a, n, S2, 128), V(net->cat2, n, S2, 384)));
    RET(Dgrad(net, 8, V(net->g_d2a, n, S2, 128), V(net->g_cat2, n, S2, 384),
              nullptr));
    UpBwdKernel<<<Blocks((long long)n * S3 * S3 * 32), kEw, 0, st>>>(
        net->g_cat2, 384, net->bb, 256, net->g_bb, 256, n, S3, S3, 256);
    // bottleneck
    RET(Wgrad(net, 7, V(net->g_bb, n, S3, 256), V(net->ba, n, S3, 256)));
    mk = V(net->ba, n, S3, 256);
    RET(Dgrad(net, 7, V(net->g_bb, n, S3, 256), V(net->g_ba, n, S3, 256),
              &mk));
    RET(Wgrad(net, 6, V(net->g_ba, n, S3, 256), V(net->p2, n, S3, 128)));
    RET(Dgrad(net, 6, V(net->g_ba, n, S3, 256), V(net->g_p2, n, S3, 128),
              nullptr));
    // encoder, level 2
    SkipBwdKernel<<<Blocks((long long)n * S2 * S2 * 16), kEw, 0, st>>>(
        net->g_cat2 + 256, 384, net->g_p2, 128, net->cat2 + 256, 384,
        net->g_e2, 128, n, S2, S2, 128);
    RET(Wgrad(net, 5, V(net->g_e2, n, S2, 128), V(net->e2a, n, S2, 128)));
    mk = V(net->e2a, n, S2, 128);
    RET(Dgrad(net, 5, V(net->g_e2, n, S2, 128), V(net->g_e2a, n, S2, 128),
              &mk));
    RET(Wgrad(net, 4, V(net->g_e2a, n, S2, 128), V(net->p1, n, S2, 64)));
    RET(Dgrad(net, 4, V(net->g_e2a, n, S2, 128), V(net->g_p1, n, S2, 64),
              nullptr));
    // level 1
    SkipBwdKernel<<<Blocks((long long)n * S1 * S1 * 8), kEw, 0, st>>>(
        net->g_cat1 + 128, 192, net->g_p1, 64, net->cat1 + 128, 192, net->g_e1,
        64, n, S1, S1, 64);
    RET(Wgrad(net, 3, V(net->g_e1, n, S1, 64), V(net->e1a, n, S1, 64)));
    mk = V(net->e1a, n, S1, 64);
    RET(Dgrad(net, 3, V(net->g_e1, n, S1, 64), V(net->g_e1a, n, S1, 64), &mk));
    RET(Wgrad(net, 2, V(net->g_e1a, n, S1, 64), V(net->p0, n, S1, 32)));
    RET(Dgrad(net, 2, V(net->g_e1a, n, S1, 64), V(net->g_p0, n, S1, 32),
              nullptr));
    // level 0
    SkipBwdKernel<<<Blocks((long long)n * S0 * S0 * 4), kEw, 0, st>>>(
        net->g_cat0 + 64, 96, net->g_p0, 32, net->cat0 + 64, 96, net->g_e0, 32,
        n, S0, S0, 32);
    RET(Wgrad(net, 1, V(net->g_e0, n, S0, 32), V(net->e0a, n, S0, 32)));
    mk = V(net->e0a, n, S0, 32);
    RET(Dgrad(net, 1, V(net->g_e0, n, S0, 32), V(net->g_e0a, n, S0, 32), &mk));
    RET(Wgrad(net, 0, V(net->g_e0a, n, S0, 32), V(net->xin, n, S0, 32)));
    NCK(cudaGetLastError());
    (void)S3;
    return kOK;
}

int CheckN(mplbnn_net* net, int n) {
    if (net == nullptr) return kInvalid;
    if (n < 1 || n > net->batch)
        return Fail(net, kInvalid,
                    "n must be in [1, batch=" + std::to_string(net->batch) +
                        "]");
    return kOK;
}

int UploadMeta(mplbnn_net* net, int ncav, const int* n,
               const long long* offset, const double* rho_scale,
               const double* u_scale) {
    if (ncav < 1 || !n || !offset || !rho_scale || !u_scale)
        return Fail(net, kInvalid, "cavity metadata missing");
    std::vector<CavMeta> h(ncav);
    for (int k = 0; k < ncav; k++) {
        if (n[k] < 2 || rho_scale[k] == 0.0 || u_scale[k] == 0.0)
            return Fail(net, kInvalid, "invalid cavity metadata");
        if (k > 0 && offset[k] != offset[k - 1] + (long long)n[k - 1] * n[k - 1])
            return Fail(net, kInvalid, "cavity offsets are not packed");
        h[k] = CavMeta{n[k], offset[k], rho_scale[k], u_scale[k]};
    }
    if (ncav > net->meta_cap) {
        if (net->meta) cudaFree(net->meta);
        net->meta = nullptr;
        NCK(cudaMalloc(&net->meta, ncav * sizeof(CavMeta)));
        net->meta_cap = ncav;
    }
    NCK(cudaMemcpyAsync(net->meta, h.data(), ncav * sizeof(CavMeta),
                        cudaMemcpyHostToDevice, net->stream));
    NCK(cudaStreamSynchronize(net->stream));
    return kOK;
}

int* PrimErrWord() {
    static int* w = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        if (cudaMalloc(&w, sizeof(int)) != cudaSuccess) w = nullptr;
    });
    return w;
}

View FromAbi(const mplbnn_view* v) {
    return View{v->ptr, v->nimg, v->h, v->w, v->c, v->ps};
}

int PrimFinish(cudaStream_t s, int* errw) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        g_prim_error = cudaGetErrorString(e);
        return kCuda;
    }
    int err = 0;
    cudaMemcpy(&err, errw, sizeof(int), cudaMemcpyDeviceToHost);
    if (err) {
        g_prim_error = "a tensor-core kernel gave up waiting on a barrier";
        cudaMemset(errw, 0, sizeof(int));
        return kTimeout;
    }
    return kOK;
}

}  // namespace

extern "C" {

const char* mplbnn_error(void) { return g_prim_error.c_str(); }

int mplbnn_conv_forward(const mplbnn_view* x, const void* w, int taps,
                        const float* bias, int relu, const mplbnn_view* y,
                        int y_f32, const mplbnn_view* mask, void* stream) {
    if (!x || !y) {
        g_prim_error = "null view";
        return kInvalid;
    }
    int* errw = PrimErrWord();
    if (!errw) {
        g_prim_error = "no device";
        return kCuda;
    }
    const View mv = mask ? FromAbi(mask) : View{};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!LaunchConv(FromAbi(x), w, taps, bias, relu, FromAbi(y), y_f32 != 0,
                    mask ? &mv : nullptr, s, errw, g_prim_error))
        return kInvalid;
    return PrimFinish(s, errw);
}

int mplbnn_conv_wgrad(const mplbnn_view* dy, const mplbnn_view* x, int taps,
                      float* dw, void* stream) {
    if (!dy || !x) {
        g_prim_error = "null view";
        return kInvalid;
    }
    int* errw = PrimErrWord();
    if (!errw) {
        g_prim_error = "no device";
        return kCuda;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!LaunchWgrad(FromAbi(dy), FromAbi(x), taps, dw, sms, s, errw,
                     g_prim_error))
        return kInvalid;
    return PrimFinish(s, errw);
}

int mplbnn_layer_count(void) { return kNumLayers; }

int mplbnn_layer_info(int layer, int* cin, int* cout, int* taps,
                      long long* w_offset, long long* b_offset) {
    if (layer < 0 || layer >= kNumLayers) return kInvalid;
    long long wo[kNumLayers], bo[kNumLayers], tot;
    LayerOffsets(wo, bo, &tot);
    if (cin) *cin = kLayers[layer].cin;
    if (cout) *cout = kLayers[layer].cout;
    if (taps) *taps = kLayers[layer].taps;
    if (w_offset) *w_offset = wo[layer];
    if (b_offset) *b_offset = bo[layer];
    return kOK;
}

int mplbnn_create(int batch, mplbnn_net** out) {
    if (!out || batch < 1) return kInvalid;
    *out = nullptr;
    mplbnn_net* net = new mplbnn_net();
    net->batch = batch;
    auto fail = [&](int rc) {
        g_prim_error = net->error;
        mplbnn_destroy(net);
        return rc;
    };
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking) !=
            cudaSuccess) {
        net->error = "no CUDA device";
        return fail(kCuda);
    }
    cudaDeviceGetAttribute(&net->sm_count, cudaDevAttrMultiProcessorCount, dev);
    LayerOffsets(net->w_off, net->b_off, &net->np);
    const long long B = batch;
    const long long P0 = B * 128 * 128, P1 = B * 64 * 64, P2 = B * 32 * 32,
                    P3 = B * 16 * 16;
    int rc = kOK;
#define A(ptr, count)                                   \
    if (rc == kOK) rc = Alloc(net, &net->ptr, (count));
    A(err_dev, 1);
    A(loss_dev, 1);
    A(params, net->np);
    A(grads, net->np);
    A(m, net->np);
    A(v, net->np);
    A(wf, net->np);
    A(wd, net->np);
    A(xin, P0 * 32);
    A(e0a, P0 * 32);
    A(cat0, P0 * 96);
    A(p0, P1 * 32);
    A(e1a, P1 * 64);
    A(cat1, P1 * 192);
    A(p1, P2 * 64);
    A(e2a, P2 * 128);
    A(cat2, P2 * 384);
    A(p2, P3 * 128);
    A(ba, P3 * 256);
    A(bb, P3 * 256);
    A(d2a, P2 * 128);
    A(d2, P2 * 128);
    A(d1a, P1 * 64);
    A(d1, P1 * 64);
    A(d0a, P0 * 32);
    A(d0, P0 * 32);
    A(pred, P0 * kOutCh);
    A(dpred, P0 * kOutCh);
    A(g_d0, P0 * 32);
    A(g_d0a, P0 * 32);
    A(g_cat0, P0 * 96);
    A(g_d1, P1 * 64);
    A(g_d1a, P1 * 64);
    A(g_cat1, P1 * 192);
    A(g_d2, P2 * 128);
    A(g_d2a, P2 * 128);
    A(g_cat2, P2 * 384);
    A(g_bb, P3 * 256);
    A(g_ba, P3 * 256);
    A(g_p2, P3 * 128);
    A(g_e2, P2 * 128);
    A(g_e2a, P2 * 128);
    A(g_p1, P2 * 64);
    A(g_e1, P1 * 64);
    A(g_e1a, P1 * 64);
    A(g_p0, P1 * 32);
    A(g_e0, P0 * 32);
    A(g_e0a, P0 * 32);
    A(cond_buf, B * 3);
    A(target_buf, P0 * 3);
#undef A
    if (rc != kOK) return fail(rc);
    if (cudaStreamSynchronize(net->stream) != cudaSuccess) {
        net->error = "initialisation failed";
        return fail(kCuda);
    }
    *out = net;
    return kOK;
}

int mplbnn_destroy(mplbnn_net* net) {
    if (!net) return kOK;
    if (net->stream) cudaStreamSynchronize(net->stream);
    for (void* p : net->allocs) cudaFree(p);
    if (net->meta) cudaFree(net->meta);
    if (net->stream) cudaStreamDestroy(net->stream);
    delete net;
    return kOK;
}

const char* mplbnn_last_error(const mplbnn_net* net) {
    return net ? net->error.c_str() : g_prim_error.c_str();
}

int mplbnn_synchronize(mplbnn_net* net) {
    if (!net) return kInvalid;
    return Sync(net);
}

long long mplbnn_param_count(const mplbnn_net* net) {
    return net ? net->np : 0;
}

int mplbnn_init_params(mplbnn_net* net, unsigned long long seed) {
    if (!net) return kInvalid;
    std::vector<float> h(net->np, 0.0f);
    std::mt19937_64 gen(seed);
    for (int l = 0; l < kNumLayers; l++) {
        const LayerSpec& s = kLayers[l];
        const double fan_in = (double)s.taps * s.cin;
        const double sd = s.relu ? std::sqrt(2.0 / fan_in)
                                 : 0.1 * std::sqrt(1.0 / fan_in);
        std::normal_distribution<double> nd(0.0, sd);
        const long long nw = (long long)s.cout * s.taps * s.cin;
        for (long long i = 0; i < nw; i++)
            h[net->w_off[l] + i] = (float)nd(gen);
    }
    return mplbnn_set_params(net, h.data());
}

int mplbnn_set_params(mplbnn_net* net, const float* params) {
    if (!net || !params) return kInvalid;
    NCK(cudaMemcpyAsync(net->params, params, net->np * sizeof(float),
                        cudaMemcpyHostToDevice, net->stream));
    NCK(cudaMemsetAsync(net->m, 0, net->np * sizeof(float), net->stream));
    NCK(cudaMemsetAsync(net->v, 0, net->np * sizeof(float), net->stream));
    net->step = 0;
    RET(RefreshWeights(net));
    return Sync(net);
}

int mplbnn_get_params(mplbnn_net* net, float* params) {
    if (!net || !params) return kInvalid;
    RET(Sync(net));
    NCK(cudaMemcpy(params, net->params, net->np * sizeof(float),
                   cudaMemcpyDeviceToHost));
    return kOK;
}

int mplbnn_get_grads(mplbnn_net* net, float* grads) {
    if (!net || !grads) return kInvalid;
    RET(Sync(net));
    NCK(cudaMemcpy(grads, net->grads, net->np * sizeof(float),
                   cudaMemcpyDeviceToHost));
    return kOK;
}

int mplbnn_forward(mplbnn_net* net, const float* cond, int n, float* pred) {
    RET(CheckN(net, n));
    if (!cond || !pred) return Fail(net, kInvalid, "null pointer");
    RET(Forward(net, cond, n));
    const long long npix = (long long)n * kGrid * kGrid;
    CompactKernel<<<Blocks(npix), kEw, 0, net->stream>>>(net->pred, npix, pred);
    NCK(cudaGetLastError());
    return Sync(net);
}

int mplbnn_loss_grad(mplbnn_net* net, const float* cond, const float* target,
                     const int* index, int n, double* loss) {
    RET(CheckN(net, n));
    if (!cond || !target) return Fail(net, kInvalid, "null pointer");
    if (index != nullptr) {
        const size_t per = (size_t)kGrid * kGrid * 3;
        for (int i = 0; i < n; i++) {
            if (index[i] < 0) return Fail(net, kInvalid, "negative index");
            NCK(cudaMemcpyAsync(net->cond_buf + 3 * i, cond + 3LL * index[i],
                                3 * sizeof(float), cudaMemcpyDeviceToDevice,
                                net->stream));
            NCK(cudaMemcpyAsync(net->target_buf + per * i,
                                target + per * index[i], per * sizeof(float),
                                cudaMemcpyDeviceToDevice, net->stream));
        }
        cond = net->cond_buf;
        target = net->target_buf;
    }
    RET(Forward(net, cond, n));
    RET(Backward(net, target, n));
    if (loss) {
        RET(Sync(net));
        double s = 0.0;
        NCK(cudaMemcpy(&s, net->loss_dev, sizeof(double),
                       cudaMemcpyDeviceToHost));
        *loss = s / (3.0 * (double)n * kGrid * kGrid);
    }
    return kOK;
}

int mplbnn_adam_step(mplbnn_net* net, float lr, float beta1, float beta2,
                     float eps) {
    if (!net) return kInvalid;
    net->step++;
    const double bc1 = 1.0 - std::pow((double)beta1, (double)net->step);
    const double bc2 = 1.0 - std::pow((double)beta2, (double)net->step);
    const float lr_t = (float)(lr * std::sqrt(bc2) / bc1);
    AdamKernel<<<Blocks(net->np), kEw, 0, net->stream>>>(
        net->params, net->grads, net->m, net->v, net->wf, net->np, lr_t, beta1,
        beta2, eps);
    NCK(cudaGetLastError());
    for (int l = 0; l < kNumLayers; l++) {
        const LayerSpec& s = kLayers[l];
        const long long nw = (long long)s.cout * s.taps * s.cin;
        FlipKernel<<<Blocks(nw), kEw, 0, net->stream>>>(
            net->params + net->w_off[l], net->wd + net->w_off[l], s.cout,
            s.taps, s.cin);
        NCK(cudaGetLastError());
    }
    return kOK;
}

int mplbnn_fields_to_grid(mplbnn_net* net, const double* rho, const double* u,
                          const double* v, int ncav, const int* n,
                          const long long* offset, const double* rho_scale,
                          const double* u_scale, float* grid) {
    if (!net || !rho || !u || !v || !grid)
        return Fail(net, kInvalid, "null pointer");
    RET(UploadMeta(net, ncav, n, offset, rho_scale, u_scale));
    const long long total = (long long)ncav * kGrid * kGrid;
    FieldsToGridKernel<<<Blocks(total), kEw, 0, net->stream>>>(
        rho, u, v, net->meta, ncav, grid);
    NCK(cudaGetLastError());
    return Sync(net);
}

int mplbnn_grid_to_fields(mplbnn_net* net, const float* grid, int ncav,
                          const int* n, const long long* offset,
                          const double* rho_scale, const double* u_scale,
                          double* rho, double* u, double* v) {
    if (!net || !rho || !u || !v || !grid)
        return Fail(net, kInvalid, "null pointer");
    RET(UploadMeta(net, ncav, n, offset, rho_scale, u_scale));
    const long long total =
        offset[ncav - 1] + (long long)n[ncav - 1] * n[ncav - 1];
    GridToFieldsKernel<<<Blocks(total), kEw, 0, net->stream>>>(
        grid, net->meta, ncav, total, rho, u, v);
    NCK(cudaGetLastError());
    return Sync(net);
}

}  // extern "C"
