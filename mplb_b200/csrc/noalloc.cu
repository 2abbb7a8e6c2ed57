// Residual sums without any device allocation.
//
// mplbgpu_residual_sums_noalloc is the allocation-free variant of the
// residual reduction behind mplbgpu_residual: the caller owns every input
// and output buffer, and the per-CTA partial sums live in the file-scope
// device array below instead of in memory obtained from cudaMalloc.  It
// exists for callers that cannot call cudaMalloc at the point where they
// need the reduction: applications that hand all device memory to their own
// pool at start-up (a framework's caching allocator, a host program with a
// fixed device-memory budget) and loops that cannot afford the device-wide
// synchronisation that allocating and freeing imply.
//
// The array is 2 x 4 x 8192 doubles (512 KiB) and every GPU that loads the
// library holds it until the process exits.  It bounds a call to 4
// variables of at most MPLBGPU_NOALLOC_MAX_NODES = 8192 x 2048 nodes.
// Every call shares the array and it keeps the last call's partials; calls
// that overlap on the GPU (different streams, or host threads) race on it.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/mplbgpu.h"

namespace {

constexpr int kVars = 4;
constexpr int kThreads = 256;
constexpr int kNodesPerThread = 8;
constexpr long long kNodesPerCta = (long long)kThreads * kNodesPerThread;
constexpr int kMaxCtas = 8192;
static_assert(kMaxCtas * kNodesPerCta == MPLBGPU_NOALLOC_MAX_NODES,
              "scratch size and the published node limit disagree");

// [variable][cta][0: sum (q - q_old)^2, 1: sum q^2]
static __device__ __align__(256) double g_noalloc_partials[kVars][kMaxCtas][2];

// Address cache, one entry per CUDA context.  Each context loads the
// library's device code separately, so the array has one address per
// context: a device's primary context after cudaDeviceReset, or a context
// a caller made with the driver API, gets its own entry.  Contexts are told
// apart by cuCtxGetId (unique for the life of the process, where a
// CUcontext handle may be reused), reached through the runtime's driver
// entry point so that the library does not link libcuda itself.
constexpr int kMaxContexts = 64;
struct ScratchEntry {
    unsigned long long ctx_id;
    double* addr;
};
std::mutex g_mu;
ScratchEntry g_scratch[kMaxContexts];
int g_nscratch = 0;

using CtxGetCurrentFn = CUresult(CUDAAPI*)(CUcontext*);
using CtxGetIdFn = CUresult(CUDAAPI*)(CUcontext, unsigned long long*);

// Id of the context current on this thread; false if there is none or the
// driver does not offer the query.
bool CurrentContextId(unsigned long long* id) {
    static CtxGetCurrentFn get_current = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000,
                                             cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    static CtxGetIdFn get_id = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000,
                                             cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetIdFn>(f);
    }();
    if (get_current == nullptr || get_id == nullptr) return false;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

// Address of the scratch array in the current context, looked up once per
// context (in practice once per device).  In host code the symbol is only
// a stand-in for the device variable, so kernels must be given this
// address, not the symbol.
cudaError_t ScratchAddress(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    unsigned long long id = 0;
    if (!CurrentContextId(&id)) {
        // no context bound to this thread yet: the lookup binds the
        // device's primary context, after which the id can be read
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess) return e;
        if (!CurrentContextId(&id)) {   // no id to key on: do not cache
            *out = static_cast<double*>(p);
            return cudaSuccess;
        }
    }
    std::lock_guard<std::mutex> lock(g_mu);
    for (int k = 0; k < g_nscratch; k++) {
        if (g_scratch[k].ctx_id == id) {
            *out = g_scratch[k].addr;
            return cudaSuccess;
        }
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess) return e;
    if (g_nscratch < kMaxContexts)
        g_scratch[g_nscratch++] = {id, static_cast<double*>(p)};
    *out = static_cast<double*>(p);
    return cudaSuccess;
}

struct VarPtrs {
    const double* q[kVars];
    double* qold[kVars];
};

// One CTA sums kNodesPerCta nodes of every variable into its slot of the
// scratch (same arithmetic as ResidualPartialKernel) and copies q to q_old.
__global__ void __launch_bounds__(kThreads)
    NoAllocPartialKernel(VarPtrs v, int nvars, long long n, double* scratch) {
    __shared__ double sd[kThreads];
    __shared__ double ss[kThreads];
    const long long base = blockIdx.x * kNodesPerCta;
    for (int m = 0; m < nvars; m++) {
        double d = 0.0, s = 0.0;
        for (int k = 0; k < kNodesPerThread; k++) {
            const long long t = base + (long long)k * kThreads + threadIdx.x;
            if (t < n) {
                const double q = v.q[m][t];
                const double dq = q - v.qold[m][t];
                d = d + dq * dq;
                s = s + q * q;
                v.qold[m][t] = q;
            }
        }
        sd[threadIdx.x] = d;
        ss[threadIdx.x] = s;
        __syncthreads();
        for (int w = kThreads / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) {
                sd[threadIdx.x] = sd[threadIdx.x] + sd[threadIdx.x + w];
                ss[threadIdx.x] = ss[threadIdx.x] + ss[threadIdx.x + w];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            double* slot = scratch + ((size_t)m * kMaxCtas + blockIdx.x) * 2;
            slot[0] = sd[0];
            slot[1] = ss[0];
        }
        __syncthreads();
    }
}

// Sums the first `nctas` partial slots of each variable in a fixed order
// into the caller's output: sums[2m] = sum (q - q_old)^2, sums[2m+1] = sum q^2.
__global__ void __launch_bounds__(kThreads)
    NoAllocFinalKernel(int nvars, int nctas, const double* scratch,
                       double* sums) {
    __shared__ double sd[kThreads];
    __shared__ double ss[kThreads];
    for (int m = 0; m < nvars; m++) {
        double d = 0.0, s = 0.0;
        for (int c = threadIdx.x; c < nctas; c += kThreads) {
            const double* slot = scratch + ((size_t)m * kMaxCtas + c) * 2;
            d = d + slot[0];
            s = s + slot[1];
        }
        sd[threadIdx.x] = d;
        ss[threadIdx.x] = s;
        __syncthreads();
        for (int w = kThreads / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) {
                sd[threadIdx.x] = sd[threadIdx.x] + sd[threadIdx.x + w];
                ss[threadIdx.x] = ss[threadIdx.x] + ss[threadIdx.x + w];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            sums[2 * m] = sd[0];
            sums[2 * m + 1] = ss[0];
        }
        __syncthreads();
    }
}

}  // namespace

extern "C" mplbgpu_status mplbgpu_residual_sums_noalloc(
    const double* const* q, double* const* q_old, int nvars, long long n,
    double* sums, void* stream) {
    if (q == nullptr || q_old == nullptr || sums == nullptr)
        return MPLBGPU_ERR_INVALID;
    if (nvars < 1 || nvars > kVars) return MPLBGPU_ERR_INVALID;
    if (n < 1 || n > MPLBGPU_NOALLOC_MAX_NODES) return MPLBGPU_ERR_INVALID;
    VarPtrs v{};
    for (int m = 0; m < nvars; m++) {
        if (q[m] == nullptr || q_old[m] == nullptr) return MPLBGPU_ERR_INVALID;
        v.q[m] = q[m];
        v.qold[m] = q_old[m];
    }
    double* scratch = nullptr;
    if (ScratchAddress(&scratch) != cudaSuccess) return MPLBGPU_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nctas = (int)((n + kNodesPerCta - 1) / kNodesPerCta);
    NoAllocPartialKernel<<<nctas, kThreads, 0, s>>>(v, nvars, n, scratch);
    if (cudaGetLastError() != cudaSuccess) return MPLBGPU_ERR_CUDA;
    NoAllocFinalKernel<<<1, kThreads, 0, s>>>(nvars, nctas, scratch, sums);
    if (cudaGetLastError() != cudaSuccess) return MPLBGPU_ERR_CUDA;
    return MPLBGPU_OK;
}
