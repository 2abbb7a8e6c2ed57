// C ABI of the B200 stream-collision path (include/mplbgpu.h).
//
// A context owns one CUDA stream (and side streams that a step forks from
// it and joins back before it returns) and, per block, two population arrays in
// the halo layout of kernels.cuh (ping-pong between steps; one array updated
// in place under the swap scheme, swap.cuh), the boundary
// tables produced by plan.cpp, the stale/deferred stores and the dense
// macroscopic fields used by the residual.  Every entry point validates its
// arguments and returns a status; CUDA errors are reported with the failing
// call in mplbgpu_last_error.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mplbgpu.h"
#include "launch.h"
#include "plan.h"

using namespace mplb;

namespace {

thread_local std::string g_create_error;

struct DevBlock {
    BlockDev dev{};
    void* pop[2] = {nullptr, nullptr};   // form T of the context
    RegionInfo* regions = nullptr;
    RegionOp* ops = nullptr;
    double* stale = nullptr;
    double* fdef = nullptr;
    int* dops_flat = nullptr;
    int4* dregions = nullptr;
    double* macro[4] = {nullptr, nullptr, nullptr, nullptr};
    double* macro_old[4] = {nullptr, nullptr, nullptr, nullptr};
    struct DOp {
        DeferredSeg* segs = nullptr;
        int nseg = 0;
        long long total = 0;
    };
    std::vector<DOp> dops;
};

struct DevHalo {          // device arrays of one copy of the halo plan
    uint8_t* prev = nullptr;
    uint8_t* ordered = nullptr;
};

}  // namespace

struct mplbgpu_ctx {
    Plan plan;
    PhysConst pc{};
    std::vector<DevBlock> blocks;
    std::vector<DevHalo> halos;
    HaloFusedDev hfd{};     // the fused transfer (copies, blocks, elements)
    unsigned halo_ctas = 0;
    int cur = 0;            // pop[cur] holds the latest g
    bool initial = true;    // pop[1 - cur] holds f^0 itself
    // swap scheme, contents of pop[0]: 0 f itself (initial or uploaded),
    // 1 the locally swapped collided state, 2 the streamed state whose
    // boundary programme is still to be applied
    int swap_state = 0;
    bool halos_pending = true;
    std::vector<bool> initialised;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // a step's independent launches (each block's step, deferred outlets)
    // on side streams forked from `stream` and joined before the halos
    static constexpr int kSides = 3;
    cudaStream_t side[kSides] = {nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[kSides] = {nullptr, nullptr, nullptr};
    int nlanes = 1;         // streams a step uses (1: no fork)
    float last_ms = 0;
    bool timing_pending = false;  // ev0/ev1 of the last step call unread
    bool begun = false;           // mplbgpu_step_begin without its finish
    long long launches = 0;
    unsigned long long step_count = 0;
    double* part = nullptr;     // reduction partials
    unsigned long long* bad = nullptr;
    double* scratch = nullptr;  // dense f staging
    size_t scratch_elems = 0;
    std::vector<RegionOp*> bc_field;  // per boundary: per-node operations
    std::string err;
};

namespace {

constexpr int kThreads = kStepThreads;
constexpr int kRedBlocks = 1024;

// Calls FN<D, T>(args...) for the context's dimension and storage form.
#define MPLB_DISPATCH(ctx, FN, ...)                                          \
    ((ctx)->plan.dim == 3                                                   \
         ? ((ctx)->plan.precision == MPLBGPU_FP64                           \
                ? FN<3, double>(__VA_ARGS__)                                \
                : (ctx)->plan.precision == MPLBGPU_FP32_SHIFTED             \
                      ? FN<3, float>(__VA_ARGS__)                           \
                      : FN<3, __half>(__VA_ARGS__))                         \
         : ((ctx)->plan.precision == MPLBGPU_FP64                           \
                ? FN<2, double>(__VA_ARGS__)                                \
                : (ctx)->plan.precision == MPLBGPU_FP32_SHIFTED             \
                      ? FN<2, float>(__VA_ARGS__)                           \
                      : FN<2, __half>(__VA_ARGS__)))
constexpr int kRedThreads = 256;

int SetErr(mplbgpu_ctx* c, int code, const std::string& m) {
    if (c) c->err = m; else g_create_error = m;
    return code;
}

#define CK(call)                                                            \
    do {                                                                    \
        cudaError_t e_ = (call);                                            \
        if (e_ != cudaSuccess)                                              \
            return SetErr(ctx, MPLBGPU_ERR_CUDA,                            \
                          std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define CK_LAUNCH_E(...)                                                    \
    do {                                                                    \
        ctx->launches++;                                                    \
        cudaError_t e_ = (__VA_ARGS__);                                     \
        if (e_ != cudaSuccess)                                              \
            return SetErr(ctx, MPLBGPU_ERR_CUDA,                            \
                          std::string("kernel launch: ") +                  \
                              cudaGetErrorString(e_));                      \
    } while (0)
#define CK_LAUNCH() CK_LAUNCH_E(cudaGetLastError())

dim3 NodeGrid(const BlockPlan& B, int dim) {
    return dim3((B.n[0] + kThreads - 1) / kThreads, B.n[1],
                dim == 3 ? B.n[2] : 1);
}

DevBlock* FindBlock(mplbgpu_ctx* ctx, int id) {
    for (size_t i = 0; i < ctx->plan.blocks.size(); i++)
        if (ctx->plan.blocks[i].id == id) return &ctx->blocks[i];
    return nullptr;
}

const BlockPlan* FindPlan(mplbgpu_ctx* ctx, int id) {
    for (const BlockPlan& B : ctx->plan.blocks)
        if (B.id == id) return &B;
    return nullptr;
}

void FreeAll(mplbgpu_ctx* c) {
    for (DevBlock& b : c->blocks) {
        cudaFree(b.pop[0]);
        cudaFree(b.pop[1]);
        cudaFree(b.regions);
        cudaFree(b.ops);
        cudaFree(b.stale);
        cudaFree(b.fdef);
        cudaFree(b.dops_flat);
        cudaFree(b.dregions);
        for (int m = 0; m < 4; m++) {
            cudaFree(b.macro[m]);
            cudaFree(b.macro_old[m]);
        }
        for (auto& d : b.dops) cudaFree(d.segs);
    }
    for (DevHalo& h : c->halos) {
        cudaFree(h.prev);
        cudaFree(h.ordered);
    }
    cudaFree(const_cast<HaloCopyDev*>(c->hfd.copies));
    cudaFree(const_cast<HaloBlockDev*>(c->hfd.blocks));
    cudaFree(const_cast<int2*>(c->hfd.ctas));
    cudaFree(const_cast<HaloElemDev*>(c->hfd.elems));
    for (RegionOp* p : c->bc_field) cudaFree(p);
    cudaFree(c->part);
    cudaFree(c->bad);
    cudaFree(c->scratch);
    for (int k = 0; k < mplbgpu_ctx::kSides; k++) {
        if (c->side[k]) cudaStreamDestroy(c->side[k]);
        if (c->join[k]) cudaEventDestroy(c->join[k]);
    }
    if (c->fork) cudaEventDestroy(c->fork);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
}

// n doubles set to v (a macroscopic field not given at initialisation).
__global__ void FillDoubleKernel(double* __restrict__ p, long long n,
                                 double v) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
         e < n; e += (long long)gridDim.x * blockDim.x)
        p[e] = v;
}

// A population array of the context's storage form set to f = 0.
cudaError_t FillZeroF(mplbgpu_ctx* c, void* p, long long popstride) {
    const int Q = c->plan.Q;
    if (c->plan.precision == MPLBGPU_FP32_SHIFTED)
        return Launch<3, float>::FillZero(c->stream, static_cast<float*>(p),
                                          popstride, Q, c->pc);
    return Launch<3, __half>::FillZero(c->stream, static_cast<__half*>(p),
                                       popstride, Q, c->pc);
}

int EnsureScratch(mplbgpu_ctx* ctx, size_t elems) {
    if (ctx->scratch_elems >= elems) return MPLBGPU_OK;
    cudaFree(ctx->scratch);
    ctx->scratch = nullptr;
    ctx->scratch_elems = 0;
    CK(cudaMalloc(&ctx->scratch, elems * sizeof(double)));
    ctx->scratch_elems = elems;
    return MPLBGPU_OK;
}

// Every halo copy of the step (Field::TransferHalos in CreateHalos order)
// in one launch.
template <int D, typename T>
int RunHalosT(mplbgpu_ctx* ctx) {
    if (!ctx->halos.empty())
        CK_LAUNCH_E(Launch<D, T>::HaloFused(ctx->stream, ctx->hfd, ctx->cur,
                                            ctx->halo_ctas));
    ctx->halos_pending = false;
    return MPLBGPU_OK;
}

int RunHalos(mplbgpu_ctx* ctx) { return MPLB_DISPATCH(ctx, RunHalosT, ctx); }

// One step of the swap scheme (single block, no halos): from f itself or
// the streamed state the node reads its own slots, from the locally swapped
// state it gathers the streamed slots.
template <int D, typename T>
int SwapStepOnce(mplbgpu_ctx* ctx) {
    ctx->pc.seed = (uint32_t)(++ctx->step_count);
    DevBlock& b = ctx->blocks[0];
    const BlockPlan& B = ctx->plan.blocks[0];
    const int st = ctx->swap_state;
    CK_LAUNCH_E(Launch<D, T>::Swap(kModeStep, st == 1, st != 0,
                                   NodeGrid(B, D), ctx->stream, b.dev, ctx->pc,
                                   static_cast<T*>(b.pop[0]), nullptr, nullptr,
                                   nullptr, nullptr));
    ctx->swap_state = st == 1 ? 2 : 1;
    ctx->initial = false;
    return MPLBGPU_OK;
}

// The launches of one step that depend on nothing else of the step - each
// block's step kernel and each block's deferred-node kernels read only the
// previous array and write disjoint nodes of the new one - go round-robin
// over the context's stream and its side streams (forked after the previous
// step's halos, joined before this step's), so that one launch's tail
// overlaps the next one's start.
template <int D, typename T>
int StepOnce(mplbgpu_ctx* ctx) {
    if (ctx->plan.swap) return SwapStepOnce<D, T>(ctx);
    const int src = ctx->cur, dst = 1 - ctx->cur;
    ctx->pc.seed = (uint32_t)(++ctx->step_count);
    const int lanes = ctx->nlanes;
    if (lanes > 1) {
        CK(cudaEventRecord(ctx->fork, ctx->stream));
        for (int k = 0; k < lanes - 1; k++)
            CK(cudaStreamWaitEvent(ctx->side[k], ctx->fork, 0));
    }
    int lane = 0;
    auto next = [&]() {
        cudaStream_t st = lane == 0 ? ctx->stream : ctx->side[lane - 1];
        lane = (lane + 1) % lanes;
        return st;
    };
    for (size_t bi = 0; bi < ctx->blocks.size(); bi++) {
        DevBlock& b = ctx->blocks[bi];
        const BlockPlan& B = ctx->plan.blocks[bi];
        const T* s = static_cast<const T*>(b.pop[src]);
        T* d = static_cast<T*>(b.pop[dst]);
        CK_LAUNCH_E(Launch<D, T>::Step(kModeStep, NodeGrid(B, D), next(),
                                       b.dev, ctx->pc, s, d, nullptr, nullptr,
                                       nullptr, nullptr));
        if (B.ndeferred > 0 && b.dev.deferred_fused) {
            const unsigned g = (unsigned)((B.ndeferred + kThreads - 1) / kThreads);
            CK_LAUNCH_E(Launch<D, T>::DeferredFused(g, next(), b.dev, ctx->pc,
                                                    s, d));
        } else if (B.ndeferred > 0) {
            // the per-boundary programme: its kernels in order on one stream
            cudaStream_t st = next();
            const unsigned g = (unsigned)((B.ndeferred + kThreads - 1) / kThreads);
            CK_LAUNCH_E(Launch<D, T>::DeferredStream(g, st, b.dev, ctx->pc, s));
            for (auto& dop : b.dops) {
                const unsigned gd =
                    (unsigned)((dop.total + kThreads - 1) / kThreads);
                CK_LAUNCH_E(Launch<D, T>::DeferredOp(gd, st, b.dev, ctx->pc, s,
                                                     dop.segs, dop.nseg,
                                                     dop.total));
            }
            CK_LAUNCH_E(Launch<D, T>::DeferredFinish(kModeStep, g, st, b.dev,
                                                     ctx->pc, d, nullptr,
                                                     nullptr, nullptr,
                                                     nullptr));
        }
    }
    if (lanes > 1) {
        for (int k = 0; k < lanes - 1; k++) {
            CK(cudaEventRecord(ctx->join[k], ctx->side[k]));
            CK(cudaStreamWaitEvent(ctx->stream, ctx->join[k], 0));
        }
    }
    ctx->cur = dst;
    ctx->initial = false;
    return RunHalosT<D, T>(ctx);
}

// First part of a step: the x faces and interior rows of every block with
// the split layout, which read no halo layer beyond a y or z face (other
// blocks do all their work in the second part).
template <int D, typename T>
int StepBeginT(mplbgpu_ctx* ctx) {
    const int src = ctx->cur, dst = 1 - ctx->cur;
    ctx->pc.seed = (uint32_t)(++ctx->step_count);
    for (size_t bi = 0; bi < ctx->blocks.size(); bi++) {
        DevBlock& b = ctx->blocks[bi];
        if (!b.dev.split) continue;
        CK_LAUNCH_E(Launch<D, T>::StepPart(
            1, ctx->stream, b.dev, ctx->pc, static_cast<const T*>(b.pop[src]),
            static_cast<T*>(b.pop[dst])));
    }
    ctx->begun = true;
    return MPLBGPU_OK;
}

// The rest of a begun step: shell rows of split blocks, whole other
// blocks, deferred nodes, then the block-to-block halos.
template <int D, typename T>
int StepFinishT(mplbgpu_ctx* ctx) {
    const int src = ctx->cur, dst = 1 - ctx->cur;
    for (size_t bi = 0; bi < ctx->blocks.size(); bi++) {
        DevBlock& b = ctx->blocks[bi];
        const BlockPlan& B = ctx->plan.blocks[bi];
        const T* s = static_cast<const T*>(b.pop[src]);
        T* d = static_cast<T*>(b.pop[dst]);
        if (b.dev.split) {
            CK_LAUNCH_E(Launch<D, T>::StepPart(2, ctx->stream, b.dev, ctx->pc,
                                               s, d));
        } else {
            CK_LAUNCH_E(Launch<D, T>::Step(kModeStep, NodeGrid(B, D),
                                           ctx->stream, b.dev, ctx->pc, s, d,
                                           nullptr, nullptr, nullptr,
                                           nullptr));
        }
        if (B.ndeferred > 0 && b.dev.deferred_fused) {
            const unsigned g = (unsigned)((B.ndeferred + kThreads - 1) / kThreads);
            CK_LAUNCH_E(Launch<D, T>::DeferredFused(g, ctx->stream, b.dev,
                                                    ctx->pc, s, d));
        } else if (B.ndeferred > 0) {
            const unsigned g = (unsigned)((B.ndeferred + kThreads - 1) / kThreads);
            CK_LAUNCH_E(Launch<D, T>::DeferredStream(g, ctx->stream, b.dev,
                                                     ctx->pc, s));
            for (auto& dop : b.dops) {
                const unsigned gd =
                    (unsigned)((dop.total + kThreads - 1) / kThreads);
                CK_LAUNCH_E(Launch<D, T>::DeferredOp(gd, ctx->stream, b.dev,
                                                     ctx->pc, s, dop.segs,
                                                     dop.nseg, dop.total));
            }
            CK_LAUNCH_E(Launch<D, T>::DeferredFinish(
                kModeStep, g, ctx->stream, b.dev, ctx->pc, d, nullptr, nullptr,
                nullptr, nullptr));
        }
    }
    ctx->cur = dst;
    ctx->initial = false;
    ctx->begun = false;
    return RunHalosT<D, T>(ctx);
}

int StepBegin(mplbgpu_ctx* ctx) { return MPLB_DISPATCH(ctx, StepBeginT, ctx); }
int StepFinish(mplbgpu_ctx* ctx) {
    return MPLB_DISPATCH(ctx, StepFinishT, ctx);
}

// Current f -> moments (kModeMacro) or point-major f (kModeF) of one block.
template <int D, typename T>
int Observe(mplbgpu_ctx* ctx, int mode, size_t bi, double* o0, double* o1,
            double* o2, double* o3) {
    DevBlock& b = ctx->blocks[bi];
    const BlockPlan& B = ctx->plan.blocks[bi];
    if (ctx->plan.swap) {
        const int st = ctx->swap_state;
        CK_LAUNCH_E(Launch<D, T>::Swap(mode, st == 1, st != 0, NodeGrid(B, D),
                                       ctx->stream, b.dev, ctx->pc,
                                       static_cast<T*>(b.pop[0]), o0, o1, o2,
                                       o3));
        return MPLBGPU_OK;
    }
    const int prev = 1 - ctx->cur;
    const T* pv = static_cast<const T*>(b.pop[prev]);
    if (ctx->initial) {
        CK_LAUNCH_E(Launch<D, T>::DirectObserve(mode, NodeGrid(B, D),
                                                ctx->stream, b.dev, ctx->pc,
                                                pv, o0, o1, o2, o3));
        return MPLBGPU_OK;
    }
    CK_LAUNCH_E(Launch<D, T>::Step(mode, NodeGrid(B, D), ctx->stream, b.dev,
                                   ctx->pc, pv, nullptr, o0, o1, o2, o3));
    if (B.ndeferred > 0) {
        const unsigned g = (unsigned)((B.ndeferred + kThreads - 1) / kThreads);
        CK_LAUNCH_E(Launch<D, T>::DeferredFinish(mode, g, ctx->stream, b.dev,
                                                 ctx->pc, nullptr, o0, o1, o2,
                                                 o3));
    }
    return MPLBGPU_OK;
}

int UpdateMacro(mplbgpu_ctx* ctx) {
    for (size_t bi = 0; bi < ctx->blocks.size(); bi++) {
        DevBlock& b = ctx->blocks[bi];
        int rc = MPLB_DISPATCH(ctx, Observe, ctx, (int)kModeMacro, bi,
                               b.macro[0], b.macro[1], b.macro[2],
                               ctx->plan.dim == 3 ? b.macro[3] : nullptr);
        if (rc != MPLBGPU_OK) return rc;
    }
    return MPLBGPU_OK;
}

int CheckReady(mplbgpu_ctx* ctx, bool allow_begun = false) {
    if (ctx->begun && !allow_begun)
        return SetErr(ctx, MPLBGPU_ERR_STATE,
                      "a step begun by mplbgpu_step_begin is not finished");
    for (size_t i = 0; i < ctx->initialised.size(); i++)
        if (!ctx->initialised[i])
            return SetErr(ctx, MPLBGPU_ERR_STATE,
                          "block " + std::to_string(ctx->plan.blocks[i].id) +
                              " has no initial state (mplbgpu_init_macro or "
                              "mplbgpu_upload_f)");
    return MPLBGPU_OK;
}

template <int D, typename T>
int InitBlock(mplbgpu_ctx* ctx, size_t bi, const double* d_rho,
              const double* d_u, const double* d_v, const double* d_w,
              const double* d_f) {
    DevBlock& b = ctx->blocks[bi];
    const BlockPlan& B = ctx->plan.blocks[bi];
    if (ctx->plan.swap) {
        CK_LAUNCH_E(Launch<D, T>::Init(NodeGrid(B, D), ctx->stream, b.dev,
                                       ctx->pc, d_rho, d_u, d_v, d_w, d_f,
                                       static_cast<T*>(b.pop[0]), nullptr));
        ctx->swap_state = 0;
        return MPLBGPU_OK;
    }
    CK_LAUNCH_E(Launch<D, T>::Init(NodeGrid(B, D), ctx->stream, b.dev,
                                   ctx->pc, d_rho, d_u, d_v, d_w, d_f,
                                   static_cast<T*>(b.pop[1 - ctx->cur]),
                                   static_cast<T*>(b.pop[ctx->cur])));
    return MPLBGPU_OK;
}

// Face of a decomposed block: the populations crossing it and the layer.
int FaceSetup(mplbgpu_ctx* ctx, int block, int surface, bool exp,
                     size_t* bi, FaceDev* fd) {
    const BlockPlan* B = FindPlan(ctx, block);
    if (!B) return SetErr(ctx, MPLBGPU_ERR_INVALID, "unknown block id");
    const int dim = ctx->plan.dim;
    if (surface < 0 || surface >= 2 * dim || !(B->cut >> surface & 1))
        return SetErr(ctx, MPLBGPU_ERR_INVALID,
                      "surface is not a cut face of the block");
    static const int axis_of[6] = {0, 0, 1, 1, 2, 2};
    static const int side_of[6] = {0, 1, 1, 0, 1, 0};   // 1: max face
    const int a = axis_of[surface], side = side_of[surface];
    *bi = (size_t)B->index;
    FaceDev& f = *fd;
    f = FaceDev{};
    f.axis = a;
    f.layer = exp ? (side ? B->n[a] - 1 : 0) : (side ? B->n[a] : -1);
    f.ua = f.va = -1;
    for (int q = 0; q < dim; q++) {
        if (q == a) continue;
        if (f.ua < 0) f.ua = q;
        else f.va = q;
    }
    f.nu = B->n[f.ua];
    f.nv = f.va >= 0 ? B->n[f.va] : 1;
    // leaving through the face (export) = entering the neighbour's halo
    // through its opposite face (import): c_a = +1 across a max face
    const int c_out = side ? 1 : -1;
    const int want = exp ? c_out : -c_out;
    f.npop = 0;
    for (int i = 0; i < ctx->plan.Q; i++) {
        const int c = dim == 3 ? comp<Lattice<3>>(i, a) : comp<Lattice<2>>(i, a);
        if (c == want) f.pop[f.npop++] = i;
    }
    return MPLBGPU_OK;
}

template <int D, typename T>
int FaceCopy(mplbgpu_ctx* ctx, size_t bi, const FaceDev& fd, bool exp,
                    void* buf) {
    DevBlock& b = ctx->blocks[bi];
    const long long total = (long long)fd.npop * fd.nu * fd.nv;
    const unsigned grid =
        (unsigned)std::min<long long>((total + 255) / 256, 4096);
    CK_LAUNCH_E(Launch<D, T>::Face(exp, grid, ctx->stream, b.dev, fd,
                                   static_cast<T*>(b.pop[ctx->cur]),
                                   static_cast<T*>(buf)));
    return MPLBGPU_OK;
}

}  // namespace

extern "C" {

mplbgpu_status mplbgpu_create(const mplbgpu_desc* desc, mplbgpu_ctx** out) {
    if (!desc || !out) return SetErr(nullptr, MPLBGPU_ERR_INVALID, "null argument");
    *out = nullptr;
    // the description is checked before the device (the plan is host
    // work), so a host without a GPU still tells a bad description apart
    std::unique_ptr<mplbgpu_ctx> c(new mplbgpu_ctx);
    std::string err;
    int rc = BuildPlan(*desc, &c->plan, &err);
    if (rc != MPLBGPU_OK) return SetErr(nullptr, rc, err);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        return SetErr(nullptr, MPLBGPU_ERR_NO_DEVICE, "no CUDA device");
    const Plan& P = c->plan;
    PhysConst& pc = c->pc;
    pc.cs = P.cs;
    pc.omc = P.omc;
    pc.tw = P.tw;
    pc.force = P.body_force == MPLBGPU_FORCE_1ST;
    pc.force_vel = P.force_velocity;
    for (int a = 0; a < 3; a++) pc.hdta[a] = P.hdta[a];
    for (int i = 0; i < kMaxQ; i++) {
        pc.cf[i] = P.cf[i];
        pc.w[i] = P.w[i];
        pc.cff[i] = (float)P.cf[i];
        pc.wf[i] = (float)P.w[i];
        pc.winvf[i] = P.w[i] > 0 ? (float)(kHalfScale / P.w[i]) : 0.0f;
        pc.wlf[i] = (float)(P.w[i] / kHalfScale);
    }
    pc.csf = (float)P.cs;
    pc.omcf = (float)P.omc;
    pc.twf = (float)P.tw;
    for (int a = 0; a < 3; a++) pc.hdtaf[a] = (float)P.hdta[a];
    for (int a = 0; a < 3; a++) pc.hdta_csf[a] = (float)(P.hdta[a] / P.cs);
    for (int i = 0; i < kMaxQ; i++) {
        pc.wcff[i] = (float)(P.w[i] * P.cf[i]);
        pc.cf256f[i] = (float)(kHalfScale * P.cf[i]);
    }
    pc.tw_omf = (float)(P.tw / (1.0 - P.omc));
    if (P.swap) {
        // KerSwapCalcBodyForce1ST3D adds the first-order force term itself
        // after the collision, not tau * omega times it
        pc.tw = 1.0;
        pc.twf = 1.0f;
        pc.tw_omf = (float)(1.0 / (1.0 - P.omc));
    }
    auto fail_cuda = [&](cudaError_t e, const char* what) {
        std::string m = std::string(what) + ": " + cudaGetErrorString(e);
        FreeAll(c.get());
        c->blocks.clear();
        c->halos.clear();
        return SetErr(nullptr, MPLBGPU_ERR_CUDA, m);
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) !=
        cudaSuccess)
        return fail_cuda(e, "cudaStreamCreate");
    if ((e = cudaEventCreate(&c->ev0)) != cudaSuccess ||
        (e = cudaEventCreate(&c->ev1)) != cudaSuccess)
        return fail_cuda(e, "cudaEventCreate");
    {
        // independent launches per step: every block's step kernel and
        // every block's deferred kernels (two-array scheme)
        int indep = 0;
        for (const BlockPlan& B : P.blocks) indep += 1 + (B.ndeferred > 0);
        c->nlanes = P.swap ? 1 : std::min(indep, mplbgpu_ctx::kSides + 1);
        for (int k = 0; k < c->nlanes - 1; k++)
            if ((e = cudaStreamCreateWithFlags(&c->side[k],
                                               cudaStreamNonBlocking)) !=
                    cudaSuccess ||
                (e = cudaEventCreateWithFlags(&c->join[k],
                                              cudaEventDisableTiming)) !=
                    cudaSuccess)
                return fail_cuda(e, "side streams");
        if (c->nlanes > 1 &&
            (e = cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming)) !=
                cudaSuccess)
            return fail_cuda(e, "side streams");
    }
    c->blocks.resize(P.blocks.size());
    c->initialised.assign(P.blocks.size(), false);
    const int Q = P.Q;
    for (size_t bi = 0; bi < P.blocks.size(); bi++) {
        const BlockPlan& B = P.blocks[bi];
        DevBlock& b = c->blocks[bi];
        const size_t popbytes = (size_t)Q * B.popstride * P.elem_bytes;
        // slack after the last population: the node pairs of the shifted
        // forms' interior compute a partner beyond the row end (and do not
        // store it), whose pulls reach up to a row and 32 nodes further
        const size_t slack = (size_t)(B.pitch + 64) * P.elem_bytes;
        for (int k = 0; k < (P.swap ? 1 : 2); k++) {
            if ((e = cudaMalloc(&b.pop[k], popbytes + slack)) != cudaSuccess)
                return fail_cuda(e, "cudaMalloc(populations)");
            // f = 0 everywhere (the reference's zero-filled dats): zero
            // bytes in FP64, h = -w in the shifted forms
            if (P.precision == MPLBGPU_FP64)
                e = cudaMemsetAsync(b.pop[k], 0, popbytes + slack, c->stream);
            else if ((e = FillZeroF(c.get(), b.pop[k], B.popstride)) ==
                     cudaSuccess)
                e = cudaMemsetAsync(static_cast<char*>(b.pop[k]) + popbytes,
                                    0, slack, c->stream);
            if (e != cudaSuccess) return fail_cuda(e, "population fill");
        }
        if ((e = cudaMalloc(&b.regions, sizeof(B.region))) != cudaSuccess ||
            (e = cudaMemcpy(b.regions, B.region, sizeof(B.region),
                            cudaMemcpyHostToDevice)) != cudaSuccess)
            return fail_cuda(e, "region table");
        if (!B.ops.empty()) {
            const size_t ob = B.ops.size() * sizeof(RegionOp);
            if ((e = cudaMalloc(&b.ops, ob)) != cudaSuccess ||
                (e = cudaMemcpy(b.ops, B.ops.data(), ob,
                                cudaMemcpyHostToDevice)) != cudaSuccess)
                return fail_cuda(e, "op table");
        }
        if (B.nstale > 0 &&
            (e = cudaMalloc(&b.stale, (size_t)B.nstale * Q * sizeof(double))) !=
                cudaSuccess)
            return fail_cuda(e, "stale store");
        std::vector<int4> dreg;
        if (B.ndeferred > 0) {
            if ((e = cudaMalloc(&b.fdef, (size_t)B.ndeferred * Q *
                                             sizeof(double))) != cudaSuccess)
                return fail_cuda(e, "deferred store");
            for (int r = 0; r < kNumRegions; r++) {
                const RegionInfo& R = B.region[r];
                if (R.cls == kDeferred)
                    dreg.push_back(make_int4(
                        r, (int)R.side_base,
                        R.ext[0] * R.ext[1] * R.ext[2], 0));
            }
            if ((e = cudaMalloc(&b.dregions, dreg.size() * sizeof(int4))) !=
                    cudaSuccess ||
                (e = cudaMemcpy(b.dregions, dreg.data(),
                                dreg.size() * sizeof(int4),
                                cudaMemcpyHostToDevice)) != cudaSuccess)
                return fail_cuda(e, "deferred regions");
            for (const DeferredOp& dop : B.dops) {
                std::vector<DeferredSeg> segs;
                long long start = 0;
                for (const DeferredSegment& s : dop.segments) {
                    const RegionInfo& R = B.region[s.region];
                    const long long cnt =
                        (long long)R.ext[0] * R.ext[1] * R.ext[2];
                    segs.push_back({s.region, s.op, start, cnt});
                    start += cnt;
                }
                DevBlock::DOp d;
                d.nseg = (int)segs.size();
                d.total = start;
                if ((e = cudaMalloc(&d.segs, segs.size() * sizeof(DeferredSeg))) !=
                        cudaSuccess ||
                    (e = cudaMemcpy(d.segs, segs.data(),
                                    segs.size() * sizeof(DeferredSeg),
                                    cudaMemcpyHostToDevice)) != cudaSuccess)
                    return fail_cuda(e, "deferred segments");
                b.dops.push_back(d);
            }
        }
        const size_t nodes = (size_t)B.nodes();
        for (int m = 0; m < P.dim + 1; m++) {
            if ((e = cudaMalloc(&b.macro[m], nodes * sizeof(double))) !=
                    cudaSuccess ||
                (e = cudaMalloc(&b.macro_old[m], nodes * sizeof(double))) !=
                    cudaSuccess)
                return fail_cuda(e, "macro fields");
            cudaMemsetAsync(b.macro[m], 0, nodes * sizeof(double), c->stream);
            cudaMemsetAsync(b.macro_old[m], 0, nodes * sizeof(double),
                            c->stream);
        }
        BlockDev& d = b.dev;
        for (int a = 0; a < 3; a++) d.n[a] = B.n[a];
        d.xoff = B.xoff;
        d.pitch = B.pitch;
        d.plane = B.plane;
        d.popstride = B.popstride;
        d.regions = b.regions;
        d.ops = b.ops;
        d.stale = b.stale;
        d.fdef = b.fdef;
        d.ndef = B.ndeferred;
        d.dregions = b.dregions;
        d.ndregions = (int)dreg.size();
        d.deferred_fused = B.deferred_fused ? 1 : 0;
        for (int r = 0; r < kNumRegions; r++) d.dops_first[r] = B.dops_first[r];
        if ((e = cudaMalloc(&b.dops_flat, B.dops_flat.size() * sizeof(int))) !=
                cudaSuccess ||
            (e = cudaMemcpy(b.dops_flat, B.dops_flat.data(),
                            B.dops_flat.size() * sizeof(int),
                            cudaMemcpyHostToDevice)) != cudaSuccess)
            return fail_cuda(e, "deferred programme");
        d.dops_flat = b.dops_flat;
        for (int i = 0; i < kMaxQ; i++) {
            d.pop_off[i] = i < Q ? (long long)i * B.popstride : 0;
            d.pull_off[i] = 0;
        }
        for (int i = 0; i < Q; i++) {
            const int cx = P.dim == 3 ? Lattice<3>::cx(i) : Lattice<2>::cx(i);
            const int cy = P.dim == 3 ? Lattice<3>::cy(i) : Lattice<2>::cy(i);
            const int cz = P.dim == 3 ? Lattice<3>::cz(i) : 0;
            d.pull_off[i] = (long long)i * B.popstride -
                            (cx + cy * B.pitch + cz * B.plane);
        }
        // 32-bit offsets from the node's own address: every access stays
        // within one population array of Q * popstride elements.  Blocks
        // beyond 2^31 elements take the 64-bit kernels;
        // MPLB_B200_WIDE_OFFSETS=1 selects them for any block, so that tests
        // can check them against the 32-bit ones on small cases.
        const long long span = (long long)Q * B.popstride;
        const char* wide = std::getenv("MPLB_B200_WIDE_OFFSETS");
        d.off32 = span < 0x7fffffffLL && !(wide && wide[0] == '1') ? 1 : 0;
        for (int i = 0; i < kMaxQ; i++) {
            d.pull_off32[i] = d.off32 ? (int)d.pull_off[i] : 0;
            d.pop_off32[i] = d.off32 ? (int)d.pop_off[i] : 0;
        }
        d.plane32 = d.off32 ? (int)B.plane : 0;
        d.pitch32 = d.off32 ? (int)B.pitch : 0;
        for (int r = 0; r < kNumRegions; r++) {
            const RegionInfo& R = B.region[r];
            d.rflags[r] = (uint8_t)((R.cls < 0 ? kPure : R.cls) |
                                    (R.fluidlike ? 4 : 0));
            d.rpull[r] = R.pull;
            d.rstale[r] = R.stale;
        }
        for (int r = 0; r < kNumRegions; r++) {
            d.swap_exch[r] = P.swap ? B.swap_exch[r] : 0u;
            for (int k = 0; k < kMaxQ; k++)
                d.swap_sigma[r][k] = P.swap ? B.swap_sigma[r][k] : (uint8_t)k;
        }
        for (int i = 0; i < kMaxQ; i++) {
            const int o = i < Q ? (P.dim == 3 ? Lattice<3>::opp(i)
                                              : Lattice<2>::opp(i))
                                : i;
            d.swap_off[i] = d.pull_off[i] + (long long)(o - i) * B.popstride;
            d.swap_off32[i] = d.off32 ? (int)d.swap_off[i] : 0;
        }
        const int center = 13;   // interior on every axis (RegionOf)
        d.split = (B.n[0] >= 3 && B.n[1] >= 3 && (P.dim == 2 || B.n[2] >= 3) &&
                   (d.rflags[center] & 3) == kPure)
                      ? 1
                      : 0;
        d.center_fluid = B.region[center].fluidlike ? 1 : 0;
    }
    if (!P.halos.empty()) {
        std::vector<HaloCopyDev> copies;
        std::vector<int2> ctas;
        for (size_t t = 0; t < P.halos.size(); t++) {
            const HaloCopy& h = P.halos[t];
            DevHalo dh;
            HaloCopyDev cd{};
            for (int a = 0; a < 3; a++) {
                cd.iter[a] = h.iter[a];
                cd.fbase[a] = h.fbase[a];
                cd.tbase[a] = h.tbase[a];
            }
            cd.pops = h.pops;
            cd.from = h.from;
            cd.to = h.to;
            cd.cells = (long long)h.iter[0] * h.iter[1] * h.iter[2];
            for (long long t0 = 0; t0 < cd.cells; t0 += kHaloCellsPerCta)
                ctas.push_back(make_int2((int)t, (int)t0));
            if (h.any_prev) {
                if ((e = cudaMalloc(&dh.prev, h.prev.size())) != cudaSuccess ||
                    (e = cudaMemcpy(dh.prev, h.prev.data(), h.prev.size(),
                                    cudaMemcpyHostToDevice)) != cudaSuccess)
                    return fail_cuda(e, "halo masks");
            }
            if ((e = cudaMalloc(&dh.ordered, h.ordered.size())) != cudaSuccess ||
                (e = cudaMemcpy(dh.ordered, h.ordered.data(), h.ordered.size(),
                                cudaMemcpyHostToDevice)) != cudaSuccess)
                return fail_cuda(e, "halo phases");
            cd.prev = dh.prev;
            cd.ordered = dh.ordered;
            copies.push_back(cd);
            c->halos.push_back(dh);
        }
        // the resolved element copies, with their element offsets
        std::vector<HaloElemDev> elems;
        for (const HaloElem& he : P.halo_elems) {
            auto elem = [&](const BlockPlan& B, long long x, long long y,
                            long long z) {
                return (long long)he.pop * B.popstride +
                       (P.dim == 3 ? z + 1 : 0) * B.plane + (y + 1) * B.pitch +
                       x + B.xoff;
            };
            HaloElemDev ed{};
            ed.s = elem(P.blocks[he.from], he.fx, he.fy, he.fz);
            ed.d = elem(P.blocks[he.to], he.tx, he.ty, he.tz);
            ed.from2 = 2 * he.from + he.prev;
            ed.to = he.to;
            elems.push_back(ed);
        }
        for (size_t m0 = 0; m0 < elems.size(); m0 += kHaloCellsPerCta)
            ctas.push_back(make_int2(-1, (int)m0));
        std::vector<HaloBlockDev> hb(c->blocks.size());
        for (size_t bi = 0; bi < c->blocks.size(); bi++) {
            const BlockPlan& B = P.blocks[bi];
            hb[bi].pitch = B.pitch;
            hb[bi].plane = B.plane;
            hb[bi].popstride = B.popstride;
            hb[bi].xoff = B.xoff;
            hb[bi].pop[0] = c->blocks[bi].pop[0];
            hb[bi].pop[1] = c->blocks[bi].pop[1];
        }
        auto upload = [&](const void* src, size_t bytes,
                          void** dst) -> cudaError_t {
            *dst = nullptr;
            if (bytes == 0) return cudaSuccess;
            cudaError_t r = cudaMalloc(dst, bytes);
            if (r != cudaSuccess) return r;
            return cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
        };
        void* p = nullptr;
        if ((e = upload(copies.data(), copies.size() * sizeof(HaloCopyDev),
                        &p)) != cudaSuccess)
            return fail_cuda(e, "halo copies");
        c->hfd.copies = static_cast<HaloCopyDev*>(p);
        if ((e = upload(hb.data(), hb.size() * sizeof(HaloBlockDev), &p)) !=
            cudaSuccess)
            return fail_cuda(e, "halo blocks");
        c->hfd.blocks = static_cast<HaloBlockDev*>(p);
        c->hfd.nblocks = (int)hb.size();
        if ((e = upload(ctas.data(), ctas.size() * sizeof(int2), &p)) !=
            cudaSuccess)
            return fail_cuda(e, "halo work");
        c->hfd.ctas = static_cast<int2*>(p);
        if ((e = upload(elems.data(), elems.size() * sizeof(HaloElemDev),
                        &p)) != cudaSuccess)
            return fail_cuda(e, "halo elements");
        c->hfd.elems = static_cast<HaloElemDev*>(p);
        c->hfd.nelems = (int)elems.size();
        c->halo_ctas = (unsigned)ctas.size();
    }
    if ((e = cudaMalloc(&c->part, 2 * kRedBlocks * sizeof(double))) !=
            cudaSuccess ||
        (e = cudaMalloc(&c->bad, sizeof(unsigned long long))) != cudaSuccess)
        return fail_cuda(e, "reduction buffers");
    if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess)
        return fail_cuda(e, "cudaStreamSynchronize");
    *out = c.release();
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_destroy(mplbgpu_ctx* ctx) {
    if (!ctx) return MPLBGPU_ERR_INVALID;
    cudaStreamSynchronize(ctx->stream);
    FreeAll(ctx);
    delete ctx;
    return MPLBGPU_OK;
}

const char* mplbgpu_last_error(const mplbgpu_ctx* ctx) {
    return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

mplbgpu_status mplbgpu_init_macro(mplbgpu_ctx* ctx, int block,
                                  const double* rho, const double* u,
                                  const double* v, const double* w) {
    if (!ctx) return MPLBGPU_ERR_INVALID;
    DevBlock* b = FindBlock(ctx, block);
    const BlockPlan* B = FindPlan(ctx, block);
    if (!b) return SetErr(ctx, MPLBGPU_ERR_INVALID, "unknown block id");
    if (ctx->begun)
        return SetErr(ctx, MPLBGPU_ERR_STATE,
                      "a step begun by mplbgpu_step_begin is not finished");
    if (!ctx->initial) {
        // a new initial state after steps: every block starts again
        std::fill(ctx->initialised.begin(), ctx->initialised.end(), false);
    }
    const int dim = ctx->plan.dim;
    const size_t nodes = (size_t)B->nodes();
    const double* src[4] = {rho, u, v, w};
    for (int m = 0; m < dim + 1; m++) {
        if (src[m]) {
            CK(cudaMemcpyAsync(b->macro[m], src[m], nodes * sizeof(double),
                               cudaMemcpyHostToDevice, ctx->stream));
        } else {
            // a field not given: rho = 1, velocity components 0
            FillDoubleKernel<<<1024, 256, 0, ctx->stream>>>(
                b->macro[m], (long long)nodes, m == 0 ? 1.0 : 0.0);
            CK_LAUNCH();
        }
        // CopyCurrentMacroVar after PreDefinedInitialCondition3D
        CK(cudaMemcpyAsync(b->macro_old[m], b->macro[m], nodes * sizeof(double),
                           cudaMemcpyDeviceToDevice, ctx->stream));
    }
    const size_t bi = (size_t)(b - ctx->blocks.data());
    int rc = MPLB_DISPATCH(ctx, InitBlock, ctx, bi, b->macro[0], b->macro[1],
                           b->macro[2], dim == 3 ? b->macro[3] : nullptr,
                           nullptr);
    if (rc != MPLBGPU_OK) return rc;
    ctx->initial = true;
    ctx->halos_pending = true;
    ctx->initialised[bi] = true;
    ctx->step_count = 0;   // a new initial state is step 0
    CK(cudaStreamSynchronize(ctx->stream));
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_upload_f(mplbgpu_ctx* ctx, int block, const double* f) {
    if (!ctx || !f) return ctx ? SetErr(ctx, MPLBGPU_ERR_INVALID, "null f")
                               : MPLBGPU_ERR_INVALID;
    DevBlock* b = FindBlock(ctx, block);
    const BlockPlan* B = FindPlan(ctx, block);
    if (!b) return SetErr(ctx, MPLBGPU_ERR_INVALID, "unknown block id");
    if (ctx->begun)
        return SetErr(ctx, MPLBGPU_ERR_STATE,
                      "a step begun by mplbgpu_step_begin is not finished");
    if (!ctx->initial)
        std::fill(ctx->initialised.begin(), ctx->initialised.end(), false);
    const size_t elems = (size_t)B->nodes() * ctx->plan.Q;
    int rc = EnsureScratch(ctx, elems);
    if (rc != MPLBGPU_OK) return rc;
    CK(cudaMemcpyAsync(ctx->scratch, f, elems * sizeof(double),
                       cudaMemcpyHostToDevice, ctx->stream));
    const size_t bi = (size_t)(b - ctx->blocks.data());
    rc = MPLB_DISPATCH(ctx, InitBlock, ctx, bi, nullptr, nullptr, nullptr,
                       nullptr, ctx->scratch);
    if (rc != MPLBGPU_OK) return rc;
    ctx->initial = true;
    ctx->halos_pending = true;
    ctx->initialised[bi] = true;
    // macro fields: moments of the uploaded f, q_old = q
    rc = MPLB_DISPATCH(ctx, Observe, ctx, (int)kModeMacro, bi, b->macro[0],
                       b->macro[1], b->macro[2],
                       ctx->plan.dim == 3 ? b->macro[3] : nullptr);
    if (rc != MPLBGPU_OK) return rc;
    for (int m = 0; m < ctx->plan.dim + 1; m++)
        CK(cudaMemcpyAsync(b->macro_old[m], b->macro[m],
                           (size_t)B->nodes() * sizeof(double),
                           cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_step(mplbgpu_ctx* ctx, int nsteps) {
    if (!ctx) return MPLBGPU_ERR_INVALID;
    if (nsteps < 0) return SetErr(ctx, MPLBGPU_ERR_INVALID, "nsteps < 0");
    int rc = CheckReady(ctx);
    if (rc != MPLBGPU_OK) return rc;
    if (ctx->halos_pending) {
        rc = RunHalos(ctx);
        if (rc != MPLBGPU_OK) return rc;
    }
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    for (int s = 0; s < nsteps; s++) {
        rc = MPLB_DISPATCH(ctx, StepOnce, ctx);
        if (rc != MPLBGPU_OK) return rc;
    }
    // no host wait: the caller's next reading call (download, residual,
    // mass, synchronize, last_step_ms) waits for the stream
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->timing_pending = true;
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_step_begin(mplbgpu_ctx* ctx) {
    if (!ctx) return MPLBGPU_ERR_INVALID;
    int rc = CheckReady(ctx);
    if (rc != MPLBGPU_OK) return rc;
    if (ctx->plan.swap)
        return SetErr(ctx, MPLBGPU_ERR_UNSUPPORTED,
                      "a step in two parts needs the two-array scheme");
    if (ctx->halos_pending) {
        rc = RunHalos(ctx);
        if (rc != MPLBGPU_OK) return rc;
    }
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    return StepBegin(ctx);
}

mplbgpu_status mplbgpu_step_finish(mplbgpu_ctx* ctx) {
    if (!ctx) return MPLBGPU_ERR_INVALID;
    if (!ctx->begun)
        return SetErr(ctx, MPLBGPU_ERR_STATE,
                      "mplbgpu_step_finish without mplbgpu_step_begin");
    int rc = StepFinish(ctx);
    if (rc != MPLBGPU_OK) return rc;
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->timing_pending = true;
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_get_stream(mplbgpu_ctx* ctx, void** stream) {
    if (!ctx || !stream) return MPLBGPU_ERR_INVALID;
    *stream = static_cast<void*>(ctx->stream);
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_step_kernel(mplbgpu_ctx* ctx, int block_id,
                                   int* kind) {
    if (!ctx || !kind) return MPLBGPU_ERR_INVALID;
    for (size_t bi = 0; bi < ctx->blocks.size(); bi++) {
        if (ctx->plan.blocks[bi].id != block_id) continue;
        const DevBlock& b = ctx->blocks[bi];
        *kind = ctx->plan.swap ? MPLBGPU_KERNEL_SWAP
                : b.dev.split  ? MPLBGPU_KERNEL_SPLIT
                               : MPLBGPU_KERNEL_NODE;
        return MPLBGPU_OK;
    }
    return SetErr(ctx, MPLBGPU_ERR_INVALID,
                  "unknown block id " + std::to_string(block_id));
}

mplbgpu_status mplbgpu_update_macro(mplbgpu_ctx* ctx) {
    if (!ctx) return MPLBGPU_ERR_INVALID;
    int rc = CheckReady(ctx);
    if (rc != MPLBGPU_OK) return rc;
    rc = UpdateMacro(ctx);
    if (rc != MPLBGPU_OK) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_residual_sums(mplbgpu_ctx* ctx, double* diff,
                                     double* sum) {
    if (!ctx || !diff || !sum) return MPLBGPU_ERR_INVALID;
    const int nv = ctx->plan.dim + 1;
    for (int m = 0; m < nv; m++) diff[m] = sum[m] = 0.0;
    std::vector<double> part(2 * kRedBlocks);
    for (int m = 0; m < nv; m++) {
        for (size_t bi = 0; bi < ctx->blocks.size(); bi++) {
            DevBlock& b = ctx->blocks[bi];
            const long long n = ctx->plan.blocks[bi].nodes();
            ResidualPartialKernel<<<kRedBlocks, kRedThreads, 0, ctx->stream>>>(
                b.macro[m], b.macro_old[m], n, ctx->part);
            CK_LAUNCH();
            CK(cudaMemcpyAsync(part.data(), ctx->part,
                               part.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            for (int k = 0; k < kRedBlocks; k++) {
                diff[m] += part[2 * k];
                sum[m] += part[2 * k + 1];
            }
        }
    }
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_residual(mplbgpu_ctx* ctx, int check_period,
                                double* per_var, double* max_residual) {
    if (!ctx) return MPLBGPU_ERR_INVALID;
    if (check_period <= 0)
        return SetErr(ctx, MPLBGPU_ERR_INVALID, "check_period must be > 0");
    const int nv = ctx->plan.dim + 1;
    double diff[4] = {0, 0, 0, 0}, sum[4] = {0, 0, 0, 0};
    int rc = mplbgpu_residual_sums(ctx, diff, sum);
    if (rc != MPLBGPU_OK) return rc;
    // GetMaximumResidual, Src/flowfield.cpp:148-158
    double mx = 0;
    for (int m = 0; m < nv; m++) {
        const double res = diff[m] / sum[m];
        if (per_var) per_var[m] = res;
        const double rel = res / (check_period * ctx->plan.dt);
        if (mx <= rel) mx = rel;
    }
    if (max_residual) *max_residual = mx;
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_download_macro(mplbgpu_ctx* ctx, int block, double* rho,
                                      double* u, double* v, double* w) {
    if (!ctx) return MPLBGPU_ERR_INVALID;
    DevBlock* b = FindBlock(ctx, block);
    const BlockPlan* B = FindPlan(ctx, block);
    if (!b) return SetErr(ctx, MPLBGPU_ERR_INVALID, "unknown block id");
    double* dst[4] = {rho, u, v, w};
    const size_t bytes = (size_t)B->nodes() * sizeof(double);
    for (int m = 0; m < ctx->plan.dim + 1; m++)
        if (dst[m])
            CK(cudaMemcpyAsync(dst[m], b->macro[m], bytes,
                               cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_download_f(mplbgpu_ctx* ctx, int block, double* f) {
    if (!ctx || !f) return ctx ? SetErr(ctx, MPLBGPU_ERR_INVALID, "null f")
                               : MPLBGPU_ERR_INVALID;
    int rc = CheckReady(ctx);
    if (rc != MPLBGPU_OK) return rc;
    DevBlock* b = FindBlock(ctx, block);
    const BlockPlan* B = FindPlan(ctx, block);
    if (!b) return SetErr(ctx, MPLBGPU_ERR_INVALID, "unknown block id");
    const size_t elems = (size_t)B->nodes() * ctx->plan.Q;
    rc = EnsureScratch(ctx, elems);
    if (rc != MPLBGPU_OK) return rc;
    const size_t bi = (size_t)(b - ctx->blocks.data());
    rc = MPLB_DISPATCH(ctx, Observe, ctx, (int)kModeF, bi, ctx->scratch,
                       nullptr, nullptr, nullptr);
    if (rc != MPLBGPU_OK) return rc;
    CK(cudaMemcpyAsync(f, ctx->scratch, elems * sizeof(double),
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_face_size(mplbgpu_ctx* ctx, int block, int surface,
                                 long long* elems, int* elem_bytes) {
    if (!ctx) return MPLBGPU_ERR_INVALID;
    size_t bi;
    FaceDev fd;
    int rc = FaceSetup(ctx, block, surface, true, &bi, &fd);
    if (rc != MPLBGPU_OK) return rc;
    if (elems) *elems = (long long)fd.npop * fd.nu * fd.nv;
    if (elem_bytes) *elem_bytes = ctx->plan.elem_bytes;
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_export_face(mplbgpu_ctx* ctx, int block, int surface,
                                   void* buf) {
    if (!ctx || !buf) return ctx ? SetErr(ctx, MPLBGPU_ERR_INVALID, "null buffer")
                                 : MPLBGPU_ERR_INVALID;
    int rc = CheckReady(ctx, true);
    if (rc != MPLBGPU_OK) return rc;
    size_t bi;
    FaceDev fd;
    rc = FaceSetup(ctx, block, surface, true, &bi, &fd);
    if (rc != MPLBGPU_OK) return rc;
    return MPLB_DISPATCH(ctx, FaceCopy, ctx, bi, fd, true, buf);
}

mplbgpu_status mplbgpu_import_face(mplbgpu_ctx* ctx, int block, int surface,
                                   const void* buf) {
    if (!ctx || !buf) return ctx ? SetErr(ctx, MPLBGPU_ERR_INVALID, "null buffer")
                                 : MPLBGPU_ERR_INVALID;
    int rc = CheckReady(ctx, true);
    if (rc != MPLBGPU_OK) return rc;
    size_t bi;
    FaceDev fd;
    rc = FaceSetup(ctx, block, surface, false, &bi, &fd);
    if (rc != MPLBGPU_OK) return rc;
    if (ctx->begun && fd.axis == 0)
        return SetErr(ctx, MPLBGPU_ERR_STATE,
                      "an x face cannot be imported while a step is begun "
                      "(its first part reads the x halo layers)");
    return MPLB_DISPATCH(ctx, FaceCopy, ctx, bi, fd, false,
                         const_cast<void*>(buf));
}

static int SumRho(mplbgpu_ctx* ctx, double* total, unsigned long long* nbad) {
    int rc = UpdateMacro(ctx);
    if (rc != MPLBGPU_OK) return rc;
    CK(cudaMemsetAsync(ctx->bad, 0, sizeof(unsigned long long), ctx->stream));
    double s = 0;
    std::vector<double> part(kRedBlocks);
    for (size_t bi = 0; bi < ctx->blocks.size(); bi++) {
        SumPartialKernel<<<kRedBlocks, kRedThreads, 0, ctx->stream>>>(
            ctx->blocks[bi].macro[0], ctx->plan.blocks[bi].nodes(), ctx->part,
            ctx->bad);
        CK_LAUNCH();
        CK(cudaMemcpyAsync(part.data(), ctx->part, part.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        for (double v : part) s += v;
    }
    CK(cudaMemcpyAsync(nbad, ctx->bad, sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *total = s;
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_mass(mplbgpu_ctx* ctx, double* mass) {
    if (!ctx || !mass) return MPLBGPU_ERR_INVALID;
    int rc = CheckReady(ctx);
    if (rc != MPLBGPU_OK) return rc;
    unsigned long long nbad = 0;
    return SumRho(ctx, mass, &nbad);
}

mplbgpu_status mplbgpu_check_health(mplbgpu_ctx* ctx) {
    if (!ctx) return MPLBGPU_ERR_INVALID;
    int rc = CheckReady(ctx);
    if (rc != MPLBGPU_OK) return rc;
    double s = 0;
    unsigned long long nbad = 0;
    rc = SumRho(ctx, &s, &nbad);
    if (rc != MPLBGPU_OK) return rc;
    if (nbad)
        return SetErr(ctx, MPLBGPU_ERR_DIVERGED,
                      std::to_string(nbad) +
                          " nodes with non-finite or non-positive density");
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_boundary_extent(mplbgpu_ctx* ctx, int boundary,
                                       int ext[3]) {
    if (!ctx || !ext) return MPLBGPU_ERR_INVALID;
    if (boundary < 0 || boundary >= (int)ctx->plan.bc_block.size() ||
        ctx->plan.bc_block[boundary] < 0)
        return SetErr(ctx, MPLBGPU_ERR_INVALID, "unknown boundary index");
    const int* r = &ctx->plan.bc_range[6 * (size_t)boundary];
    for (int a = 0; a < 3; a++) ext[a] = r[2 * a + 1] - r[2 * a];
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_set_boundary_velocity(mplbgpu_ctx* ctx, int boundary,
                                             const double* u, const double* v,
                                             const double* w) {
    if (!ctx) return MPLBGPU_ERR_INVALID;
    int ext[3];
    int rc = mplbgpu_boundary_extent(ctx, boundary, ext);
    if (rc != MPLBGPU_OK) return rc;
    if (ctx->plan.swap)
        return SetErr(ctx, MPLBGPU_ERR_UNSUPPORTED,
                      "per-node wall velocities are not available under the "
                      "swap scheme");
    const int bi = ctx->plan.bc_block[boundary];
    BlockPlan& B = ctx->plan.blocks[bi];
    DevBlock& b = ctx->blocks[bi];
    const int* r = &ctx->plan.bc_range[6 * (size_t)boundary];
    const size_t cnt = (size_t)ext[0] * ext[1] * ext[2];
    const bool clear = !u && !v && !w;
    std::vector<RegionOp> node_ops;
    if (!clear) {
        std::vector<double> packed(3 * cnt, 0.0);
        const double* src[3] = {u, v, ctx->plan.dim == 3 ? w : nullptr};
        for (int c = 0; c < 3; c++)
            if (src[c])
                for (size_t k = 0; k < cnt; k++) packed[3 * k + c] = src[c][k];
        for (double x : packed)
            if (!std::isfinite(x))
                return SetErr(ctx, MPLBGPU_ERR_INVALID,
                              "non-finite wall velocity");
        std::string err;
        rc = BoundaryNodeOps(ctx->plan, boundary, packed.data(), &node_ops,
                             &err);
        if (rc != MPLBGPU_OK) return SetErr(ctx, rc, err);
    } else if (ctx->plan.bc_scheme[boundary] != MPLBGPU_BC_EQM_DIFFUSE_REFL &&
               ctx->plan.bc_scheme[boundary] !=
                   MPLBGPU_BC_HALFWAY_BOUNCE_BACK) {
        return SetErr(ctx, MPLBGPU_ERR_UNSUPPORTED,
                      "per-node velocities need an EQMDiffuseRefl or halfway "
                      "bounce-back boundary");
    }
    // no kernel of this context may read the op tables while they change
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->bc_field.size() < ctx->plan.bc_block.size())
        ctx->bc_field.resize(ctx->plan.bc_block.size(), nullptr);
    RegionOp*& dev = ctx->bc_field[boundary];
    CK(cudaFree(dev));
    dev = nullptr;
    if (!clear) {
        const size_t bytes = node_ops.size() * sizeof(RegionOp);
        CK(cudaMalloc(&dev, bytes));
        CK(cudaMemcpy(dev, node_ops.data(), bytes, cudaMemcpyHostToDevice));
    }
    for (RegionOp& op : B.ops) {
        if (op.bc != boundary) continue;
        op.node_ops = dev;
        for (int a = 0; a < 3; a++) {
            op.forg[a] = r[2 * a];
            op.fext[a] = ext[a];
        }
    }
    CK(cudaMemcpy(b.ops, B.ops.data(), B.ops.size() * sizeof(RegionOp),
                  cudaMemcpyHostToDevice));
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_set_step(mplbgpu_ctx* ctx, long long step) {
    if (!ctx) return MPLBGPU_ERR_INVALID;
    if (step < 0) return SetErr(ctx, MPLBGPU_ERR_INVALID, "step < 0");
    ctx->step_count = (unsigned long long)step;
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_synchronize(mplbgpu_ctx* ctx) {
    if (!ctx) return MPLBGPU_ERR_INVALID;
    CK(cudaStreamSynchronize(ctx->stream));
    return MPLBGPU_OK;
}

long long mplbgpu_launch_count(const mplbgpu_ctx* ctx) {
    return ctx ? ctx->launches : 0;
}

mplbgpu_status mplbgpu_last_step_ms(mplbgpu_ctx* ctx, float* ms) {
    if (!ctx || !ms) return MPLBGPU_ERR_INVALID;
    if (ctx->timing_pending) {
        CK(cudaEventSynchronize(ctx->ev1));
        CK(cudaEventElapsedTime(&ctx->last_ms, ctx->ev0, ctx->ev1));
        ctx->timing_pending = false;
    }
    *ms = ctx->last_ms;
    return MPLBGPU_OK;
}

}  // extern "C"
