// Batched cavities behind the C ABI (mplbgpu_batch_*, include/mplbgpu.h).
//
// All cavities live in one pair of population arrays; a step advances every
// active tile.  Steps run in chunks: either a CUDA graph that replays
// `chunk` one-step launches, or one cooperative persistent launch of
// `chunk` steps with a bounded grid barrier between steps (itself captured
// in a graph when the driver allows it).  Every check period the moments
// of the last step feed a per-cavity residual (the reference's
// CalcResidualError + GetMaximumResidual on each cavity); converged cavities
// leave the active tile list.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/mplbgpu.h"
#include "batch_kernels.cuh"
#include "lattice.h"

using namespace mplb;

// The launchers are instantiated in kernels_f64.cu / kernels_lp.cu with the
// floating-point contraction rules of their forms.
extern template struct mplb::BatchLaunch<double>;
extern template struct mplb::BatchLaunch<float>;

struct mplbgpu_batch {
    int precision = MPLBGPU_FP32_SHIFTED;
    std::vector<mplbgpu_cavity> cav;
    std::vector<BatchCav> hcav;
    long long total_nodes = 0;
    long long pop_elems = 0;
    BatchCav* dcav = nullptr;
    void* pop[2] = {nullptr, nullptr};
    int cur = 0;                       // pop[cur] holds the latest g
    double* macro[3] = {nullptr, nullptr, nullptr};
    double* macro_old[3] = {nullptr, nullptr, nullptr};
    int4* tiles_all = nullptr;
    int4* tiles_active = nullptr;
    int* ntiles_dev = nullptr;
    int ntiles_all = 0;
    int ntiles_active = 0;
    double* part = nullptr;
    int4* ranges = nullptr;
    double* res = nullptr;
    unsigned* sync_count = nullptr;
    unsigned* sync_gen = nullptr;
    int* sync_err = nullptr;
    std::vector<int> active;           // active cavity indices, in order
    std::vector<int> first_tile;       // per cavity, in tiles_all
    std::vector<int> ntile;            // per cavity
    mplbgpu_batch_tuning tune{128, 0, 100, 8};
    PhysConst pc{};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // [macro on last step]
    bool graph_ok = true;
    double device_ms = 0;
    long long node_updates = 0;
    long long launches = 0;
    unsigned long long seed = 1;
    bool initialised = false;
    long long wait_limit = (long long)1 << 26;  // grid barrier polls
    std::string err;
};

namespace {

thread_local std::string g_batch_create_error;

int BErr(mplbgpu_batch* b, int code, const std::string& m) {
    if (b) b->err = m; else g_batch_create_error = m;
    return code;
}

#define BCK(call)                                                            \
    do {                                                                     \
        cudaError_t e_ = (call);                                             \
        if (e_ != cudaSuccess)                                               \
            return BErr(b, MPLBGPU_ERR_CUDA,                                 \
                        std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

BatchDev MakeDev(mplbgpu_batch* b) {
    BatchDev d{};
    d.cavs = b->dcav;
    d.tiles = b->tiles_active;
    d.ntiles = b->ntiles_dev;
    d.tile_nodes = b->tune.tile_nodes;
    for (int m = 0; m < 3; m++) {
        d.macro[m] = b->macro[m];
        d.macro_old[m] = b->macro_old[m];
    }
    return d;
}

void DropGraphs(mplbgpu_batch* b) {
    for (auto& g : b->graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

int BuildTiles(mplbgpu_batch* b) {
    const int tn = b->tune.tile_nodes;
    std::vector<int4> tiles;
    const long long unit = 128 / (b->precision == MPLBGPU_FP64 ? 8 : 4);
    b->first_tile.assign(b->cav.size(), 0);
    b->ntile.assign(b->cav.size(), 0);
    for (size_t c = 0; c < b->cav.size(); c++) {
        const long long nn = (long long)b->cav[c].n * b->cav[c].n;
        b->first_tile[c] = (int)tiles.size();
        // cavity offsets are multiples of 128 bytes (mplbgpu_batch_create)
        const int base = (int)(b->hcav[c].base / unit);
        for (long long k = 0; k < nn; k += tn)
            tiles.push_back(make_int4((int)c, (int)k, b->cav[c].n, base));
        b->ntile[c] = (int)tiles.size() - b->first_tile[c];
    }
    cudaFree(b->tiles_all);
    cudaFree(b->tiles_active);
    cudaFree(b->part);
    b->tiles_all = b->tiles_active = nullptr;
    b->part = nullptr;
    b->ntiles_all = (int)tiles.size();
    BCK(cudaMalloc(&b->tiles_all, tiles.size() * sizeof(int4)));
    BCK(cudaMalloc(&b->tiles_active, tiles.size() * sizeof(int4)));
    BCK(cudaMalloc(&b->part, tiles.size() * 6 * sizeof(double)));
    BCK(cudaMemcpy(b->tiles_all, tiles.data(), tiles.size() * sizeof(int4),
                   cudaMemcpyHostToDevice));
    DropGraphs(b);
    return MPLBGPU_OK;
}

// Active tiles and per-cavity tile ranges from b->active.
int UploadActive(mplbgpu_batch* b) {
    std::vector<int4> ranges;
    int pos = 0;
    for (int c : b->active) {
        ranges.push_back(make_int4(c, pos, b->ntile[c], 0));
        BCK(cudaMemcpyAsync(b->tiles_active + pos, b->tiles_all + b->first_tile[c],
                            b->ntile[c] * sizeof(int4), cudaMemcpyDeviceToDevice,
                            b->stream));
        pos += b->ntile[c];
    }
    // one-step graphs are captured with one CTA per active tile
    if (pos != b->ntiles_active && !b->tune.persistent) DropGraphs(b);
    b->ntiles_active = pos;
    BCK(cudaMemcpyAsync(b->ntiles_dev, &b->ntiles_active, sizeof(int),
                        cudaMemcpyHostToDevice, b->stream));
    if (!ranges.empty())
        BCK(cudaMemcpyAsync(b->ranges, ranges.data(), ranges.size() * sizeof(int4),
                            cudaMemcpyHostToDevice, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    return MPLBGPU_OK;
}

// One-step launches: one CTA per active tile (the hardware keeps the SMs
// full and a finished CTA's slot goes to the next tile; a grid-stride loop
// over tiles serialised each CTA's dependent tile -> cavity -> population
// loads).  Persistent launches: the co-resident CTA count.
int Grid(mplbgpu_batch* b, bool persistent) {
    if (!persistent) return std::max(1, b->ntiles_active);
    int dev = 0, sms = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per = std::max(1, b->tune.ctas_per_sm);
    if (persistent) {
        int maxres = 1;
        if (b->precision == MPLBGPU_FP64)
            BatchLaunch<double>::MaxCoResident(
                b->tune.tile_nodes / BatchNodesPerThread<double>(), &maxres);
        else
            BatchLaunch<float>::MaxCoResident(
                b->tune.tile_nodes / BatchNodesPerThread<float>(), &maxres);
        per = std::min(per, std::max(1, maxres));
    }
    return sms * per;
}

template <typename T>
int LaunchChunk(mplbgpu_batch* b, int nsteps, bool macro_last) {
    const BatchDev d = MakeDev(b);
    T* P0 = static_cast<T*>(b->pop[0]);
    T* P1 = static_cast<T*>(b->pop[1]);
    const int threads = b->tune.tile_nodes / BatchNodesPerThread<T>();
    if (b->tune.persistent) {
        const GridSync gs{b->sync_count, b->sync_gen, b->sync_err,
                          b->wait_limit};
        T* a = b->cur == 0 ? P0 : P1;
        T* c = b->cur == 0 ? P1 : P0;
        cudaError_t e = BatchLaunch<T>::Persistent(Grid(b, true), threads,
                                                   b->stream, d, b->pc, a, c,
                                                   nsteps, macro_last ? 1 : 0,
                                                   gs);
        b->launches++;
        if (e != cudaSuccess)
            return BErr(b, MPLBGPU_ERR_CUDA,
                        std::string("persistent launch: ") + cudaGetErrorString(e));
        b->pc.seed += nsteps;
    } else {
        const int grid = Grid(b, false);
        for (int s = 0; s < nsteps; s++) {
            const T* src = (b->cur ^ (s & 1)) == 0 ? P0 : P1;
            T* dst = (b->cur ^ (s & 1)) == 0 ? P1 : P0;
            cudaError_t e = BatchLaunch<T>::Step(macro_last && s == nsteps - 1,
                                                 grid, threads, b->stream, d,
                                                 b->pc, b->ntiles_active, src,
                                                 dst);
            b->launches++;
            b->pc.seed += 1;
            if (e != cudaSuccess)
                return BErr(b, MPLBGPU_ERR_CUDA,
                            std::string("step launch: ") + cudaGetErrorString(e));
        }
    }
    if (nsteps & 1) b->cur ^= 1;
    return MPLBGPU_OK;
}

int Chunk(mplbgpu_batch* b, int nsteps, bool macro_last) {
    return b->precision == MPLBGPU_FP64 ? LaunchChunk<double>(b, nsteps, macro_last)
                                        : LaunchChunk<float>(b, nsteps, macro_last);
}

// A chunk of `tune.chunk` steps replayed from a CUDA graph (captured on
// first use; the active tile list lives in device memory, so a persistent
// graph stays valid when cavities converge; one-step graphs are captured
// again when the active tile count, their grid, changes).
int GraphChunk(mplbgpu_batch* b, bool macro_last) {
    const int n = b->tune.chunk;
    cudaGraphExec_t& g = b->graph[macro_last ? 1 : 0];
    if (b->graph_ok && g == nullptr && b->cur == 0) {
        cudaGraph_t graph = nullptr;
        const unsigned long long seed0 = b->pc.seed;
        const long long l0 = b->launches;
        if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) ==
            cudaSuccess) {
            int rc = Chunk(b, n, macro_last);
            cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
            if (rc == MPLBGPU_OK && e == cudaSuccess &&
                cudaGraphInstantiate(&g, graph, 0) == cudaSuccess) {
                cudaGraphDestroy(graph);
            } else {
                if (graph) cudaGraphDestroy(graph);
                g = nullptr;
                b->graph_ok = false;
                cudaGetLastError();
            }
        } else {
            b->graph_ok = false;
            cudaGetLastError();
        }
        b->pc.seed = seed0;
        b->launches = l0;
        if (n & 1) b->cur ^= 1;  // the capture did not run the steps
    }
    if (g != nullptr && b->cur == 0) {
        BCK(cudaGraphLaunch(g, b->stream));
        b->launches += b->tune.persistent ? 1 : n;
        b->pc.seed += n;
        if (n & 1) b->cur ^= 1;
        return MPLBGPU_OK;
    }
    return Chunk(b, n, macro_last);
}

int CheckSync(mplbgpu_batch* b) {
    int err = 0;
    BCK(cudaMemcpyAsync(&err, b->sync_err, sizeof(int), cudaMemcpyDeviceToHost,
                        b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    if (err) {
        cudaMemsetAsync(b->sync_err, 0, sizeof(int), b->stream);
        cudaMemsetAsync(b->sync_count, 0, sizeof(unsigned), b->stream);
        // the CTAs that gave up left their steps undone: the fields are a
        // mix of steps, so the batch needs a new initial state
        b->initialised = false;
        return BErr(b, MPLBGPU_ERR_TIMEOUT,
                    "a grid barrier of the persistent kernel gave up waiting "
                    "(the batch must be initialised again)");
    }
    return MPLBGPU_OK;
}

// Advances the active cavities by nsteps; moments written on the last step
// when macro_last.
int Advance(mplbgpu_batch* b, long long nsteps, bool macro_last) {
    long long done = 0;
    const int chunk = std::max(2, b->tune.chunk);
    while (nsteps - done >= chunk) {
        const bool last = macro_last && nsteps - done == chunk;
        int rc = GraphChunk(b, last);
        if (rc != MPLBGPU_OK) return rc;
        done += chunk;
    }
    if (nsteps > done) {
        int rc = Chunk(b, (int)(nsteps - done), macro_last);
        if (rc != MPLBGPU_OK) return rc;
    }
    long long active_nodes = 0;
    for (int c : b->active) active_nodes += (long long)b->cav[c].n * b->cav[c].n;
    b->node_updates += active_nodes * nsteps;
    return b->tune.persistent ? CheckSync(b) : MPLBGPU_OK;
}

void FreeBatch(mplbgpu_batch* b) {
    DropGraphs(b);
    cudaFree(b->dcav);
    cudaFree(b->pop[0]);
    cudaFree(b->pop[1]);
    for (int m = 0; m < 3; m++) {
        cudaFree(b->macro[m]);
        cudaFree(b->macro_old[m]);
    }
    cudaFree(b->tiles_all);
    cudaFree(b->tiles_active);
    cudaFree(b->ntiles_dev);
    cudaFree(b->part);
    cudaFree(b->ranges);
    cudaFree(b->res);
    cudaFree(b->sync_count);
    cudaFree(b->sync_gen);
    cudaFree(b->sync_err);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
}

}  // namespace

extern "C" {

mplbgpu_status mplbgpu_batch_create(const mplbgpu_cavity* cavities, int ncav,
                                    int precision, mplbgpu_batch** out) {
    mplbgpu_batch* b = nullptr;
    if (!cavities || !out || ncav < 1)
        return BErr(nullptr, MPLBGPU_ERR_INVALID, "no cavities");
    *out = nullptr;
    if (precision != MPLBGPU_FP64 && precision != MPLBGPU_FP32_SHIFTED)
        return BErr(nullptr, MPLBGPU_ERR_UNSUPPORTED,
                    "batched cavities run in FP64 or shifted FP32");
    b = new mplbgpu_batch;
    b->precision = precision;
    b->cav.assign(cavities, cavities + ncav);
    const double CS = std::sqrt(3.0);
    using L = Lattice<2>;
    const double w[3] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 36.0};
    const int esize = precision == MPLBGPU_FP64 ? 8 : 4;
    const long long align = 128 / esize;
    long long base = 0, mbase = 0;
    for (int c = 0; c < ncav; c++) {
        const mplbgpu_cavity& cv = cavities[c];
        if (cv.n < 3 || cv.n > 46340) {
            delete b;
            return BErr(nullptr, MPLBGPU_ERR_INVALID, "cavity side must be 3..46340");
        }
        const double dt = 1.0 / ((cv.n - 1) * CS);
        if (!(cv.tau_ref + 0.5 * dt > 0)) {
            delete b;
            return BErr(nullptr, MPLBGPU_ERR_INVALID, "tau_ref + dt/2 must be > 0");
        }
        BatchCav h{};
        h.base = base;
        h.mbase = mbase;
        h.n = cv.n;
        const double omega = dt / (cv.tau_ref + 0.5 * dt);
        h.omc = 1 - omega;
        h.omcf = (float)h.omc;
        h.ninv = 1.0f / (float)cv.n;
        h.dt = dt;
        for (int i = 0; i < 9; i++) {
            // 2 w_i (c_i . u_lid) in the halfway bounce-back's operation order
            const double cu = CS * (double)L::cx(i) * cv.lid_u +
                              CS * (double)L::cy(i) * 0.0;
            h.lidb[i] = 2.0 * w[L::wclass(i)] * cu;
            h.lidbf[i] = (float)h.lidb[i];
        }
        b->hcav.push_back(h);
        const long long nn = (long long)cv.n * cv.n;
        base += ((9 * nn + align - 1) / align) * align;
        mbase += nn;
    }
    if (base / align > 0x7fffffffLL) {   // tiles hold the offset in 32 bits
        delete b;
        return BErr(nullptr, MPLBGPU_ERR_INVALID, "batch too large");
    }
    // the cavities are checked before the device is looked for
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        delete b;
        return BErr(nullptr, MPLBGPU_ERR_NO_DEVICE, "no CUDA device");
    }
    b->pop_elems = base;
    b->total_nodes = mbase;
    mplbgpu_batch* bb = b;
    auto fail = [&](int code, const std::string& m) {
        FreeBatch(bb);
        delete bb;
        return BErr(nullptr, code, m);
    };
    cudaError_t e;
#define CRE(call)                                                  \
    if ((e = (call)) != cudaSuccess)                               \
        return fail(MPLBGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e));
    CRE(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    CRE(cudaEventCreate(&b->ev0));
    CRE(cudaEventCreate(&b->ev1));
    CRE(cudaMalloc(&b->dcav, ncav * sizeof(BatchCav)));
    CRE(cudaMemcpy(b->dcav, b->hcav.data(), ncav * sizeof(BatchCav),
                   cudaMemcpyHostToDevice));
    for (int k = 0; k < 2; k++) CRE(cudaMalloc(&b->pop[k], (size_t)base * esize));
    for (int m = 0; m < 3; m++) {
        CRE(cudaMalloc(&b->macro[m], (size_t)mbase * sizeof(double)));
        CRE(cudaMalloc(&b->macro_old[m], (size_t)mbase * sizeof(double)));
    }
    CRE(cudaMalloc(&b->ntiles_dev, sizeof(int)));
    CRE(cudaMalloc(&b->ranges, ncav * sizeof(int4)));
    CRE(cudaMalloc(&b->res, ncav * sizeof(double)));
    CRE(cudaMalloc(&b->sync_count, sizeof(unsigned)));
    CRE(cudaMalloc(&b->sync_gen, sizeof(unsigned)));
    CRE(cudaMalloc(&b->sync_err, sizeof(int)));
    CRE(cudaMemset(b->sync_count, 0, sizeof(unsigned)));
    CRE(cudaMemset(b->sync_gen, 0, sizeof(unsigned)));
    CRE(cudaMemset(b->sync_err, 0, sizeof(int)));
#undef CRE
    PhysConst& pc = b->pc;
    pc.cs = CS;
    pc.csf = (float)CS;
    for (int i = 0; i < 9; i++) {
        pc.w[i] = w[L::wclass(i)];
        pc.wf[i] = (float)pc.w[i];
        pc.winvf[i] = (float)(kHalfScale / pc.w[i]);
        pc.wlf[i] = (float)(pc.w[i] / kHalfScale);
    }
    pc.seed = 1;
    if (BuildTiles(b) != MPLBGPU_OK) {
        std::string m = b->err;
        return fail(MPLBGPU_ERR_CUDA, m);
    }
    for (int c = 0; c < ncav; c++) b->active.push_back(c);
    if (UploadActive(b) != MPLBGPU_OK) {
        std::string m = b->err;
        return fail(MPLBGPU_ERR_CUDA, m);
    }
    *out = b;
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_batch_destroy(mplbgpu_batch* b) {
    if (!b) return MPLBGPU_ERR_INVALID;
    cudaStreamSynchronize(b->stream);
    FreeBatch(b);
    delete b;
    return MPLBGPU_OK;
}

const char* mplbgpu_batch_last_error(const mplbgpu_batch* b) {
    return b ? b->err.c_str() : g_batch_create_error.c_str();
}

mplbgpu_status mplbgpu_batch_set_tuning(mplbgpu_batch* b,
                                        const mplbgpu_batch_tuning* t) {
    if (!b || !t) return MPLBGPU_ERR_INVALID;
    if (t->tile_nodes != 64 && t->tile_nodes != 128 && t->tile_nodes != 256)
        return BErr(b, MPLBGPU_ERR_INVALID, "tile_nodes must be 64, 128 or 256");
    if (b->precision != MPLBGPU_FP64 &&
        t->tile_nodes < 32 * BatchNodesPerThread<float>())
        return BErr(b, MPLBGPU_ERR_INVALID,
                    "tile_nodes too small for the FP32 form's nodes per thread");
    if (t->chunk < 2 || (t->chunk & 1))
        return BErr(b, MPLBGPU_ERR_INVALID, "chunk must be even and >= 2");
    if (t->persistent < 0 || t->persistent > 1)
        return BErr(b, MPLBGPU_ERR_INVALID, "persistent must be 0 or 1");
    if (t->ctas_per_sm < 1 || t->ctas_per_sm > 32)
        return BErr(b, MPLBGPU_ERR_INVALID, "ctas_per_sm must be 1..32");
    const bool retile = t->tile_nodes != b->tune.tile_nodes;
    b->tune = *t;
    DropGraphs(b);
    b->graph_ok = true;
    if (retile) {
        int rc = BuildTiles(b);
        if (rc != MPLBGPU_OK) return rc;
        return UploadActive(b);
    }
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_batch_set_wait_limit(mplbgpu_batch* b,
                                            long long polls) {
    if (!b) return MPLBGPU_ERR_INVALID;
    if (polls < 1)
        return BErr(b, MPLBGPU_ERR_INVALID, "the wait limit must be >= 1");
    b->wait_limit = polls;
    DropGraphs(b);   // captured persistent launches carry the old limit
    b->graph_ok = true;
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_batch_get_tuning(mplbgpu_batch* b,
                                        mplbgpu_batch_tuning* t) {
    if (!b || !t) return MPLBGPU_ERR_INVALID;
    *t = b->tune;
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_batch_init(mplbgpu_batch* b, const double* rho,
                                  const double* u, const double* v) {
    if (!b) return MPLBGPU_ERR_INVALID;
    const double* src[3] = {rho, u, v};
    std::vector<double> fill;
    for (int m = 0; m < 3; m++) {
        if (src[m]) {
            BCK(cudaMemcpyAsync(b->macro[m], src[m], b->total_nodes * sizeof(double),
                                cudaMemcpyDefault, b->stream));
        } else {
            fill.assign(b->total_nodes, m == 0 ? 1.0 : 0.0);
            BCK(cudaMemcpyAsync(b->macro[m], fill.data(),
                                b->total_nodes * sizeof(double),
                                cudaMemcpyHostToDevice, b->stream));
            BCK(cudaStreamSynchronize(b->stream));
        }
        BCK(cudaMemcpyAsync(b->macro_old[m], b->macro[m],
                            b->total_nodes * sizeof(double),
                            cudaMemcpyDeviceToDevice, b->stream));
    }
    b->cur = 0;
    b->active.clear();
    for (size_t c = 0; c < b->cav.size(); c++) b->active.push_back((int)c);
    int rc = UploadActive(b);
    if (rc != MPLBGPU_OK) return rc;
    const BatchDev d = MakeDev(b);
    cudaError_t e;
    if (b->precision == MPLBGPU_FP64)
        e = BatchLaunch<double>::Init(Grid(b, false), b->tune.tile_nodes, b->stream,
                                      d, b->pc, b->tiles_all, b->ntiles_all,
                                      static_cast<double*>(b->pop[0]));
    else
        e = BatchLaunch<float>::Init(Grid(b, false), b->tune.tile_nodes, b->stream,
                                     d, b->pc, b->tiles_all, b->ntiles_all,
                                     static_cast<float*>(b->pop[0]));
    b->launches++;
    if (e != cudaSuccess)
        return BErr(b, MPLBGPU_ERR_CUDA, std::string("init: ") + cudaGetErrorString(e));
    BCK(cudaStreamSynchronize(b->stream));
    b->initialised = true;
    b->device_ms = 0;
    b->node_updates = 0;
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_batch_step(mplbgpu_batch* b, int nsteps) {
    if (!b || nsteps < 0) return MPLBGPU_ERR_INVALID;
    if (!b->initialised) return BErr(b, MPLBGPU_ERR_STATE, "batch not initialised");
    BCK(cudaEventRecord(b->ev0, b->stream));
    int rc = Advance(b, nsteps, true);
    if (rc != MPLBGPU_OK) return rc;
    BCK(cudaEventRecord(b->ev1, b->stream));
    BCK(cudaEventSynchronize(b->ev1));
    float ms = 0;
    BCK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    b->device_ms += ms;
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_batch_run(mplbgpu_batch* b, long long max_steps,
                                 int check_period, double criterion,
                                 long long* steps, double* residual,
                                 int* converged) {
    if (!b || check_period < 1 || max_steps < 0) return MPLBGPU_ERR_INVALID;
    if (!b->initialised) return BErr(b, MPLBGPU_ERR_STATE, "batch not initialised");
    const size_t ncav = b->cav.size();
    std::vector<long long> st(ncav, 0);
    std::vector<double> rs(ncav, NAN);
    std::vector<int> cv(ncav, 0);
    std::vector<double> hres(ncav);
    long long done = 0;
    while (!b->active.empty() && done < max_steps) {
        const long long n = std::min<long long>(check_period, max_steps - done);
        BCK(cudaEventRecord(b->ev0, b->stream));
        int rc = Advance(b, n, true);
        if (rc != MPLBGPU_OK) return rc;
        done += n;
        const BatchDev d = MakeDev(b);
        BatchResidualPartialKernel<<<std::max(1, std::min(b->ntiles_active, 65535)),
                                     b->tune.tile_nodes, 0, b->stream>>>(d, b->part);
        BatchResidualFinalKernel<<<((int)b->active.size() + 127) / 128, 128, 0,
                                   b->stream>>>(d, b->part, b->ranges,
                                                (int)b->active.size(),
                                                (int)n, b->res);
        b->launches += 2;
        BCK(cudaGetLastError());
        BCK(cudaEventRecord(b->ev1, b->stream));
        BCK(cudaMemcpyAsync(hres.data(), b->res, b->active.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, b->stream));
        BCK(cudaStreamSynchronize(b->stream));
        float ms = 0;
        BCK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        b->device_ms += ms;
        std::vector<int> still;
        for (size_t k = 0; k < b->active.size(); k++) {
            const int c = b->active[k];
            st[c] += n;
            rs[c] = hres[k];
            if (std::isnan(hres[k])) cv[c] = -1;   // diverged: dropped
            else if (n == check_period && hres[k] < criterion) cv[c] = 1;
            else still.push_back(c);
        }
        if (still.size() != b->active.size()) {
            b->active = still;
            rc = UploadActive(b);
            if (rc != MPLBGPU_OK) return rc;
        }
    }
    for (size_t c = 0; c < ncav; c++) {
        if (steps) steps[c] = st[c];
        if (residual) residual[c] = rs[c];
        if (converged) converged[c] = cv[c];
    }
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_batch_download_macro(mplbgpu_batch* b, double* rho,
                                            double* u, double* v) {
    if (!b) return MPLBGPU_ERR_INVALID;
    double* dst[3] = {rho, u, v};
    for (int m = 0; m < 3; m++)
        if (dst[m])
            BCK(cudaMemcpyAsync(dst[m], b->macro[m], b->total_nodes * sizeof(double),
                                cudaMemcpyDefault, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    return MPLBGPU_OK;
}

mplbgpu_status mplbgpu_batch_stats(mplbgpu_batch* b, double* device_ms,
                                   long long* node_updates,
                                   long long* launches) {
    if (!b) return MPLBGPU_ERR_INVALID;
    if (device_ms) *device_ms = b->device_ms;
    if (node_updates) *node_updates = b->node_updates;
    if (launches) *launches = b->launches;
    return MPLBGPU_OK;
}

}  // extern "C"
