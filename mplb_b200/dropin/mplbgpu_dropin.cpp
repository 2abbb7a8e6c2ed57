// Drop-in glue between MPLB's setup/iteration API and the C ABI
// (include/mplbgpu.h).  See mplbgpu_dropin.h.
#include "mplbgpu_dropin.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

#include "boundary.h"
#include "flowfield.h"
#include "model.h"
#include "mplbgpu.h"
#include "scheme.h"

namespace mplbgpu_dropin {
namespace {

mplbgpu_ctx* g_ctx = nullptr;

void Check(mplbgpu_status st, const char* what) {
    if (st != MPLBGPU_OK) {
        ops_printf("MPLB B200 path: %s failed (%d): %s\n", what, st,
                   mplbgpu_last_error(g_ctx));
        std::fflush(stdout);
        assert(st == MPLBGPU_OK);
        std::abort();
    }
}

int Precision() {
    const char* p = std::getenv("MPLB_B200_PRECISION");
    if (p == nullptr) return MPLBGPU_FP64;
    const std::string s{p};
    if (s == "fp32") return MPLBGPU_FP32_SHIFTED;
    if (s == "fp16") return MPLBGPU_FP16_SHIFTED;
    return MPLBGPU_FP64;
}

const Component& TheComponent() {
    if (g_Components().size() != 1) {
        ops_printf("MPLB B200 path: exactly one component is supported\n");
        assert(g_Components().size() == 1);
    }
    return g_Components().begin()->second;
}

long long Nodes(const Block& block) {
    long long n = 1;
    for (int s : block.Size()) n *= s;
    return n;
}

// Index (0 rho, 1 u, 2 v, 3 w) of a macroscopic variable type, or -1.
int MacroSlot(int type) {
    switch (type) {
        case Variable_Rho: return 0;
        case Variable_U: case Variable_U_Force: return 1;
        case Variable_V: case Variable_V_Force: return 2;
        case Variable_W: case Variable_W_Force: return 3;
        default: return -1;
    }
}

void Create(Real time) {
    const Component& compo = TheComponent();
    std::vector<mplbgpu_block> blocks;
    std::vector<mplbgpu_connection> conns;
    for (const auto& idBlock : g_Block()) {
        const Block& block = idBlock.second;
        mplbgpu_block b{};
        b.id = block.ID();
        for (int a = 0; a < 3; a++)
            b.size[a] = a < SpaceDim() ? block.Size().at(a) : 1;
        blocks.push_back(b);
        for (const auto& sn : block.Neighbors()) {
            mplbgpu_connection c{};
            c.from_block = block.ID();
            c.from_surface = (int)sn.first;
            c.to_block = sn.second.blockId;
            c.to_surface = (int)sn.second.surface;
            c.type = (int)sn.second.type;
            conns.push_back(c);
        }
    }
    std::vector<mplbgpu_boundary> bcs;
    for (const BlockBoundary& bb : BlockBoundaries()) {
        mplbgpu_boundary b{};
        b.block = bb.blockIndex;
        b.surface = (int)bb.boundarySurface;
        b.scheme = (int)bb.boundaryScheme;
        b.vertex_type = (int)bb.boundaryType;
        for (size_t k = 0; k < bb.givenVars.size() && k < 3; k++)
            b.given[k] = bb.givenVars[k];
        bcs.push_back(b);
    }
    mplbgpu_desc d{};
    d.abi_version = MPLBGPU_ABI_VERSION;
    d.space_dim = SpaceDim();
    d.lattice = NUMXI;
    d.precision = Precision();
    d.nblocks = (int)blocks.size();
    d.blocks = blocks.data();
    d.nconnections = (int)conns.size();
    d.connections = conns.data();
    d.nboundaries = (int)bcs.size();
    d.boundaries = bcs.data();
    d.tau_ref = compo.tauRef;
    d.dt = TimeStep();
    d.cs = SoundSpeed();
    // the _Swap force types add the same first-order term after the
    // collision instead of inside it; the scheme tells the two apart
    d.body_force = (compo.bodyForceType == BodyForce_1st ||
                    compo.bodyForceType == BodyForce_1st_Swap)
                       ? MPLBGPU_FORCE_1ST
                       : MPLBGPU_FORCE_NONE;
    d.scheme = (int)Scheme();
    d.force_velocity =
        compo.macroVars.count(Variable_U_Force) ? 1 : 0;
    // uniform body acceleration: the force field's first node
    if (g_MacroBodyforce().count(compo.id)) {
        const Block& first = g_Block().begin()->second;
        std::vector<Real> acc((size_t)Nodes(first) * SpaceDim());
        ops_dat_fetch_data(g_MacroBodyforce().at(compo.id).at(first.ID()), 0,
                           reinterpret_cast<char*>(acc.data()));
        for (int a = 0; a < SpaceDim(); a++) d.accel[a] = acc[a];
    }
    Check(mplbgpu_create(&d, &g_ctx), "mplbgpu_create");
    for (const auto& idBlock : g_Block()) {
        const Block& block = idBlock.second;
        if (time == 0) {
            // fresh start: f is feq of the initial macroscopic fields
            // (PreDefinedInitialCondition3D), which are also the residual's
            // previous values; rebuilding f from them keeps both
            std::vector<Real> q[4];
            const double* p[4] = {nullptr, nullptr, nullptr, nullptr};
            for (const auto& tv : compo.macroVars) {
                const int m = MacroSlot(tv.first);
                if (m < 0 || m > SpaceDim()) continue;
                q[m].resize((size_t)Nodes(block));
                ops_dat_fetch_data(g_MacroVars().at(tv.second.id).at(block.ID()),
                                   0, reinterpret_cast<char*>(q[m].data()));
                p[m] = q[m].data();
            }
            Check(mplbgpu_init_macro(g_ctx, block.ID(), p[0], p[1], p[2], p[3]),
                  "mplbgpu_init_macro");
            continue;
        }
        // restart: the distributions as read back by the reference
        std::vector<Real> f((size_t)Nodes(block) * NUMXI);
        ops_dat_fetch_data(g_f().at(block.ID()), 0,
                           reinterpret_cast<char*>(f.data()));
        Check(mplbgpu_upload_f(g_ctx, block.ID(), f.data()), "mplbgpu_upload_f");
    }
    // a restart continues from its CurrentTimeStep (time = step * dt)
    if (time != 0)
        Check(mplbgpu_set_step(g_ctx, std::llround(time / TimeStep())),
              "mplbgpu_set_step");
}

}  // namespace

bool Active() { return g_ctx != nullptr; }

void StreamCollision(const Real time) {
    if (g_ctx == nullptr) Create(time);
    Check(mplbgpu_step(g_ctx, 1), "mplbgpu_step");
}

void SwapStreamCollision(const Real time) { StreamCollision(time); }

void UpdateMacroVars() {
    Check(mplbgpu_update_macro(g_ctx), "mplbgpu_update_macro");
    const Component& compo = TheComponent();
    const char* sync = std::getenv("MPLB_B200_SYNC_F");
    const bool syncf = sync == nullptr || sync[0] != '0';
    for (const auto& idBlock : g_Block()) {
        const Block& block = idBlock.second;
        const size_t n = (size_t)Nodes(block);
        std::vector<Real> q[4];
        for (auto& v : q) v.resize(n);
        Check(mplbgpu_download_macro(g_ctx, block.ID(), q[0].data(),
                                     q[1].data(), q[2].data(), q[3].data()),
              "mplbgpu_download_macro");
        for (const auto& tv : compo.macroVars) {
            const int m = MacroSlot(tv.first);
            if (m < 0 || m > SpaceDim()) continue;
            ops_dat_set_data(g_MacroVars().at(tv.second.id).at(block.ID()), 0,
                             reinterpret_cast<char*>(q[m].data()));
        }
        if (syncf) {
            std::vector<Real> f(n * NUMXI);
            Check(mplbgpu_download_f(g_ctx, block.ID(), f.data()),
                  "mplbgpu_download_f");
            ops_dat_set_data(g_f().at(block.ID()), 0,
                             reinterpret_cast<char*>(f.data()));
        }
    }
}

void CalcResidualError() {
    double per[4] = {0, 0, 0, 0};
    double mx = 0;
    Check(mplbgpu_residual(g_ctx, 1, per, &mx), "mplbgpu_residual");
    const Component& compo = TheComponent();
    for (const auto& tv : compo.macroVars) {
        const int m = MacroSlot(tv.first);
        if (m >= 0 && m <= SpaceDim()) g_ResidualError().at(tv.second.id) = per[m];
    }
}

void Synchronize() {
    if (g_ctx) Check(mplbgpu_synchronize(g_ctx), "mplbgpu_synchronize");
}

void Release() {
    if (g_ctx) mplbgpu_destroy(g_ctx);
    g_ctx = nullptr;
}

}  // namespace mplbgpu_dropin
