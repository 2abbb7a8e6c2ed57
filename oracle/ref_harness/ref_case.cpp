/*
 * Reference-case driver (TEST INFRASTRUCTURE ONLY).
 *
 * Runs the reference solver's own setup and time-step code, compiled against
 * the sequential OPS stand-in in ../ops_shim, on a case described in the
 * reference's JSON configuration format (Src/configuration.cpp:152-223), and
 * dumps the state for parity checks.  The setup sequence follows the apps'
 * simulate(const Configuration&) (Apps/3DCavity/lbm3d_cavity.cpp:151-185),
 * the time loop follows Iterate(criterion, checkPeriod)
 * (Src/evolution.cpp:102-135) but runs a fixed number of steps.
 *
 * Extra JSON keys read here (the reference leaves these to app code):
 *   "InitialMacroVars": {"rho": r, "u": u, "v": v, "w": w}   uniform start
 *   "BodyAcceleration": [ax, ay(, az)]                       uniform force
 *                       (set once before the first step and at every step)
 *
 * usage: ref_case <config.json> <outdir> <steps> [timing_steps]
 *   writes <outdir>/<var>_b<id>.f64 (moments after the last step, points
 *   ordered z,y,x), f_b<id>.f64 (distributions, point-major, 19 or 9 per
 *   point) and residual.txt (step, max residual, per-variable residuals at
 *   every check period).  With timing_steps > 0 it instead times that many
 *   StreamCollision calls after <steps> warm-up calls and prints
 *   "seconds <t> cells <n>".
 */
#include <chrono>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "mplb.h"
#include "ops_seq_v2.h"
#ifdef MPLB_DROPIN
// Built with MPLB_DROPIN the same driver runs the B200 path through the
// drop-in glue (mplb_b200/dropin) in place of the reference's
// StreamCollision / UpdateMacroVars / CalcResidualError.
#include "mplbgpu_dropin.h"
#endif

namespace {
Real g_rho0{1}, g_u0{0}, g_v0{0}, g_w0{0};
std::vector<Real> g_accel{0, 0, 0};
}  // namespace

#ifdef OPS_3D
void KerHarnessInitMacro(ACC<Real>& rho, ACC<Real>& u, ACC<Real>& v,
                         ACC<Real>& w, const Real* init) {
    rho(0, 0, 0) = init[0];
    u(0, 0, 0) = init[1];
    v(0, 0, 0) = init[2];
    w(0, 0, 0) = init[3];
}
void KerHarnessSetAccel(ACC<Real>& a, const Real* g) {
    a(0, 0, 0, 0) = g[0];
    a(1, 0, 0, 0) = g[1];
    a(2, 0, 0, 0) = g[2];
}
#endif
#ifdef OPS_2D
void KerHarnessInitMacro(ACC<Real>& rho, ACC<Real>& u, ACC<Real>& v,
                         const Real* init) {
    rho(0, 0) = init[0];
    u(0, 0) = init[1];
    v(0, 0) = init[2];
}
void KerHarnessSetAccel(ACC<Real>& a, const Real* g) {
    a(0, 0, 0) = g[0];
    a(1, 0, 0) = g[1];
}
#endif

void SetInitialMacrosVars() {
    const Real init[4]{g_rho0, g_u0, g_v0, g_w0};
    for (auto& idBlock : g_Block()) {
        const Block& block{idBlock.second};
        std::vector<int> rng(block.WholeRange().begin(),
                             block.WholeRange().end());
        const int b{block.ID()};
        for (auto& idCompo : g_Components()) {
            const Component& compo{idCompo.second};
            const int rhoId{compo.macroVars.at(Variable_Rho).id};
            ops_par_loop(
                KerHarnessInitMacro, "KerHarnessInitMacro", block.Get(),
                SpaceDim(), rng.data(),
                ops_arg_dat(g_MacroVars().at(rhoId).at(b), 1, LOCALSTENCIL,
                            "double", OPS_RW),
                ops_arg_dat(g_MacroVars().at(compo.uId).at(b), 1,
                            LOCALSTENCIL, "double", OPS_RW),
                ops_arg_dat(g_MacroVars().at(compo.vId).at(b), 1,
                            LOCALSTENCIL, "double", OPS_RW),
#ifdef OPS_3D
                ops_arg_dat(g_MacroVars().at(compo.wId).at(b), 1,
                            LOCALSTENCIL, "double", OPS_RW),
#endif
                ops_arg_gbl(init, 4, "double", OPS_READ));
        }
    }
}

void UpdateMacroscopicBodyForce(const Real /*time*/) {
    for (auto& idBlock : g_Block()) {
        const Block& block{idBlock.second};
        std::vector<int> rng(block.WholeRange().begin(),
                             block.WholeRange().end());
        const int b{block.ID()};
        for (auto& force : g_MacroBodyforce()) {
            ops_par_loop(KerHarnessSetAccel, "KerHarnessSetAccel",
                         block.Get(), SpaceDim(), rng.data(),
                         ops_arg_dat(force.second.at(b), SpaceDim(),
                                     LOCALSTENCIL, "double", OPS_WRITE),
                         ops_arg_gbl(g_accel.data(), 3, "double", OPS_READ));
        }
    }
}

static void UpdateMacro() {
#ifdef MPLB_DROPIN
    if (mplbgpu_dropin::Active()) {
        mplbgpu_dropin::UpdateMacroVars();
        return;
    }
#endif
#ifdef OPS_3D
    UpdateMacroVars3D();
#else
    UpdateMacroVars();
#endif
}

// The case's "SchemeType": Scheme_StreamCollision_Swap selects the
// reference's one-array swap step (Src/evolution.cpp:195-252).
bool g_swapScheme{false};

static void Step(Real time) {
#ifdef MPLB_DROPIN
    mplbgpu_dropin::StreamCollision(time);
#else
    if (g_swapScheme) {
        SwapStreamCollision(time);
        return;
    }
    StreamCollision(time);
#endif
}

static void Residual() {
#ifdef MPLB_DROPIN
    if (mplbgpu_dropin::Active()) {
        mplbgpu_dropin::CalcResidualError();
        return;
    }
#endif
    CalcResidualError();
}

static void DumpDat(ops_dat dat, const Block& block, const std::string& path) {
    const std::vector<int>& n{block.Size()};
    const int nz{SpaceDim() == 3 ? n.at(2) : 1};
    std::ofstream out(path, std::ios::binary);
    for (int k = 0; k < nz; k++) {
        for (int j = 0; j < n.at(1); j++) {
            for (int i = 0; i < n.at(0); i++) {
                const char* p = ops_shim_point_ptr(dat, i, j, k);
                out.write(p, (std::streamsize)dat->dim * dat->elem_size);
            }
        }
    }
}

int main(int argc, const char** argv) {
    if (argc < 4) {
        std::fprintf(stderr,
                     "usage: %s config.json outdir steps [timing_steps]\n",
                     argv[0]);
        return 2;
    }
    ops_init(argc, argv, 1);
    std::string configFile{argv[1]};
    const std::string outDir{argv[2]};
    const long steps{std::atol(argv[3])};
    const long timingSteps{argc > 4 ? std::atol(argv[4]) : 0};

    ReadConfiguration(configFile);
    const Configuration& config{Config()};
    const nlohmann::json& js{JsonConfig()};
    g_swapScheme = config.schemeType == Scheme_StreamCollision_Swap;
    if (js.contains("InitialMacroVars")) {
        const auto& im = js["InitialMacroVars"];
        if (im.contains("rho")) g_rho0 = im["rho"].get<Real>();
        if (im.contains("u")) g_u0 = im["u"].get<Real>();
        if (im.contains("v")) g_v0 = im["v"].get<Real>();
        if (im.contains("w")) g_w0 = im["w"].get<Real>();
    }
    if (js.contains("BodyAcceleration")) {
        std::vector<Real> a = js["BodyAcceleration"].get<std::vector<Real>>();
        for (size_t i = 0; i < a.size() && i < 3; i++) g_accel[i] = a[i];
    }

    DefineCase(config.caseName, config.spaceDim, config.transient);
    DefineBlocks(config.blockIds, config.blockNames, config.blockSize,
                 config.meshSize, config.startPos);
    if (!config.fromBlockIds.empty()) {
        DefineBlockConnection(config.fromBlockIds, config.fromBoundarySurface,
                              config.toBlockIds, config.toBoundarySurface,
                              config.blockConnectionType);
    }
    DefineComponents(config.compoNames, config.compoIds, config.lattNames,
                     config.tauRef, 0);
    DefineMacroVars(config.macroVarTypes, config.macroVarNames,
                    config.macroVarIds, config.macroCompoIds, 0);
    DefineCollision(config.CollisionTypes, config.CollisionCompoIds);
    DefineBodyForce(config.bodyForceTypes, config.bodyForceCompoIds);
    DefineScheme(config.schemeType);
    DefineInitialCondition(config.initialTypes, config.initialConditionCompoId);
    for (auto& bc : config.blockBoundaryConfig) {
        if (bc.boundaryScheme == BoundaryScheme::None &&
            bc.boundaryType == VertexType::VirtualBoundary) {
            DefineBlockBoundary(bc.blockIndex, bc.componentID,
                                bc.boundarySurface, bc.boundaryType);
        } else {
            DefineBlockBoundary(bc.blockIndex, bc.componentID,
                                bc.boundarySurface, bc.boundaryScheme,
                                bc.macroVarTypesatBoundary, bc.givenVars,
                                bc.boundaryType);
        }
    }
    Partition();
    SetInitialMacrosVars();
#ifdef OPS_3D
    PreDefinedInitialCondition3D();
#else
    PreDefinedInitialCondition();
#endif
    SetTimeStep(config.meshSize / SoundSpeed());
    // The uniform acceleration field is in place from the first step (the
    // apps' hook is otherwise first called after step 1's moments).
    UpdateMacroscopicBodyForce(0);

    if (timingSteps > 0) {
        for (long it = 0; it < steps; it++) Step(it * TimeStep());
        const auto t0 = std::chrono::steady_clock::now();
        for (long it = 0; it < timingSteps; it++) {
            Step((steps + it) * TimeStep());
        }
#ifdef MPLB_DROPIN
        mplbgpu_dropin::Synchronize();   // the GPU steps are queued only
#endif
        const auto t1 = std::chrono::steady_clock::now();
        long cells{0};
        for (auto& idBlock : g_Block()) {
            long c{1};
            for (int s : idBlock.second.Size()) c *= s;
            cells += c;
        }
        std::printf("seconds %.9f cells %ld steps %ld\n",
                    std::chrono::duration<double>(t1 - t0).count(), cells,
                    timingSteps);
        return 0;
    }

    std::ofstream res(outDir + "/residual.txt");
    res.precision(17);
    for (long it = 0; it < steps; it++) {
        Step(it * TimeStep());
        const long done{it + 1};
        if (!config.transient && done % (long)config.checkPeriod == 0) {
            UpdateMacro();
            Residual();
            const Real maxRes{GetMaximumResidual(config.checkPeriod)};
            res << done << " " << maxRes;
            for (auto& e : g_ResidualError()) res << " " << e.second;
            res << "\n";
        }
    }
    UpdateMacro();
    for (auto& idBlock : g_Block()) {
        const Block& block{idBlock.second};
        const int b{block.ID()};
        for (auto& idCompo : g_Components()) {
            for (auto& mv : idCompo.second.macroVars) {
                DumpDat(g_MacroVars().at(mv.second.id).at(b), block,
                        outDir + "/" + mv.second.name + "_b" +
                            std::to_string(b) + ".f64");
            }
        }
        DumpDat(g_f().at(b), block,
                outDir + "/f_b" + std::to_string(b) + ".f64");
    }
    ops_exit();
    return 0;
}
