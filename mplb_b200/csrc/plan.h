// Host-side planning of the fused stream-collision step.
//
// MPLB assigns every node a VertexType and a VertexGeometryType
// (PrepareFlowField, Src/flowfield.cpp:224-244) and applies boundary
// kernels surface by surface in definition order (ImplementBoundary3D,
// Src/boundary.cpp:379-386).  Every node range the reference uses (bulk,
// halo shells, faces, edges, corners, the VirtualBoundary-shrunk faces) is
// a union of the 3^D "regions" of a block - each axis split into
// {first node, interior, last node} - so all per-node semantics are
// resolved here once per region:
//   PURE     : fluid-like node with no boundary kernel: pull all Q
//              populations, moments, BGK collision.
//   LOCAL    : boundary node whose boundary kernels only read the node
//              itself: pulled populations + a short in-register program of
//              EQMDiffuseRefl / halfway bounce-back operations.
//   DEFERRED : node whose program reads a neighbour's post-boundary value
//              (ExtrapolPressure1ST) or is read by one: processed by the
//              sequential deferred kernels on an explicit f store.
// The halo transfer plan reproduces Field::CreateHalos order
// (Src/field.h:215-395), copying only populations that point into the
// destination block.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mplbgpu.h"

namespace mplb {

constexpr int kMaxQ = 19;
constexpr int kMaxOps = 4;
constexpr int kNumRegions = 27;

enum NodeClass : int { kPure = 0, kLocal = 1, kDeferred = 2 };
// kOpZero: FDPeriodic, which sets every population of the node to the
// value of a halo cell of f that no step writes (zero)
enum OpKind : int { kOpEqm = 1, kOpHbb = 2, kOpExtrapol = 3, kOpZero = 4 };

// One boundary operation specialised to one region's geometry.  All FP64
// constants that depend only on the boundary's given values are computed
// here in the reference's operation order.
struct RegionOp {
    int kind;
    int bc;             // index of the boundary (definition order)
    uint32_t in_mask;   // EQM: incoming;  EXTRAPOL: copied populations
    uint32_t out_mask;  // EQM: outgoing;  HBB: bounced populations
    uint32_t par_mask;  // EQM: parallel
    int nb_axis;        // EXTRAPOL copy source axis (-1: none)
    int nb_sign;
    double denom;       // EQM: (1 - deltaRho) - rhoParallel
    double win;         // EQM: sum of the incoming weights (shifted forms)
    double c0;          // EQM: 2 win - denom, so rhoWall - 1 =
                        //      (c0 + 2 sum_in h) / denom (shifted forms)
    double am1[kMaxQ];  // EQM: a - 1 per parallel population (shifted)
    double rho_given;   // EXTRAPOL
    double a[kMaxQ];    // EQM: feq(1,u_w)/w per parallel population (res)
    double b[kMaxQ];    // EQM: c.u_w per outgoing; HBB: 2 w (c.u_w)
    // the shifted forms' FP32 copies: 1 / (float)denom, (float)c0 and the
    // arrays above rounded to float (SetFloatConsts)
    float invf, c0f;
    float am1f[kMaxQ], af[kMaxQ], bf[kMaxQ];
    // EQM / HBB with a wall velocity per node (mplbgpu_set_boundary_velocity):
    // this operation evaluated for every node of the boundary's surface
    // range (x fastest, from node forg) with that node's velocity; null:
    // the constants above (uniform given values) hold for every node
    const RegionOp* node_ops;
    int forg[3];
    int fext[3];
};

struct RegionInfo {
    int cls;            // NodeClass; -1 for an empty region
    int vt;             // VertexType
    int vg;             // VertexGeometryType
    int fluidlike;      // Fluid or MDPeriodic: body force + force velocity
    uint32_t pull;      // populations taken from the upstream node
    uint32_t stale;     // LOCAL: populations neither pulled nor written
    int nops;
    int op[kMaxOps];    // indices into BlockPlan::ops
    int ext[3];         // node extent of the region per axis
    int org[3];         // first node of the region per axis
    long long side_base;  // first index in the stale or deferred store
};

struct DeferredSegment {
    int region;
    int op;             // index into BlockPlan::ops
};

struct DeferredOp {     // one boundary (definition order) on deferred nodes
    std::vector<DeferredSegment> segments;
};

struct BlockPlan {
    int id;
    int index;          // position in id order
    int cut;            // bit s: surface s continues in another context
    int n[3];
    int xoff;           // element index of x = 0 inside a row
    long long pitch;    // elements per row
    long long plane;    // elements per z plane (with y halo)
    long long popstride;// elements per population (with halos)
    RegionInfo region[kNumRegions];
    std::vector<RegionOp> ops;
    long long nstale;   // nodes with a stale store
    long long ndeferred;
    std::vector<DeferredOp> dops;
    // every deferred node's programme in one pass is possible when no
    // ExtrapolPressure1ST of a deferred node reads a deferred neighbour:
    // per deferred region its operations (definition order, -1 ended)
    bool deferred_fused = false;
    std::vector<int> dops_flat;
    int dops_first[kNumRegions] = {};
    std::vector<int> allops[kNumRegions];  // every op of a region (host)
    // swap scheme: per region, slot k of a node holds population
    // swap_sigma[r][k] of the collided node after its local swap, and
    // swap_exch[r] bit k says that slot k lives at slot opp(k) of the
    // upstream node x - c_k instead of the node's own slot k
    uint8_t swap_sigma[kNumRegions][kMaxQ];
    uint32_t swap_exch[kNumRegions];
    bool any_deferred() const { return ndeferred > 0; }
    long long nodes() const { return (long long)n[0] * n[1] * n[2]; }
};

struct HaloCopy {
    int from, to;       // block indices (id order)
    int axis;
    int to_low;         // 1: destination layer is -1 (from Right/Top/Front)
    int iter[3];
    int fbase[3];
    int tbase[3];
    uint32_t pops;      // populations copied
    std::vector<uint8_t> prev;  // per box cell: read the previous array
    bool any_prev;
    // Fused transfer (all copies in one launch): a cell whose source no
    // earlier copy writes and whose destination no other copy writes is
    // copied by its box; the others (`ordered`) are left to the resolved
    // element copies of Plan::halo_elems.
    std::vector<uint8_t> ordered;   // per box cell: 1 = resolved elsewhere
    long long nordered = 0;
};

// One population of one halo cell whose value the copies of a step produce
// through more than one copy (a destination written twice, a source
// written earlier): the final value's origin, resolved by following the
// copies in definition order, so that it can be copied directly and in any
// order (the origin is a place no copy of the step writes, read from the
// current array, or from the previous one where the reference reads a
// value that a later copy overwrites).
struct HaloElem {
    int to, tx, ty, tz;       // destination block and node (halo included)
    int from, fx, fy, fz;     // origin block and node
    int pop;
    int prev;                 // 1: the origin is read from the previous array
};

struct Plan {
    std::vector<HaloElem> halo_elems;   // resolved element copies
    int dim = 3;
    int Q = 19;
    int precision = MPLBGPU_FP64;
    int elem_bytes = 8;
    double cs = 0, tau = 0, dt = 0;
    double omega = 0;   // dt / (tau + dt/2)
    double omc = 0;     // 1 - omega
    double tw = 0;      // tau * omega
    int body_force = 0;
    int force_velocity = 0;
    double accel[3] = {0, 0, 0};
    double hdta[3] = {0, 0, 0};  // dt * a / 2
    double cf[kMaxQ] = {};       // CS c_i . a  (CalcBodyForce sum)
    double w[kMaxQ] = {};
    int swap = 0;       // Scheme_StreamCollision_Swap: one population array
    std::vector<BlockPlan> blocks;  // sorted by id
    std::vector<HaloCopy> halos;
    // per boundary (definition order): its block's index and its surface
    // range [r0, r1) x [r2, r3) x [r4, r5) (Block::BoundarySurfaceRange)
    std::vector<int> bc_block;
    std::vector<int> bc_range;
    std::vector<int> bc_scheme;
    std::vector<int> bc_surface;
};

// Builds the plan; returns MPLBGPU_OK or an error code with a message.
int BuildPlan(const mplbgpu_desc& desc, Plan* plan, std::string* err);

// Boundary `boundary` (EQMDiffuseRefl or halfway bounce-back) evaluated
// per node of its surface range with a per-node wall velocity `uvw`
// (u, v, w per node, x fastest): each node's operation has the masks of its
// region and the constants of its own velocity, computed as the uniform
// operations are.
int BoundaryNodeOps(const Plan& P, int boundary, const double* uvw,
                    std::vector<RegionOp>* out, std::string* err);

// Region of coordinate v on an axis of n nodes: 0 first, 2 last, 1 inside.
inline int RegionCoord(int v, int n) {
    return v == 0 ? 0 : (v == n - 1 ? 2 : 1);
}

}  // namespace mplb
