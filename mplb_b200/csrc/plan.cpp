// Host-side planning of the fused stream-collision step (see plan.h).
// Compiled with -ffp-contract=off: the FP64 constants below are computed in
// the reference's operation order so that kernels using them reproduce the
// reference bit for bit.
#include "plan.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>

#include "lattice.h"

namespace mplb {
namespace {

constexpr int kVtFluid = MPLBGPU_VT_FLUID;
constexpr int kVtMD = MPLBGPU_VT_MDPERIODIC;
constexpr int kVtVB = MPLBGPU_VT_VIRTUAL_BOUNDARY;
constexpr int kVtSolid = MPLBGPU_VT_IMMERSED_SOLID;

enum { kDvIncoming = 1, kDvOutgoing = 2, kDvParallel = 3, kDvInvalid = -1 };

struct Lat {
    int D, Q;
    int c[kMaxQ][3];
    int opp[kMaxQ];
    double w[kMaxQ];
};

template <int D>
void FillLat(Lat* L) {
    using LL = Lattice<D>;
    L->D = D;
    L->Q = LL::Q;
    for (int i = 0; i < LL::Q; i++) {
        L->c[i][0] = LL::cx(i);
        L->c[i][1] = LL::cy(i);
        L->c[i][2] = LL::cz(i);
        L->opp[i] = LL::opp(i);
    }
    // SetupD2Q9Latt / SetupD3Q19Latt, Src/model.cpp:99-131
    double cls[3];
    if (D == 2) {
        cls[0] = 4.0 / 9.0;
        cls[1] = 1.0 / 9.0;
        cls[2] = 1.0 / 36.0;
    } else {
        cls[0] = 1 / ((double)3);
        cls[1] = 1 / ((double)18);
        cls[2] = 1 / ((double)36);
    }
    for (int i = 0; i < LL::Q; i++) L->w[i] = cls[LL::wclass(i)];
}

// CalcBGKFeq(l, rho, u, v[, w], T = 1, polyOrder = 2) / (w_l rho):
// the bracket "res" of Src/model_host_device.h:34-82, same operation order.
double FeqRes(const Lat& L, double CS, int l, const double* u) {
    const double T = 1;
    const double XI0 = L.c[l][0], XI1 = L.c[l][1], XI2 = L.c[l][2];
    double cu, c2, u2;
    if (L.D == 2) {
        cu = (CS * XI0 * u[0] + CS * XI1 * u[1]);
        c2 = (CS * XI0 * CS * XI0 + CS * XI1 * CS * XI1);
        u2 = u[0] * u[0] + u[1] * u[1];
    } else {
        cu = (CS * XI0 * u[0] + CS * XI1 * u[1] + CS * XI2 * u[2]);
        c2 = (CS * XI0 * CS * XI0 + CS * XI1 * CS * XI1 + CS * XI2 * CS * XI2);
        u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    }
    const double cu2 = cu * cu;
    return 1.0 + cu + 0.5 * (cu2 - u2 + (T - 1.0) * (c2 - L.D));
}

// Block::RangeStart / RangeEnd (Src/block.cpp:14-97), including the
// TopBack/TopFront y-range left whole by the OP_3D test at Src/block.cpp:35.
void SurfaceRange(int dim, const int n[3], int s, int r[6]) {
    for (int a = 0; a < 3; a++) {
        r[2 * a] = 0;
        r[2 * a + 1] = n[a];
    }
    const bool d3 = dim == 3;
    if (s == MPLBGPU_RIGHT || s == MPLBGPU_RIGHT_TOP ||
        s == MPLBGPU_RIGHT_BOTTOM ||
        (d3 && (s == MPLBGPU_RIGHT_FRONT || s == MPLBGPU_RIGHT_BACK)))
        r[0] = n[0] - 1;
    if (s == MPLBGPU_LEFT || s == MPLBGPU_LEFT_BOTTOM || s == MPLBGPU_LEFT_TOP ||
        (d3 && (s == MPLBGPU_LEFT_FRONT || s == MPLBGPU_LEFT_BACK)))
        r[1] = 1;
    if (s == MPLBGPU_TOP || s == MPLBGPU_LEFT_TOP || s == MPLBGPU_RIGHT_TOP)
        r[2] = n[1] - 1;
    if (s == MPLBGPU_BOTTOM || s == MPLBGPU_LEFT_BOTTOM ||
        s == MPLBGPU_RIGHT_BOTTOM ||
        (d3 && (s == MPLBGPU_BOTTOM_BACK || s == MPLBGPU_BOTTOM_FRONT)))
        r[3] = 1;
    if (d3) {
        if (s == MPLBGPU_FRONT || s == MPLBGPU_LEFT_FRONT ||
            s == MPLBGPU_RIGHT_FRONT || s == MPLBGPU_TOP_FRONT ||
            s == MPLBGPU_BOTTOM_FRONT)
            r[4] = n[2] - 1;
        if (s == MPLBGPU_BACK || s == MPLBGPU_LEFT_BACK ||
            s == MPLBGPU_RIGHT_BACK || s == MPLBGPU_TOP_BACK ||
            s == MPLBGPU_BOTTOM_BACK)
            r[5] = 1;
    }
}

bool ValidSurface(int dim, int s) {
    switch (s) {
        case MPLBGPU_LEFT: case MPLBGPU_RIGHT: case MPLBGPU_TOP:
        case MPLBGPU_BOTTOM: case MPLBGPU_LEFT_TOP: case MPLBGPU_LEFT_BOTTOM:
        case MPLBGPU_RIGHT_TOP: case MPLBGPU_RIGHT_BOTTOM:
            return true;
        case MPLBGPU_FRONT: case MPLBGPU_BACK: case MPLBGPU_LEFT_BACK:
        case MPLBGPU_LEFT_FRONT: case MPLBGPU_RIGHT_BACK:
        case MPLBGPU_RIGHT_FRONT: case MPLBGPU_TOP_BACK:
        case MPLBGPU_TOP_FRONT: case MPLBGPU_BOTTOM_BACK:
        case MPLBGPU_BOTTOM_FRONT:
            return dim == 3;
        default:
            return false;
    }
}

// Faces making up a surface or edge: axis and side (0 min, 1 max).
int SurfaceFaces(int s, int axis[2], int side[2]) {
    struct F { int s, a, sd; };
    static const F tab[] = {
        {MPLBGPU_LEFT, 0, 0}, {MPLBGPU_RIGHT, 0, 1}, {MPLBGPU_BOTTOM, 1, 0},
        {MPLBGPU_TOP, 1, 1}, {MPLBGPU_BACK, 2, 0}, {MPLBGPU_FRONT, 2, 1},
        {MPLBGPU_LEFT_BACK, 0, 0}, {MPLBGPU_LEFT_BACK, 2, 0},
        {MPLBGPU_LEFT_FRONT, 0, 0}, {MPLBGPU_LEFT_FRONT, 2, 1},
        {MPLBGPU_RIGHT_BACK, 0, 1}, {MPLBGPU_RIGHT_BACK, 2, 0},
        {MPLBGPU_RIGHT_FRONT, 0, 1}, {MPLBGPU_RIGHT_FRONT, 2, 1},
        {MPLBGPU_TOP_BACK, 1, 1}, {MPLBGPU_TOP_BACK, 2, 0},
        {MPLBGPU_TOP_FRONT, 1, 1}, {MPLBGPU_TOP_FRONT, 2, 1},
        {MPLBGPU_BOTTOM_BACK, 1, 0}, {MPLBGPU_BOTTOM_BACK, 2, 0},
        {MPLBGPU_BOTTOM_FRONT, 1, 0}, {MPLBGPU_BOTTOM_FRONT, 2, 1},
        {MPLBGPU_LEFT_TOP, 0, 0}, {MPLBGPU_LEFT_TOP, 1, 1},
        {MPLBGPU_LEFT_BOTTOM, 0, 0}, {MPLBGPU_LEFT_BOTTOM, 1, 0},
        {MPLBGPU_RIGHT_TOP, 0, 1}, {MPLBGPU_RIGHT_TOP, 1, 1},
        {MPLBGPU_RIGHT_BOTTOM, 0, 1}, {MPLBGPU_RIGHT_BOTTOM, 1, 0},
    };
    int n = 0;
    for (const F& f : tab) {
        if (f.s == s && n < 2) {
            axis[n] = f.a;
            side[n] = f.sd;
            n++;
        }
    }
    return n;
}

bool InRange(const int p[3], const int r[6]) {
    return p[0] >= r[0] && p[0] < r[1] && p[1] >= r[2] && p[1] < r[3] &&
           p[2] >= r[4] && p[2] < r[5];
}

// Surface (BoundarySurface) of the min (side 0) or max (side 1) face of an
// axis.
int FaceSurface(int axis, int side) {
    static const int tab[3][2] = {{MPLBGPU_LEFT, MPLBGPU_RIGHT},
                                  {MPLBGPU_BOTTOM, MPLBGPU_TOP},
                                  {MPLBGPU_BACK, MPLBGPU_FRONT}};
    return tab[axis][side];
}

// Boundary faces of a node: axes on which it is the first/last node, with
// the inward sign (+1 on the first node: the "P" codes).  Faces in `cut`
// (bit s: surface s continues into a block of another context) are not
// boundaries: the node is interior there.
int NodeFaces(int dim, const int n[3], const int p[3], int axis[3],
              int sign[3], int cut = 0) {
    int k = 0;
    for (int a = 0; a < dim; a++) {
        if (p[a] == 0 && !(cut >> FaceSurface(a, 0) & 1)) {
            axis[k] = a;
            sign[k++] = 1;
        } else if (p[a] == n[a] - 1 && !(cut >> FaceSurface(a, 1) & 1)) {
            axis[k] = a;
            sign[k++] = -1;
        }
    }
    return k;
}

// VertexGeometryType of a node from its position: the code written last by
// SetBlockGeometryProperty (Src/flowfield_wrapper.cpp:291-623).
int GeometryCode(int dim, const int n[3], const int p[3], int cut = 0) {
    int axis[3], sign[3];
    const int k = NodeFaces(dim, n, p, axis, sign, cut);
    auto face = [](int a, int s) { return 10 * (a + 1) + (s > 0 ? 0 : 1); };
    if (k == 0) return 0;
    if (k == 1) return face(axis[0], sign[0]);
    if (k == 2) return face(axis[0], sign[0]) * 1000 + face(axis[1], sign[1]) * 10;
    return face(axis[0], sign[0]) * 100000 + face(axis[1], sign[1]) * 1000 +
           face(axis[2], sign[2]) * 10;
}

// FindBdyDvType / FindBdyDvType3D, Src/boundary_host_device.h:47-706, in
// inward components; 3D corners keep the reference's labelling.
int DvType(const Lat& L, int nf, const int axis[3], const int sign[3], int l) {
    int c[3];
    for (int q = 0; q < nf; q++) c[q] = sign[q] * L.c[l][axis[q]];
    if (nf == 1) return c[0] < 0 ? kDvIncoming : (c[0] == 0 ? kDvParallel
                                                              : kDvOutgoing);
    if (nf == 2) {
        if ((c[0] <= 0 && c[1] < 0) || (c[0] < 0 && c[1] == 0))
            return kDvIncoming;
        if ((c[0] >= 0 && c[1] > 0) || (c[0] > 0 && c[1] == 0))
            return kDvOutgoing;
        return kDvParallel;
    }
    if (nf == 3) {
        if (c[0] == 0 && c[1] == 0 && c[2] == 0) return kDvParallel;
        if (c[0] <= 0 && c[1] <= 0 && c[2] <= 0) return kDvOutgoing;
        if (c[0] >= 0 && c[1] >= 0 && c[2] >= 0) return kDvIncoming;
        return kDvParallel;
    }
    return kDvInvalid;
}

bool FluidLike(int vt) { return vt == kVtFluid || vt == kVtMD; }
bool PullsAll(int vt) { return vt == kVtFluid || vt == kVtMD || vt == kVtVB; }

// FP32 copies of an operation's constants for the shifted forms, rounded
// as the device would round them (IEEE division and conversions).
void SetFloatConsts(RegionOp& op) {
    op.invf = op.denom != 0.0 ? 1.0f / (float)op.denom : 0.0f;
    op.c0f = (float)op.c0;
    for (int l = 0; l < kMaxQ; l++) {
        op.am1f[l] = (float)op.am1[l];
        op.af[l] = (float)op.a[l];
        op.bf[l] = (float)op.b[l];
    }
}

// EQMDiffuseRefl constants (KerCutCellEQMDiffuseRefl(3D),
// Src/boundary_kernel.inc:534-613, 1184-1276).
RegionOp MakeEqm(const Lat& L, double CS, int nf, const int axis[3],
                 const int sign[3], const double* given) {
    RegionOp op{};
    op.kind = kOpEqm;
    op.nb_axis = -1;
    const double u = given[0], v = given[1], w = L.D == 3 ? given[2] : 0.0;
    const double uw[3] = {u, v, w};
    double rhoParallel = 0, deltaRho = 0;
    for (int l = 0; l < L.Q; l++) {
        const double cx = CS * (double)L.c[l][0];
        const double cy = CS * (double)L.c[l][1];
        const double cz = CS * (double)L.c[l][2];
        const double cu = L.D == 3 ? (cx * u + cy * v + cz * w)
                                   : (cx * u + cy * v);
        switch (DvType(L, nf, axis, sign, l)) {
            case kDvIncoming:
                op.in_mask |= 1u << l;
                op.win += L.w[l];
                break;
            case kDvOutgoing:
                op.out_mask |= 1u << l;
                deltaRho += (2 * L.w[l]) * cu;
                op.b[l] = cu;
                break;
            case kDvParallel:
                op.par_mask |= 1u << l;
                rhoParallel += L.w[l] * 1 * FeqRes(L, CS, l, uw);
                op.a[l] = FeqRes(L, CS, l, uw);
                break;
            default:
                break;
        }
    }
    op.denom = 1 - deltaRho - rhoParallel;
    op.c0 = 2 * op.win - op.denom;
    for (int l = 0; l < L.Q; l++)
        if (op.par_mask >> l & 1u) op.am1[l] = op.a[l] - 1.0;
    SetFloatConsts(op);
    return op;
}

// KerCutCellExtrapolPressure1ST(3D), Src/boundary_kernel.inc:404-488,
// 894-1182: copy mask and source neighbour for the surface being treated.
RegionOp MakeExtrapol(const Lat& L, int nf, const int axis[3],
                      const int sign[3], int surface, double rho_given) {
    RegionOp op{};
    op.kind = kOpExtrapol;
    op.rho_given = rho_given;
    op.nb_axis = -1;
    int sa[2], ss[2];
    const int sf = SurfaceFaces(surface, sa, ss);
    const bool face = sf == 1 && (surface == MPLBGPU_LEFT ||
                                  surface == MPLBGPU_RIGHT ||
                                  surface == MPLBGPU_TOP ||
                                  surface == MPLBGPU_BOTTOM ||
                                  surface == MPLBGPU_FRONT ||
                                  surface == MPLBGPU_BACK);
    if (nf == 1) {
        op.nb_axis = axis[0];
        op.nb_sign = sign[0];
    } else if (face) {
        const int want = ss[0] == 0 ? 1 : -1;
        for (int q = 0; q < nf; q++) {
            if (axis[q] == sa[0] && sign[q] == want) {
                op.nb_axis = axis[q];
                op.nb_sign = sign[q];
            }
        }
    }
    for (int l = 0; l < L.Q; l++) {
        int c[3] = {0, 0, 0};
        for (int q = 0; q < nf; q++) c[q] = sign[q] * L.c[l][axis[q]];
        bool copy = false;
        if (nf == 1) copy = c[0] > 0;
        if (nf == 2) copy = (c[0] >= 0 && c[1] > 0) || (c[0] > 0 && c[1] == 0);
        if (nf == 3)
            copy = (c[0] >= 0 && c[1] >= 0 && c[2] >= 0) &&
                   (c[0] != 0 || c[1] != 0 || c[2] != 0);
        if (copy && op.nb_axis >= 0) op.in_mask |= 1u << l;
    }
    return op;
}

// Halfway bounce-back of this path: populations whose upstream node lies
// beyond one of the surface's faces.
RegionOp MakeHbb(const Lat& L, double CS, const int n[3], const int p[3],
                 int surface, const double* given) {
    RegionOp op{};
    op.kind = kOpHbb;
    op.nb_axis = -1;
    int sa[2], ss[2];
    const int sf = SurfaceFaces(surface, sa, ss);
    for (int l = 0; l < L.Q; l++) {
        bool beyond = false;
        for (int q = 0; q < sf; q++) {
            const int s = p[sa[q]] - L.c[l][sa[q]];
            beyond = beyond || (ss[q] ? (s > n[sa[q]] - 1) : (s < 0));
        }
        if (!beyond) continue;
        op.out_mask |= 1u << l;
        double cu = CS * (double)L.c[l][0] * given[0] +
                    CS * (double)L.c[l][1] * given[1];
        if (L.D == 3) cu = cu + CS * (double)L.c[l][2] * given[2];
        op.b[l] = 2.0 * L.w[l] * cu;
    }
    SetFloatConsts(op);
    return op;
}

// Swap scheme of the reference (KerLocalSwap3D / KerSwapStream3D,
// Src/scheme_kernel.inc:959-1398).  A node exchanges its population l + Q/2
// with population l of x + c_l (l = 1..Q/2) when it is fluid-like
// (Fluid, MDPeriodic, VirtualBoundary) or, for a boundary-typed node, when
// c_l has no component pointing out of any of its faces.
bool SwapExchanges(const Lat& L, int vt, int nf, const int axis[3],
                   const int sign[3], int l) {
    if (vt == kVtSolid) return false;
    if (PullsAll(vt)) return true;
    if (nf == 0) return false;
    for (int q = 0; q < nf; q++)
        if (sign[q] * L.c[l][axis[q]] < 0) return false;
    return true;
}

// The node's local swap as a map from slots to the collided populations.
// Fluid-like nodes swap each population with its opposite; a boundary-typed
// node walks l = 1..Q-1 in order over the directions with no inward
// component (pointing out of or along its faces): a direction lying in all
// of its faces is exchanged with its opposite (the walk meets both members
// of the pair, so the pair ends where it began), any other direction takes
// a copy of its opposite slot.
void SwapLocal(const Lat& L, int vt, int nf, const int axis[3],
               const int sign[3], uint8_t* sigma) {
    const int half = (L.Q - 1) / 2;
    for (int k = 0; k < kMaxQ; k++) sigma[k] = (uint8_t)(k < L.Q ? k : 0);
    if (vt == kVtSolid) return;
    if (PullsAll(vt)) {
        for (int l = 1; l <= half; l++) std::swap(sigma[l], sigma[l + half]);
        return;
    }
    for (int l = 1; l < L.Q && nf > 0; l++) {
        bool out = true, along = true;
        for (int q = 0; q < nf; q++) {
            const int c = sign[q] * L.c[l][axis[q]];
            if (c > 0) out = false;
            if (c != 0) along = false;
        }
        if (!out) continue;
        if (along) std::swap(sigma[l], sigma[L.opp[l]]);
        else sigma[l] = sigma[L.opp[l]];
    }
}

// Exchange masks and local-swap maps of every region.  In pull form slot k
// (k <= Q/2) of x comes from the upstream node x - c_k when that node
// exchanges direction k, slot k > Q/2 when x itself exchanges direction
// k - Q/2 (it then lives at slot k - Q/2 = opp(k) of x + c_(k - Q/2) =
// x - c_k).  Within a region the upstream node may sit in different
// regions; the plan is accepted only where they all agree.
int PlanSwap(const Lat& L, BlockPlan& B, std::string* err) {
    const int half = (L.Q - 1) / 2;
    for (int r = 0; r < kNumRegions; r++) {
        const RegionInfo& R = B.region[r];
        B.swap_exch[r] = 0;
        for (int k = 0; k < kMaxQ; k++) B.swap_sigma[r][k] = (uint8_t)k;
        if (R.cls < 0) continue;
        int axis[3], sign[3];
        const int nf = NodeFaces(3, B.n, R.org, axis, sign);
        SwapLocal(L, R.vt, nf, axis, sign, B.swap_sigma[r]);
        for (int k = 0; k < L.Q; k++) {
            const int sg = B.swap_sigma[r][k];
            if (sg != k && sg != L.opp[k]) {
                *err = "local swap moves a population across directions";
                return MPLBGPU_ERR_UNSUPPORTED;
            }
        }
        const int rc[3] = {r % 3, (r / 3) % 3, r / 9};
        for (int k = 1; k < L.Q; k++) {
            if (k > half) {
                const int l = k - half;
                if (!SwapExchanges(L, R.vt, nf, axis, sign, l)) continue;
                for (int a = 0; a < 3; a++) {
                    const int c = L.c[l][a];
                    if ((rc[a] == 0 && c < 0) || (rc[a] == 2 && c > 0)) {
                        *err = "the swap scheme would exchange with a halo "
                               "node (a fluid-like node on the block "
                               "boundary)";
                        return MPLBGPU_ERR_UNSUPPORTED;
                    }
                }
                B.swap_exch[r] |= 1u << k;
                continue;
            }
            // upstream node z = x - c_k: its possible regions per axis
            int opts[3][2], nopt[3];
            bool outside = false;
            for (int a = 0; a < 3; a++) {
                const int c = L.c[k][a];
                nopt[a] = 0;
                if (rc[a] == 0) {
                    if (c > 0) outside = true;
                    else opts[a][nopt[a]++] = c < 0 ? 1 : 0;
                } else if (rc[a] == 2) {
                    if (c < 0) outside = true;
                    else opts[a][nopt[a]++] = c > 0 ? 1 : 2;
                } else {
                    opts[a][nopt[a]++] = 1;
                    if (c > 0) opts[a][nopt[a]++] = 0;
                    if (c < 0) opts[a][nopt[a]++] = 2;
                }
            }
            if (outside) continue;
            int exchanges = -1;
            for (int i0 = 0; i0 < nopt[0]; i0++)
                for (int i1 = 0; i1 < nopt[1]; i1++)
                    for (int i2 = 0; i2 < nopt[2]; i2++) {
                        const int zr = opts[0][i0] + 3 * opts[1][i1] +
                                       9 * opts[2][i2];
                        const RegionInfo& Z = B.region[zr];
                        if (Z.cls < 0) continue;
                        int za[3], zs[3];
                        const int zf = NodeFaces(3, B.n, Z.org, za, zs);
                        const int e = SwapExchanges(L, Z.vt, zf, za, zs, k);
                        if (exchanges >= 0 && exchanges != e) {
                            *err = "swap exchange pattern differs within a "
                                   "region";
                            return MPLBGPU_ERR_UNSUPPORTED;
                        }
                        exchanges = e;
                    }
            if (exchanges == 1) B.swap_exch[r] |= 1u << k;
        }
    }
    return MPLBGPU_OK;
}

bool Dispatched(int scheme) {
    return scheme == MPLBGPU_BC_EQM_DIFFUSE_REFL ||
           scheme == MPLBGPU_BC_EXTRAPOL_PRESSURE_1ST ||
           scheme == MPLBGPU_BC_HALFWAY_BOUNCE_BACK ||
           scheme == MPLBGPU_BC_FDPERIODIC;
}

// KerCutCellPeriodic(3D) (Src/boundary_kernel.inc:615-719, 1278-1666): the
// copies f(node) = f(node + off) it makes at a node of geometry vg for the
// boundary surface being treated, in its order (the edge and corner cases
// compare the surface with face values, a few of them with a face other
// than the one the offset crosses).  Returns the number of copies.
int FdPeriodicCopies(int vg, int surface, int off[3][3]) {
    int n = 0;
    auto add = [&](bool when, int x, int y, int z) {
        if (!when) return;
        off[n][0] = x;
        off[n][1] = y;
        off[n][2] = z;
        n++;
    };
    const bool L = surface == MPLBGPU_LEFT, R = surface == MPLBGPU_RIGHT,
               T = surface == MPLBGPU_TOP, B = surface == MPLBGPU_BOTTOM,
               F = surface == MPLBGPU_FRONT, K = surface == MPLBGPU_BACK;
    switch (vg) {
        case 10: add(true, -1, 0, 0); break;                 // IP
        case 11: add(true, 1, 0, 0); break;                  // IM
        case 20: add(true, 0, -1, 0); break;                 // JP
        case 21: add(true, 0, 1, 0); break;                  // JM
        case 30: add(true, 0, 0, -1); break;                 // KP
        case 31: add(true, 0, 0, 1); break;                  // KM
        case 10200: add(L, -1, 0, 0); add(B, 0, -1, 0); break;   // IPJP
        case 10210: add(L, -1, 0, 0); add(T, 0, 1, 0); break;    // IPJM
        case 11200: add(R, 1, 0, 0); add(B, 0, -1, 0); break;    // IMJP
        case 11210: add(R, 1, 0, 0); add(T, 0, 1, 0); break;     // IMJM
        case 10300: add(L, -1, 0, 0); add(K, 0, 0, -1); break;   // IPKP
        case 10310: add(R, -1, 0, 0); add(F, 0, 0, 1); break;    // IPKM
        case 11300: add(R, 1, 0, 0); add(K, 0, 0, -1); break;    // IMKP
        case 11310: add(R, 1, 0, 0); add(F, 0, 0, 1); break;     // IMKM
        case 20300: add(B, 0, -1, 0); add(K, 0, 0, -1); break;   // JPKP
        case 20310: add(B, 0, -1, 0); add(F, 0, 0, 1); break;    // JPKM
        case 21300: add(T, 0, 1, 0); add(F, 0, 0, -1); break;    // JMKP
        case 21310: add(T, 0, 1, 0); add(F, 0, 0, 1); break;     // JMKM
        case 1020300:                                             // IPJPKP
            add(L, -1, 0, 0); add(B, 0, -1, 0); add(K, 0, 0, -1); break;
        case 1020310:                                             // IPJPKM
            add(L, -1, 0, 0); add(B, 0, -1, 0); add(F, 0, 0, 1); break;
        case 1021300:                                             // IPJMKP
            add(L, -1, 0, 0); add(T, 0, 1, 0); add(K, 0, 0, -1); break;
        case 1021310:                                             // IPJMKM
            add(T, -1, 0, 0); add(T, 0, 1, 0); add(F, 0, 0, 1); break;
        case 1120300:                                             // IMJPKP
            add(R, 1, 0, 0); add(B, 0, -1, 0); add(K, 0, 0, -1); break;
        case 1120310:                                             // IMJPKM
            add(R, 1, 0, 0); add(B, 0, -1, 0); add(F, 0, 0, 1); break;
        case 1121300:                                             // IMJMKP
            add(R, 1, 0, 0); add(T, 0, 1, 0); add(K, 0, 0, -1); break;
        case 1121310:                                             // IMJMKM
            add(R, 1, 0, 0); add(T, 0, 1, 0); add(F, 0, 0, 1); break;
        default:
            break;
    }
    return n;
}

}  // namespace

int BuildPlan(const mplbgpu_desc& d, Plan* plan, std::string* err) {
    auto fail = [&](int code, const std::string& m) {
        *err = m;
        return code;
    };
    if (d.abi_version != MPLBGPU_ABI_VERSION)
        return fail(MPLBGPU_ERR_INVALID, "abi_version mismatch");
    if (!((d.space_dim == 2 && d.lattice == MPLBGPU_D2Q9) ||
          (d.space_dim == 3 && d.lattice == MPLBGPU_D3Q19)))
        return fail(MPLBGPU_ERR_UNSUPPORTED,
                    "only D2Q9 (2D) and D3Q19 (3D) are supported");
    if (d.precision < MPLBGPU_FP64 || d.precision > MPLBGPU_FP16_SHIFTED)
        return fail(MPLBGPU_ERR_INVALID, "unknown precision");
    if (d.nblocks < 1 || !d.blocks)
        return fail(MPLBGPU_ERR_INVALID, "no blocks");
    if (!(d.dt > 0) || !(d.cs > 0) || !(d.tau_ref + 0.5 * d.dt > 0))
        return fail(MPLBGPU_ERR_INVALID, "dt, cs and tau must be positive");
    if (d.body_force != MPLBGPU_FORCE_NONE && d.body_force != MPLBGPU_FORCE_1ST)
        return fail(MPLBGPU_ERR_UNSUPPORTED, "unknown body force type");
    if (d.scheme != 0 && d.scheme != MPLBGPU_SCHEME_STREAM_COLLISION &&
        d.scheme != MPLBGPU_SCHEME_STREAM_COLLISION_SWAP)
        return fail(MPLBGPU_ERR_UNSUPPORTED, "unknown scheme");
    const bool swap = d.scheme == MPLBGPU_SCHEME_STREAM_COLLISION_SWAP;
    if (swap && (d.space_dim != 3 || d.nblocks != 1 || d.nconnections != 0))
        return fail(MPLBGPU_ERR_UNSUPPORTED,
                    "the swap scheme runs on one 3D block without "
                    "connections (the reference's swap kernels are 3D)");

    Plan& P = *plan;
    P.dim = d.space_dim;
    P.Q = d.lattice;
    P.precision = d.precision;
    P.elem_bytes = d.precision == MPLBGPU_FP64 ? 8
                   : d.precision == MPLBGPU_FP32_SHIFTED ? 4 : 2;
    P.cs = d.cs;
    P.tau = d.tau_ref;
    P.dt = d.dt;
    // KerCollideBGKIsothermal3D, Src/model_kernel.inc:428-438
    const double tau = d.tau_ref;
    P.omega = d.dt / (tau + 0.5 * d.dt);
    P.omc = 1 - P.omega;
    P.tw = tau * P.omega;
    P.body_force = d.body_force;
    P.force_velocity = d.force_velocity ? 1 : 0;
    P.swap = swap ? 1 : 0;
    Lat L{};
    if (P.dim == 2) FillLat<2>(&L); else FillLat<3>(&L);
    for (int a = 0; a < 3; a++) {
        P.accel[a] = a < P.dim ? d.accel[a] : 0.0;
        // KerCalcUForce3D: u += dt * a / 2
        P.hdta[a] = (d.dt * P.accel[a] / 2);
    }
    for (int l = 0; l < P.Q; l++) {
        P.w[l] = L.w[l];
        // CalcBodyForce, Src/model_host_device.h:25-32
        double cf = 0;
        for (int a = 0; a < P.dim; a++)
            cf += d.cs * (double)L.c[l][a] * P.accel[a];
        P.cf[l] = cf;
    }

    // blocks in id order (the reference keeps them in a std::map)
    std::vector<int> order(d.nblocks);
    for (int i = 0; i < d.nblocks; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int x, int y) {
        return d.blocks[x].id < d.blocks[y].id;
    });
    for (int i = 1; i < d.nblocks; i++)
        if (d.blocks[order[i]].id == d.blocks[order[i - 1]].id)
            return fail(MPLBGPU_ERR_INVALID, "duplicate block id");
    const int xoff = 32 / P.elem_bytes;
    P.blocks.resize(d.nblocks);
    for (int i = 0; i < d.nblocks; i++) {
        BlockPlan& B = P.blocks[i];
        const mplbgpu_block& src = d.blocks[order[i]];
        B.id = src.id;
        B.index = i;
        B.cut = src.cut;
        if (B.cut != 0) {
            if (B.cut & ~((1 << (2 * P.dim)) - 1))
                return fail(MPLBGPU_ERR_INVALID,
                            "cut faces outside the block's dimension");
            if (d.nconnections != 0 || swap)
                return fail(MPLBGPU_ERR_UNSUPPORTED,
                            "decomposed (cut) blocks take no connections "
                            "and the two-array scheme");
        }
        for (int a = 0; a < 3; a++) {
            B.n[a] = a < P.dim ? src.size[a] : 1;
            if (a < P.dim && B.n[a] < 2)
                return fail(MPLBGPU_ERR_INVALID,
                            "every block needs at least 2 nodes per axis");
        }
        B.xoff = xoff;
        B.pitch = ((xoff + B.n[0] + 1 + xoff - 1) / xoff) * xoff;
        B.plane = B.pitch * (B.n[1] + 2);
        const long long zs = P.dim == 3 ? B.n[2] + 2 : 1;
        const long long ps = B.plane * zs;
        const long long align = 256 / P.elem_bytes;
        B.popstride = ((ps + align - 1) / align) * align;
    }
    auto blockIndex = [&](int id) {
        for (const BlockPlan& B : P.blocks)
            if (B.id == id) return B.index;
        return -1;
    };

    // boundaries
    for (int k = 0; k < d.nboundaries; k++) {
        const mplbgpu_boundary& bc = d.boundaries[k];
        if (blockIndex(bc.block) < 0)
            return fail(MPLBGPU_ERR_INVALID, "boundary on an unknown block");
        if (!ValidSurface(P.dim, bc.surface))
            return fail(MPLBGPU_ERR_INVALID, "invalid boundary surface");
        if (bc.scheme == MPLBGPU_BC_FDPERIODIC && swap)
            return fail(MPLBGPU_ERR_UNSUPPORTED,
                        "FDPeriodic with the swap scheme");
        if (bc.vertex_type == kVtSolid ||
            bc.vertex_type == MPLBGPU_VT_IMMERSED_BOUNDARY)
            return fail(MPLBGPU_ERR_UNSUPPORTED,
                        "immersed-solid boundary node types are not supported");
        if (bc.scheme == MPLBGPU_BC_HALFWAY_BOUNCE_BACK) {
            int sa[2], ss[2];
            if (SurfaceFaces(bc.surface, sa, ss) < 1)
                return fail(MPLBGPU_ERR_INVALID, "bad bounce-back surface");
        }
        {
            const int cut = P.blocks[blockIndex(bc.block)].cut;
            int sa[2], ss[2];
            const int nsf = SurfaceFaces(bc.surface, sa, ss);
            for (int q = 0; q < nsf; q++)
                if (cut >> FaceSurface(sa[q], ss[q]) & 1)
                    return fail(MPLBGPU_ERR_INVALID,
                                "boundary condition on a cut face");
        }
    }

    // regions
    for (BlockPlan& B : P.blocks) {
        long long stale_nodes = 0, deferred_nodes = 0;
        for (int r = 0; r < kNumRegions; r++) {
            RegionInfo& R = B.region[r];
            R = RegionInfo{};
            const int rc[3] = {r % 3, (r / 3) % 3, r / 9};
            bool empty = false;
            for (int a = 0; a < 3; a++) {
                if (a >= P.dim) {
                    R.org[a] = 0;
                    R.ext[a] = 1;
                    if (rc[a] != 1) empty = true;
                    continue;
                }
                const int n = B.n[a];
                if (rc[a] == 0) { R.org[a] = 0; R.ext[a] = 1; }
                if (rc[a] == 2) { R.org[a] = n - 1; R.ext[a] = 1; }
                if (rc[a] == 1) { R.org[a] = 1; R.ext[a] = n - 2; }
                if (R.ext[a] <= 0) empty = true;
            }
            if (empty) {
                R.cls = -1;
                continue;
            }
            const int* p = R.org;
            // node type: bulk Fluid, faces unset (0), then every boundary in
            // definition order (SetBulkandHaloNodesType /
            // SetBoundaryNodeType, Src/flowfield_wrapper.cpp:625-788)
            bool bulk = true;
            for (int a = 0; a < P.dim; a++)
                bulk = bulk &&
                       (p[a] >= 1 || (B.cut >> FaceSurface(a, 0) & 1)) &&
                       (p[a] < B.n[a] - 1 || (B.cut >> FaceSurface(a, 1) & 1));
            int vt = bulk ? kVtFluid : 0;
            for (int k = 0; k < d.nboundaries; k++) {
                const mplbgpu_boundary& bc = d.boundaries[k];
                if (bc.block != B.id) continue;
                int rg[6];
                SurfaceRange(P.dim, B.n, bc.surface, rg);
                if (bc.vertex_type == kVtVB) {
                    const int s = bc.surface;
                    if (s == MPLBGPU_LEFT || s == MPLBGPU_RIGHT) {
                        rg[2]++; rg[3]--;
                        if (P.dim == 3) { rg[4]++; rg[5]--; }
                    }
                    if (s == MPLBGPU_TOP || s == MPLBGPU_BOTTOM) {
                        rg[0]++; rg[1]--;
                        if (P.dim == 3) { rg[4]++; rg[5]--; }
                    }
                    if (P.dim == 3 &&
                        (s == MPLBGPU_FRONT || s == MPLBGPU_BACK)) {
                        rg[0]++; rg[1]--; rg[2]++; rg[3]--;
                    }
                }
                if (InRange(p, rg)) vt = bc.vertex_type;
            }
            R.vt = vt;
            R.vg = GeometryCode(P.dim, B.n, p, B.cut);
            R.fluidlike = FluidLike(vt) ? 1 : 0;
            int axis[3], sign[3];
            const int nf = NodeFaces(P.dim, B.n, p, axis, sign, B.cut);
            // KerStream3D selection, Src/scheme_kernel.inc:1400-2051
            uint32_t pull = 0;
            for (int l = 0; l < P.Q; l++) {
                bool take = PullsAll(vt);
                const bool rest = L.c[l][0] == 0 && L.c[l][1] == 0 &&
                                  L.c[l][2] == 0;
                if (!take && (rest || nf > 0)) {
                    take = true;
                    if (!rest)
                        for (int q = 0; q < nf; q++)
                            if (sign[q] * L.c[l][axis[q]] > 0) take = false;
                }
                if (take) pull |= 1u << l;
            }
            R.pull = pull;
            // boundary programme, definition order
            std::vector<RegionOp> prog;
            for (int k = 0; k < d.nboundaries; k++) {
                const mplbgpu_boundary& bc = d.boundaries[k];
                if (bc.block != B.id || !Dispatched(bc.scheme)) continue;
                int rg[6];
                SurfaceRange(P.dim, B.n, bc.surface, rg);
                if (!InRange(p, rg)) continue;
                if (bc.scheme == MPLBGPU_BC_FDPERIODIC) {
                    // every copy reads a halo cell of f (the offsets point
                    // out of the block at the nodes of the surface): one
                    // that no step transfers or writes, zero from the
                    // start, so a node with any copy ends with f = 0
                    int off[3][3];
                    const int nc = FdPeriodicCopies(R.vg, bc.surface, off);
                    if (nc == 0) continue;
                    for (int c = 0; c < nc; c++)
                        for (int a = 0; a < P.dim; a++) {
                            if (off[c][a] == 0) continue;
                            const int q = p[a] + off[c][a];
                            if (R.ext[a] != 1 || (q >= 0 && q < B.n[a]))
                                return fail(MPLBGPU_ERR_UNSUPPORTED,
                                            "FDPeriodic copying from inside "
                                            "the block");
                        }
                    RegionOp op{};
                    op.kind = kOpZero;
                    op.nb_axis = -1;
                    op.out_mask = (1u << P.Q) - 1u;
                    prog.push_back(op);
                } else if (bc.scheme == MPLBGPU_BC_EQM_DIFFUSE_REFL) {
                    prog.push_back(MakeEqm(L, P.cs, nf, axis, sign, bc.given));
                } else if (bc.scheme == MPLBGPU_BC_EXTRAPOL_PRESSURE_1ST) {
                    prog.push_back(MakeExtrapol(L, nf, axis, sign, bc.surface,
                                                bc.given[0]));
                } else {
                    prog.push_back(MakeHbb(L, P.cs, B.n, p, bc.surface,
                                           bc.given));
                }
                prog.back().bc = k;
            }
            bool extrapol = false;
            uint32_t written = 0, readfirst = 0;
            for (const RegionOp& op : prog) {
                if (op.kind == kOpExtrapol) extrapol = true;
                if (op.kind == kOpEqm) {
                    uint32_t reads = op.in_mask;
                    for (int l = 0; l < P.Q; l++)
                        if (op.out_mask >> l & 1u) reads |= 1u << L.opp[l];
                    readfirst |= reads & ~written;
                    written |= op.out_mask | op.par_mask;
                } else if (op.kind == kOpHbb || op.kind == kOpZero) {
                    written |= op.out_mask;
                }
            }
            const uint32_t all = (P.Q == 32) ? ~0u : ((1u << P.Q) - 1u);
            if (prog.empty() && PullsAll(vt)) {
                R.cls = kPure;
            } else if (extrapol || (int)prog.size() > kMaxOps ||
                       (readfirst & ~pull & written) != 0) {
                R.cls = kDeferred;
            } else {
                R.cls = kLocal;
            }
            R.stale = all & ~pull & ~written;
            R.nops = 0;
            for (const RegionOp& op : prog) {
                if (R.nops < kMaxOps) R.op[R.nops++] = (int)B.ops.size();
                B.allops[r].push_back((int)B.ops.size());
                B.ops.push_back(op);
            }
        }
        // An ExtrapolPressure1ST reads its inner neighbour's post-boundary
        // f: the deferred kernel takes it from the store when the
        // neighbour is deferred, re-pulls it when the neighbour is pure,
        // and re-evaluates it (pull, stale store, the neighbour's boundary
        // operations defined before this one) when the neighbour is local.
        // A local neighbour is materialised all the same when a population
        // the extrapolation copies is none of those - neither pulled nor
        // stale nor written by an earlier operation: the reference has the
        // neighbour's value of the previous step there, which only the
        // deferred store keeps.
        for (int r = 0; r < kNumRegions; r++) {
            const RegionInfo& R = B.region[r];
            if (R.cls != kDeferred) continue;
            for (int oi : B.allops[r]) {
                const RegionOp& op = B.ops[oi];
                if (op.kind != kOpExtrapol || op.nb_axis < 0) continue;
                int q[3] = {R.org[0], R.org[1], R.org[2]};
                q[op.nb_axis] += op.nb_sign;
                int rc[3];
                for (int a = 0; a < 3; a++)
                    rc[a] = a < P.dim ? RegionCoord(q[a], B.n[a]) : 1;
                const int nr = rc[0] + 3 * rc[1] + 9 * rc[2];
                RegionInfo& N = B.region[nr];
                if (N.cls != kLocal) continue;
                uint32_t avail = N.pull | N.stale;
                for (int ni : B.allops[nr]) {
                    const RegionOp& nop = B.ops[ni];
                    if (nop.bc >= op.bc) break;
                    avail |= nop.out_mask;
                    if (nop.kind == kOpEqm) avail |= nop.par_mask;
                }
                if (op.in_mask & ~avail) N.cls = kDeferred;
            }
        }
        for (int r = 0; r < kNumRegions; r++) {
            RegionInfo& R = B.region[r];
            const long long cnt = (long long)R.ext[0] * R.ext[1] * R.ext[2];
            R.side_base = -1;
            if (R.cls == kLocal && R.stale != 0) {
                R.side_base = stale_nodes;
                stale_nodes += cnt;
            } else if (R.cls == kDeferred) {
                R.side_base = deferred_nodes;
                deferred_nodes += cnt;
            }
        }
        B.nstale = stale_nodes;
        B.ndeferred = deferred_nodes;
        // the deferred programme in one pass: independent unless an
        // extrapolation reads a deferred neighbour
        B.deferred_fused = B.ndeferred > 0;
        B.dops_flat.clear();
        for (int r = 0; r < kNumRegions; r++) {
            const RegionInfo& R = B.region[r];
            B.dops_first[r] = (int)B.dops_flat.size();
            if (R.cls != kDeferred) continue;
            for (int oi : B.allops[r]) {
                const RegionOp& op = B.ops[oi];
                B.dops_flat.push_back(oi);
                if (op.kind != kOpExtrapol || op.nb_axis < 0) continue;
                int q[3] = {R.org[0], R.org[1], R.org[2]};
                q[op.nb_axis] += op.nb_sign;
                int rc[3];
                for (int a = 0; a < 3; a++)
                    rc[a] = a < P.dim ? RegionCoord(q[a], B.n[a]) : 1;
                if (B.region[rc[0] + 3 * rc[1] + 9 * rc[2]].cls == kDeferred)
                    B.deferred_fused = false;
            }
            B.dops_flat.push_back(-1);
        }
        if (B.dops_flat.empty()) B.dops_flat.push_back(-1);
        // deferred programme: every boundary, in definition order, on the
        // deferred regions it covers
        if (B.ndeferred > 0) {
            for (int k = 0; k < d.nboundaries; k++) {
                const mplbgpu_boundary& bc = d.boundaries[k];
                if (bc.block != B.id || !Dispatched(bc.scheme)) continue;
                int rg[6];
                SurfaceRange(P.dim, B.n, bc.surface, rg);
                DeferredOp dop;
                for (int r = 0; r < kNumRegions; r++) {
                    const RegionInfo& R = B.region[r];
                    if (R.cls != kDeferred || !InRange(R.org, rg)) continue;
                    int axis[3], sign[3];
                    const int nf =
                        NodeFaces(P.dim, B.n, R.org, axis, sign, B.cut);
                    RegionOp op;
                    if (bc.scheme == MPLBGPU_BC_EQM_DIFFUSE_REFL)
                        op = MakeEqm(L, P.cs, nf, axis, sign, bc.given);
                    else if (bc.scheme == MPLBGPU_BC_EXTRAPOL_PRESSURE_1ST)
                        op = MakeExtrapol(L, nf, axis, sign, bc.surface,
                                          bc.given[0]);
                    else
                        op = MakeHbb(L, P.cs, B.n, R.org, bc.surface,
                                     bc.given);
                    op.bc = k;
                    dop.segments.push_back({r, (int)B.ops.size()});
                    B.ops.push_back(op);
                }
                if (!dop.segments.empty()) B.dops.push_back(dop);
            }
        }
    }

    // swap scheme: node-local boundary programmes (EQMDiffuseRefl or no
    // kernel), at least three nodes per axis
    if (P.swap) {
        BlockPlan& B = P.blocks[0];
        for (int a = 0; a < 3; a++)
            if (B.n[a] < 3)
                return fail(MPLBGPU_ERR_UNSUPPORTED,
                            "the swap scheme needs at least 3 nodes per axis");
        for (int r = 0; r < kNumRegions; r++) {
            if ((int)B.allops[r].size() > kMaxOps)
                return fail(MPLBGPU_ERR_UNSUPPORTED,
                            "too many boundary conditions on one node");
            for (int oi : B.allops[r])
                if (B.ops[oi].kind != kOpEqm)
                    return fail(MPLBGPU_ERR_UNSUPPORTED,
                                "the swap scheme takes node-local boundary "
                                "conditions only (EQMDiffuseRefl)");
        }
        const RegionInfo& C = B.region[13];
        if (!C.fluidlike || !B.allops[13].empty())
            return fail(MPLBGPU_ERR_UNSUPPORTED,
                        "the swap scheme needs a fluid interior");
        int rc = PlanSwap(L, B, err);
        if (rc != MPLBGPU_OK) return rc;
    }

    // halo transfers: Field::CreateHalos order, Src/field.h:215-395
    for (const BlockPlan& FB : P.blocks) {
        for (int s = 0; s <= 5; s++) {
            for (int c = 0; c < d.nconnections; c++) {
                const mplbgpu_connection& cn = d.connections[c];
                if (cn.from_block != FB.id || cn.from_surface != s) continue;
                const int ti = blockIndex(cn.to_block);
                if (ti < 0)
                    return fail(MPLBGPU_ERR_INVALID,
                                "connection to an unknown block");
                const BlockPlan& TB = P.blocks[ti];
                const int axis = s < 2 ? 0 : (s < 4 ? 1 : 2);
                if (axis >= P.dim)
                    return fail(MPLBGPU_ERR_INVALID,
                                "connection surface not in this dimension");
                HaloCopy h;
                h.from = FB.index;
                h.to = ti;
                h.axis = axis;
                const bool maxside = s == MPLBGPU_RIGHT || s == MPLBGPU_TOP ||
                                     s == MPLBGPU_FRONT;
                const int disp = (cn.type == MPLBGPU_VT_FDPERIODIC ||
                                  cn.type == kVtMD || cn.type == kVtVB) ? -1
                                                                        : 0;
                for (int a = 0; a < 3; a++) {
                    const int hd = a < P.dim ? 1 : 0;
                    h.iter[a] = FB.n[a] + 2 * hd;
                    h.fbase[a] = -hd;
                    h.tbase[a] = -hd;
                    if (a != axis && a < P.dim && FB.n[a] != TB.n[a])
                        return fail(MPLBGPU_ERR_INVALID,
                                    "connected blocks differ in size");
                }
                h.iter[axis] = 1;
                if (maxside) {
                    h.fbase[axis] = FB.n[axis] + disp;
                    h.tbase[axis] = -1;
                    h.to_low = 1;
                } else {
                    h.fbase[axis] = 0;
                    h.tbase[axis] = TB.n[axis];
                    h.to_low = 0;
                }
                h.pops = 0;
                for (int l = 0; l < P.Q; l++)
                    if (L.c[l][axis] == (h.to_low ? 1 : -1)) h.pops |= 1u << l;
                h.any_prev = false;
                P.halos.push_back(h);
            }
        }
    }
    // A source cell that a later transfer of the same step overwrites, and
    // no earlier one did, still holds last step's value in the reference.
    for (size_t t = 0; t < P.halos.size(); t++) {
        HaloCopy& h = P.halos[t];
        const BlockPlan& FB = P.blocks[h.from];
        const long long cells = (long long)h.iter[0] * h.iter[1] * h.iter[2];
        h.prev.assign(cells, 0);
        for (long long cidx = 0; cidx < cells; cidx++) {
            const int i = (int)(cidx % h.iter[0]);
            const int j = (int)((cidx / h.iter[0]) % h.iter[1]);
            const int k = (int)(cidx / ((long long)h.iter[0] * h.iter[1]));
            const int sp[3] = {h.fbase[0] + i, h.fbase[1] + j, h.fbase[2] + k};
            bool inside = true;
            for (int a = 0; a < P.dim; a++)
                inside = inside && sp[a] >= 0 && sp[a] < FB.n[a];
            if (inside) continue;
            bool before = false, after = false;
            for (size_t u = 0; u < P.halos.size(); u++) {
                const HaloCopy& o = P.halos[u];
                if (u == t || o.to != h.from) continue;
                bool in = true;
                for (int a = 0; a < 3; a++)
                    in = in && sp[a] >= o.tbase[a] &&
                         sp[a] < o.tbase[a] + o.iter[a];
                if (!in) continue;
                if (u < t) before = true; else after = true;
            }
            if (!before && after) {
                h.prev[cidx] = 1;
                h.any_prev = true;
            }
        }
        if (!h.any_prev) h.prev.clear();
    }
    // Phases of the fused transfer.  A cell must run in definition order
    // when its destination is written by more than one copy, or when its
    // source (a halo cell) is written by an earlier copy of the step; every
    // other cell reads a value no copy of this step changes (a block node, a
    // halo cell no copy writes, or one only a later copy writes, which
    // `prev` sends to the previous array) and writes a cell no other copy
    // writes, so the cells can run in any order.
    {
        // first writer (copy index) and number of writers per halo cell
        std::map<std::pair<int, long long>, std::pair<int, int>> writers;
        auto cell = [&](int blk, int x, int y, int z) {
            const BlockPlan& B = P.blocks[blk];
            const long long a0 = B.n[0] + 2, a1 = B.n[1] + 2;
            return std::make_pair(
                blk, ((long long)(z + 1) * a1 + (y + 1)) * a0 + (x + 1));
        };
        for (size_t t = 0; t < P.halos.size(); t++) {
            const HaloCopy& h = P.halos[t];
            for (int k = 0; k < h.iter[2]; k++)
                for (int j = 0; j < h.iter[1]; j++)
                    for (int i = 0; i < h.iter[0]; i++) {
                        auto& w = writers[cell(h.to, h.tbase[0] + i,
                                               h.tbase[1] + j,
                                               h.tbase[2] + k)];
                        if (w.second++ == 0) w.first = (int)t;
                    }
        }
        for (size_t t = 0; t < P.halos.size(); t++) {
            HaloCopy& h = P.halos[t];
            const long long cells =
                (long long)h.iter[0] * h.iter[1] * h.iter[2];
            h.ordered.assign(cells, 0);
            h.nordered = 0;
            long long cidx = 0;
            for (int k = 0; k < h.iter[2]; k++)
                for (int j = 0; j < h.iter[1]; j++)
                    for (int i = 0; i < h.iter[0]; i++, cidx++) {
                        const auto& dw = writers[cell(h.to, h.tbase[0] + i,
                                                      h.tbase[1] + j,
                                                      h.tbase[2] + k)];
                        bool ord = dw.second > 1;
                        const auto sw = writers.find(cell(
                            h.from, h.fbase[0] + i, h.fbase[1] + j,
                            h.fbase[2] + k));
                        if (sw != writers.end() && sw->second.first < (int)t)
                            ord = true;
                        if (ord) {
                            h.ordered[cidx] = 1;
                            h.nordered++;
                        }
                    }
        }
        // Resolved element copies: the copies run symbolically in
        // definition order, each written element remembering where its
        // value comes from (an element written earlier in the step passes
        // on its own origin); the elements of the ordered cells' final
        // writes are then copied from those origins directly.
        struct Origin {
            int blk, x, y, z, prev;
        };
        std::map<std::pair<std::pair<int, long long>, int>, Origin> origin;
        std::map<std::pair<std::pair<int, long long>, int>, HaloElem> finals;
        for (size_t t = 0; t < P.halos.size(); t++) {
            const HaloCopy& h = P.halos[t];
            long long cidx = 0;
            std::vector<std::pair<std::pair<std::pair<int, long long>, int>,
                                  Origin>>
                writes;
            for (int k = 0; k < h.iter[2]; k++)
                for (int j = 0; j < h.iter[1]; j++)
                    for (int i = 0; i < h.iter[0]; i++, cidx++) {
                        const int fx = h.fbase[0] + i, fy = h.fbase[1] + j,
                                  fz = h.fbase[2] + k;
                        const int tx = h.tbase[0] + i, ty = h.tbase[1] + j,
                                  tz = h.tbase[2] + k;
                        const auto dc = cell(h.to, tx, ty, tz);
                        const auto sc = cell(h.from, fx, fy, fz);
                        const int pv = h.any_prev && h.prev[cidx] ? 1 : 0;
                        for (int q = 0; q < P.Q; q++) {
                            if (!(h.pops >> q & 1u)) continue;
                            auto so = origin.find({sc, q});
                            const Origin o =
                                so != origin.end()
                                    ? so->second
                                    : Origin{h.from, fx, fy, fz, pv};
                            writes.push_back({{dc, q}, o});
                            if (h.ordered[cidx])
                                finals[{dc, q}] = HaloElem{
                                    h.to, tx, ty, tz, o.blk, o.x, o.y, o.z,
                                    q, o.prev};
                        }
                    }
            // this copy's writes take effect after its reads
            for (const auto& w : writes) origin[w.first] = w.second;
        }
        P.halo_elems.clear();
        for (const auto& f : finals) P.halo_elems.push_back(f.second);
    }
    // surface range of every boundary, for per-node wall velocities
    P.bc_block.assign(d.nboundaries, -1);
    P.bc_range.assign(6 * (size_t)d.nboundaries, 0);
    P.bc_scheme.assign(d.nboundaries, 0);
    P.bc_surface.assign(d.nboundaries, 0);
    for (int k = 0; k < d.nboundaries; k++) {
        P.bc_scheme[k] = d.boundaries[k].scheme;
        P.bc_surface[k] = d.boundaries[k].surface;
        for (const BlockPlan& B : P.blocks) {
            if (B.id != d.boundaries[k].block) continue;
            P.bc_block[k] = B.index;
            SurfaceRange(P.dim, B.n, d.boundaries[k].surface,
                         &P.bc_range[6 * (size_t)k]);
        }
    }
    return MPLBGPU_OK;
}

int BoundaryNodeOps(const Plan& P, int k, const double* uvw,
                    std::vector<RegionOp>* out, std::string* err) {
    if (k < 0 || k >= (int)P.bc_block.size() || P.bc_block[k] < 0) {
        *err = "unknown boundary index";
        return MPLBGPU_ERR_INVALID;
    }
    const int scheme = P.bc_scheme[k];
    if (scheme != MPLBGPU_BC_EQM_DIFFUSE_REFL &&
        scheme != MPLBGPU_BC_HALFWAY_BOUNCE_BACK) {
        *err = "per-node velocities need an EQMDiffuseRefl or halfway "
               "bounce-back boundary";
        return MPLBGPU_ERR_UNSUPPORTED;
    }
    const BlockPlan& B = P.blocks[P.bc_block[k]];
    const int* r = &P.bc_range[6 * (size_t)k];
    Lat L{};
    if (P.dim == 2) FillLat<2>(&L); else FillLat<3>(&L);
    out->clear();
    size_t idx = 0;
    for (int z = r[4]; z < r[5]; z++)
        for (int y = r[2]; y < r[3]; y++)
            for (int x = r[0]; x < r[1]; x++, idx++) {
                const int p[3] = {x, y, z};
                int axis[3], sign[3];
                const int nf = NodeFaces(P.dim, B.n, p, axis, sign, B.cut);
                const double* g = uvw + 3 * idx;
                RegionOp op = scheme == MPLBGPU_BC_EQM_DIFFUSE_REFL
                                  ? MakeEqm(L, P.cs, nf, axis, sign, g)
                                  : MakeHbb(L, P.cs, B.n, p, P.bc_surface[k],
                                            g);
                op.bc = k;
                out->push_back(op);
            }
    return MPLBGPU_OK;
}

}  // namespace mplb
