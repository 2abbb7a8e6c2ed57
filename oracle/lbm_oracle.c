/*
 * CPU restatement of MPLB's stream-collision step (TEST INFRASTRUCTURE ONLY;
 * see lbm_oracle.h).  Each routine names the reference code it restates.
 * Compile with -ffp-contract=off: the arithmetic is written in the
 * reference's operation order so results are bitwise reproducible.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* VertexType, Src/flowfield_host_device.h:21-37 */
enum { VT_FLUID = 10, VT_MDPERIODIC = 13, VT_FDPERIODIC = 15,
       VT_IMMERSED_SOLID = -1, VT_VIRTUAL_BOUNDARY = -3 };
/* VertexGeometryType subset, Src/flowfield_host_device.h:77-144 */
enum { VG_FLUID = 0, VG_IMMERSED_SOLID = -1 };
/* BndryDvType, Src/boundary_host_device.h:34-39 */
enum { DV_INCOMING = 1, DV_OUTGOING = 2, DV_PARALLEL = 3, DV_INVALID = -1 };

typedef struct {
    int id;
    int n[3];     /* interior nodes per axis (n[2] = 1 in 2D) */
    int h[3];     /* halo depth per axis */
    int a[3];     /* allocated points per axis */
    double* f;
    double* fs;   /* fStage */
    double* mac[4];
    double* old[4];
    int* vt;
    int* vg;
} oblock;

typedef struct {
    int from, to;
    int iter[3], fbase[3], tbase[3];
} ohalo;

struct lbm_oracle {
    int dim, Q, nmac;
    double cs, tau, dt;
    int body_force, force_vel;
    int swap;     /* Scheme_StreamCollision_Swap */
    double accel[3];
    double xi[19 * 3];
    double w[19];
    int opp[19];
    int nb;
    oblock* b;
    int nbc;
    mplbgpu_boundary* bc;
    double** bc_field; /* per boundary: (u, v, w) per node of its range or
                          NULL (a new-build extension of GivenVars) */
    int nhalo;
    ohalo* halo;
};

static oblock* find_block(lbm_oracle* o, int id);

static char g_err[256];
const char* lbmo_error(void) { return g_err; }
static int fail(const char* msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return -1;
}

static size_t pidx(const oblock* b, int i, int j, int k) {
    return ((size_t)(k + b->h[2]) * (size_t)b->a[1] + (size_t)(j + b->h[1])) *
               (size_t)b->a[0] +
           (size_t)(i + b->h[0]);
}

/* SetupD2Q9Latt / SetupD3Q19Latt / FindReverseXi, Src/model.cpp:82-131 */
static void setup_lattice(lbm_oracle* o) {
    if (o->Q == 9) {
        const double t00 = 4.0 / 9.0, t01 = 1.0 / 9.0, t11 = 1.0 / 36.0;
        const double t[9] = {t00, t11, t01, t11, t01, t11, t01, t11, t01};
        const int cx[9] = {0, -1, -1, -1, 0, 1, 1, 1, 0};
        const int cy[9] = {0, 1, 0, -1, -1, -1, 0, 1, 1};
        const int op[9] = {0, 5, 6, 7, 8, 1, 2, 3, 4};
        for (int l = 0; l < 9; l++) {
            o->xi[l * 2] = cx[l];
            o->xi[l * 2 + 1] = cy[l];
            o->w[l] = t[l];
            o->opp[l] = op[l];
        }
    } else {
        const double t000 = 1 / ((double)3), t001 = 1 / ((double)18),
                     t011 = 1 / ((double)36);
        const double t[19] = {t000, t001, t001, t001, t011, t011, t011,
                              t011, t011, t011, t001, t001, t001, t011,
                              t011, t011, t011, t011, t011};
        const int cx[19] = {0, -1, 0, 0, -1, -1, -1, -1, 0, 0,
                            1, 0, 0, 1, 1, 1, 1, 0, 0};
        const int cy[19] = {0, 0, -1, 0, -1, 1, 0, 0, -1, -1,
                            0, 1, 0, 1, -1, 0, 0, 1, 1};
        const int cz[19] = {0, 0, 0, -1, 0, 0, -1, 1, -1, 1,
                            0, 0, 1, 0, 0, 1, -1, 1, -1};
        for (int l = 0; l < 19; l++) {
            o->xi[l * 3] = cx[l];
            o->xi[l * 3 + 1] = cy[l];
            o->xi[l * 3 + 2] = cz[l];
            o->w[l] = t[l];
        }
        for (int i = 0; i < 19; i++) {
            for (int j = 0; j < 19; j++) {
                int rev = 1;
                for (int k = 0; k < 3; k++) {
                    rev = rev && (o->xi[i * 3 + k] + o->xi[j * 3 + k] == 0.0);
                }
                if (rev) {
                    o->opp[i] = j;
                    break;
                }
            }
        }
    }
}

static int C(const lbm_oracle* o, int l, int axis) {
    return axis < o->dim ? (int)o->xi[l * o->dim + axis] : 0;
}

/* CalcBGKFeq, Src/model_host_device.h:34-82 (T = 1, polyOrder = 2) */
static double feq(const lbm_oracle* o, int l, double rho, double u, double v,
                  double w) {
    const double CS = o->cs;
    const int D = o->dim;
    const double* XI = o->xi;
    const double T = 1;
    double cu, c2, u2;
    if (D == 2) {
        cu = (CS * XI[l * D] * u + CS * XI[l * D + 1] * v);
        c2 = (CS * XI[l * D] * CS * XI[l * D] +
              CS * XI[l * D + 1] * CS * XI[l * D + 1]);
        u2 = u * u + v * v;
    } else {
        cu = (CS * XI[l * D] * u + CS * XI[l * D + 1] * v +
              CS * XI[l * D + 2] * w);
        c2 = (CS * XI[l * D] * CS * XI[l * D] +
              CS * XI[l * D + 1] * CS * XI[l * D + 1] +
              CS * XI[l * D + 2] * CS * XI[l * D + 2]);
        u2 = u * u + v * v + w * w;
    }
    const double cu2 = cu * cu;
    const double res = 1.0 + cu + 0.5 * (cu2 - u2 + (T - 1.0) * (c2 - D));
    return o->w[l] * rho * res;
}

/* Block::RangeStart/RangeEnd, Src/block.cpp:14-97.  The y-range of the
 * TopBack/TopFront edges is left whole: the reference guards that test with
 * the undefined macro OP_3D (Src/block.cpp:35). */
static void surface_range(const lbm_oracle* o, const oblock* b, int s,
                          int r[6]) {
    for (int a = 0; a < 3; a++) {
        r[2 * a] = 0;
        r[2 * a + 1] = b->n[a];
    }
    const int d3 = o->dim == 3;
    if (s == MPLBGPU_RIGHT || s == MPLBGPU_RIGHT_TOP ||
        s == MPLBGPU_RIGHT_BOTTOM ||
        (d3 && (s == MPLBGPU_RIGHT_FRONT || s == MPLBGPU_RIGHT_BACK)))
        r[0] = b->n[0] - 1;
    if (s == MPLBGPU_LEFT || s == MPLBGPU_LEFT_BOTTOM || s == MPLBGPU_LEFT_TOP ||
        (d3 && (s == MPLBGPU_LEFT_FRONT || s == MPLBGPU_LEFT_BACK)))
        r[1] = 1;
    if (s == MPLBGPU_TOP || s == MPLBGPU_LEFT_TOP || s == MPLBGPU_RIGHT_TOP)
        r[2] = b->n[1] - 1;
    if (s == MPLBGPU_BOTTOM || s == MPLBGPU_LEFT_BOTTOM ||
        s == MPLBGPU_RIGHT_BOTTOM ||
        (d3 && (s == MPLBGPU_BOTTOM_BACK || s == MPLBGPU_BOTTOM_FRONT)))
        r[3] = 1;
    if (d3) {
        if (s == MPLBGPU_FRONT || s == MPLBGPU_LEFT_FRONT ||
            s == MPLBGPU_RIGHT_FRONT || s == MPLBGPU_TOP_FRONT ||
            s == MPLBGPU_BOTTOM_FRONT)
            r[4] = b->n[2] - 1;
        if (s == MPLBGPU_BACK || s == MPLBGPU_LEFT_BACK ||
            s == MPLBGPU_RIGHT_BACK || s == MPLBGPU_TOP_BACK ||
            s == MPLBGPU_BOTTOM_BACK)
            r[5] = 1;
    }
}

static int valid_surface(int dim, int s) {
    switch (s) {
        case MPLBGPU_LEFT: case MPLBGPU_RIGHT: case MPLBGPU_TOP:
        case MPLBGPU_BOTTOM: case MPLBGPU_LEFT_TOP: case MPLBGPU_LEFT_BOTTOM:
        case MPLBGPU_RIGHT_TOP: case MPLBGPU_RIGHT_BOTTOM:
            return 1;
        case MPLBGPU_FRONT: case MPLBGPU_BACK: case MPLBGPU_LEFT_BACK:
        case MPLBGPU_LEFT_FRONT: case MPLBGPU_RIGHT_BACK:
        case MPLBGPU_RIGHT_FRONT: case MPLBGPU_TOP_BACK: case MPLBGPU_TOP_FRONT:
        case MPLBGPU_BOTTOM_BACK: case MPLBGPU_BOTTOM_FRONT:
            return dim == 3;
        default:
            return 0;
    }
}

static void fill_int(const oblock* b, int* field, const int r[6], int value) {
    for (int k = r[4]; k < r[5]; k++)
        for (int j = r[2]; j < r[3]; j++)
            for (int i = r[0]; i < r[1]; i++) field[pidx(b, i, j, k)] = value;
}

/* Geometry code of a surface/edge/corner: faces 10*(axis+1) + (minus side),
 * edges A*1000 + B*10, corners A*100000 + B*1000 + C*10 (inner "_I"
 * codes), Src/flowfield_host_device.h:77-144. */
static int face_code(int axis, int maxside) { return 10 * (axis + 1) + maxside; }

/* SetBlockGeometryProperty, Src/flowfield_wrapper.cpp:291-623 */
static void set_geometry(const lbm_oracle* o, oblock* b) {
    int r[6];
    const int nx = b->n[0], ny = b->n[1], nz = b->n[2];
    const int d3 = o->dim == 3;
    int bulk[6] = {1, nx - 1, 1, ny - 1, d3 ? 1 : 0, d3 ? nz - 1 : 1};
    fill_int(b, b->vg, bulk, VG_FLUID);
    /* halo shells */
    for (int a = 0; a < o->dim; a++) {
        for (int side = 0; side < 2; side++) {
            int hr[6] = {-b->h[0], nx + b->h[0], -b->h[1], ny + b->h[1],
                         -b->h[2], nz + b->h[2]};
            if (side == 0) {
                hr[2 * a] = -1;
                hr[2 * a + 1] = 0;
            } else {
                hr[2 * a] = b->n[a];
                hr[2 * a + 1] = b->n[a] + 1;
            }
            fill_int(b, b->vg, hr, VG_IMMERSED_SOLID);
        }
    }
    /* faces (Bottom, Top, Left, Right, Back, Front) */
    const int faces[6] = {MPLBGPU_BOTTOM, MPLBGPU_TOP, MPLBGPU_LEFT,
                          MPLBGPU_RIGHT, MPLBGPU_BACK, MPLBGPU_FRONT};
    const int codes[6] = {face_code(1, 0), face_code(1, 1), face_code(0, 0),
                          face_code(0, 1), face_code(2, 0), face_code(2, 1)};
    for (int f = 0; f < (d3 ? 6 : 4); f++) {
        surface_range(o, b, faces[f], r);
        fill_int(b, b->vg, r, codes[f]);
    }
    /* edges (2D corners): every pair of axes, both sides */
    for (int a0 = 0; a0 < o->dim; a0++) {
        for (int a1 = a0 + 1; a1 < o->dim; a1++) {
            for (int s0 = 0; s0 < 2; s0++) {
                for (int s1 = 0; s1 < 2; s1++) {
                    int er[6] = {0, nx, 0, ny, 0, nz};
                    er[2 * a0] = s0 ? b->n[a0] - 1 : 0;
                    er[2 * a0 + 1] = s0 ? b->n[a0] : 1;
                    er[2 * a1] = s1 ? b->n[a1] - 1 : 0;
                    er[2 * a1 + 1] = s1 ? b->n[a1] : 1;
                    fill_int(b, b->vg, er,
                             face_code(a0, s0) * 1000 + face_code(a1, s1) * 10);
                }
            }
        }
    }
    if (d3) {
        for (int s0 = 0; s0 < 2; s0++)
            for (int s1 = 0; s1 < 2; s1++)
                for (int s2 = 0; s2 < 2; s2++) {
                    int cr[6] = {s0 ? nx - 1 : 0, s0 ? nx : 1,
                                 s1 ? ny - 1 : 0, s1 ? ny : 1,
                                 s2 ? nz - 1 : 0, s2 ? nz : 1};
                    fill_int(b, b->vg, cr,
                             face_code(0, s0) * 100000 +
                                 face_code(1, s1) * 1000 +
                                 face_code(2, s2) * 10);
                }
    }
}

/* Splits a geometry code into its faces: returns the number of axes (0 for
 * VG_Fluid and halo codes) with axis[] and sign[] (+1 for the "P" side,
 * i.e. the normal points to +axis). */
static int decode_vg(int code, int axis[3], int sign[3]) {
    if (code <= 0) return 0;
    int parts[3], n = 0;
    if (code >= 1000000) {
        parts[0] = code / 100000;
        parts[1] = (code / 1000) % 100;
        parts[2] = (code / 10) % 100;
        n = 3;
    } else if (code >= 10000) {
        parts[0] = code / 1000;
        parts[1] = (code / 10) % 100;
        n = 2;
    } else {
        parts[0] = code;
        n = 1;
    }
    for (int p = 0; p < n; p++) {
        axis[p] = parts[p] / 10 - 1;
        sign[p] = (parts[p] % 10) ? -1 : 1;
    }
    return n;
}

/* FindBdyDvType / FindBdyDvType3D, Src/boundary_host_device.h:47-706, inner
 * codes.  Faces: by the sign of the inward component.  Edges: incoming if
 * (a <= 0 && b < 0) || (a < 0 && b == 0) in inward components.  3D corners
 * keep the reference's labelling: all inward components <= 0 is Outgoing,
 * all >= 0 is Incoming. */
static int bdy_dv_type(const lbm_oracle* o, int vg, int l) {
    int axis[3], sign[3];
    const int n = decode_vg(vg, axis, sign);
    int c[3];
    for (int p = 0; p < n; p++) c[p] = sign[p] * C(o, l, axis[p]);
    if (n == 1) {
        return c[0] < 0 ? DV_INCOMING : (c[0] == 0 ? DV_PARALLEL : DV_OUTGOING);
    }
    if (n == 2) {
        if ((c[0] <= 0 && c[1] < 0) || (c[0] < 0 && c[1] == 0))
            return DV_INCOMING;
        if ((c[0] >= 0 && c[1] > 0) || (c[0] > 0 && c[1] == 0))
            return DV_OUTGOING;
        return DV_PARALLEL;
    }
    if (n == 3) {
        if (c[0] == 0 && c[1] == 0 && c[2] == 0) return DV_PARALLEL;
        if (c[0] <= 0 && c[1] <= 0 && c[2] <= 0) return DV_OUTGOING;
        if (c[0] >= 0 && c[1] >= 0 && c[2] >= 0) return DV_INCOMING;
        return DV_PARALLEL;
    }
    return DV_INVALID;
}

/* Stream selection of KerStream / KerStream3D for boundary-typed nodes,
 * Src/scheme_kernel.inc:53-221, 1400-2051: pull direction l when every
 * inward component of c_l is <= 0 (faces: one, edges: both, corners: all). */
static int is_fluidlike(int vt);

static int stream_pulls(const lbm_oracle* o, int vg, int l) {
    int axis[3], sign[3];
    const int n = decode_vg(vg, axis, sign);
    if (n == 0) return 0;
    for (int p = 0; p < n; p++) {
        if (sign[p] * C(o, l, axis[p]) > 0) return 0;
    }
    return 1;
}

int lbmo_create(const mplbgpu_desc* d, lbm_oracle** out) {
    *out = NULL;
    if (!d || d->abi_version != MPLBGPU_ABI_VERSION) return fail("abi");
    if (!((d->space_dim == 2 && d->lattice == MPLBGPU_D2Q9) ||
          (d->space_dim == 3 && d->lattice == MPLBGPU_D3Q19)))
        return fail("lattice/dimension");
    if (d->nblocks < 1) return fail("no blocks");
    for (int i = 0; i < d->nblocks; i++)
        if (d->blocks[i].cut != 0)
            return fail("decomposed (cut) blocks are not restated here");
    lbm_oracle* o = (lbm_oracle*)calloc(1, sizeof(lbm_oracle));
    o->dim = d->space_dim;
    o->Q = d->lattice;
    o->nmac = d->space_dim + 1;
    o->cs = d->cs;
    o->tau = d->tau_ref;
    o->dt = d->dt;
    o->body_force = d->body_force;
    o->force_vel = d->force_velocity;
    o->swap = d->scheme == MPLBGPU_SCHEME_STREAM_COLLISION_SWAP;
    if (d->scheme != 0 && d->scheme != MPLBGPU_SCHEME_STREAM_COLLISION &&
        !o->swap) {
        free(o);
        return fail("unknown scheme");
    }
    if (o->swap && (d->space_dim != 3 || d->nblocks != 1 ||
                    d->nconnections != 0)) {
        free(o);
        return fail("the swap scheme runs on one 3D block without "
                    "connections");
    }
    for (int a = 0; a < 3; a++) o->accel[a] = d->accel[a];
    setup_lattice(o);
    /* blocks sorted by id: the reference keeps them in a std::map */
    o->nb = d->nblocks;
    o->b = (oblock*)calloc((size_t)o->nb, sizeof(oblock));
    for (int i = 0; i < o->nb; i++) o->b[i].id = d->blocks[i].id;
    for (int i = 0; i < o->nb; i++) {
        for (int j = i + 1; j < o->nb; j++) {
            if (o->b[j].id < o->b[i].id) {
                oblock t = o->b[i];
                o->b[i] = o->b[j];
                o->b[j] = t;
            }
        }
    }
    for (int i = 0; i < o->nb; i++) {
        oblock* b = &o->b[i];
        const mplbgpu_block* src = NULL;
        for (int j = 0; j < d->nblocks; j++)
            if (d->blocks[j].id == b->id) src = &d->blocks[j];
        for (int a = 0; a < 3; a++) {
            b->n[a] = a < o->dim ? src->size[a] : 1;
            b->h[a] = a < o->dim ? 1 : 0;
            b->a[a] = b->n[a] + 2 * b->h[a];
            if (b->n[a] < (a < o->dim ? 2 : 1)) {
                lbmo_destroy(o);
                return fail("block too small");
            }
        }
        const size_t pts = (size_t)b->a[0] * b->a[1] * b->a[2];
        b->f = (double*)calloc(pts * o->Q, sizeof(double));
        b->fs = (double*)calloc(pts * o->Q, sizeof(double));
        for (int m = 0; m < o->nmac; m++) {
            b->mac[m] = (double*)calloc(pts, sizeof(double));
            b->old[m] = (double*)calloc(pts, sizeof(double));
        }
        b->vt = (int*)calloc(pts, sizeof(int));
        b->vg = (int*)calloc(pts, sizeof(int));
    }
    /* boundaries, in definition order */
    o->nbc = d->nboundaries;
    o->bc = (mplbgpu_boundary*)calloc((size_t)(o->nbc + 1),
                                      sizeof(mplbgpu_boundary));
    o->bc_field = (double**)calloc((size_t)(o->nbc + 1), sizeof(double*));
    for (int i = 0; i < o->nbc; i++) {
        o->bc[i] = d->boundaries[i];
        if (!valid_surface(o->dim, o->bc[i].surface)) {
            lbmo_destroy(o);
            return fail("bad surface");
        }
        if (o->bc[i].scheme == MPLBGPU_BC_FDPERIODIC && o->swap) {
            lbmo_destroy(o);
            return fail("FDPeriodic with the swap scheme");
        }
        if (o->swap && (o->bc[i].scheme == MPLBGPU_BC_EXTRAPOL_PRESSURE_1ST ||
                        o->bc[i].scheme == MPLBGPU_BC_HALFWAY_BOUNCE_BACK)) {
            lbmo_destroy(o);
            return fail("the swap scheme takes node-local boundary "
                        "conditions only");
        }
        int found = 0;
        for (int j = 0; j < o->nb; j++) found |= o->b[j].id == o->bc[i].block;
        if (!found) {
            lbmo_destroy(o);
            return fail("boundary on unknown block");
        }
    }
    /* Field::CreateHalos, Src/field.h:215-395: blocks by id, neighbours by
     * surface value; each connection copies this block's face layer into
     * the neighbour's halo. */
    o->halo = (ohalo*)calloc((size_t)(d->nconnections + 1), sizeof(ohalo));
    o->nhalo = 0;
    for (int bi = 0; bi < o->nb; bi++) {
        for (int s = 0; s <= 5; s++) {
            for (int c = 0; c < d->nconnections; c++) {
                const mplbgpu_connection* cn = &d->connections[c];
                if (cn->from_block != o->b[bi].id || cn->from_surface != s)
                    continue;
                int ti = -1;
                for (int j = 0; j < o->nb; j++)
                    if (o->b[j].id == cn->to_block) ti = j;
                if (ti < 0) {
                    lbmo_destroy(o);
                    return fail("connection to unknown block");
                }
                const oblock* fb = &o->b[bi];
                const oblock* tb = &o->b[ti];
                const int axis = s < 2 ? 0 : (s < 4 ? 1 : 2);
                if (axis >= o->dim) {
                    lbmo_destroy(o);
                    return fail("bad connection surface");
                }
                const int maxside = (s == MPLBGPU_RIGHT || s == MPLBGPU_TOP ||
                                     s == MPLBGPU_FRONT);
                const int disp = (cn->type == MPLBGPU_VT_FDPERIODIC ||
                                  cn->type == MPLBGPU_VT_MDPERIODIC ||
                                  cn->type == MPLBGPU_VT_VIRTUAL_BOUNDARY)
                                     ? -1
                                     : 0;
                ohalo* h = &o->halo[o->nhalo++];
                h->from = bi;
                h->to = ti;
                for (int a = 0; a < 3; a++) {
                    h->iter[a] = fb->n[a] + 2 * fb->h[a];
                    h->fbase[a] = -fb->h[a];
                    h->tbase[a] = -tb->h[a];
                    if (a != axis && a < o->dim && fb->n[a] != tb->n[a]) {
                        lbmo_destroy(o);
                        return fail("connected blocks differ in size");
                    }
                }
                h->iter[axis] = 1;
                if (maxside) {
                    h->fbase[axis] = fb->n[axis] + disp;
                    h->tbase[axis] = -1;
                } else {
                    h->fbase[axis] = 0;
                    h->tbase[axis] = tb->n[axis];
                }
            }
        }
    }
    /* PrepareFlowField, Src/flowfield.cpp:224-244 */
    for (int bi = 0; bi < o->nb; bi++) {
        oblock* b = &o->b[bi];
        set_geometry(o, b);
        /* SetBulkandHaloNodesType, Src/flowfield_wrapper.cpp:671-788 */
        const int d3 = o->dim == 3;
        int bulk[6] = {1, b->n[0] - 1, 1, b->n[1] - 1, d3 ? 1 : 0,
                       d3 ? b->n[2] - 1 : 1};
        fill_int(b, b->vt, bulk, VT_FLUID);
        for (int a = 0; a < o->dim; a++) {
            for (int side = 0; side < 2; side++) {
                int hr[6] = {-b->h[0], b->n[0] + b->h[0], -b->h[1],
                             b->n[1] + b->h[1], -b->h[2], b->n[2] + b->h[2]};
                hr[2 * a] = side ? b->n[a] : -1;
                hr[2 * a + 1] = side ? b->n[a] + 1 : 0;
                fill_int(b, b->vt, hr, VT_IMMERSED_SOLID);
            }
        }
    }
    /* SetBoundaryNodeType, Src/flowfield_wrapper.cpp:625-669 */
    for (int i = 0; i < o->nbc; i++) {
        const mplbgpu_boundary* bc = &o->bc[i];
        oblock* b = NULL;
        for (int j = 0; j < o->nb; j++)
            if (o->b[j].id == bc->block) b = &o->b[j];
        int r[6];
        surface_range(o, b, bc->surface, r);
        if (bc->vertex_type == MPLBGPU_VT_VIRTUAL_BOUNDARY) {
            const int s = bc->surface;
            if (s == MPLBGPU_LEFT || s == MPLBGPU_RIGHT) {
                r[2]++; r[3]--;
                if (o->dim == 3) { r[4]++; r[5]--; }
            }
            if (s == MPLBGPU_TOP || s == MPLBGPU_BOTTOM) {
                r[0]++; r[1]--;
                if (o->dim == 3) { r[4]++; r[5]--; }
            }
            if (o->dim == 3 && (s == MPLBGPU_FRONT || s == MPLBGPU_BACK)) {
                r[0]++; r[1]--; r[2]++; r[3]--;
            }
        }
        fill_int(b, b->vt, r, bc->vertex_type);
    }
    if (o->swap) {
        /* a fluid-like node on the block boundary would swap with its halo */
        const oblock* b = &o->b[0];
        for (int k = 0; k < b->n[2]; k++)
            for (int j = 0; j < b->n[1]; j++)
                for (int i = 0; i < b->n[0]; i++) {
                    if (i > 0 && i < b->n[0] - 1 && j > 0 &&
                        j < b->n[1] - 1 && k > 0 && k < b->n[2] - 1)
                        continue;
                    const int vt = b->vt[pidx(b, i, j, k)];
                    if (is_fluidlike(vt) || vt == VT_VIRTUAL_BOUNDARY) {
                        lbmo_destroy(o);
                        return fail("the swap scheme needs a boundary "
                                    "condition on every block face");
                    }
                }
    }
    *out = o;
    return 0;
}

void lbmo_destroy(lbm_oracle* o) {
    if (!o) return;
    for (int i = 0; i < o->nb; i++) {
        oblock* b = &o->b[i];
        free(b->f);
        free(b->fs);
        for (int m = 0; m < 4; m++) {
            free(b->mac[m]);
            free(b->old[m]);
        }
        free(b->vt);
        free(b->vg);
    }
    free(o->b);
    for (int i = 0; i < o->nbc; i++) free(o->bc_field[i]);
    free(o->bc_field);
    free(o->bc);
    free(o->halo);
    free(o);
}

int lbmo_boundary_extent(lbm_oracle* o, int boundary, int ext[3]) {
    if (boundary < 0 || boundary >= o->nbc) return fail("unknown boundary");
    oblock* b = find_block(o, o->bc[boundary].block);
    if (!b) return fail("unknown block");
    int r[6];
    surface_range(o, b, o->bc[boundary].surface, r);
    for (int a = 0; a < 3; a++) ext[a] = r[2 * a + 1] - r[2 * a];
    return 0;
}

int lbmo_set_boundary_velocity(lbm_oracle* o, int boundary, const double* u,
                               const double* v, const double* w) {
    int ext[3];
    if (lbmo_boundary_extent(o, boundary, ext) != 0) return -1;
    const int s = o->bc[boundary].scheme;
    if (s != MPLBGPU_BC_EQM_DIFFUSE_REFL && s != MPLBGPU_BC_HALFWAY_BOUNCE_BACK)
        return fail("per-node velocity on a boundary without a wall kernel");
    if (o->swap) return fail("per-node velocity under the swap scheme");
    free(o->bc_field[boundary]);
    o->bc_field[boundary] = NULL;
    if (!u && !v && !w) return 0;
    const size_t cnt = (size_t)ext[0] * ext[1] * ext[2];
    double* f = (double*)calloc(3 * cnt, sizeof(double));
    const double* src[3] = {u, v, o->dim == 3 ? w : NULL};
    for (int c = 0; c < 3; c++)
        if (src[c])
            for (size_t k = 0; k < cnt; k++) f[3 * k + c] = src[c][k];
    o->bc_field[boundary] = f;
    return 0;
}

static oblock* find_block(lbm_oracle* o, int id) {
    for (int i = 0; i < o->nb; i++)
        if (o->b[i].id == id) return &o->b[i];
    return NULL;
}

static int is_fluidlike(int vt) {
    return vt == VT_FLUID || vt == VT_MDPERIODIC;
}

/* UpdateMacroVars3D / UpdateMacroVars with KerCalcDensity3D, KerCalcU3D...
 * and the Variable_U_Force family, Src/model_kernel.inc:570-759 */
static void update_macro(lbm_oracle* o) {
    const double CS = o->cs;
    const int D = o->dim, Q = o->Q;
    for (int bi = 0; bi < o->nb; bi++) {
        oblock* b = &o->b[bi];
        for (int k = 0; k < b->n[2]; k++)
            for (int j = 0; j < b->n[1]; j++)
                for (int i = 0; i < b->n[0]; i++) {
                    const size_t p = pidx(b, i, j, k);
                    const int vt = b->vt[p];
                    if (vt == VT_IMMERSED_SOLID) continue;
                    const double* f = &b->f[p * Q];
                    double rho = 0;
                    for (int l = 0; l < Q; l++) rho += f[l];
                    b->mac[0][p] = rho;
                    for (int a = 0; a < D; a++) {
                        double u = 0;
                        for (int l = 0; l < Q; l++)
                            u += CS * o->xi[l * D + a] * f[l];
                        u /= b->mac[0][p];
                        if (o->force_vel && is_fluidlike(vt)) {
                            u += (o->dt * o->accel[a] / 2);
                        }
                        b->mac[1 + a][p] = u;
                    }
                }
    }
}

int lbmo_update_macro(lbm_oracle* o) {
    update_macro(o);
    return 0;
}

/* CopyCurrentMacroVar, Src/flowfield_wrapper.cpp:10-29 */
static void copy_macro(lbm_oracle* o) {
    for (int bi = 0; bi < o->nb; bi++) {
        oblock* b = &o->b[bi];
        for (int k = 0; k < b->n[2]; k++)
            for (int j = 0; j < b->n[1]; j++)
                for (int i = 0; i < b->n[0]; i++) {
                    const size_t p = pidx(b, i, j, k);
                    for (int m = 0; m < o->nmac; m++) b->old[m][p] = b->mac[m][p];
                }
    }
}

int lbmo_init_macro(lbm_oracle* o, int block, const double* rho,
                    const double* u, const double* v, const double* w) {
    oblock* b = find_block(o, block);
    if (!b) return fail("unknown block");
    const double* src[4] = {rho, u, v, w};
    size_t n = 0;
    for (int k = 0; k < b->n[2]; k++)
        for (int j = 0; j < b->n[1]; j++)
            for (int i = 0; i < b->n[0]; i++, n++) {
                const size_t p = pidx(b, i, j, k);
                for (int m = 0; m < o->nmac; m++) {
                    b->mac[m][p] = src[m] ? src[m][n] : (m == 0 ? 1.0 : 0.0);
                }
                /* KerInitialiseBGK2nd(3D), Src/model_kernel.inc:193-219,
                 * 352-380 */
                if (b->vt[p] != VT_IMMERSED_SOLID) {
                    for (int l = 0; l < o->Q; l++) {
                        b->f[p * o->Q + l] =
                            feq(o, l, b->mac[0][p], b->mac[1][p], b->mac[2][p],
                                o->dim == 3 ? b->mac[3][p] : 0.0);
                    }
                }
            }
    copy_macro(o);
    return 0;
}

int lbmo_set_f(lbm_oracle* o, int block, const double* f) {
    oblock* b = find_block(o, block);
    if (!b) return fail("unknown block");
    size_t n = 0;
    for (int k = 0; k < b->n[2]; k++)
        for (int j = 0; j < b->n[1]; j++)
            for (int i = 0; i < b->n[0]; i++, n++) {
                memcpy(&b->f[pidx(b, i, j, k) * o->Q], &f[n * o->Q],
                       sizeof(double) * o->Q);
            }
    return 0;
}

/* KerCutCellPeriodic(3D), Src/boundary_kernel.inc:615-719, 1278-1666:
 * f(node) = f(node + off) for every population, for the offsets the
 * kernel's switch takes at a node of geometry vg when it treats `surface`
 * (edge and corner cases compare the surface with face values).  The
 * sources are halo cells of f, which the step never writes. */
static int fd_copies(int vg, int surface, int off[3][3]) {
    int n = 0;
#define FD_ADD(cond, x, y, z)                                               \
    do {                                                                    \
        if (cond) {                                                         \
            off[n][0] = (x);                                                \
            off[n][1] = (y);                                                \
            off[n][2] = (z);                                                \
            n++;                                                            \
        }                                                                   \
    } while (0)
    const int L = surface == MPLBGPU_LEFT, R = surface == MPLBGPU_RIGHT,
              T = surface == MPLBGPU_TOP, B = surface == MPLBGPU_BOTTOM,
              F = surface == MPLBGPU_FRONT, K = surface == MPLBGPU_BACK;
    switch (vg) {
        case 10: FD_ADD(1, -1, 0, 0); break;
        case 11: FD_ADD(1, 1, 0, 0); break;
        case 20: FD_ADD(1, 0, -1, 0); break;
        case 21: FD_ADD(1, 0, 1, 0); break;
        case 30: FD_ADD(1, 0, 0, -1); break;
        case 31: FD_ADD(1, 0, 0, 1); break;
        case 10200: FD_ADD(L, -1, 0, 0); FD_ADD(B, 0, -1, 0); break;
        case 10210: FD_ADD(L, -1, 0, 0); FD_ADD(T, 0, 1, 0); break;
        case 11200: FD_ADD(R, 1, 0, 0); FD_ADD(B, 0, -1, 0); break;
        case 11210: FD_ADD(R, 1, 0, 0); FD_ADD(T, 0, 1, 0); break;
        case 10300: FD_ADD(L, -1, 0, 0); FD_ADD(K, 0, 0, -1); break;
        case 10310: FD_ADD(R, -1, 0, 0); FD_ADD(F, 0, 0, 1); break;
        case 11300: FD_ADD(R, 1, 0, 0); FD_ADD(K, 0, 0, -1); break;
        case 11310: FD_ADD(R, 1, 0, 0); FD_ADD(F, 0, 0, 1); break;
        case 20300: FD_ADD(B, 0, -1, 0); FD_ADD(K, 0, 0, -1); break;
        case 20310: FD_ADD(B, 0, -1, 0); FD_ADD(F, 0, 0, 1); break;
        case 21300: FD_ADD(T, 0, 1, 0); FD_ADD(F, 0, 0, -1); break;
        case 21310: FD_ADD(T, 0, 1, 0); FD_ADD(F, 0, 0, 1); break;
        case 1020300:
            FD_ADD(L, -1, 0, 0); FD_ADD(B, 0, -1, 0); FD_ADD(K, 0, 0, -1);
            break;
        case 1020310:
            FD_ADD(L, -1, 0, 0); FD_ADD(B, 0, -1, 0); FD_ADD(F, 0, 0, 1);
            break;
        case 1021300:
            FD_ADD(L, -1, 0, 0); FD_ADD(T, 0, 1, 0); FD_ADD(K, 0, 0, -1);
            break;
        case 1021310:
            FD_ADD(T, -1, 0, 0); FD_ADD(T, 0, 1, 0); FD_ADD(F, 0, 0, 1);
            break;
        case 1120300:
            FD_ADD(R, 1, 0, 0); FD_ADD(B, 0, -1, 0); FD_ADD(K, 0, 0, -1);
            break;
        case 1120310:
            FD_ADD(R, 1, 0, 0); FD_ADD(B, 0, -1, 0); FD_ADD(F, 0, 0, 1);
            break;
        case 1121300:
            FD_ADD(R, 1, 0, 0); FD_ADD(T, 0, 1, 0); FD_ADD(K, 0, 0, -1);
            break;
        case 1121310:
            FD_ADD(R, 1, 0, 0); FD_ADD(T, 0, 1, 0); FD_ADD(F, 0, 0, 1);
            break;
        default:
            break;
    }
#undef FD_ADD
    return n;
}

static void bc_fdperiodic(lbm_oracle* o, oblock* b, const int r[6],
                          int surface) {
    const int Q = o->Q;
    for (int k = r[4]; k < r[5]; k++)
        for (int j = r[2]; j < r[3]; j++)
            for (int i = r[0]; i < r[1]; i++) {
                const size_t p = pidx(b, i, j, k);
                int off[3][3];
                const int nc = fd_copies(b->vg[p], surface, off);
                for (int c = 0; c < nc; c++) {
                    const size_t q = pidx(b, i + off[c][0], j + off[c][1],
                                          k + off[c][2]);
                    for (int l = 0; l < Q; l++)
                        b->f[p * Q + l] = b->f[q * Q + l];
                }
            }
}

/* KerCutCellEQMDiffuseRefl(3D), Src/boundary_kernel.inc:534-613,1184-1276 */
/* Wall velocity of node (i, j, k) of range r: the boundary's uniform
 * GivenVars, or its entry of a per-node field over the range (x fastest;
 * not in the reference, whose GivenVars are uniform). */
static const double* wall_velocity(const double* given, const double* field,
                                   const int r[6], int i, int j, int k) {
    if (!field) return given;
    const size_t idx = ((size_t)(k - r[4]) * (size_t)(r[3] - r[2]) +
                        (size_t)(j - r[2])) * (size_t)(r[1] - r[0]) +
                       (size_t)(i - r[0]);
    return &field[3 * idx];
}

static void bc_eqm(lbm_oracle* o, oblock* b, const int r[6],
                   const double* given, const double* field) {
    const double CS = o->cs;
    const int D = o->dim, Q = o->Q;
    for (int k = r[4]; k < r[5]; k++)
        for (int j = r[2]; j < r[3]; j++)
            for (int i = r[0]; i < r[1]; i++) {
                const double* g = wall_velocity(given, field, r, i, j, k);
                const double u = g[0], v = g[1], w = D == 3 ? g[2] : 0.0;
                const size_t p = pidx(b, i, j, k);
                const int vg = b->vg[p];
                double* f = &b->f[p * Q];
                int outgoing[19], parallel[19];
                int nout = 0, npar = 0;
                double rhoIncoming = 0, rhoParallel = 0, deltaRho = 0;
                for (int l = 0; l < Q; l++) {
                    const double cx = CS * o->xi[l * D];
                    const double cy = CS * o->xi[l * D + 1];
                    const double cz = D == 3 ? CS * o->xi[l * D + 2] : 0.0;
                    switch (bdy_dv_type(o, vg, l)) {
                        case DV_INCOMING:
                            rhoIncoming += f[l];
                            break;
                        case DV_OUTGOING:
                            outgoing[nout++] = l;
                            if (D == 3)
                                deltaRho += (2 * o->w[l]) *
                                            (cx * u + cy * v + cz * w);
                            else
                                deltaRho += (2 * o->w[l]) * (cx * u + cy * v);
                            break;
                        case DV_PARALLEL:
                            parallel[npar++] = l;
                            rhoParallel += feq(o, l, 1, u, v, w);
                            break;
                        default:
                            break;
                    }
                }
                const double rhoWall =
                    2 * rhoIncoming / (1 - deltaRho - rhoParallel);
                for (int n = 0; n < npar; n++) {
                    f[parallel[n]] = feq(o, parallel[n], rhoWall, u, v, w);
                }
                for (int n = 0; n < nout; n++) {
                    const int l = outgoing[n];
                    const double cx = CS * o->xi[l * D];
                    const double cy = CS * o->xi[l * D + 1];
                    const double cz = D == 3 ? CS * o->xi[l * D + 2] : 0.0;
                    if (D == 3)
                        f[l] = f[o->opp[l]] + 2 * rhoWall * o->w[l] *
                                                  (cx * u + cy * v + cz * w);
                    else
                        f[l] = f[o->opp[l]] +
                               2 * rhoWall * o->w[l] * (cx * u + cy * v);
                }
            }
}

static int surface_face(int surface, int* axis, int* sign) {
    switch (surface) {
        case MPLBGPU_LEFT: *axis = 0; *sign = 1; return 1;
        case MPLBGPU_RIGHT: *axis = 0; *sign = -1; return 1;
        case MPLBGPU_BOTTOM: *axis = 1; *sign = 1; return 1;
        case MPLBGPU_TOP: *axis = 1; *sign = -1; return 1;
        case MPLBGPU_BACK: *axis = 2; *sign = 1; return 1;
        case MPLBGPU_FRONT: *axis = 2; *sign = -1; return 1;
        default: return 0;
    }
}

/* KerCutCellExtrapolPressure1ST(3D), Src/boundary_kernel.inc:404-488,
 * 894-1182.  Faces copy the inward-pointing populations from the inner
 * neighbour; edges and corners do so only along the axis of the surface
 * being treated.  Every population but the last is then rescaled. */
static void bc_extrapol(lbm_oracle* o, oblock* b, const int r[6],
                        int surface, double rhoGiven) {
    const int Q = o->Q;
    int saxis = -1, ssign = 0;
    const int isface = surface_face(surface, &saxis, &ssign);
    for (int k = r[4]; k < r[5]; k++)
        for (int j = r[2]; j < r[3]; j++)
            for (int i = r[0]; i < r[1]; i++) {
                const size_t p = pidx(b, i, j, k);
                const int vg = b->vg[p];
                int axis[3], sign[3];
                const int n = decode_vg(vg, axis, sign);
                double* f = &b->f[p * Q];
                double rho = 0;
                for (int l = 0; l < Q; l++) {
                    int c[3] = {0, 0, 0};
                    for (int q = 0; q < n; q++) c[q] = sign[q] * C(o, l, axis[q]);
                    int copy = 0;
                    if (n == 1) {
                        copy = c[0] > 0;
                    } else if (n == 2) {
                        copy = (c[0] >= 0 && c[1] > 0) || (c[0] > 0 && c[1] == 0);
                    } else if (n == 3) {
                        copy = (c[0] >= 0 && c[1] >= 0 && c[2] >= 0) &&
                               (c[0] != 0 || c[1] != 0 || c[2] != 0);
                    }
                    if (copy) {
                        int ax = -1, sg = 0;
                        if (n == 1) {
                            ax = axis[0];
                            sg = sign[0];
                        } else if (isface) {
                            for (int q = 0; q < n; q++)
                                if (axis[q] == saxis && sign[q] == ssign) {
                                    ax = axis[q];
                                    sg = sign[q];
                                }
                        }
                        if (ax >= 0) {
                            int s3[3] = {i, j, k};
                            s3[ax] += sg;
                            f[l] = b->f[pidx(b, s3[0], s3[1], s3[2]) * Q + l];
                        }
                    }
                    rho += f[l];
                }
                const double ratio = rhoGiven / rho;
                for (int l = 0; l < Q - 1; l++) f[l] *= ratio;
            }
}

/* Faces of a surface or edge (Src/boundary_host_device.h:7-29): axis and
 * side (0 = min, 1 = max). */
static int surface_sides(int s, int axis[2], int side[2]) {
    int n = 0;
    if (s == MPLBGPU_LEFT || s == MPLBGPU_LEFT_BACK || s == MPLBGPU_LEFT_FRONT ||
        s == MPLBGPU_LEFT_TOP || s == MPLBGPU_LEFT_BOTTOM) {
        axis[n] = 0; side[n++] = 0;
    }
    if (s == MPLBGPU_RIGHT || s == MPLBGPU_RIGHT_BACK ||
        s == MPLBGPU_RIGHT_FRONT || s == MPLBGPU_RIGHT_TOP ||
        s == MPLBGPU_RIGHT_BOTTOM) {
        axis[n] = 0; side[n++] = 1;
    }
    if (s == MPLBGPU_BOTTOM || s == MPLBGPU_BOTTOM_BACK ||
        s == MPLBGPU_BOTTOM_FRONT || s == MPLBGPU_LEFT_BOTTOM ||
        s == MPLBGPU_RIGHT_BOTTOM) {
        axis[n] = 1; side[n++] = 0;
    }
    if (s == MPLBGPU_TOP || s == MPLBGPU_TOP_BACK || s == MPLBGPU_TOP_FRONT ||
        s == MPLBGPU_LEFT_TOP || s == MPLBGPU_RIGHT_TOP) {
        axis[n] = 1; side[n++] = 1;
    }
    if (s == MPLBGPU_BACK || s == MPLBGPU_LEFT_BACK || s == MPLBGPU_RIGHT_BACK ||
        s == MPLBGPU_TOP_BACK || s == MPLBGPU_BOTTOM_BACK) {
        axis[n] = 2; side[n++] = 0;
    }
    if (s == MPLBGPU_FRONT || s == MPLBGPU_LEFT_FRONT ||
        s == MPLBGPU_RIGHT_FRONT || s == MPLBGPU_TOP_FRONT ||
        s == MPLBGPU_BOTTOM_FRONT) {
        axis[n] = 2; side[n++] = 1;
    }
    return n;
}

/* Link-wise halfway bounce-back of this path (no reference kernel): a
 * population whose upstream node x - c_l lies beyond one of the surface's
 * faces takes the node's own post-collision opposite population plus
 * 2 w_l (c_l . u_wall); the wall sits half a spacing beyond the face. */
static void bc_halfway_bb(lbm_oracle* o, oblock* b, const int r[6],
                          int surface, const double* given,
                          const double* field) {
    const double CS = o->cs;
    const int D = o->dim, Q = o->Q;
    int axis[2], side[2];
    const int nf = surface_sides(surface, axis, side);
    for (int k = r[4]; k < r[5]; k++)
        for (int j = r[2]; j < r[3]; j++)
            for (int i = r[0]; i < r[1]; i++) {
                const size_t p = pidx(b, i, j, k);
                const int x[3] = {i, j, k};
                const double* g = wall_velocity(given, field, r, i, j, k);
                for (int l = 0; l < Q; l++) {
                    int beyond = 0;
                    for (int q = 0; q < nf; q++) {
                        const int s = x[axis[q]] - C(o, l, axis[q]);
                        beyond |= side[q] ? (s > b->n[axis[q]] - 1) : (s < 0);
                    }
                    if (!beyond) continue;
                    double cu = CS * o->xi[l * D] * g[0] +
                                CS * o->xi[l * D + 1] * g[1];
                    if (D == 3) cu = cu + CS * o->xi[l * D + 2] * g[2];
                    b->f[p * Q + l] =
                        b->fs[p * Q + o->opp[l]] + 2.0 * o->w[l] * cu;
                }
            }
}

static void one_step(lbm_oracle* o) {
    const int Q = o->Q, D = o->dim;
    const double CS = o->cs;
    /* UpdateMacroVars3D */
    update_macro(o);
    for (int bi = 0; bi < o->nb; bi++) {
        oblock* b = &o->b[bi];
        /* CopyBlockEnvelopDistribution(fStage, f),
         * Src/flowfield_wrapper.cpp:113-232 */
        const int faces[6] = {MPLBGPU_LEFT, MPLBGPU_RIGHT, MPLBGPU_BOTTOM,
                              MPLBGPU_TOP, MPLBGPU_BACK, MPLBGPU_FRONT};
        for (int fidx = 0; fidx < 2 * D; fidx++) {
            int r[6];
            surface_range(o, b, faces[fidx], r);
            for (int k = r[4]; k < r[5]; k++)
                for (int j = r[2]; j < r[3]; j++)
                    for (int i = r[0]; i < r[1]; i++) {
                        const size_t p = pidx(b, i, j, k);
                        memcpy(&b->fs[p * Q], &b->f[p * Q], sizeof(double) * Q);
                    }
        }
        const double tau = o->tau;
        const double dtOvertauPlusdt = o->dt / (tau + 0.5 * o->dt);
        for (int k = 0; k < b->n[2]; k++)
            for (int j = 0; j < b->n[1]; j++)
                for (int i = 0; i < b->n[0]; i++) {
                    const size_t p = pidx(b, i, j, k);
                    const int vt = b->vt[p];
                    double* fs = &b->fs[p * Q];
                    const double* f = &b->f[p * Q];
                    /* KerCalcBodyForce1ST3D / KerCalcBodyForceNone3D,
                     * Src/model_kernel.inc:504-541 with CalcBodyForce,
                     * Src/model_host_device.h:25-32 */
                    if (is_fluidlike(vt)) {
                        for (int l = 0; l < Q; l++) {
                            if (o->body_force == MPLBGPU_FORCE_1ST) {
                                double cf = 0;
                                for (int a = 0; a < D; a++)
                                    cf += CS * o->xi[l * D + a] * o->accel[a];
                                fs[l] = o->w[l] * b->mac[0][p] * cf;
                            } else {
                                fs[l] = 0;
                            }
                        }
                    }
                    /* KerCollideBGKIsothermal3D, Src/model_kernel.inc:410-455 */
                    if (vt == VT_IMMERSED_SOLID) continue;
                    const double rho = b->mac[0][p], u = b->mac[1][p],
                                 v = b->mac[2][p],
                                 w = D == 3 ? b->mac[3][p] : 0.0;
                    for (int l = 0; l < Q; l++) {
                        const double fe = feq(o, l, rho, u, v, w);
                        if (is_fluidlike(vt)) {
                            fs[l] = fe + (1 - dtOvertauPlusdt) * (f[l] - fe) +
                                    tau * dtOvertauPlusdt * fs[l];
                        } else {
                            fs[l] = fe + (1 - dtOvertauPlusdt) * (f[l] - fe);
                        }
                    }
                }
    }
    /* TransferHalos of fStage, Src/flowfield.cpp:294-302 */
    for (int hI = 0; hI < o->nhalo; hI++) {
        const ohalo* h = &o->halo[hI];
        const oblock* fb = &o->b[h->from];
        oblock* tb = &o->b[h->to];
        for (int k = 0; k < h->iter[2]; k++)
            for (int j = 0; j < h->iter[1]; j++)
                for (int i = 0; i < h->iter[0]; i++) {
                    const size_t ps = pidx(fb, h->fbase[0] + i,
                                           h->fbase[1] + j, h->fbase[2] + k);
                    const size_t pd = pidx(tb, h->tbase[0] + i,
                                           h->tbase[1] + j, h->tbase[2] + k);
                    memcpy(&tb->fs[pd * Q], &fb->fs[ps * Q], sizeof(double) * Q);
                }
    }
    /* KerStream / KerStream3D */
    for (int bi = 0; bi < o->nb; bi++) {
        oblock* b = &o->b[bi];
        for (int k = 0; k < b->n[2]; k++)
            for (int j = 0; j < b->n[1]; j++)
                for (int i = 0; i < b->n[0]; i++) {
                    const size_t p = pidx(b, i, j, k);
                    const int vt = b->vt[p];
                    if (vt == VT_IMMERSED_SOLID) continue;
                    const int pullAll = vt == VT_FLUID || vt == VT_MDPERIODIC ||
                                        vt == VT_VIRTUAL_BOUNDARY;
                    for (int l = 0; l < Q; l++) {
                        const int cx = C(o, l, 0), cy = C(o, l, 1),
                                  cz = C(o, l, 2);
                        const int rest = cx == 0 && cy == 0 && cz == 0;
                        if (pullAll || rest || stream_pulls(o, b->vg[p], l)) {
                            b->f[p * Q + l] =
                                b->fs[pidx(b, i - cx, j - cy, k - cz) * Q + l];
                        }
                    }
                }
    }
    /* ImplementBoundary3D, Src/boundary.cpp:379-386 */
    for (int i = 0; i < o->nbc; i++) {
        const mplbgpu_boundary* bc = &o->bc[i];
        oblock* b = find_block(o, bc->block);
        int r[6];
        surface_range(o, b, bc->surface, r);
        switch (bc->scheme) {
            case MPLBGPU_BC_EQM_DIFFUSE_REFL:
                bc_eqm(o, b, r, bc->given, o->bc_field[i]);
                break;
            case MPLBGPU_BC_EXTRAPOL_PRESSURE_1ST:
                bc_extrapol(o, b, r, bc->surface, bc->given[0]);
                break;
            case MPLBGPU_BC_HALFWAY_BOUNCE_BACK:
                bc_halfway_bb(o, b, r, bc->surface, bc->given,
                              o->bc_field[i]);
                break;
            case MPLBGPU_BC_FDPERIODIC:
                bc_fdperiodic(o, b, r, bc->surface);
                break;
            default:
                break; /* TreatBlockBoundary3D: no kernel dispatched */
        }
    }
}

/* KerLocalSwap3D, Src/scheme_kernel.inc:959-1194, on one node.  Fluid-like
 * nodes exchange each population with its opposite (l <-> l + half).  A
 * boundary-typed node walks l = 1..Q-1 in order over the directions that
 * point outward or along its faces (every inward component <= 0): a
 * direction lying in all of its faces is exchanged with its opposite (the
 * walk meets both members of such a pair, so the pair ends where it began),
 * any other takes a copy of its opposite.  Geometry codes without faces
 * leave the node alone. */
static void swap_local(const lbm_oracle* o, int vt, int vg, double* f) {
    const int Q = o->Q, half = (Q - 1) / 2;
    if (vt == VT_IMMERSED_SOLID) return;
    if (is_fluidlike(vt) || vt == VT_VIRTUAL_BOUNDARY) {
        for (int l = 1; l <= half; l++) {
            const double t = f[l];
            f[l] = f[l + half];
            f[l + half] = t;
        }
        return;
    }
    int axis[3], sign[3];
    const int n = decode_vg(vg, axis, sign);
    for (int l = 1; l < Q && n > 0; l++) {
        int outward = 1, along = 1;
        for (int p = 0; p < n; p++) {
            const int c = sign[p] * C(o, l, axis[p]);
            if (c > 0) outward = 0;
            if (c != 0) along = 0;
        }
        if (!outward) continue;
        if (along) {
            const double t = f[l];
            f[l] = f[o->opp[l]];
            f[o->opp[l]] = t;
        } else {
            f[l] = f[o->opp[l]];
        }
    }
}

/* KerSwapStream3D, Src/scheme_kernel.inc:1196-1398: node x exchanges its
 * population l + half with population l of x + c_l, for l = 1..half; a
 * boundary-typed node only for directions with every inward component >= 0
 * (those whose opposite does not point into the node from outside). */
static int swap_streams(const lbm_oracle* o, int vt, int vg, int l) {
    if (vt == VT_IMMERSED_SOLID) return 0;
    if (is_fluidlike(vt) || vt == VT_VIRTUAL_BOUNDARY) return 1;
    int axis[3], sign[3];
    const int n = decode_vg(vg, axis, sign);
    if (n == 0) return 0;
    for (int p = 0; p < n; p++)
        if (sign[p] * C(o, l, axis[p]) < 0) return 0;
    return 1;
}

/* SwapStreamCollision, Src/evolution.cpp:195-252: moments, in-place
 * collision (KerSwapCollideBGKIsothermal3D, Src/model_kernel.inc:385-408),
 * body force added after it (KerSwapCalcBodyForce1ST3D, :543-568), local
 * swap, swap streaming, boundary conditions on f. */
static void swap_step(lbm_oracle* o) {
    const int Q = o->Q, D = o->dim, half = (Q - 1) / 2;
    const double CS = o->cs;
    update_macro(o);
    oblock* b = &o->b[0];
    const double tau = o->tau;
    const double dtOvertauPlusdt = o->dt / (tau + 0.5 * o->dt);
    for (int k = 0; k < b->n[2]; k++)
        for (int j = 0; j < b->n[1]; j++)
            for (int i = 0; i < b->n[0]; i++) {
                const size_t p = pidx(b, i, j, k);
                double* f = &b->f[p * Q];
                const double rho = b->mac[0][p], u = b->mac[1][p],
                             v = b->mac[2][p], w = b->mac[3][p];
                for (int l = 0; l < Q; l++) {
                    const double fe = feq(o, l, rho, u, v, w);
                    f[l] = fe + (1 - dtOvertauPlusdt) * (f[l] - fe);
                }
                if (o->body_force == MPLBGPU_FORCE_1ST &&
                    is_fluidlike(b->vt[p])) {
                    for (int l = 0; l < Q; l++) {
                        double cf = 0;
                        for (int a = 0; a < D; a++)
                            cf += CS * o->xi[l * D + a] * o->accel[a];
                        f[l] += o->w[l] * b->mac[0][p] * cf;
                    }
                }
            }
    for (int k = 0; k < b->n[2]; k++)
        for (int j = 0; j < b->n[1]; j++)
            for (int i = 0; i < b->n[0]; i++) {
                const size_t p = pidx(b, i, j, k);
                swap_local(o, b->vt[p], b->vg[p], &b->f[p * Q]);
            }
    for (int k = 0; k < b->n[2]; k++)
        for (int j = 0; j < b->n[1]; j++)
            for (int i = 0; i < b->n[0]; i++) {
                const size_t p = pidx(b, i, j, k);
                for (int l = 1; l <= half; l++) {
                    if (!swap_streams(o, b->vt[p], b->vg[p], l)) continue;
                    const size_t q = pidx(b, i + C(o, l, 0), j + C(o, l, 1),
                                          k + C(o, l, 2));
                    const double t = b->f[p * Q + l + half];
                    b->f[p * Q + l + half] = b->f[q * Q + l];
                    b->f[q * Q + l] = t;
                }
            }
    for (int i = 0; i < o->nbc; i++) {
        const mplbgpu_boundary* bc = &o->bc[i];
        int r[6];
        surface_range(o, b, bc->surface, r);
        if (bc->scheme == MPLBGPU_BC_EQM_DIFFUSE_REFL)
            bc_eqm(o, b, r, bc->given, NULL);
    }
}

int lbmo_step(lbm_oracle* o, int nsteps) {
    for (int s = 0; s < nsteps; s++) {
        if (o->swap) swap_step(o);
        else one_step(o);
    }
    return 0;
}

/* CalcResidualError + GetMaximumResidual, Src/flowfield_wrapper.cpp:31-89,
 * Src/flowfield.cpp:148-158 */
int lbmo_residual(lbm_oracle* o, int check_period, double* per_var,
                  double* max_residual) {
    double diff[4] = {0, 0, 0, 0}, sum[4] = {0, 0, 0, 0};
    for (int m = 0; m < o->nmac; m++) {
        for (int bi = 0; bi < o->nb; bi++) {
            oblock* b = &o->b[bi];
            for (int k = 0; k < b->n[2]; k++)
                for (int j = 0; j < b->n[1]; j++)
                    for (int i = 0; i < b->n[0]; i++) {
                        const size_t p = pidx(b, i, j, k);
                        diff[m] = diff[m] + (b->mac[m][p] - b->old[m][p]) *
                                                (b->mac[m][p] - b->old[m][p]);
                    }
        }
    }
    copy_macro(o);
    for (int m = 0; m < o->nmac; m++) {
        for (int bi = 0; bi < o->nb; bi++) {
            oblock* b = &o->b[bi];
            for (int k = 0; k < b->n[2]; k++)
                for (int j = 0; j < b->n[1]; j++)
                    for (int i = 0; i < b->n[0]; i++) {
                        const size_t p = pidx(b, i, j, k);
                        sum[m] = sum[m] + (b->mac[m][p]) * (b->mac[m][p]);
                    }
        }
    }
    double maxRes = 0;
    for (int m = 0; m < o->nmac; m++) {
        const double res = diff[m] / sum[m];
        if (per_var) per_var[m] = res;
        const double rel = res / (check_period * o->dt);
        if (maxRes <= rel) maxRes = rel;
    }
    if (max_residual) *max_residual = maxRes;
    return 0;
}

int lbmo_get_macro(lbm_oracle* o, int block, double* rho, double* u,
                   double* v, double* w) {
    oblock* b = find_block(o, block);
    if (!b) return fail("unknown block");
    double* dst[4] = {rho, u, v, w};
    size_t n = 0;
    for (int k = 0; k < b->n[2]; k++)
        for (int j = 0; j < b->n[1]; j++)
            for (int i = 0; i < b->n[0]; i++, n++) {
                const size_t p = pidx(b, i, j, k);
                for (int m = 0; m < o->nmac; m++)
                    if (dst[m]) dst[m][n] = b->mac[m][p];
            }
    return 0;
}

int lbmo_get_f(lbm_oracle* o, int block, double* f) {
    oblock* b = find_block(o, block);
    if (!b) return fail("unknown block");
    size_t n = 0;
    for (int k = 0; k < b->n[2]; k++)
        for (int j = 0; j < b->n[1]; j++)
            for (int i = 0; i < b->n[0]; i++, n++) {
                memcpy(&f[n * o->Q], &b->f[pidx(b, i, j, k) * o->Q],
                       sizeof(double) * o->Q);
            }
    return 0;
}

int lbmo_get_node_info(lbm_oracle* o, int block, int* node_type,
                       int* geometry) {
    oblock* b = find_block(o, block);
    if (!b) return fail("unknown block");
    size_t n = 0;
    for (int k = 0; k < b->n[2]; k++)
        for (int j = 0; j < b->n[1]; j++)
            for (int i = 0; i < b->n[0]; i++, n++) {
                const size_t p = pidx(b, i, j, k);
                if (node_type) node_type[n] = b->vt[p];
                if (geometry) geometry[n] = b->vg[p];
            }
    return 0;
}
