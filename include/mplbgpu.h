/*
 * mplbgpu.h - C ABI of the B200 lattice Boltzmann stream-collision path.
 *
 * The path replaces one MPLB time step, StreamCollision()
 * (Src/evolution.cpp:137-193: moments, body force, BGK collision, halo
 * transfer, streaming, boundary conditions), and the check-period calls that
 * Iterate() makes around it (UpdateMacroVars3D/UpdateMacroVars,
 * CalcResidualError, GetMaximumResidual: Src/evolution.cpp:102-135,
 * Src/flowfield_wrapper.cpp:31-89, Src/flowfield.cpp:148-158).
 *
 * A context is built from a description of what the reference's setup API
 * holds after Partition(): the blocks (DefineBlocks, Src/flowfield.cpp:189),
 * the block connections (DefineBlockConnection, Src/flowfield.cpp:258-283),
 * the boundary list in definition order (DefineBlockBoundary,
 * Src/boundary.cpp:61-130), the lattice (DefineComponents, Src/model.cpp:208),
 * tauRef, TimeStep() and the body-force type.  Every enum value below is the
 * reference's own value, so a descriptor can be filled field by field from
 * Block, Neighbor and BlockBoundary (Src/block.h:55-104, Src/boundary.h:85-93).
 *
 * Plain pointers and sizes only; all device memory belongs to the context.
 * Host arrays are dense, z slowest and x fastest over a block's nodes
 * (size[0] x size[1] x size[2], size[2] = 1 in 2D); distributions are
 * point-major with Q = 9 or 19 values per node in the reference's lattice
 * order (SetupD2Q9Latt / SetupD3Q19Latt, Src/model.cpp:99-131).
 *
 * All calls return an mplbgpu_status; there are no exceptions across the ABI.
 * One context is driven by one host thread at a time.
 */
#ifndef MPLBGPU_H
#define MPLBGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define MPLBGPU_ABI_VERSION 3

typedef int mplbgpu_status;
enum {
    MPLBGPU_OK = 0,
    MPLBGPU_ERR_INVALID = 1,     /* bad argument or inconsistent description */
    MPLBGPU_ERR_UNSUPPORTED = 2, /* valid reference input this path rejects */
    MPLBGPU_ERR_CUDA = 3,        /* CUDA runtime error (message has detail)  */
    MPLBGPU_ERR_DIVERGED = 4,    /* non-finite or non-positive density seen  */
    MPLBGPU_ERR_TIMEOUT = 5,     /* a bounded device wait gave up            */
    MPLBGPU_ERR_NO_DEVICE = 6,   /* no usable CUDA device                    */
    MPLBGPU_ERR_STATE = 7        /* call out of order (e.g. step before init) */
};

/* BoundarySurface, Src/boundary_host_device.h:7-29 */
enum {
    MPLBGPU_LEFT = 0, MPLBGPU_RIGHT = 1, MPLBGPU_TOP = 2, MPLBGPU_BOTTOM = 3,
    MPLBGPU_FRONT = 4, MPLBGPU_BACK = 5,
    MPLBGPU_LEFT_BACK = 50, MPLBGPU_LEFT_FRONT = 40,
    MPLBGPU_RIGHT_BACK = 51, MPLBGPU_RIGHT_FRONT = 41,
    MPLBGPU_TOP_BACK = 52, MPLBGPU_TOP_FRONT = 42,
    MPLBGPU_BOTTOM_BACK = 53, MPLBGPU_BOTTOM_FRONT = 43,
    MPLBGPU_LEFT_TOP = 20, MPLBGPU_LEFT_BOTTOM = 30,
    MPLBGPU_RIGHT_TOP = 21, MPLBGPU_RIGHT_BOTTOM = 31
};

/* VertexType, Src/flowfield_host_device.h:21-37 */
enum {
    MPLBGPU_VT_FLUID = 10, MPLBGPU_VT_INLET = 11, MPLBGPU_VT_OUTLET = 12,
    MPLBGPU_VT_MDPERIODIC = 13, MPLBGPU_VT_SYMMETRY = 14,
    MPLBGPU_VT_FDPERIODIC = 15, MPLBGPU_VT_WALL = 1000,
    MPLBGPU_VT_IMMERSED_SOLID = -1, MPLBGPU_VT_IMMERSED_BOUNDARY = -2,
    MPLBGPU_VT_VIRTUAL_BOUNDARY = -3
};

/* BoundaryScheme, Src/boundary.h:70-83, plus one scheme of this path. */
enum {
    MPLBGPU_BC_KINETIC_DIFFUSE_WALL = 11,
    MPLBGPU_BC_KINETIC_SPECULAR_WALL = 12,
    MPLBGPU_BC_EXTRAPOL_PRESSURE_1ST = 16,
    MPLBGPU_BC_EXTRAPOL_PRESSURE_2ND = 17,
    MPLBGPU_BC_MDPERIODIC = 18,
    MPLBGPU_BC_FDPERIODIC = 19,
    MPLBGPU_BC_BOUNCE_BACK = 20, /* reference: no kernel dispatched (no-op) */
    MPLBGPU_BC_FREE_FLUX = 21,
    MPLBGPU_BC_ZOUHE_VELOCITY = 22,
    MPLBGPU_BC_EQN_NOSLIP = 23,
    MPLBGPU_BC_EQM_DIFFUSE_REFL = 24,
    MPLBGPU_BC_NONE = -1,
    /* Not in the reference: link-wise halfway bounce-back with a moving-wall
     * correction (the wall sits half a spacing outside the surface nodes). */
    MPLBGPU_BC_HALFWAY_BOUNCE_BACK = 100
};

enum { MPLBGPU_D2Q9 = 9, MPLBGPU_D3Q19 = 19 };

/* Storage/arithmetic forms of the distributions. */
enum {
    MPLBGPU_FP64 = 0,          /* reference arithmetic, FP64 storage          */
    MPLBGPU_FP32_SHIFTED = 1,  /* stores f_i - w_i in FP32, FP32 arithmetic   */
    MPLBGPU_FP16_SHIFTED = 2   /* stores f_i - w_i in FP16, FP32 arithmetic   */
};

/* BodyForceType, Src/model.h:101-106 */
enum { MPLBGPU_FORCE_NONE = 0, MPLBGPU_FORCE_1ST = 1 };

/* SchemeType, Src/scheme.h:67-72.  The swap scheme stands for the
 * reference's one-array trio Scheme_StreamCollision_Swap +
 * Collision_BGKIsothermal2nd_Swap + BodyForce_{None,1st}_Swap
 * (SwapStreamCollision, Src/evolution.cpp:195-252): D3Q19, one block
 * without connections, every block-boundary node under EQMDiffuseRefl. */
enum {
    MPLBGPU_SCHEME_STREAM_COLLISION = 10,      /* 0 means the same */
    MPLBGPU_SCHEME_STREAM_COLLISION_SWAP = 11
};

typedef struct {
    int id;       /* block id as given to DefineBlocks */
    int size[3];  /* nodes per axis; size[2] = 1 for 2D */
    int cut;      /* bit s set: surface s (MPLBGPU_LEFT..MPLBGPU_BACK) is not
                     a boundary but continues into a block held by another
                     context (decomposition of one block over GPUs, the
                     job OPS's MPI partition does for the reference); its
                     halo layer is filled with mplbgpu_import_face.  0 for
                     the reference's own blocks. */
} mplbgpu_block;

typedef struct {  /* one entry of DefineBlockConnection */
    int from_block;
    int from_surface;
    int to_block;
    int to_surface;
    int type;     /* VertexType: VirtualBoundary, MDPeriodic, FDPeriodic */
} mplbgpu_connection;

typedef struct {  /* one DefineBlockBoundary call, in call order */
    int block;
    int surface;
    int scheme;       /* BoundaryScheme */
    int vertex_type;  /* VertexType written to the surface's nodes */
    double given[3];  /* GivenVars: (u, v[, w]) for walls, (rho) for
                         ExtrapolPressure1ST, unused otherwise */
} mplbgpu_boundary;

typedef struct {
    int abi_version;  /* MPLBGPU_ABI_VERSION */
    int space_dim;    /* 2 or 3 */
    int lattice;      /* MPLBGPU_D2Q9 (2D) or MPLBGPU_D3Q19 (3D) */
    int precision;    /* MPLBGPU_FP64 / _FP32_SHIFTED / _FP16_SHIFTED */
    int nblocks;
    const mplbgpu_block* blocks;
    int nconnections;
    const mplbgpu_connection* connections;
    int nboundaries;
    const mplbgpu_boundary* boundaries;
    double tau_ref;   /* Component::tauRef */
    double dt;        /* TimeStep() */
    double cs;        /* SoundSpeed(), sqrt(3) for D2Q9/D3Q19 */
    int body_force;   /* BodyForceType */
    double accel[3];  /* uniform body acceleration (MPLB units) */
    int force_velocity; /* 1 when the velocity moments are Variable_U_Force
                           etc.: u += dt*a/2 at Fluid/MDPeriodic nodes */
    int scheme;       /* SchemeType (DefineScheme, Src/scheme.cpp:92-110) */
} mplbgpu_desc;

typedef struct mplbgpu_ctx mplbgpu_ctx;

/* Builds node classification, boundary tables and halo plans, allocates the
 * device state (Partition + DefineScheme + PrepareFlowField).  The
 * description is checked before the device is looked for: a bad one gives
 * MPLBGPU_ERR_INVALID / _UNSUPPORTED even where there is no GPU. */
mplbgpu_status mplbgpu_create(const mplbgpu_desc* desc, mplbgpu_ctx** out);
mplbgpu_status mplbgpu_destroy(mplbgpu_ctx* ctx);

/* Message for the last failed call on ctx (ctx may be NULL for create). */
const char* mplbgpu_last_error(const mplbgpu_ctx* ctx);

/* Initial macroscopic state of one block followed by f = feq(rho, u)
 * (app SetInitialMacrosVars + PreDefinedInitialCondition3D,
 * Src/model_wrapper.cpp:347-391).  Any of u, v, w may be NULL (zero);
 * rho NULL means 1. */
mplbgpu_status mplbgpu_init_macro(mplbgpu_ctx* ctx, int block,
                                  const double* rho, const double* u,
                                  const double* v, const double* w);

/* Replaces the distributions of one block (restart from saved f).  The
 * context's step count is left as it is; a restart sets it with
 * mplbgpu_set_step. */
mplbgpu_status mplbgpu_upload_f(mplbgpu_ctx* ctx, int block, const double* f);

/* nsteps calls of StreamCollision().  The kernels are queued on the
 * context's stream and the call returns without waiting for them (a launch
 * error is returned at once; a fault during the steps is returned by the
 * next call that waits: a download, residual, mass, health check,
 * mplbgpu_synchronize or mplbgpu_last_step_ms).  Calling it once per time
 * step, as StreamCollision() is called, costs no host round trip. */
mplbgpu_status mplbgpu_step(mplbgpu_ctx* ctx, int nsteps);

/* One step in two calls, for decomposed blocks whose cut faces come from
 * another GPU: mplbgpu_step_begin queues the part of the step that reads
 * no halo layer beyond a y or z face (the x faces and interior rows of
 * every block), mplbgpu_step_finish the rest (the rows on a y or z face,
 * deferred boundary nodes, block-to-block halos).  Between the two only
 * mplbgpu_export_face and mplbgpu_import_face of y and z faces are
 * accepted (other calls return MPLBGPU_ERR_STATE), so a face transfer on
 * another stream overlaps the interior's computation when the import waits
 * for it.  begin + finish is one mplbgpu_step(ctx, 1), bit for bit.
 * Two-array scheme only. */
mplbgpu_status mplbgpu_step_begin(mplbgpu_ctx* ctx);
mplbgpu_status mplbgpu_step_finish(mplbgpu_ctx* ctx);

/* The context's CUDA stream (a cudaStream_t), for ordering a caller's own
 * work (a face transfer, an event) with the context's. */
mplbgpu_status mplbgpu_get_stream(mplbgpu_ctx* ctx, void** stream);

/* Which step kernel a block runs (a diagnostic; no reference counterpart):
 * one thread per node (blocks with a non-pure interior or an extent below
 * 3), the split step (shell rows, x faces and interior nodes in separate
 * CTAs) or the swap scheme's. */
enum {
    MPLBGPU_KERNEL_NODE = 0,
    MPLBGPU_KERNEL_SPLIT = 1,
    MPLBGPU_KERNEL_SWAP = 2
};
mplbgpu_status mplbgpu_step_kernel(mplbgpu_ctx* ctx, int block_id, int* kind);

/* Moments of the current f into the context's macro fields
 * (UpdateMacroVars3D / UpdateMacroVars). */
mplbgpu_status mplbgpu_update_macro(mplbgpu_ctx* ctx);

/* CalcResidualError + GetMaximumResidual(check_period): per variable
 * (rho, u, v[, w]) sum((q - q_old)^2) / sum(q^2) over all blocks, then the
 * maximum of those divided by check_period * dt; q_old becomes q.  per_var
 * (space_dim + 1 entries) may be NULL. */
mplbgpu_status mplbgpu_residual(mplbgpu_ctx* ctx, int check_period,
                                double* per_var, double* max_residual);

/* Copies of the macro fields / distributions of one block to the host. */
mplbgpu_status mplbgpu_download_macro(mplbgpu_ctx* ctx, int block,
                                      double* rho, double* u, double* v,
                                      double* w);
mplbgpu_status mplbgpu_download_f(mplbgpu_ctx* ctx, int block, double* f);

/* Decomposed blocks (cut faces).  Before each mplbgpu_step the caller moves,
 * for every cut face, the populations leaving the neighbouring context's
 * block through its opposite face into this block's halo layer:
 *   mplbgpu_face_size   elements (and bytes per element, the storage form's)
 *                       of one face buffer: the populations crossing the
 *                       face, population-major, then the face's nodes with
 *                       the lower in-plane axis fastest;
 *   mplbgpu_export_face the populations leaving through `surface` from the
 *                       block's layer next to it, into device buffer `buf`;
 *   mplbgpu_import_face `buf` (the neighbour's export through the opposite
 *                       face) into the halo layer beyond `surface`.
 * Both run on the context's stream (mplbgpu_synchronize before handing the
 * buffer to another stream).  A block split into slabs this way steps bit
 * for bit as the whole block does. */
mplbgpu_status mplbgpu_face_size(mplbgpu_ctx* ctx, int block, int surface,
                                 long long* elems, int* elem_bytes);
mplbgpu_status mplbgpu_export_face(mplbgpu_ctx* ctx, int block, int surface,
                                   void* buf);
mplbgpu_status mplbgpu_import_face(mplbgpu_ctx* ctx, int block, int surface,
                                   const void* buf);

/* The residual's sums over this context's nodes (CalcResidualError before
 * the division, Src/flowfield_wrapper.cpp:31-89): per variable
 * diff = sum((q - q_old)^2) and sum = sum(q^2) (space_dim + 1 entries
 * each); q_old becomes q.  Decomposed runs add them over contexts. */
mplbgpu_status mplbgpu_residual_sums(mplbgpu_ctx* ctx, double* diff,
                                     double* sum);

/* Wall velocity per node for one boundary: no counterpart in the
 * reference, whose BlockBoundary carries one uniform GivenVars per surface
 * (Src/boundary.h:85-93); used for an inlet with a perturbed velocity
 * profile.  `boundary` indexes desc.boundaries (definition order) and must
 * be an EQMDiffuseRefl or halfway bounce-back boundary.  The arrays hold
 * one value (MPLB units, like GivenVars) per node of the boundary's
 * surface range (Block::BoundarySurfaceRange, Src/block.cpp:17-97, the
 * range its kernel runs over), x fastest then y then z, extent from
 * mplbgpu_boundary_extent; NULL components are zero, all three NULL go
 * back to the uniform given values.  Each node's wall constants are then
 * evaluated from its own velocity in the operation order of the uniform
 * case, so a field of equal values steps bit for bit as `given` does.
 * Not available under the swap scheme (MPLBGPU_ERR_UNSUPPORTED). */
mplbgpu_status mplbgpu_boundary_extent(mplbgpu_ctx* ctx, int boundary,
                                       int ext[3]);
mplbgpu_status mplbgpu_set_boundary_velocity(mplbgpu_ctx* ctx, int boundary,
                                             const double* u, const double* v,
                                             const double* w);

/* FP64 sum of rho over all nodes of all blocks, from the current f. */
mplbgpu_status mplbgpu_mass(mplbgpu_ctx* ctx, double* mass);

/* Scans the current state for non-finite or non-positive density:
 * MPLBGPU_OK or MPLBGPU_ERR_DIVERGED. */
mplbgpu_status mplbgpu_check_health(mplbgpu_ctx* ctx);

/* Number of steps the current state has taken: 0 after
 * mplbgpu_init_macro, advanced by mplbgpu_step; a restart from saved f
 * sets it to the checkpoint's step (the reference's CurrentTimeStep,
 * Src/model.cpp:299-309).  The FP16 storage form draws its stochastic
 * rounding from it, so a restarted FP16 run takes the draws of the
 * uninterrupted one. */
mplbgpu_status mplbgpu_set_step(mplbgpu_ctx* ctx, long long step);

/* Waits for all work issued on the context's stream. */
mplbgpu_status mplbgpu_synchronize(mplbgpu_ctx* ctx);

/* Number of kernel launches the context has issued since creation. */
long long mplbgpu_launch_count(const mplbgpu_ctx* ctx);

/* Device time of the most recent mplbgpu_step call's kernels (ms); waits
 * for them to finish. */
mplbgpu_status mplbgpu_last_step_ms(mplbgpu_ctx* ctx, float* ms);

/* ---------------------------------------------------------------------
 * Batched cavities (no counterpart in the reference, which runs one case
 * per process): many independent square D2Q9 lid-driven cavities of
 * different sizes advanced together.  Each cavity is the single-block
 * case with halfway bounce-back on its four walls and a lid moving along
 * +x; its residual is the reference's CalcResidualError +
 * GetMaximumResidual on that cavity, with dt = 1 / ((n - 1) sqrt(3)).
 * ------------------------------------------------------------------- */
typedef struct {
    int n;           /* nodes per side */
    double lid_u;    /* lid speed in MPLB units (sqrt(3) x lattice units) */
    double tau_ref;  /* MPLB tauRef (tau_L = tauRef / dt + 1/2) */
} mplbgpu_cavity;

typedef struct {
    int tile_nodes;  /* nodes per tile: 64, 128 or 256; a CTA has one
                        thread per node in FP64 and one per two nodes in
                        FP32 */
    int persistent;  /* 1: one cooperative launch per chunk of steps with a
                        bounded grid barrier between steps; 0: one launch
                        per step, a chunk replayed from a CUDA graph */
    int chunk;       /* steps per chunk (even) */
    int ctas_per_sm; /* CTAs per SM of the persistent launches (at most
                        the co-resident count) */
} mplbgpu_batch_tuning;

typedef struct mplbgpu_batch mplbgpu_batch;

/* precision: MPLBGPU_FP64 or MPLBGPU_FP32_SHIFTED.  The cavities are checked
 * before the device is looked for. */
mplbgpu_status mplbgpu_batch_create(const mplbgpu_cavity* cavities, int ncav,
                                    int precision, mplbgpu_batch** out);
mplbgpu_status mplbgpu_batch_destroy(mplbgpu_batch* b);
const char* mplbgpu_batch_last_error(const mplbgpu_batch* b);
mplbgpu_status mplbgpu_batch_set_tuning(mplbgpu_batch* b,
                                        const mplbgpu_batch_tuning* t);
mplbgpu_status mplbgpu_batch_get_tuning(mplbgpu_batch* b,
                                        mplbgpu_batch_tuning* t);
/* Polls a grid barrier of the persistent launch makes before it gives up
 * (default 2^26, several seconds): the kernel then records an error and
 * returns, and the step or run call reports MPLBGPU_ERR_TIMEOUT; the batch
 * is then uninitialised (MPLBGPU_ERR_STATE until mplbgpu_batch_init), its
 * fields being a mix of steps.  Small limits let a test exercise that
 * path. */
mplbgpu_status mplbgpu_batch_set_wait_limit(mplbgpu_batch* b,
                                            long long polls);
/* Initial macroscopic fields of every cavity, packed cavity after cavity
 * (n*n values each, y slowest), in host or device memory; NULL means
 * rho = 1 / u = v = 0.  f = feq, every cavity active again. */
mplbgpu_status mplbgpu_batch_init(mplbgpu_batch* b, const double* rho,
                                  const double* u, const double* v);
/* nsteps steps of every active cavity; moments of the last step are kept. */
mplbgpu_status mplbgpu_batch_step(mplbgpu_batch* b, int nsteps);
/* Steps every active cavity, check_period at a time, until its residual is
 * below criterion or max_steps have passed.  Per cavity (arrays of ncav,
 * each may be NULL): steps taken, last residual, and 1 if converged, 0 if
 * not within max_steps, -1 if it diverged (NaN residual; the cavity is
 * dropped at that check; unlike the reference's GetMaximumResidual, which
 * skips NaN ratios and so reports a diverged run as converged). */
mplbgpu_status mplbgpu_batch_run(mplbgpu_batch* b, long long max_steps,
                                 int check_period, double criterion,
                                 long long* steps, double* residual,
                                 int* converged);
/* Moments of the last step or check, packed like mplbgpu_batch_init, into
 * host or device memory. */
mplbgpu_status mplbgpu_batch_download_macro(mplbgpu_batch* b, double* rho,
                                            double* u, double* v);
/* Device time, node updates and kernel launches since the last init. */
mplbgpu_status mplbgpu_batch_stats(mplbgpu_batch* b, double* device_ms,
                                   long long* node_updates,
                                   long long* launches);

/* Residual sums that allocate nothing (no counterpart in the reference).
 * For callers that cannot call cudaMalloc where they need the reduction -
 * programs that give all device memory to their own pool at start-up, or
 * loops that cannot take the device-wide synchronisation that allocating
 * and freeing cause.  The caller owns every buffer: q[v] and q_old[v]
 * (v < nvars <= 4) are device arrays of n doubles, sums a device array of
 * 2 * nvars doubles that receives sum((q - q_old)^2) and sum(q^2) per
 * variable; q_old is overwritten with q.  Per-CTA partial sums go to a
 * fixed 512 KiB device array inside the library (held on every GPU that
 * loads it until exit), which limits n to MPLBGPU_NOALLOC_MAX_NODES; larger
 * n is rejected with MPLBGPU_ERR_INVALID.  The first call in a CUDA context
 * (in practice, the first call on each device) looks up that array's
 * address in the current context; make it before any stream capture.  Work is queued on `stream` (a cudaStream_t, NULL for the
 * default stream).  All calls share the array: calls that overlap on the
 * GPU race. */
#define MPLBGPU_NOALLOC_MAX_NODES 16777216LL
mplbgpu_status mplbgpu_residual_sums_noalloc(const double* const* q,
                                             double* const* q_old, int nvars,
                                             long long n, double* sums,
                                             void* stream);

#ifdef __cplusplus
}
#endif
#endif /* MPLBGPU_H */
