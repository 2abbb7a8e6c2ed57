/*
 * CPU restatement of MPLB's stream-collision step (TEST INFRASTRUCTURE ONLY).
 *
 * Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
 * the checker of the CUDA path; never linked into the product.  It follows
 * the reference's unfused sequence one loop at a time, on its own arrays,
 * with the reference's operation order so that its FP64 results are bitwise
 * equal to the reference compiled with -ffp-contract=off.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include "../include/mplbgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lbm_oracle lbm_oracle;

/* 0 on success; negative on an invalid or unsupported description. */
int lbmo_create(const mplbgpu_desc* desc, lbm_oracle** out);
void lbmo_destroy(lbm_oracle* o);
const char* lbmo_error(void);

/* SetInitialMacrosVars (per node, NULL = 1 for rho, 0 for velocities) then
 * PreDefinedInitialCondition(3D) and CopyCurrentMacroVar. */
int lbmo_init_macro(lbm_oracle* o, int block, const double* rho,
                    const double* u, const double* v, const double* w);
/* f of one block, point-major, interior nodes. */
int lbmo_set_f(lbm_oracle* o, int block, const double* f);
int lbmo_step(lbm_oracle* o, int nsteps);
int lbmo_update_macro(lbm_oracle* o);
int lbmo_residual(lbm_oracle* o, int check_period, double* per_var,
                  double* max_residual);
int lbmo_get_macro(lbm_oracle* o, int block, double* rho, double* u,
                   double* v, double* w);
int lbmo_get_f(lbm_oracle* o, int block, double* f);
/* Per-node wall velocity of an EQMDiffuseRefl / halfway bounce-back
 * boundary over its surface range (x fastest; NULL components zero, all
 * NULL: back to GivenVars), as mplbgpu_set_boundary_velocity. */
int lbmo_boundary_extent(lbm_oracle* o, int boundary, int ext[3]);
int lbmo_set_boundary_velocity(lbm_oracle* o, int boundary, const double* u,
                               const double* v, const double* w);
/* Node type / geometry property of one block's interior nodes. */
int lbmo_get_node_info(lbm_oracle* o, int block, int* node_type,
                       int* geometry);

#ifdef __cplusplus
}
#endif
#endif
