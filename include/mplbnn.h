/*
 * mplbnn.h — the learned warm start of the batched cavity solver.
 *
 * No reference counterpart: the reference has no learned component.  A
 * 4-level convolutional encoder-decoder maps a cavity's (Reynolds number,
 * lid speed, grid side) to its normalised steady state (rho, u, v) on a
 * 128 x 128 grid; the batched solver (mplbgpu_batch_*) is then started from
 * that field instead of rest.  Forward and backward passes run on the
 * sm_100a tensor cores (tcgen05 MMAs, TMA-fed, accumulators in tensor
 * memory) in bf16 with fp32 accumulation and fp32 master weights (Adam).
 *
 * Pointers documented as "device" are CUDA device addresses; every other
 * pointer is host memory.  Calls on one network are not re-entrant; the
 * network runs on its own CUDA stream (mplbnn_synchronize waits for it).
 */
#ifndef MPLBNN_H
#define MPLBNN_H

#ifdef __cplusplus
extern "C" {
#endif

#define MPLBNN_ABI_VERSION 1
#define MPLBNN_GRID 128          /* network grid side */
#define MPLBNN_COND 3            /* conditioning scalars per cavity */
#define MPLBNN_FIELDS 3          /* predicted fields: rho, u, v (normalised) */

/* A bf16 (or fp32 where stated) NHWC activation view: channel c of pixel
 * (img, y, x) sits at ptr[((img * h + y) * w + x) * ps + c]. */
typedef struct {
    void* ptr;               /* device */
    int nimg, h, w, c;
    long long ps;            /* elements between consecutive pixels, >= c */
} mplbnn_view;

/* ---- primitives (tensor-core convolutions) ------------------------------ */

/* y = act(conv(x, w) + bias) [* (mask > 0)]: w is bf16 [y.c][taps][x.c]
 * (device), taps 9 (3x3, zero padding 1) or 1; bias fp32 [y.c] (device) or
 * NULL; relu 0/1; y bf16, or fp32 when y_f32; mask a bf16 view shaped like y
 * or NULL.  Requires x.c and y.c multiples of 16, ps multiples of 8 (4 for
 * fp32), w <= 128 dividing 128, h * w a multiple of 128. */
int mplbnn_conv_forward(const mplbnn_view* x, const void* w, int taps,
                        const float* bias, int relu, const mplbnn_view* y,
                        int y_f32, const mplbnn_view* mask, void* stream);

/* dw[n][t][c] += sum over pixels p of dy[p][n] * x[p + offset(t)][c]
 * (dw fp32 device, [dy.c][taps][x.c]). */
int mplbnn_conv_wgrad(const mplbnn_view* dy, const mplbnn_view* x, int taps,
                      float* dw, void* stream);

/* Last error of the primitives (per thread). */
const char* mplbnn_error(void);

/* ---- the network --------------------------------------------------------- */

typedef struct mplbnn_net mplbnn_net;

/* Buffers for up to `batch` cavities per pass. */
int mplbnn_create(int batch, mplbnn_net** out);
int mplbnn_destroy(mplbnn_net* net);
const char* mplbnn_last_error(const mplbnn_net* net);
int mplbnn_synchronize(mplbnn_net* net);

/* Parameters: fp32, per layer W[cout][taps][cin] then b[cout], layers in
 * order (mplbnn_layer_info). */
long long mplbnn_param_count(const mplbnn_net* net);
int mplbnn_layer_count(void);
int mplbnn_layer_info(int layer, int* cin, int* cout, int* taps,
                      long long* w_offset, long long* b_offset);
int mplbnn_init_params(mplbnn_net* net, unsigned long long seed);
int mplbnn_set_params(mplbnn_net* net, const float* params);
int mplbnn_get_params(mplbnn_net* net, float* params);
int mplbnn_get_grads(mplbnn_net* net, float* grads);

/* cond: n x 3 fp32 (device), each in [0, 1]: (ln(Re / 100) / ln 32,
 * (U - 0.02) / 0.06, (N - 64) / 192).  pred: n x 128 x 128 x 3 fp32
 * (device), normalised fields. */
int mplbnn_forward(mplbnn_net* net, const float* cond, int n, float* pred);

/* Forward + backward of the mean squared error against target (128 x 128 x
 * 3 fp32 per sample, device); gradients stay in the network.  With index
 * (host, n sample numbers) the n samples cond[index[i]], target[index[i]]
 * are gathered first; with index NULL the first n are used.  loss (host)
 * may be NULL (no synchronisation). */
int mplbnn_loss_grad(mplbnn_net* net, const float* cond, const float* target,
                     const int* index, int n, double* loss);

/* One Adam step on the current gradients (step counter kept inside). */
int mplbnn_adam_step(mplbnn_net* net, float lr, float beta1, float beta2,
                     float eps);

/* ---- fields between the cavities and the network grid -------------------- */

/* Packed cavity fields (device fp64, cavity k's n_k^2 nodes from offset[k],
 * row-major y then x, node centres at ((i + 1/2) / n_k, (j + 1/2) / n_k))
 * resampled bilinearly to the 128 x 128 grid (centres at (i + 1/2) / 128)
 * and normalised: (rho - 1) / rho_scale[k], u / u_scale[k], v / u_scale[k].
 * grid: ncav x 128 x 128 x 3 fp32 (device).  n, offset, rho_scale, u_scale
 * are host arrays. */
int mplbnn_fields_to_grid(mplbnn_net* net, const double* rho, const double* u,
                          const double* v, int ncav, const int* n,
                          const long long* offset, const double* rho_scale,
                          const double* u_scale, float* grid);

/* The inverse: grid fields resampled to each cavity's nodes and scaled back
 * (rho = 1 + rho_scale * g0, u = u_scale * g1, v = u_scale * g2). */
int mplbnn_grid_to_fields(mplbnn_net* net, const float* grid, int ncav,
                          const int* n, const long long* offset,
                          const double* rho_scale, const double* u_scale,
                          double* rho, double* u, double* v);

#ifdef __cplusplus
}
#endif

#endif /* MPLBNN_H */
