/*
 * adh_sw2_gnn.h -- C ABI of the learned Newton initial guess: a per-node
 * message-passing network over the mesh's node graph (BF16 weights, FP32
 * accumulation) with its forward, backward and Adam kernels for sm_100a.
 *
 * No counterpart in the reference: the reference starts every Newton solve from
 * the previous time step (initialize_system, src/newton/newton_tools.c:35-37).
 * The network's output goes through sw2g_set_guess / sw2g_newton_opts.use_guess
 * (adh_sw2_gpu.h), which keeps the previous step whenever its residual is smaller.
 *
 * All pointers are device pointers; `stream` is a cudaStream_t (NULL: default
 * stream).  Row-major [node][feature] FP32 activations; H = 64 hidden features,
 * aggregation output 4H = 256.  Return values: 0 (or a count, sw2n_mse) on
 * success, -1 bad argument, -2 launch error.
 *
 * Graph arguments: indptr [n+1], nbr [nnz] (symmetric node graph, no self
 * loops), rev [nnz] (slot of the reverse edge), wx, wy [nnz] = (x_j - x_i) /
 * (L deg_i), inv_deg [n], swx, swy [n] = row sums of wx, wy.
 */
#ifndef ADH_SW2_GNN_H
#define ADH_SW2_GNN_H
#ifdef __cplusplus
extern "C" {
#endif

/* X[i] = [E_i, mean_j E_j, sum_j wx_ij (E_j - E_i), sum_j wy_ij (E_j - E_i)]  (E [n][64] -> X [n][256]) */
int sw2n_agg_fwd(int n, const int *indptr, const int *nbr, const int *rev, const float *wx, const float *wy,
                 const float *inv_deg, const float *swx, const float *swy, const float *E, float *X, void *stream);
/* dE += the adjoint of sw2n_agg_fwd applied to dX (a gather: no atomics) */
int sw2n_agg_bwd(int n, const int *indptr, const int *nbr, const int *rev, const float *wx, const float *wy,
                 const float *inv_deg, const float *swx, const float *swy, const float *dX, float *dE, void *stream);
/* Y = act(W X + b) (+ R); W [out][in] BF16, in <= 256 and a multiple of 4, out <= 64; act 1 = SiLU;
 * Z (optional) receives the pre-activation */
int sw2n_dense_fwd(int n, int in, int out, const void *W_bf16, const float *b, const float *X, const float *R, int act,
                   float *Z, float *Y, void *stream);
/* dZ = dY * act'(Z); dX = W^T dZ (dX optional); gW [out*in + out] = (sum_i dZ_i X_i^T, sum_i dZ_i);
 * part: ceil(n / nodes_per_block) * (out*in + out) floats of block partials */
int sw2n_dense_bwd(int n, int in, int out, const void *W_bf16, const float *X, const float *Z, const float *dY, int act,
                   float *dZ, float *dX, int nodes_per_block, float *part, float *gW, void *stream);
/* Adam step t (>= 1) on FP32 master weights w with gradient g, moments m, v; refreshes the BF16 copy */
int sw2n_adam(int count, float *w, const float *g, float *m, float *v, void *w_bf16, float lr, float b1, float b2,
              float eps, int t, void *stream);
int sw2n_to_bf16(int count, const float *w, void *w_bf16, void *stream);
/* network inputs F [n][8] = ([h, u, v, dh, du, dv, z_bed, wet] - mu) / sd from the FP64 states [3n] */
int sw2n_features(int n, const double *sol, const double *sol_prev, const double *z, const float *mu, const float *sd,
                  float *F, void *stream);
/* training targets T [n][3] = (sol_next - 2 sol + sol_prev) / scale: the correction to linear extrapolation;
 * M [n] = 1 where h > min_depth in sol and sol_next (where the guess uses the network), else 0 */
int sw2n_targets(int n, const double *sol_next, const double *sol, const double *sol_prev, const float *scale,
                 double min_depth, float *T, float *M, void *stream);
/* masked mean squared error: dY = 2 M (Y - T) / (3n); returns the number of partial sums written to part
 * (their sum is the loss) */
int sw2n_mse(int n, const float *Y, const float *T, const float *M, float *dY, float *part, void *stream);
/* Ys_i = (Y_i + sum_j Y_j) / (deg_i + 1) over 3 channels, and its adjoint (Y != Ys) */
int sw2n_smooth3(int n, const int *indptr, const int *nbr, const float *Y, float *Ys, void *stream);
int sw2n_smooth3_adj(int n, const int *indptr, const int *nbr, const float *dYs, float *dY, void *stream);
/* guess [3n] (FP64) = 2 sol - sol_prev + scale * Y per node; nodes with h <= min_depth in sol or in the
 * guess keep sol (the guess does not move the wet/dry front) */
int sw2n_apply_guess(int n, const double *sol, const double *sol_prev, const float *Y, const float *scale,
                     double min_depth, double *guess, void *stream);

#ifdef __cplusplus
}
#endif
#endif
