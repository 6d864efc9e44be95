// Linear-algebra kernels for the SW2 Newton step: norms, check_diag / Dirichlet /
// row scaling (src/la/matrix_utilities.c, src/la/scale_linear_system.c), the 3x3
// nodal block-Jacobi preconditioner that replaces the reference's full UMFPACK LU
// (src/la/bcgstab_solver.c:371-420), and the reference's left-preconditioned
// BiCGStab (bcgstab_solver.c:65-330) with every scalar kept on the device.
//
// B200 mapping:
//  * SpMV is node-centric on the reference CSR: the three rows of a node share one
//    column pattern, so a group of 8 lanes walks the node's neighbour slots, reads
//    each 3x3 block as three 24-byte runs (coalesced across the group), gathers the
//    neighbour's three x values once, and reduces with shuffles.  The block-Jacobi
//    apply and the dot products of the BiCGStab step are fused into the same pass.
//  * Reductions are two-phase: each block writes a partial, the last block to
//    finish sums the partials in block order and updates the scalars, so results
//    are deterministic and no host round trip happens inside the iteration.
//  * Grids are a fixed multiple of the SM count (grid-stride loops), which also
//    bounds the partial arrays.
#include <cmath>
#include "sw2_launch.h"

namespace sw2 {

#define SW2_DBL_EPS 2.220446049250313080847e-16

static int g_num_sms = 0;
static int grid_for(long work, int threads) {
    if (g_num_sms == 0) {
        int dev = 0; cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0) g_num_sms = 148;
    }
    long need = (work + threads - 1) / threads;
    long cap = 8L * g_num_sms;
    if (cap > kMaxBlocks) cap = kMaxBlocks;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double ld_part(const Reduce& R, int i) { return __ldcg(R.partial + i); }

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0) for (int i = 0; i < NT / 32; i++) t += sh[i];
    return t;   // valid in thread 0
}
template <int NT>
__device__ __forceinline__ double block_max(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0) for (int i = 0; i < NT / 32; i++) t = fmax(t, sh[i]);
    return t;
}
// Publish this block's partials; returns true in thread 0 of the last block, which
// then reads every partial through ld_part (L1-bypassing loads).
__device__ __forceinline__ bool last_block(Reduce R, const double* vals, int nv) {
    __shared__ bool is_last;
    if (threadIdx.x == 0) {
        for (int i = 0; i < nv; i++) R.partial[blockIdx.x * 4 + i] = vals[i];
        __threadfence();
        unsigned int t = atomicInc(R.counter, gridDim.x - 1);   // the last block wraps it back to 0
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    return is_last && threadIdx.x == 0;
}

// ---------------------------------------------------------------- Newton norms
__global__ void __launch_bounds__(256) k_norms(int n, const double* __restrict__ res, const double* __restrict__ dsol,
                                               const int* __restrict__ bc_mask, Reduce R) {
    __shared__ double sh[8];
    double mx = 0, l2 = 0, im = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (bc_mask[i] == 1) continue;
        double a = fabs(res[i]);
        mx = fmax(mx, a);
        l2 += res[i] * res[i];
        im = fmax(im, fabs(dsol[i]));
    }
    double v[3];
    v[0] = block_max<256>(mx, sh); v[1] = block_sum<256>(l2, sh); v[2] = block_max<256>(im, sh);
    if (last_block(R, v, 3)) {
        double a = 0, b = 0, c = 0;
        for (int k = 0; k < (int)gridDim.x; k++) {
            a = fmax(a, ld_part(R, 4 * k)); b += ld_part(R, 4 * k + 1); c = fmax(c, ld_part(R, 4 * k + 2));
        }
        R.out[0] = a; R.out[1] = b; R.out[2] = c;
    }
}
void launch_norms(int n, const double* res, const double* dsol, const int* bc_mask, Reduce R, cudaStream_t st) {
    k_norms<<<grid_for(n, 256), 256, 0, st>>>(n, res, dsol, bc_mask, R);
}

// ---------------------------------------------------------------- Dirichlet + scaling
// check_diag (matrix_utilities.c:120): |A_ii| < DBL_EPSILON makes the row Dirichlet.
__global__ void k_check_diag(int n, const int* __restrict__ diag, const double* __restrict__ vals, int* __restrict__ bc_mask) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    if (fabs(vals[diag[r]]) < SW2_DBL_EPS) bc_mask[r] = 1;
}
void launch_check_diag(const BlockCSR& A, const double* vals, int* bc_mask, cudaStream_t st) {
    k_check_diag<<<(A.n + 255) / 256, 256, 0, st>>>(A.n, A.diag, vals, bc_mask);
}

// apply_Dirichlet_BC (matrix_utilities.c:42-118) then the row part of
// scale_linear_system (scale_linear_system.c:31-95): both only touch row r.
__global__ void k_dirichlet_rowscale(int n, const int* __restrict__ indptr, const int* __restrict__ cols,
                                     const int* __restrict__ bc_mask, double* __restrict__ vals, double* __restrict__ b,
                                     double* __restrict__ x, double* __restrict__ scale) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int k0 = indptr[r], k1 = indptr[r + 1];
    const bool dirichlet_row = bc_mask[r] == 1;
    double mx = 0;
    for (int k = k0; k < k1; k++) {
        const int c = cols[k];
        double v = vals[k];
        if (bc_mask[c] == 1) v = 0.0;
        if (dirichlet_row) v = (c == r) ? 1.0 : 0.0;
        vals[k] = v;
        double t = fabs(v);
        if (t > mx) mx = t;
    }
    if (dirichlet_row) b[r] = 0.0;
    const double small = SW2_DBL_EPS, small_factor = 1.0 / sqrt(small);
    const double s = (mx < small) ? small_factor : 1.0 / sqrt(fabs(mx));
    scale[r] = s;
    b[r] *= s;
    x[r] /= s;
}
void launch_dirichlet_rowscale(const BlockCSR& A, const int* bc_mask, double* vals, double* b, double* x,
                               double* scale, cudaStream_t st) {
    k_dirichlet_rowscale<<<(A.n + 255) / 256, 256, 0, st>>>(A.n, A.indptr, A.cols, bc_mask, vals, b, x, scale);
}

// vals_ij *= s_i * s_j (scale_linear_system.c:97-121)
__global__ void k_scale_vals(int n, const int* __restrict__ indptr, const int* __restrict__ cols,
                             const double* __restrict__ scale, double* __restrict__ vals) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const double sr = scale[r];
    for (int k = indptr[r]; k < indptr[r + 1]; k++) vals[k] *= sr * scale[cols[k]];
}
void launch_scale_vals(const BlockCSR& A, const double* scale, double* vals, cudaStream_t st) {
    k_scale_vals<<<(A.n + 255) / 256, 256, 0, st>>>(A.n, A.indptr, A.cols, scale, vals);
}

// 3x3 nodal block-Jacobi: Gauss-Jordan with partial pivoting on the node's
// diagonal block; a singular block falls back to the identity.
__global__ void k_bj_setup(int nnodes, const int* __restrict__ indptr, const int* __restrict__ diag,
                           const double* __restrict__ vals, double* __restrict__ inv) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nnodes) return;
    double m[3][6];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const int p = diag[3 * a + r] - r;   // position of column 3a in row 3a+r
#pragma unroll
        for (int c = 0; c < 3; c++) { m[r][c] = vals[p + c]; m[r][3 + c] = (r == c) ? 1.0 : 0.0; }
    }
    bool ok = true;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        int p = c; double pv = fabs(m[c][c]);
#pragma unroll
        for (int r = c + 1; r < 3; r++) if (fabs(m[r][c]) > pv) { pv = fabs(m[r][c]); p = r; }
        if (pv == 0.0) { ok = false; break; }
        if (p != c) {
#pragma unroll
            for (int k = 0; k < 6; k++) {
                double t0 = m[c][k], t1 = (p == 1 ? m[1][k] : m[2][k]);
                m[c][k] = t1;
                if (p == 1) m[1][k] = t0; else m[2][k] = t0;
            }
        }
        const double d = m[c][c];
#pragma unroll
        for (int k = 0; k < 6; k++) m[c][k] /= d;
#pragma unroll
        for (int r = 0; r < 3; r++) {
            if (r == c) continue;
            const double f = m[r][c];
#pragma unroll
            for (int k = 0; k < 6; k++) m[r][k] -= f * m[c][k];
        }
    }
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) inv[9 * a + 3 * r + c] = ok ? m[r][3 + c] : (r == c ? 1.0 : 0.0);
}
void launch_bj_setup(const BlockCSR& A, const double* vals, double* inv, cudaStream_t st) {
    k_bj_setup<<<(A.nnodes + 127) / 128, 128, 0, st>>>(A.nnodes, A.indptr, A.diag, vals, inv);
}

// ---------------------------------------------------------------- SpMV + block-Jacobi
// y = M^-1 (A x) for node a, computed by the 8 lanes of a group; every lane of the
// group returns the result.
template <class VT>
__device__ __forceinline__ void node_spmv_bj(const BlockCSR& A, const VT* __restrict__ vals, const VT* __restrict__ inv,
                                             const VT* __restrict__ x, int a, bool valid, int g8, VT z[3]) {
    double y0 = 0, y1 = 0, y2 = 0;
    const int rs = valid ? A.indptr[3 * a] : 0;
    const int len = valid ? A.indptr[3 * a + 1] - rs : 0;
    const int s0 = valid ? A.bptr[a] : 0, deg = valid ? A.bptr[a + 1] - s0 : 0;
    for (int j = g8; j < deg; j += 8) {
        const int b = A.bcol[s0 + j];
        const double xb0 = x[3 * b], xb1 = x[3 * b + 1], xb2 = x[3 * b + 2];
        const VT* v0 = vals + rs + 3 * j;
        y0 += (double)v0[0] * xb0 + (double)v0[1] * xb1 + (double)v0[2] * xb2;
        const VT* v1 = v0 + len;
        y1 += (double)v1[0] * xb0 + (double)v1[1] * xb1 + (double)v1[2] * xb2;
        const VT* v2 = v1 + len;
        y2 += (double)v2[0] * xb0 + (double)v2[1] * xb1 + (double)v2[2] * xb2;
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
        y0 += __shfl_xor_sync(0xffffffffu, y0, o);
        y1 += __shfl_xor_sync(0xffffffffu, y1, o);
        y2 += __shfl_xor_sync(0xffffffffu, y2, o);
    }
    if (!valid) { z[0] = z[1] = z[2] = (VT)0; return; }
    const VT* M = inv + 9 * a;
    z[0] = (VT)((double)M[0] * y0 + (double)M[1] * y1 + (double)M[2] * y2);
    z[1] = (VT)((double)M[3] * y0 + (double)M[4] * y1 + (double)M[5] * y2);
    z[2] = (VT)((double)M[6] * y0 + (double)M[7] * y1 + (double)M[8] * y2);
}

// b <- M^-1 b ; x <- b    (bcgstab_solver.c:137-143)
template <class VT>
__global__ void k_bicg_init1(int nnodes, KrylovVecs<VT> V) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nnodes) return;
    const VT* M = V.inv + 9 * a;
    double b0 = V.b[3 * a], b1 = V.b[3 * a + 1], b2 = V.b[3 * a + 2];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        VT z = (VT)((double)M[3 * r] * b0 + (double)M[3 * r + 1] * b1 + (double)M[3 * r + 2] * b2);
        V.b[3 * a + r] = z; V.x[3 * a + r] = z;
    }
}

// r = b - M^-1 A x ; q = p = r ; rnorm, bnorm, rho   (bcgstab_solver.c:144-205)
template <class VT>
__global__ void __launch_bounds__(256) k_bicg_init2(BlockCSR A, KrylovVecs<VT> V, KrylovScalars* S, Reduce R) {
    __shared__ double sh[8];
    const int g8 = threadIdx.x & 7;
    double rmax = 0, bmax = 0, rr = 0;
    const int sub = (threadIdx.x & 31) >> 3;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 4; base < A.nnodes; base += nw * 4) {
        const int a = base + sub;
        const bool valid = a < A.nnodes;
        VT z[3];
        node_spmv_bj(A, V.vals, V.inv, V.x, a, valid, g8, z);
        if (g8 == 0 && valid) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                VT r = V.b[3 * a + k] + (VT)-1 * z[k];
                V.r[3 * a + k] = r; V.q[3 * a + k] = r; V.p[3 * a + k] = r; V.Ap[3 * a + k] = 0;
                rmax = fmax(rmax, fabs((double)r)); bmax = fmax(bmax, fabs((double)V.b[3 * a + k]));
                rr += (double)r * (double)r;
            }
        }
    }
    double v[3];
    v[0] = block_max<256>(rmax, sh); v[1] = block_max<256>(bmax, sh); v[2] = block_sum<256>(rr, sh);
    if (last_block(R, v, 3)) {
        double a = 0, b = 0, c = 0;
        for (int k = 0; k < (int)gridDim.x; k++) { a = fmax(a, ld_part(R, 4 * k)); b = fmax(b, ld_part(R, 4 * k + 1)); c += ld_part(R, 4 * k + 2); }
        S->rnorm = a; S->bnorm = b; S->rho = c;
        S->rhop = 1.0; S->alpha = 1.0; S->omega = 1.0; S->beta = 0.0; S->it = 0; S->status = 0;
        S->done = (a > (S->tol + b * S->rtol)) ? 0 : 1;
        if (!isfinite(a) || !isfinite(c)) { S->status = 2; S->done = 1; }
    }
}

// Ap = M^-1 A p ; gamma = q.Ap ; alpha = rho / gamma
template <class VT>
__global__ void __launch_bounds__(256) k_bicg_spmv_p(BlockCSR A, KrylovVecs<VT> V, KrylovScalars* S, Reduce R) {
    if (S->done) return;
    __shared__ double sh[8];
    const int g8 = threadIdx.x & 7;
    double qa = 0;
    const int sub = (threadIdx.x & 31) >> 3;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 4; base < A.nnodes; base += nw * 4) {
        const int a = base + sub;
        const bool valid = a < A.nnodes;
        VT z[3];
        node_spmv_bj(A, V.vals, V.inv, V.p, a, valid, g8, z);
        if (g8 == 0 && valid) {
#pragma unroll
            for (int k = 0; k < 3; k++) { V.Ap[3 * a + k] = z[k]; qa += (double)V.q[3 * a + k] * (double)z[k]; }
        }
    }
    double v[1];
    v[0] = block_sum<256>(qa, sh);
    if (last_block(R, v, 1)) {
        double g = 0;
        for (int k = 0; k < (int)gridDim.x; k++) g += ld_part(R, 4 * k);
        S->gamma = g;
        if (g == 0.0 || !isfinite(g)) { S->status = 1; S->done = 1; }
        else S->alpha = S->rho / g;
    }
}

// s = r - alpha Ap
template <class VT>
__global__ void k_bicg_s(int n, KrylovVecs<VT> V, const KrylovScalars* S) {
    if (S->done) return;
    const VT alpha = (VT)S->alpha;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        V.s[i] = V.r[i] + -alpha * V.Ap[i];
}

// As = M^-1 A s ; omega = As.s / As.As ; rho' = -omega As.q ; beta' = rho' alpha / (rho omega)
template <class VT>
__global__ void __launch_bounds__(256) k_bicg_spmv_s(BlockCSR A, KrylovVecs<VT> V, KrylovScalars* S, Reduce R) {
    if (S->done) return;
    __shared__ double sh[8];
    const int g8 = threadIdx.x & 7;
    double ss = 0, aa = 0, aq = 0;
    const int sub = (threadIdx.x & 31) >> 3;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 4; base < A.nnodes; base += nw * 4) {
        const int a = base + sub;
        const bool valid = a < A.nnodes;
        VT z[3];
        node_spmv_bj(A, V.vals, V.inv, V.s, a, valid, g8, z);
        if (g8 == 0 && valid) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                V.As[3 * a + k] = z[k];
                const double zk = (double)z[k];
                ss += zk * (double)V.s[3 * a + k]; aa += zk * zk; aq += zk * (double)V.q[3 * a + k];
            }
        }
    }
    double v[3];
    v[0] = block_sum<256>(ss, sh); v[1] = block_sum<256>(aa, sh); v[2] = block_sum<256>(aq, sh);
    if (last_block(R, v, 3)) {
        double a = 0, b = 0, c = 0;
        for (int k = 0; k < (int)gridDim.x; k++) { a += ld_part(R, 4 * k); b += ld_part(R, 4 * k + 1); c += ld_part(R, 4 * k + 2); }
        if (b == 0.0) {            // s == 0: x + alpha p is the solution
            S->omega = 0.0; S->status = 3;
        } else {
            const double om = a / b;
            S->omega = om;
            S->rhop = S->rho;
            S->rho = -1.0 * om * c;
            S->beta = (S->rho * S->alpha) / (S->rhop * om);
        }
    }
}

// x += alpha p ; x += omega s ; r = s - omega As ; p' = (p - omega Ap) beta' + r ; rnorm
template <class VT>
__global__ void __launch_bounds__(256) k_bicg_update(int n, KrylovVecs<VT> V, KrylovScalars* S, Reduce R) {
    if (S->done) return;
    __shared__ double sh[8];
    const bool s_zero = S->status == 3 || S->status == 5;
    const VT alpha = (VT)S->alpha, omega = (VT)S->omega, beta = (VT)S->beta;
    double rmax = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        VT x = V.x[i] + alpha * V.p[i];
        VT r;
        if (s_zero) {
            r = V.s[i];
        } else {
            x = x + omega * V.s[i];
            r = V.s[i] + -omega * V.As[i];
            VT p = V.p[i] + -omega * V.Ap[i];
            p = p * beta;
            V.p[i] = p + (VT)1 * r;
        }
        V.x[i] = x; V.r[i] = r;
        rmax = fmax(rmax, fabs((double)r));
    }
    double v[1];
    v[0] = block_max<256>(rmax, sh);
    if (last_block(R, v, 1)) {
        double m = 0;
        for (int k = 0; k < (int)gridDim.x; k++) m = fmax(m, ld_part(R, 4 * k));
        S->rnorm = m;
        S->it += 1;
        if (S->status == 3) { S->status = 0; S->done = 1; }
        if (S->status == 5) { S->status = 1; S->done = 1; }
        if (!(m > (S->tol + S->bnorm * S->rtol)) || S->it >= S->max_it) S->done = 1;
        if (!isfinite(m)) { S->status = 2; S->done = 1; }
    }
}

template <class VT>
void launch_bicg_init(const BlockCSR& A, KrylovVecs<VT> V, KrylovScalars* S, Reduce R, cudaStream_t st) {
    k_bicg_init1<VT><<<(A.nnodes + 255) / 256, 256, 0, st>>>(A.nnodes, V);
    k_bicg_init2<VT><<<grid_for(8L * A.nnodes, 256), 256, 0, st>>>(A, V, S, R);
}
template <class VT>
void launch_bicg_iteration(const BlockCSR& A, KrylovVecs<VT> V, KrylovScalars* S, Reduce R, cudaStream_t st) {
    const int gs = grid_for(8L * A.nnodes, 256);
    const int gv = grid_for(A.n, 256);
    k_bicg_spmv_p<VT><<<gs, 256, 0, st>>>(A, V, S, R);
    k_bicg_s<VT><<<gv, 256, 0, st>>>(A.n, V, S);
    k_bicg_spmv_s<VT><<<gs, 256, 0, st>>>(A, V, S, R);
    k_bicg_update<VT><<<gv, 256, 0, st>>>(A.n, V, S, R);
}
template void launch_bicg_init<double>(const BlockCSR&, KrylovVecs<double>, KrylovScalars*, Reduce, cudaStream_t);
template void launch_bicg_init<float>(const BlockCSR&, KrylovVecs<float>, KrylovScalars*, Reduce, cudaStream_t);
template void launch_bicg_iteration<double>(const BlockCSR&, KrylovVecs<double>, KrylovScalars*, Reduce, cudaStream_t);
template void launch_bicg_iteration<float>(const BlockCSR&, KrylovVecs<float>, KrylovScalars*, Reduce, cudaStream_t);

// t = b - A x ; max |M^-1 t|   (FP64 refinement residual)
__global__ void __launch_bounds__(256) k_resid_pnorm(BlockCSR A, const double* __restrict__ vals, const double* __restrict__ inv,
                                                     const double* __restrict__ x, const double* __restrict__ b,
                                                     double* __restrict__ t, Reduce R) {
    __shared__ double sh[8];
    const int g8 = threadIdx.x & 7, sub = (threadIdx.x & 31) >> 3;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    double zmax = 0;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 4; base < A.nnodes; base += nw * 4) {
        const int a = base + sub;
        const bool valid = a < A.nnodes;
        double y0 = 0, y1 = 0, y2 = 0;
        const int rs = valid ? A.indptr[3 * a] : 0;
        const int len = valid ? A.indptr[3 * a + 1] - rs : 0;
        const int s0 = valid ? A.bptr[a] : 0, deg = valid ? A.bptr[a + 1] - s0 : 0;
        for (int j = g8; j < deg; j += 8) {
            const int bb = A.bcol[s0 + j];
            const double xb0 = x[3 * bb], xb1 = x[3 * bb + 1], xb2 = x[3 * bb + 2];
            const double* v0 = vals + rs + 3 * j;
            y0 += v0[0] * xb0 + v0[1] * xb1 + v0[2] * xb2;
            const double* v1 = v0 + len;
            y1 += v1[0] * xb0 + v1[1] * xb1 + v1[2] * xb2;
            const double* v2 = v1 + len;
            y2 += v2[0] * xb0 + v2[1] * xb1 + v2[2] * xb2;
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
            y0 += __shfl_xor_sync(0xffffffffu, y0, o);
            y1 += __shfl_xor_sync(0xffffffffu, y1, o);
            y2 += __shfl_xor_sync(0xffffffffu, y2, o);
        }
        if (g8 == 0 && valid) {
            const double t0 = b[3 * a] - y0, t1 = b[3 * a + 1] - y1, t2 = b[3 * a + 2] - y2;
            t[3 * a] = t0; t[3 * a + 1] = t1; t[3 * a + 2] = t2;
            const double* M = inv + 9 * a;
            zmax = fmax(zmax, fabs(M[0] * t0 + M[1] * t1 + M[2] * t2));
            zmax = fmax(zmax, fabs(M[3] * t0 + M[4] * t1 + M[5] * t2));
            zmax = fmax(zmax, fabs(M[6] * t0 + M[7] * t1 + M[8] * t2));
        }
    }
    double v[1];
    v[0] = block_max<256>(zmax, sh);
    if (last_block(R, v, 1)) {
        double mm = 0;
        for (int k = 0; k < (int)gridDim.x; k++) mm = fmax(mm, ld_part(R, 4 * k));
        R.out[0] = mm;
    }
}
void launch_resid_pnorm(const BlockCSR& A, const double* vals, const double* inv, const double* x, const double* b,
                        double* t, Reduce R, cudaStream_t st) {
    k_resid_pnorm<<<grid_for(8L * A.nnodes, 256), 256, 0, st>>>(A, vals, inv, x, b, t, R);
}

// ---------------------------------------------------------------- vector helpers
// unscale_linear_system (scale_linear_system.c:137): x = (x + x0) * s
__global__ void k_unscale(int n, const double* __restrict__ x0, const double* __restrict__ s, double* __restrict__ x) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = x[i] + x0[i];
    x[i] = v * s[i];
}
void launch_unscale(int n, const double* x0, const double* scale, double* x, cudaStream_t st) {
    k_unscale<<<(n + 255) / 256, 256, 0, st>>>(n, x0, scale, x);
}
__global__ void k_axpy(int n, double a, const double* __restrict__ x, double* __restrict__ y) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += a * x[i];
}
void launch_axpy(int n, double a, const double* x, double* y, cudaStream_t st) {
    k_axpy<<<(n + 255) / 256, 256, 0, st>>>(n, a, x, y);
}
__global__ void k_scal(int n, double a, double* __restrict__ x) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] *= a;
}
void launch_scal(int n, double a, double* x, cudaStream_t st) {
    k_scal<<<(n + 255) / 256, 256, 0, st>>>(n, a, x);
}
__global__ void k_to_float(int n, const double* __restrict__ s, float* __restrict__ d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = (float)s[i];
}
__global__ void k_to_double(int n, const float* __restrict__ s, double* __restrict__ d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = (double)s[i];
}
void launch_to_float(int n, const double* src, float* dst, cudaStream_t st) {
    k_to_float<<<(n + 255) / 256, 256, 0, st>>>(n, src, dst);
}
void launch_to_double(int n, const float* src, double* dst, cudaStream_t st) {
    k_to_double<<<(n + 255) / 256, 256, 0, st>>>(n, src, dst);
}

}  // namespace sw2

namespace sw2 {
// dst[i] = src[i] where mask[i] == 1 (initialize_dirichlet_bc, src/newton/newton_tools.c:130)
__global__ void k_masked_copy(int n, const int* __restrict__ mask, const double* __restrict__ src, double* __restrict__ dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && mask[i] == 1) dst[i] = src[i];
}
void launch_masked_copy(int n, const int* mask, const double* src, double* dst, cudaStream_t st) {
    k_masked_copy<<<(n + 255) / 256, 256, 0, st>>>(n, mask, src, dst);
}
}  // namespace sw2

// ======================================================================
// BiCGStab with an explicit preconditioner apply (multicolour block ILU).
// Per iteration: Ap = M^-1 (A p); alpha; s; As = M^-1 (A s); omega, rho, beta;
// update -- the recurrences of bcgstab_solver.c:210-310.
namespace sw2 {

int grid_for_nodes(long nodes) { return grid_for(8L * nodes, 256); }
int grid_resident(long work_items, int blocks_per_sm) {
    grid_for(1, 256);   // fills g_num_sms
    long need = (work_items + 255) / 256;
    long cap = (long)blocks_per_sm * g_num_sms;
    if (cap > kMaxBlocks) cap = kMaxBlocks;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

template <class VT>
__global__ void __launch_bounds__(256, kSweepBlocksPerSM) k_spmv(BlockCSR A, const VT* __restrict__ vals, const VT* __restrict__ x,
                                              VT* __restrict__ y, const int* __restrict__ skip) {
    if (skip && *skip) return;
    // lanes per node: 8 for FP64 values; 2 for FP32, whose half-size rows need more neighbour
    // blocks in flight per lane (the same choice as the AMG level-0 kernels, measured there)
    constexpr int LANES = sizeof(VT) == 4 ? 2 : 8, PER_WARP = 32 / LANES;
    const int g8 = threadIdx.x & (LANES - 1), sub = (threadIdx.x & 31) / LANES;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * PER_WARP; base < A.nnodes; base += nw * PER_WARP) {
        const int a = base + sub;
        const bool valid = a < A.nnodes;
        double y0 = 0, y1 = 0, y2 = 0;
        const int rs = valid ? A.indptr[3 * a] : 0;
        const int len = valid ? A.indptr[3 * a + 1] - rs : 0;
        const int s0 = valid ? A.bptr[a] : 0, deg = valid ? A.bptr[a + 1] - s0 : 0;
#pragma unroll 2
        for (int j = g8; j < deg; j += LANES) {
            const int b = A.bcol[s0 + j];
            const double xb0 = x[3 * b], xb1 = x[3 * b + 1], xb2 = x[3 * b + 2];
            const VT* v0 = vals + rs + 3 * j;
            y0 += (double)v0[0] * xb0 + (double)v0[1] * xb1 + (double)v0[2] * xb2;
            const VT* v1 = v0 + len;
            y1 += (double)v1[0] * xb0 + (double)v1[1] * xb1 + (double)v1[2] * xb2;
            const VT* v2 = v1 + len;
            y2 += (double)v2[0] * xb0 + (double)v2[1] * xb1 + (double)v2[2] * xb2;
        }
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1) {
            y0 += __shfl_xor_sync(0xffffffffu, y0, o);
            y1 += __shfl_xor_sync(0xffffffffu, y1, o);
            y2 += __shfl_xor_sync(0xffffffffu, y2, o);
        }
        if (g8 == 0 && valid) { y[3 * a] = (VT)y0; y[3 * a + 1] = (VT)y1; y[3 * a + 2] = (VT)y2; }
    }
}
// lanes per node of k_spmv (must match LANES inside it) and its one-wave grid
template <class VT> static int spmv_grid(int nnodes) {
    return grid_resident((long)nnodes * (sizeof(VT) == 4 ? 2 : 8), kSweepBlocksPerSM);
}

template <class VT>
__global__ void k_copy(int n, const VT* __restrict__ a, VT* __restrict__ b) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

// r = b - r (r holds M^-1 A x) ; q = p = r ; Ap = 0 ; rnorm, bnorm, rho
template <class VT>
__global__ void __launch_bounds__(256) k_bicg_init_pc(int n, KrylovVecs<VT> V, KrylovScalars* S, Reduce R) {
    __shared__ double sh[8];
    double rmax = 0, bmax = 0, rr = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const VT r = V.b[i] + (VT)-1 * V.r[i];
        V.r[i] = r; V.q[i] = r; V.p[i] = r; V.Ap[i] = 0;
        rmax = fmax(rmax, fabs((double)r)); bmax = fmax(bmax, fabs((double)V.b[i]));
        rr += (double)r * (double)r;
    }
    double v[3];
    v[0] = block_max<256>(rmax, sh); v[1] = block_max<256>(bmax, sh); v[2] = block_sum<256>(rr, sh);
    if (last_block(R, v, 3)) {
        double a = 0, b = 0, c = 0;
        for (int k = 0; k < (int)gridDim.x; k++) { a = fmax(a, ld_part(R, 4 * k)); b = fmax(b, ld_part(R, 4 * k + 1)); c += ld_part(R, 4 * k + 2); }
        S->rnorm = a; S->bnorm = b; S->rho = c;
        S->rhop = 1.0; S->alpha = 1.0; S->omega = 1.0; S->beta = 0.0; S->it = 0; S->status = 0;
        S->done = (a > (S->tol + b * S->rtol)) ? 0 : 1;
        if (!isfinite(a) || !isfinite(c)) { S->status = 2; S->done = 1; }
    }
}

// gamma = q.Ap ; alpha = rho / gamma
template <class VT>
__global__ void __launch_bounds__(256) k_bicg_alpha(int n, KrylovVecs<VT> V, KrylovScalars* S, Reduce R) {
    if (S->done) return;
    __shared__ double sh[8];
    double qa = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        qa += (double)V.q[i] * (double)V.Ap[i];
    double v[1];
    v[0] = block_sum<256>(qa, sh);
    if (last_block(R, v, 1)) {
        double g = 0;
        for (int k = 0; k < (int)gridDim.x; k++) g += ld_part(R, 4 * k);
        S->gamma = g;
        if (g == 0.0 || !isfinite(g)) { S->status = 1; S->done = 1; }
        else S->alpha = S->rho / g;
    }
}

// omega = As.s / As.As ; rho' = -omega As.q ; beta'
template <class VT>
__global__ void __launch_bounds__(256) k_bicg_omega(int n, KrylovVecs<VT> V, KrylovScalars* S, Reduce R) {
    if (S->done) return;
    __shared__ double sh[8];
    double ss = 0, aa = 0, aq = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double z = (double)V.As[i];
        ss += z * (double)V.s[i]; aa += z * z; aq += z * (double)V.q[i];
    }
    double v[3];
    v[0] = block_sum<256>(ss, sh); v[1] = block_sum<256>(aa, sh); v[2] = block_sum<256>(aq, sh);
    if (last_block(R, v, 3)) {
        double a = 0, b = 0, c = 0;
        for (int k = 0; k < (int)gridDim.x; k++) { a += ld_part(R, 4 * k); b += ld_part(R, 4 * k + 1); c += ld_part(R, 4 * k + 2); }
        if (b == 0.0) { S->omega = 0.0; S->status = 3; }
        else {
            const double om = a / b;
            const double rho_new = -1.0 * om * c;
            const double beta = (rho_new * S->alpha) / (S->rho * om);
            if (om == 0.0 || rho_new == 0.0 || !isfinite(om) || !isfinite(beta)) {
                S->omega = 0.0; S->status = 5;   // breakdown: take the half step x += alpha p, then stop
            } else {
                S->omega = om; S->rhop = S->rho; S->rho = rho_new; S->beta = beta;
            }
        }
    }
}

void launch_spmv64(const BlockCSR& A, const double* vals, const double* x, double* y, cudaStream_t st) {
    k_spmv<double><<<spmv_grid<double>(A.nnodes), 256, 0, st>>>(A, vals, x, y, nullptr);
}

template <class VT>
__global__ void k_cast_skip(int n, const VT* __restrict__ a, float* __restrict__ b, const int* __restrict__ skip) {
    if (skip && *skip) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = (float)a[i];
}
template <class VT>
__global__ void k_uncast_skip(int n, const float* __restrict__ a, VT* __restrict__ b, const int* __restrict__ skip) {
    if (skip && *skip) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = (VT)a[i];
}

template <class VT>
void precond_apply(const BlockCSR& A, const PrecondOp<VT>& P, VT* y, const int* skip, cudaStream_t st) {
    if (P.mixed) {
        PrecondOp<float> P32;
        P32.kind = P.kind; P32.ilu = P.ilu; P32.lu = P.lu32; P32.dinv = P.dinv32; P32.amg = P.amg; P32.vals = P.vals32;
        const int g = grid_for(A.n, 256);
        k_cast_skip<VT><<<g, 256, 0, st>>>(A.n, y, P.tmp32, skip);
        precond_apply<float>(A, P32, P.tmp32, skip, st);
        k_uncast_skip<VT><<<g, 256, 0, st>>>(A.n, P.tmp32, y, skip);
        return;
    }
    if (P.kind == 2) {
        amg_apply<VT>(A, *P.amg, P.vals, y, skip, st);
    } else {
        IluHost Hs = *P.ilu; Hs.view.skip = skip;
        launch_bilu_apply<VT>(A, Hs, P.lu, P.dinv, y, st);
    }
}
template void precond_apply<double>(const BlockCSR&, const PrecondOp<double>&, double*, const int*, cudaStream_t);
template void precond_apply<float>(const BlockCSR&, const PrecondOp<float>&, float*, const int*, cudaStream_t);

template <class VT>
__global__ void k_copy_skip(int n, const VT* __restrict__ a, VT* __restrict__ b, const int* __restrict__ skip) {
    if (skip && *skip) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

// Left preconditioning (the reference's form, bcgstab_solver.c:65-330): the
// recurrences run on M^-1 A and M^-1 b, so the stopping test sees preconditioned
// residuals.  Right preconditioning runs the same recurrences on A M^-1 with the
// plain b (x holds y, and x = M^-1 y is taken after the loop), so the stopping
// test sees the true residual of the scaled system -- needed when M is an
// approximate multilevel operator whose M^-1 r can be small while r is not.  Both
// start from x0 = M^-1 b.
template <class VT>
void launch_bicg_init_pc(const BlockCSR& A, const PrecondOp<VT>& P, KrylovVecs<VT> V, KrylovScalars* S, Reduce R,
                         cudaStream_t st) {
    const int gv = grid_for(A.n, 256);
    if (P.right) {
        k_copy<VT><<<gv, 256, 0, st>>>(A.n, V.b, V.x);                // y = b
        k_copy<VT><<<gv, 256, 0, st>>>(A.n, V.x, V.z);
        precond_apply<VT>(A, P, V.z, nullptr, st);                    // z = M^-1 y
        k_spmv<VT><<<spmv_grid<VT>(A.nnodes), 256, 0, st>>>(A, V.vals, V.z, V.r, nullptr);
    } else {
        precond_apply<VT>(A, P, V.b, nullptr, st);                    // b <- M^-1 b
        k_copy<VT><<<gv, 256, 0, st>>>(A.n, V.b, V.x);                // x = b
        k_spmv<VT><<<spmv_grid<VT>(A.nnodes), 256, 0, st>>>(A, V.vals, V.x, V.r, nullptr);
        precond_apply<VT>(A, P, V.r, nullptr, st);                    // r <- M^-1 A x
    }
    k_bicg_init_pc<VT><<<gv, 256, 0, st>>>(A.n, V, S, R);
}
template <class VT>
void copy_skip(int n, const VT* a, VT* b, const int* skip, cudaStream_t st) {
    k_copy_skip<VT><<<grid_for(n, 256), 256, 0, st>>>(n, a, b, skip);
}
template <class VT>
void spmv_skip(const BlockCSR& A, const VT* vals, const VT* x, VT* y, const int* skip, cudaStream_t st) {
    k_spmv<VT><<<spmv_grid<VT>(A.nnodes), 256, 0, st>>>(A, vals, x, y, skip);
}
template void copy_skip<double>(int, const double*, double*, const int*, cudaStream_t);
template void copy_skip<float>(int, const float*, float*, const int*, cudaStream_t);
template void spmv_skip<double>(const BlockCSR&, const double*, const double*, double*, const int*, cudaStream_t);
template void spmv_skip<float>(const BlockCSR&, const float*, const float*, float*, const int*, cudaStream_t);

template <class VT>
void launch_bicg_iteration_pc(const BlockCSR& A, const PrecondOp<VT>& P, KrylovVecs<VT> V, KrylovScalars* S, Reduce R,
                              cudaStream_t st) {
    const int gv = grid_for(A.n, 256), gs = spmv_grid<VT>(A.nnodes);
    const int* done = &S->done;
    if (P.right) {
        k_copy_skip<VT><<<gv, 256, 0, st>>>(A.n, V.p, V.z, done);
        precond_apply<VT>(A, P, V.z, done, st);
        k_spmv<VT><<<gs, 256, 0, st>>>(A, V.vals, V.z, V.Ap, done);
    } else {
        k_spmv<VT><<<gs, 256, 0, st>>>(A, V.vals, V.p, V.Ap, done);
        precond_apply<VT>(A, P, V.Ap, done, st);
    }
    k_bicg_alpha<VT><<<gv, 256, 0, st>>>(A.n, V, S, R);
    k_bicg_s<VT><<<gv, 256, 0, st>>>(A.n, V, S);
    if (P.right) {
        k_copy_skip<VT><<<gv, 256, 0, st>>>(A.n, V.s, V.z, done);
        precond_apply<VT>(A, P, V.z, done, st);
        k_spmv<VT><<<gs, 256, 0, st>>>(A, V.vals, V.z, V.As, done);
    } else {
        k_spmv<VT><<<gs, 256, 0, st>>>(A, V.vals, V.s, V.As, done);
        precond_apply<VT>(A, P, V.As, done, st);
    }
    k_bicg_omega<VT><<<gv, 256, 0, st>>>(A.n, V, S, R);
    k_bicg_update<VT><<<gv, 256, 0, st>>>(A.n, V, S, R);
}
template void launch_bicg_init_pc<double>(const BlockCSR&, const PrecondOp<double>&, KrylovVecs<double>, KrylovScalars*, Reduce, cudaStream_t);
template void launch_bicg_init_pc<float>(const BlockCSR&, const PrecondOp<float>&, KrylovVecs<float>, KrylovScalars*, Reduce, cudaStream_t);
template void launch_bicg_iteration_pc<double>(const BlockCSR&, const PrecondOp<double>&, KrylovVecs<double>, KrylovScalars*, Reduce, cudaStream_t);
template void launch_bicg_iteration_pc<float>(const BlockCSR&, const PrecondOp<float>&, KrylovVecs<float>, KrylovScalars*, Reduce, cudaStream_t);

}  // namespace sw2

namespace sw2 {
__global__ void __launch_bounds__(256) k_spmv_sub(BlockCSR A, const double* __restrict__ vals, const double* __restrict__ x,
                                                  const double* __restrict__ b, double* __restrict__ t) {
    const int g8 = threadIdx.x & 7, sub = (threadIdx.x & 31) >> 3;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 4; base < A.nnodes; base += nw * 4) {
        const int a = base + sub;
        const bool valid = a < A.nnodes;
        double y0 = 0, y1 = 0, y2 = 0;
        const int rs = valid ? A.indptr[3 * a] : 0;
        const int len = valid ? A.indptr[3 * a + 1] - rs : 0;
        const int s0 = valid ? A.bptr[a] : 0, deg = valid ? A.bptr[a + 1] - s0 : 0;
        for (int j = g8; j < deg; j += 8) {
            const int bb = A.bcol[s0 + j];
            const double xb0 = x[3 * bb], xb1 = x[3 * bb + 1], xb2 = x[3 * bb + 2];
            const double* v0 = vals + rs + 3 * j;
            y0 += v0[0] * xb0 + v0[1] * xb1 + v0[2] * xb2;
            const double* v1 = v0 + len;
            y1 += v1[0] * xb0 + v1[1] * xb1 + v1[2] * xb2;
            const double* v2 = v1 + len;
            y2 += v2[0] * xb0 + v2[1] * xb1 + v2[2] * xb2;
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
            y0 += __shfl_xor_sync(0xffffffffu, y0, o);
            y1 += __shfl_xor_sync(0xffffffffu, y1, o);
            y2 += __shfl_xor_sync(0xffffffffu, y2, o);
        }
        if (g8 == 0 && valid) { t[3 * a] = b[3 * a] - y0; t[3 * a + 1] = b[3 * a + 1] - y1; t[3 * a + 2] = b[3 * a + 2] - y2; }
    }
}
void launch_spmv_sub(const BlockCSR& A, const double* vals, const double* x, const double* b, double* t, cudaStream_t st) {
    k_spmv_sub<<<grid_for_nodes(A.nnodes), 256, 0, st>>>(A, vals, x, b, t);
}
__global__ void k_bj_apply(int nnodes, const double* __restrict__ inv, double* __restrict__ z) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nnodes) return;
    const double* M = inv + 9 * a;
    const double z0 = z[3 * a], z1 = z[3 * a + 1], z2 = z[3 * a + 2];
    z[3 * a] = M[0] * z0 + M[1] * z1 + M[2] * z2;
    z[3 * a + 1] = M[3] * z0 + M[4] * z1 + M[5] * z2;
    z[3 * a + 2] = M[6] * z0 + M[7] * z1 + M[8] * z2;
}
void launch_bj_apply(int nnodes, const double* inv, double* z, cudaStream_t st) {
    k_bj_apply<<<(nnodes + 255) / 256, 256, 0, st>>>(nnodes, inv, z);
}
__global__ void __launch_bounds__(256) k_maxabs(int n, const double* __restrict__ z, Reduce R) {
    __shared__ double sh[8];
    double m = 0, bad = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double a = fabs(z[i]);
        if (!isfinite(a)) bad = 1; else m = fmax(m, a);
    }
    double v[2];
    v[0] = block_max<256>(m, sh); v[1] = block_max<256>(bad, sh);
    if (last_block(R, v, 2)) {
        double a = 0, b = 0;
        for (int k = 0; k < (int)gridDim.x; k++) { a = fmax(a, ld_part(R, 4 * k)); b = fmax(b, ld_part(R, 4 * k + 1)); }
        R.out[0] = b > 0 ? NAN : a;   // a non-finite entry is reported, not hidden by fmax
    }
}
__global__ void __launch_bounds__(256) k_maxabs_unscaled(int n, const double* __restrict__ t, const double* __restrict__ sc,
                                                         Reduce R) {
    __shared__ double sh[8];
    double m = 0, bad = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double a = fabs(t[i] / sc[i]);
        if (!isfinite(a)) bad = 1; else m = fmax(m, a);
    }
    double v[2];
    v[0] = block_max<256>(m, sh); v[1] = block_max<256>(bad, sh);
    if (last_block(R, v, 2)) {
        double a = 0, b = 0;
        for (int k = 0; k < (int)gridDim.x; k++) { a = fmax(a, ld_part(R, 4 * k)); b = fmax(b, ld_part(R, 4 * k + 1)); }
        R.out[0] = b > 0 ? NAN : a;
    }
}
__global__ void k_inv_scale(int n, const double* __restrict__ s, double* __restrict__ rw) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) rw[i] = 1.0 / s[i];
}
void launch_inv_scale(int n, const double* scale, double* rw, cudaStream_t st) {
    k_inv_scale<<<grid_for(n, 256), 256, 0, st>>>(n, scale, rw);
}
void launch_maxabs_unscaled(int n, const double* t, const double* scale, Reduce R, cudaStream_t st) {
    k_maxabs_unscaled<<<grid_for(n, 256), 256, 0, st>>>(n, t, scale, R);
}
void launch_maxabs(int n, const double* z, Reduce R, cudaStream_t st) {
    k_maxabs<<<grid_for(n, 256), 256, 0, st>>>(n, z, R);
}
}  // namespace sw2
