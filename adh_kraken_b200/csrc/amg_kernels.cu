// Aggregation AMG preconditioner for the scaled 3x3-block SW2 Jacobian.
//
// Why: at the Courant numbers of a fine wet/dry beach (gravity-wave CFL ~ 120 at
// 14 m spacing and dt = 120 s) the SUPG-stabilised Jacobian is an elliptic
// system -- the h-h block is Laplacian-like with a small mass shift and the
// momentum block carries a grad-div-like part -- so 3x3 block-Jacobi stalls and
// zero-fill block ILU is numerically unstable.  The reference sidesteps this with
// a full UMFPACK LU per Newton iteration (src/la/bcgstab_solver.c:371-420).  This
// preconditioner is a multilevel method over the same node blocks:
//   * levels: greedy node aggregation (a node with no aggregated neighbour seeds an
//     aggregate with its whole neighbourhood; leftovers join a neighbour's); the
//     prolongation is piecewise constant per variable, so every coarse 3x3 block is
//     the plain sum of the fine blocks it covers (Galerkin R A P with R = P^T);
//   * smoother: damped 3x3 block-Jacobi (omega = kAmgOmega), kAmgNu sweeps before
//     and after the coarse correction, with an l1 fix-up of the blocks where plain
//     block-Jacobi amplifies (the wet/dry front, the inflow boundary); the coarsest
//     level gets kAmgCoarseSweeps sweeps inside one CTA;
//   * one V-cycle is a fixed linear operator, as BiCGStab requires.
// Level 0 is the reference CSR itself (node-centric kernels as in the SpMV); the
// coarse levels are block CSR with 9 values per block.
//
// Everything is deterministic: coarse values and restrictions are gathers in a
// fixed order (no atomics), so a run is reproducible bit for bit.
#include <cmath>
#include "sw2_launch.h"

namespace sw2 {

static inline int nb(long n, int t) { return (int)((n + t - 1) / t); }

// ---------------------------------------------------------------- numeric set-up (FP64)
// coarse block q of level 1 = sum of the level-0 slots gsrc[gptr[q] .. gptr[q+1])
// (slot k holds rows 3i..3i+2 at vals[boff[k] + v*blen[k] + 0..2])
__global__ void k_galerkin0(int nbc, const int* __restrict__ gptr, const int* __restrict__ gsrc,
                            const int* __restrict__ boff, const int* __restrict__ blen, const double* __restrict__ vals,
                            double* __restrict__ coarse) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nbc) return;
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int t = gptr[q]; t < gptr[q + 1]; t++) {
        const int k = gsrc[t];
        const double* v = vals + boff[k];
        const int L = blen[k];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) s[3 * r + c] += v[r * L + c];
    }
#pragma unroll
    for (int e = 0; e < 9; e++) coarse[9 * (size_t)q + e] = s[e];
}

// coarse block q of level l+1 = sum of the level-l blocks gsrc[gptr[q] .. gptr[q+1])
__global__ void k_galerkin(int nbc, const int* __restrict__ gptr, const int* __restrict__ gsrc,
                           const double* __restrict__ fine, double* __restrict__ coarse) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nbc) return;
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int t = gptr[q]; t < gptr[q + 1]; t++) {
        const double* v = fine + 9 * (size_t)gsrc[t];
#pragma unroll
        for (int e = 0; e < 9; e++) s[e] += v[e];
    }
#pragma unroll
    for (int e = 0; e < 9; e++) coarse[9 * (size_t)q + e] = s[e];
}

// 3x3 inverse by cofactors; false (and the identity) when the block is singular
__device__ __forceinline__ bool inv3(const double* a, double* o) {
    const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    const double scale = fabs(a[0]) + fabs(a[4]) + fabs(a[8]);
    if (!(fabs(det) > 1e-300 && fabs(det) > 1e-14 * scale * scale * scale) || !isfinite(det)) {
        for (int e = 0; e < 9; e++) o[e] = (e % 4 == 0) ? 1.0 : 0.0;
        return false;
    }
    const double r = 1.0 / det;
    o[0] = c00 * r; o[1] = (a[2] * a[7] - a[1] * a[8]) * r; o[2] = (a[1] * a[5] - a[2] * a[4]) * r;
    o[3] = c01 * r; o[4] = (a[0] * a[8] - a[2] * a[6]) * r; o[5] = (a[2] * a[3] - a[0] * a[5]) * r;
    o[6] = c02 * r; o[7] = (a[1] * a[6] - a[0] * a[7]) * r; o[8] = (a[0] * a[4] - a[1] * a[3]) * r;
    return true;
}

// Smoother block of one node: the inverse of its diagonal 3x3 block, with an l1
// fix-up where plain block-Jacobi would amplify.  A row whose diagonal is small
// against the rest of its row (|a_vv| < kAmgL1Theta * off_v, shallow nodes at the
// wet/dry front) gets off_v added to its diagonal; a node whose local Jacobi gain
// ||D^-1||_inf * max_v off_v exceeds kAmgGainMax (nearly singular blocks, e.g.
// at the inflow boundary) gets that for all three rows.  off_v = sum of |a| of
// row v outside the diagonal block.
// Returns true when the block the smoother uses is much weaker than the plain inverse
// (sum of |entries| below kPatchFlagRatio of it, or no plain inverse at all): block-Jacobi
// barely moves such a node, so the chunk correction takes it over.
__device__ __forceinline__ bool l1_block_inverse(const double* a_in, const double* off, double* o) {
    double a[9];
#pragma unroll
    for (int e = 0; e < 9; e++) a[e] = a_in[e];
    bool fix[3], any = false;
#pragma unroll
    for (int v = 0; v < 3; v++) { fix[v] = fabs(a[4 * v]) < kAmgL1Theta * off[v]; any |= fix[v]; }
    const bool ok = inv3(a, o);
    double gain = 0.0;
    if (ok) {
        const double offmax = fmax(off[0], fmax(off[1], off[2]));
        for (int v = 0; v < 3; v++) gain = fmax(gain, (fabs(o[3 * v]) + fabs(o[3 * v + 1]) + fabs(o[3 * v + 2])) * offmax);
    }
    if (!ok || gain > kAmgGainMax) { fix[0] = fix[1] = fix[2] = true; any = true; }
    if (!any) return false;
    double plain = 0.0;
#pragma unroll
    for (int e = 0; e < 9; e++) plain += fabs(o[e]);
#pragma unroll
    for (int v = 0; v < 3; v++)
        if (fix[v]) a[4 * v] += (a[4 * v] >= 0.0 ? off[v] : -off[v]);
    inv3(a, o);
    double fixed = 0.0;
#pragma unroll
    for (int e = 0; e < 9; e++) fixed += fabs(o[e]);
    return !ok || fixed < kPatchFlagRatio * plain;
}

// level 0: diagonal blocks and off-block row sums read from the reference CSR
__global__ void k_amg_dinv0(BlockCSR A, const double* __restrict__ vals, double* __restrict__ dinv, int* __restrict__ flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.nnodes) return;
    const int rs = A.indptr[3 * i], len = A.indptr[3 * i + 1] - rs;
    const int dslot = (A.diag[3 * i] - rs) / 3;
    double blk[9], off[3] = {0, 0, 0};
    for (int v = 0; v < 3; v++) {
        const double* row = vals + rs + v * len;
        for (int q = 0; q < len; q++) {
            if (q / 3 == dslot) blk[3 * v + (q - 3 * dslot)] = row[q];
            else off[v] += fabs(row[q]);
        }
    }
    const bool weak = l1_block_inverse(blk, off, dinv + 9 * (size_t)i);
    if (flag) flag[i] = weak ? 1 : 0;
}

// coarse levels (block CSR)
__global__ void k_bsr_dinv(int n, const int* __restrict__ bptr, const int* __restrict__ dpos,
                           const double* __restrict__ val, double* __restrict__ dinv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double off[3] = {0, 0, 0};
    for (int q = bptr[i]; q < bptr[i + 1]; q++) {
        if (q == dpos[i]) continue;
        const double* v = val + 9 * (size_t)q;
        for (int r = 0; r < 3; r++) off[r] += fabs(v[3 * r]) + fabs(v[3 * r + 1]) + fabs(v[3 * r + 2]);
    }
    l1_block_inverse(val + 9 * (size_t)dpos[i], off, dinv + 9 * (size_t)i);
}

__global__ void k_cast32(long n, const double* __restrict__ a, float* __restrict__ b) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) b[i] = (float)a[i];
}

// ---------------------------------------------------------------- V-cycle kernels
// y = w * Dinv b (a smoothing sweep from a zero start), per node
template <class VT>
__global__ void k_amg_scale(int nn, const VT* __restrict__ dinv, const VT* __restrict__ b, VT* __restrict__ y, double w,
                            const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const VT* D = dinv + 9 * (size_t)i;
    const double b0 = b[3 * i], b1 = b[3 * i + 1], b2 = b[3 * i + 2];
    y[3 * i] = (VT)(w * ((double)D[0] * b0 + (double)D[1] * b1 + (double)D[2] * b2));
    y[3 * i + 1] = (VT)(w * ((double)D[3] * b0 + (double)D[4] * b1 + (double)D[5] * b2));
    y[3 * i + 2] = (VT)(w * ((double)D[6] * b0 + (double)D[7] * b1 + (double)D[8] * b2));
}

// Level 0 (reference CSR): LANES lanes per node walk its neighbour slots.
// MODE 0: r = b - A x ;  MODE 1: y = x + w Dinv (b - A x)
template <class VT, int MODE, int LANES>
__global__ void __launch_bounds__(256, kSweepBlocksPerSM) k_amg_l0(BlockCSR A, const VT* __restrict__ vals, const VT* __restrict__ dinv,
                                                const VT* __restrict__ b, const VT* __restrict__ x, VT* __restrict__ y,
                                                double w, const int* __restrict__ skip) {
    if (skip && *skip) return;
    constexpr int PER_WARP = 32 / LANES;
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
            const int c = A.bcol[s0 + j];
            const double x0 = x[3 * c], x1 = x[3 * c + 1], x2 = x[3 * c + 2];
            const VT* v0 = vals + rs + 3 * j;
            y0 += (double)v0[0] * x0 + (double)v0[1] * x1 + (double)v0[2] * x2;
            const VT* v1 = v0 + len;
            y1 += (double)v1[0] * x0 + (double)v1[1] * x1 + (double)v1[2] * x2;
            const VT* v2 = v1 + len;
            y2 += (double)v2[0] * x0 + (double)v2[1] * x1 + (double)v2[2] * x2;
        }
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1) {
            y0 += __shfl_xor_sync(0xffffffffu, y0, o);
            y1 += __shfl_xor_sync(0xffffffffu, y1, o);
            y2 += __shfl_xor_sync(0xffffffffu, y2, o);
        }
        if (g8 == 0 && valid) {
            const double r0 = (double)b[3 * a] - y0, r1 = (double)b[3 * a + 1] - y1, r2 = (double)b[3 * a + 2] - y2;
            if (MODE == 0) {
                y[3 * a] = (VT)r0; y[3 * a + 1] = (VT)r1; y[3 * a + 2] = (VT)r2;
            } else {
                const VT* D = dinv + 9 * (size_t)a;
                y[3 * a] = (VT)((double)x[3 * a] + w * ((double)D[0] * r0 + (double)D[1] * r1 + (double)D[2] * r2));
                y[3 * a + 1] = (VT)((double)x[3 * a + 1] + w * ((double)D[3] * r0 + (double)D[4] * r1 + (double)D[5] * r2));
                y[3 * a + 2] = (VT)((double)x[3 * a + 2] + w * ((double)D[6] * r0 + (double)D[7] * r1 + (double)D[8] * r2));
            }
        }
    }
}

static int l0_grid(int nnodes, int lanes) { return grid_resident((long)nnodes * lanes, kSweepBlocksPerSM); }
// lanes per node of the level-0 kernels, measured on the 4M beach (B200, 2M nodes, ~7 neighbours)
// with a grid of 8 blocks per SM: FP32 values 2 lanes (0.198 ms per sweep) vs 4 (0.226) vs 8
// (0.265); FP64 4 lanes (0.304 ms) vs 8 (0.315).  Fewer lanes per node keep more independent
// loads in flight per lane, which the latency-bound neighbour gathers need.  With the one-wave
// grid (6 blocks per SM) the FP32 sweep takes 0.181 ms.
template <class VT> struct L0Lanes { static constexpr int value = 4; };
template <> struct L0Lanes<float> { static constexpr int value = 2; };

// Coarse levels (block CSR, 9 values per block), same modes, 8 lanes per row.
template <class VT, int MODE>
__global__ void __launch_bounds__(256, kSweepBlocksPerSM) k_amg_bsr(int n, const int* __restrict__ bptr, const int* __restrict__ bcol,
                                                 const VT* __restrict__ val, const VT* __restrict__ dinv,
                                                 const VT* __restrict__ b, const VT* __restrict__ x, VT* __restrict__ y,
                                                 double w, const int* __restrict__ skip) {
    if (skip && *skip) return;
    constexpr int LANES = sizeof(VT) == 4 ? 4 : 8, PER_WARP = 32 / LANES;   // coarse rows hold ~10 blocks
    const int g8 = threadIdx.x & (LANES - 1), sub = (threadIdx.x & 31) / LANES;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * PER_WARP; base < n; base += nw * PER_WARP) {
        const int a = base + sub;
        const bool valid = a < n;
        double y0 = 0, y1 = 0, y2 = 0;
        const int q0 = valid ? bptr[a] : 0, q1 = valid ? bptr[a + 1] : 0;
#pragma unroll 2
        for (int q = q0 + g8; q < q1; q += LANES) {
            const int c = bcol[q];
            const double x0 = x[3 * c], x1 = x[3 * c + 1], x2 = x[3 * c + 2];
            const VT* v = val + 9 * (size_t)q;
            y0 += (double)v[0] * x0 + (double)v[1] * x1 + (double)v[2] * x2;
            y1 += (double)v[3] * x0 + (double)v[4] * x1 + (double)v[5] * x2;
            y2 += (double)v[6] * x0 + (double)v[7] * x1 + (double)v[8] * x2;
        }
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1) {
            y0 += __shfl_xor_sync(0xffffffffu, y0, o);
            y1 += __shfl_xor_sync(0xffffffffu, y1, o);
            y2 += __shfl_xor_sync(0xffffffffu, y2, o);
        }
        if (g8 == 0 && valid) {
            const double r0 = (double)b[3 * a] - y0, r1 = (double)b[3 * a + 1] - y1, r2 = (double)b[3 * a + 2] - y2;
            if (MODE == 0) {
                y[3 * a] = (VT)r0; y[3 * a + 1] = (VT)r1; y[3 * a + 2] = (VT)r2;
            } else {
                const VT* D = dinv + 9 * (size_t)a;
                y[3 * a] = (VT)((double)x[3 * a] + w * ((double)D[0] * r0 + (double)D[1] * r1 + (double)D[2] * r2));
                y[3 * a + 1] = (VT)((double)x[3 * a + 1] + w * ((double)D[3] * r0 + (double)D[4] * r1 + (double)D[5] * r2));
                y[3 * a + 2] = (VT)((double)x[3 * a + 2] + w * ((double)D[6] * r0 + (double)D[7] * r1 + (double)D[8] * r2));
            }
        }
    }
}

// bc[I] = sum of r over the members of aggregate I (fixed member order)
template <class VT>
__global__ void k_amg_restrict(int nc, const int* __restrict__ mptr, const int* __restrict__ mem, const VT* __restrict__ r,
                               VT* __restrict__ bc, const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= nc) return;
    double s0 = 0, s1 = 0, s2 = 0;
    for (int t = mptr[I]; t < mptr[I + 1]; t++) {
        const int i = mem[t];
        s0 += (double)r[3 * i]; s1 += (double)r[3 * i + 1]; s2 += (double)r[3 * i + 2];
    }
    bc[3 * I] = (VT)s0; bc[3 * I + 1] = (VT)s1; bc[3 * I + 2] = (VT)s2;
}

// x += P xc (piecewise constant per variable)
template <class VT>
__global__ void k_amg_prolong(int n3, const int* __restrict__ agg, const VT* __restrict__ xc, VT* __restrict__ x,
                              const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n3) return;
    const int i = d / 3, v = d - 3 * i;
    x[d] = (VT)((double)x[d] + (double)xc[3 * agg[i] + v]);
}

// coarsest level: `sweeps` damped block-Jacobi sweeps from zero inside one CTA
template <class VT>
__global__ void __launch_bounds__(1024) k_amg_coarsest(int n, const int* __restrict__ bptr, const int* __restrict__ bcol,
                                                       const VT* __restrict__ val, const VT* __restrict__ dinv,
                                                       const VT* __restrict__ b, VT* __restrict__ x, VT* __restrict__ t,
                                                       double w, int sweeps, const int* __restrict__ skip) {
    if (skip && *skip) return;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const VT* D = dinv + 9 * (size_t)i;
        const double b0 = b[3 * i], b1 = b[3 * i + 1], b2 = b[3 * i + 2];
        x[3 * i] = (VT)(w * ((double)D[0] * b0 + (double)D[1] * b1 + (double)D[2] * b2));
        x[3 * i + 1] = (VT)(w * ((double)D[3] * b0 + (double)D[4] * b1 + (double)D[5] * b2));
        x[3 * i + 2] = (VT)(w * ((double)D[6] * b0 + (double)D[7] * b1 + (double)D[8] * b2));
    }
    __syncthreads();
    for (int s = 1; s < sweeps; s++) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double r0 = b[3 * i], r1 = b[3 * i + 1], r2 = b[3 * i + 2];
            for (int q = bptr[i]; q < bptr[i + 1]; q++) {
                const int c = bcol[q];
                const double x0 = x[3 * c], x1 = x[3 * c + 1], x2 = x[3 * c + 2];
                const VT* v = val + 9 * (size_t)q;
                r0 -= (double)v[0] * x0 + (double)v[1] * x1 + (double)v[2] * x2;
                r1 -= (double)v[3] * x0 + (double)v[4] * x1 + (double)v[5] * x2;
                r2 -= (double)v[6] * x0 + (double)v[7] * x1 + (double)v[8] * x2;
            }
            const VT* D = dinv + 9 * (size_t)i;
            t[3 * i] = (VT)((double)x[3 * i] + w * ((double)D[0] * r0 + (double)D[1] * r1 + (double)D[2] * r2));
            t[3 * i + 1] = (VT)((double)x[3 * i + 1] + w * ((double)D[3] * r0 + (double)D[4] * r1 + (double)D[5] * r2));
            t[3 * i + 2] = (VT)((double)x[3 * i + 2] + w * ((double)D[6] * r0 + (double)D[7] * r1 + (double)D[8] * r2));
        }
        __syncthreads();
        for (int d = threadIdx.x; d < 3 * n; d += blockDim.x) x[d] = t[d];
        __syncthreads();
    }
}

template <class VT>
__global__ void k_amg_copy(int n, const VT* __restrict__ a, VT* __restrict__ b, const int* __restrict__ skip) {
    if (skip && *skip) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

// ---------------------------------------------------------------- chunk corrections (level 0)
// One CTA per chunk (grid-stride): the chunk's dense block of the scaled level-0 matrix
// (its nodes' rows and columns; couplings to nodes outside the chunk are left out) is
// inverted by Gauss-Jordan elimination with partial pivoting in shared memory, and the
// rows of the chunk's own dofs (own nodes come first) are written in FP64 and FP32.  A
// zero pivot leaves the chunk's rows at zero (no correction) and is counted.
constexpr int kPatchMaxDof = 3 * kPatchMaxNodes;
__global__ void __launch_bounds__(256) k_patch_invert(BlockCSR A, PatchDev P, const double* __restrict__ vals,
                                                      int nchunks) {
    extern __shared__ double sm[];                 // [m * m], m = 3 * chunk nodes
    __shared__ int nodes[kPatchMaxNodes];
    __shared__ int piv[kPatchMaxDof];
    __shared__ double colk[kPatchMaxDof];
    __shared__ int s_p, s_bad;
    __shared__ double s_pinv;
    for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const int p0 = P.chunk_ptr[c], ne = P.chunk_ptr[c + 1] - p0, own = P.own_cnt[c];
        const int m = 3 * ne;
        for (int t = threadIdx.x; t < ne; t += blockDim.x) nodes[t] = P.ext_node[p0 + t];
        for (int t = threadIdx.x; t < m * m; t += blockDim.x) sm[t] = 0.0;
        if (threadIdx.x == 0) s_bad = 0;
        __syncthreads();
        for (int t = threadIdx.x; t < ne * 32; t += blockDim.x) {   // (chunk node, neighbour slot)
            const int ia = t >> 5, q = t & 31;
            const int a = nodes[ia];
            const int s0 = A.bptr[a], deg = A.bptr[a + 1] - s0;
            if (q >= deg) continue;
            const int b = A.bcol[s0 + q];
            int ib = -1;
            for (int k = 0; k < ne; k++)
                if (nodes[k] == b) { ib = k; break; }
            if (ib < 0) continue;
            const int rs = A.indptr[3 * a], len = A.indptr[3 * a + 1] - rs;
#pragma unroll
            for (int v = 0; v < 3; v++)
#pragma unroll
                for (int w = 0; w < 3; w++) sm[(3 * ia + v) * m + 3 * ib + w] = vals[rs + v * len + 3 * q + w];
        }
        __syncthreads();
        for (int k = 0; k < m; k++) {
            if (threadIdx.x < 32) {                    // pivot: largest |a_ik|, i >= k (lowest index on ties)
                double best = -1.0;
                int bi = k;
                for (int i = k + threadIdx.x; i < m; i += 32) {
                    const double v = fabs(sm[i * m + k]);
                    if (v > best) { best = v; bi = i; }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double ov = __shfl_xor_sync(0xffffffffu, best, o);
                    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                    if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
                }
                if (threadIdx.x == 0) {
                    s_p = bi; piv[k] = bi;
                    if (!(best > 1e-300) || !isfinite(best)) s_bad = 1;
                }
            }
            __syncthreads();
            if (s_bad) break;
            const int p = s_p;
            if (p != k)
                for (int j = threadIdx.x; j < m; j += blockDim.x) {
                    const double t0 = sm[k * m + j];
                    sm[k * m + j] = sm[p * m + j];
                    sm[p * m + j] = t0;
                }
            __syncthreads();
            if (threadIdx.x == 0) s_pinv = 1.0 / sm[k * m + k];
            __syncthreads();
            const double pinv = s_pinv;
            for (int j = threadIdx.x; j < m; j += blockDim.x) sm[k * m + j] = (j == k) ? pinv : sm[k * m + j] * pinv;
            for (int i = threadIdx.x; i < m; i += blockDim.x) colk[i] = sm[i * m + k];
            __syncthreads();
            for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
                const int i = t / m, j = t - i * m;
                if (i == k) continue;
                sm[t] = (j == k) ? -colk[i] * pinv : sm[t] - colk[i] * sm[k * m + j];
            }
            __syncthreads();
        }
        const int ro = 3 * own;
        double* R = P.r64 + P.rofs[c];
        float* R32 = P.r32 + P.rofs[c];
        if (s_bad) {
            for (int t = threadIdx.x; t < ro * m; t += blockDim.x) { R[t] = 0.0; R32[t] = 0.0f; }
            if (threadIdx.x == 0) atomicAdd(P.failed, 1);
            __syncthreads();
            continue;
        }
        for (int k = m - 1; k >= 0; k--) {           // undo the row interchanges on the columns
            const int p = piv[k];
            if (p != k)
                for (int i = threadIdx.x; i < m; i += blockDim.x) {
                    const double t0 = sm[i * m + k];
                    sm[i * m + k] = sm[i * m + p];
                    sm[i * m + p] = t0;
                }
            __syncthreads();
        }
        for (int t = threadIdx.x; t < ro * m; t += blockDim.x) { R[t] = sm[t]; R32[t] = (float)sm[t]; }
        __syncthreads();
    }
}

// e = b - A x at every chunk node (entries of all chunks; a node in several chunks is
// evaluated once per chunk)
template <class VT>
__global__ void __launch_bounds__(256) k_patch_resid(BlockCSR A, const VT* __restrict__ vals, const VT* __restrict__ b,
                                                     const VT* __restrict__ x, PatchDev P, VT* __restrict__ e,
                                                     const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int ne = P.counts[1];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ne; t += gridDim.x * blockDim.x) {
        const int a = P.ext_node[t];
        const int rs = A.indptr[3 * a], len = A.indptr[3 * a + 1] - rs;
        const int s0 = A.bptr[a], deg = A.bptr[a + 1] - s0;
        double y0 = 0, y1 = 0, y2 = 0;
        for (int j = 0; j < deg; j++) {
            const int c = A.bcol[s0 + j];
            const double x0 = x[3 * c], x1 = x[3 * c + 1], x2 = x[3 * c + 2];
            const VT* v0 = vals + rs + 3 * j;
            y0 += (double)v0[0] * x0 + (double)v0[1] * x1 + (double)v0[2] * x2;
            const VT* v1 = v0 + len;
            y1 += (double)v1[0] * x0 + (double)v1[1] * x1 + (double)v1[2] * x2;
            const VT* v2 = v1 + len;
            y2 += (double)v2[0] * x0 + (double)v2[1] * x1 + (double)v2[2] * x2;
        }
        e[3 * t] = (VT)((double)b[3 * a] - y0);
        e[3 * t + 1] = (VT)((double)b[3 * a + 1] - y1);
        e[3 * t + 2] = (VT)((double)b[3 * a + 2] - y2);
    }
}

template <class VT> struct PatchBuf;
template <> struct PatchBuf<double> {
    static const double* r(const PatchDev& P) { return P.r64; }
    static double* e(const PatchDev& P) { return P.e64; }
};
template <> struct PatchBuf<float> {
    static const float* r(const PatchDev& P) { return P.r32; }
    static float* e(const PatchDev& P) { return P.e32; }
};

// x[own dofs of chunk c] += R_c e_c; the own nodes of different chunks are disjoint
template <class VT>
__global__ void __launch_bounds__(256) k_patch_apply(PatchDev P, const VT* __restrict__ R, const VT* __restrict__ e,
                                                     VT* __restrict__ x, const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int nch = P.counts[0];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int c = blockIdx.x; c < nch; c += gridDim.x) {
        const int p0 = P.chunk_ptr[c], m = 3 * (P.chunk_ptr[c + 1] - p0), ro = 3 * P.own_cnt[c];
        const VT* Rc = R + P.rofs[c];
        const VT* ec = e + 3 * (size_t)p0;
        for (int i = warp; i < ro; i += nw) {
            double acc = 0.0;
            for (int j = lane; j < m; j += 32) acc += (double)Rc[(size_t)i * m + j] * (double)ec[j];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) {
                const int node = P.ext_node[p0 + i / 3];
                const int d = 3 * node + i % 3;
                x[d] = (VT)((double)x[d] + acc);
            }
        }
    }
}

void patch_invert(const BlockCSR& A, const PatchDev& P, const double* vals, int nchunks, cudaStream_t st) {
    if (nchunks <= 0) return;
    static bool attr = false;
    const int smem = kPatchMaxDof * kPatchMaxDof * (int)sizeof(double);
    if (!attr) {
        cudaFuncSetAttribute(k_patch_invert, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        attr = true;
    }
    k_patch_invert<<<P.grid, 256, smem, st>>>(A, P, vals, nchunks);
}

// ---------------------------------------------------------------- host side
void amg_setup(const BlockCSR& A, const AmgHost& H, const AssemblyMaps& maps, const double* vals, cudaStream_t st) {
    k_amg_dinv0<<<nb(A.nnodes, 128), 128, 0, st>>>(A, vals, H.dinv0_64, H.patch.flag);
    for (int l = 1; l < H.nlev; l++) {
        const AmgLevel& C = H.lev[l];
        const AmgLink& K = H.link[l - 1];
        if (l == 1)
            k_galerkin0<<<nb(C.nb, 128), 128, 0, st>>>(C.nb, K.gptr, K.gsrc, maps.boff, maps.blen, vals, C.val64);
        else
            k_galerkin<<<nb(C.nb, 128), 128, 0, st>>>(C.nb, K.gptr, K.gsrc, H.lev[l - 1].val64, C.val64);
        k_bsr_dinv<<<nb(C.n, 128), 128, 0, st>>>(C.n, C.bptr, C.dpos, C.val64, C.dinv64);
    }
    k_cast32<<<1184, 256, 0, st>>>(9L * A.nnodes, H.dinv0_64, H.dinv0_32);
    for (int l = 1; l < H.nlev; l++) {   // FP32 copies for the FP32 Krylov path
        const AmgLevel& C = H.lev[l];
        k_cast32<<<1184, 256, 0, st>>>(9L * C.nb, C.val64, C.val32);
        k_cast32<<<1184, 256, 0, st>>>(9L * C.n, C.dinv64, C.dinv32);
    }
}

template <class VT>
static void smooth_or_resid(const BlockCSR& A, const AmgLevel& L, int l, const VT* vals0, const VT* dinv, const VT* b,
                            const VT* x, VT* y, bool resid, const int* skip, cudaStream_t st) {
    if (l == 0) {
        constexpr int LN = L0Lanes<VT>::value;
        if (resid) k_amg_l0<VT, 0, LN><<<l0_grid(A.nnodes, LN), 256, 0, st>>>(A, vals0, dinv, b, x, y, 0.0, skip);
        else k_amg_l0<VT, 1, LN><<<l0_grid(A.nnodes, LN), 256, 0, st>>>(A, vals0, dinv, b, x, y, kAmgOmega, skip);
    } else {
        const VT* val = AmgBuf<VT>::val(L);
        const int gb = grid_resident((long)L.n * (sizeof(VT) == 4 ? 4 : 8), kSweepBlocksPerSM);   // k_amg_bsr's lanes
        if (resid) k_amg_bsr<VT, 0><<<gb, 256, 0, st>>>(L.n, L.bptr, L.bcol, val, dinv, b, x, y, 0.0, skip);
        else k_amg_bsr<VT, 1><<<gb, 256, 0, st>>>(L.n, L.bptr, L.bcol, val, dinv, b, x, y, kAmgOmega, skip);
    }
}

// one V-cycle at level l: x <- V(b); level 0 uses the CSR values passed in
template <class VT>
void amg_patch_correct(const BlockCSR& A, const AmgHost& H, const VT* vals0, const VT* b, VT* y, const int* skip,
                       cudaStream_t st);
template <class VT>
static void vcycle(const BlockCSR& A, const AmgHost& H, int l, const VT* vals0, const VT* b, VT* x, const int* skip,
                   cudaStream_t st) {
    const AmgLevel& L = H.lev[l];
    const int n = (l == 0) ? A.nnodes : L.n;
    const VT* dinv = (l == 0) ? AmgBuf<VT>::dinv0(H) : AmgBuf<VT>::dinv(L);
    VT* t = AmgBuf<VT>::t(L);
    VT* r = AmgBuf<VT>::r(L);
    if (l == H.nlev - 1) {
        k_amg_coarsest<VT><<<1, 1024, 0, st>>>(n, L.bptr, L.bcol, AmgBuf<VT>::val(L), dinv, b, x, t, kAmgOmega,
                                               kAmgCoarseSweeps, skip);
        return;
    }
    // pre-smoothing: the sweeps alternate between t and x so that the last lands in x
    VT* cur = (kAmgNu % 2 == 1) ? x : t;
    k_amg_scale<VT><<<nb(n, 256), 256, 0, st>>>(n, dinv, b, cur, kAmgOmega, skip);
    for (int s = 1; s < kAmgNu; s++) {
        VT* nxt = (cur == x) ? t : x;
        smooth_or_resid<VT>(A, L, l, vals0, dinv, b, cur, nxt, false, skip, st);
        cur = nxt;
    }
    if (l == 0 && H.patch.mode == 2) amg_patch_correct<VT>(A, H, vals0, b, cur, skip, st);
    // coarse correction
    const AmgLevel& C = H.lev[l + 1];
    const AmgLink& K = H.link[l];
    smooth_or_resid<VT>(A, L, l, vals0, dinv, b, cur, r, true, skip, st);
    k_amg_restrict<VT><<<nb(C.n, 128), 128, 0, st>>>(C.n, K.mptr, K.mem, r, AmgBuf<VT>::b(C), skip);
    vcycle<VT>(A, H, l + 1, vals0, AmgBuf<VT>::b(C), AmgBuf<VT>::x(C), skip, st);
    k_amg_prolong<VT><<<nb(3L * n, 256), 256, 0, st>>>(3 * n, K.agg, AmgBuf<VT>::x(C), cur, skip);
    // post-smoothing
    for (int s = 0; s < kAmgNu; s++) {
        VT* nxt = (cur == x) ? t : x;
        smooth_or_resid<VT>(A, L, l, vals0, dinv, b, cur, nxt, false, skip, st);
        cur = nxt;
    }
    if (l == 0 && H.patch.mode == 2) amg_patch_correct<VT>(A, H, vals0, b, cur, skip, st);
    if (cur != x) k_amg_copy<VT><<<nb(3L * n, 256), 256, 0, st>>>(3 * n, cur, x, skip);
}

void amg_smooth0_once(const BlockCSR& A, const AmgHost& H, const double* vals, const double* b, const double* x, double* y,
                      cudaStream_t st) {
    constexpr int LN = L0Lanes<double>::value;
    k_amg_l0<double, 1, LN><<<l0_grid(A.nnodes, LN), 256, 0, st>>>(A, vals, H.dinv0_64, b, x, y, kAmgOmega, nullptr);
}

void amg_smooth0_once32(const BlockCSR& A, const AmgHost& H, const float* vals, const float* b, const float* x, float* y,
                        cudaStream_t st) {
    constexpr int LN = L0Lanes<float>::value;
    k_amg_l0<float, 1, LN><<<l0_grid(A.nnodes, LN), 256, 0, st>>>(A, vals, H.dinv0_32, b, x, y, kAmgOmega, nullptr);
}

template <class VT>
void amg_patch_correct(const BlockCSR& A, const AmgHost& H, const VT* vals0, const VT* b, VT* y, const int* skip,
                       cudaStream_t st);
template <class VT>
void amg_apply(const BlockCSR& A, const AmgHost& H, const VT* vals0, VT* y, const int* skip, cudaStream_t st) {
    VT* b0 = AmgBuf<VT>::b(H.lev[0]);
    k_amg_copy<VT><<<1184, 256, 0, st>>>(3 * A.nnodes, y, b0, skip);
    vcycle<VT>(A, H, 0, vals0, b0, y, skip, st);
    if (H.patch.mode == 1) amg_patch_correct<VT>(A, H, vals0, b0, y, skip, st);
}

template <class VT>
void amg_patch_correct(const BlockCSR& A, const AmgHost& H, const VT* vals0, const VT* b, VT* y, const int* skip,
                       cudaStream_t st) {
    if (!H.patch.flag) return;   // chunk corrections on the flagged nodes (counts read on the device)
    const PatchDev& P = H.patch;
    k_patch_resid<VT><<<P.grid, 256, 0, st>>>(A, vals0, b, y, P, PatchBuf<VT>::e(P), skip);
    k_patch_apply<VT><<<P.grid, 256, 0, st>>>(P, PatchBuf<VT>::r(P), PatchBuf<VT>::e(P), y, skip);
}
template void amg_patch_correct<double>(const BlockCSR&, const AmgHost&, const double*, const double*, double*,
                                        const int*, cudaStream_t);
template void amg_patch_correct<float>(const BlockCSR&, const AmgHost&, const float*, const float*, float*,
                                       const int*, cudaStream_t);
template void amg_apply<double>(const BlockCSR&, const AmgHost&, const double*, double*, const int*, cudaStream_t);
template void amg_apply<float>(const BlockCSR&, const AmgHost&, const float*, float*, const int*, cudaStream_t);

}  // namespace sw2
