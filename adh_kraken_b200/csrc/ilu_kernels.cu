// Multicolour 3x3 block ILU(0) preconditioner and the BiCGStab iteration that
// uses it.
//
// Why: the reference preconditions BiCGStab with a full UMFPACK LU
// (src/la/bcgstab_solver.c:371-420), so its Krylov solve converges at once.  On
// wet/dry meshes the 3x3 nodal block-Jacobi substitute stalls (thousands of
// iterations, then a wild iterate), while block ILU(0) over the node graph keeps
// the iteration count in the tens.  A natural-order ILU sweep is a long chain of
// dependent rows; a greedy colouring of the node graph (same-colour nodes never
// share an element) turns each sweep into one parallel kernel per colour.
//
// Storage: the factor overwrites a copy of the scaled CSR values in the same
// layout (L blocks in the slots of lower-coloured neighbours, U blocks in the
// others), plus the inverted diagonal block of every node.  Lower/upper is
// decided by colour: neighbour b is "lower" for node i iff colour(b) < colour(i).
#include <cmath>
#include "sw2_launch.h"

namespace sw2 {

#define ILU_MAXDEG 32   // neighbour slots per node handled by the factorisation (checked at set-up)

__device__ __forceinline__ void mm33(const double* a, const double* b, double* c) {
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int k = 0; k < 3; k++) c[3 * r + k] = a[3 * r] * b[k] + a[3 * r + 1] * b[3 + k] + a[3 * r + 2] * b[6 + k];
}

__device__ __forceinline__ void inv33(const double* a, double* inv) {
    double m[3][6];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) { m[r][c] = a[3 * r + c]; m[r][3 + c] = (r == c) ? 1.0 : 0.0; }
    bool ok = true;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        int p = c; double pv = fabs(m[c][c]);
#pragma unroll
        for (int r = c + 1; r < 3; r++) if (fabs(m[r][c]) > pv) { pv = fabs(m[r][c]); p = r; }
        if (!(pv > 0.0)) { ok = false; break; }
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
        for (int c = 0; c < 3; c++) inv[3 * r + c] = ok ? m[r][3 + c] : (r == c ? 1.0 : 0.0);
}

// block (node i, slot j) of a CSR-layout value array: rows rs + v*len, columns 3j..3j+2
__device__ __forceinline__ void ld_blk(const double* LU, int rs, int len, int j, double* b) {
#pragma unroll
    for (int v = 0; v < 3; v++)
#pragma unroll
        for (int w = 0; w < 3; w++) b[3 * v + w] = LU[rs + v * len + 3 * j + w];
}
__device__ __forceinline__ void st_blk(double* LU, int rs, int len, int j, const double* b) {
#pragma unroll
    for (int v = 0; v < 3; v++)
#pragma unroll
        for (int w = 0; w < 3; w++) LU[rs + v * len + 3 * j + w] = b[3 * v + w];
}

// IKJ block ILU(0) for the nodes of one colour.  Rows of lower colours are final.
__global__ void k_bilu_factor(BlockCSR A, IluView P, int cbeg, int cend, double* __restrict__ LU,
                              double* __restrict__ dinv) {
    const int t = cbeg + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cend) return;
    const int i = P.color_nodes[t];
    const int ci = P.node_color[i];
    const int rs = A.indptr[3 * i], len = A.indptr[3 * i + 1] - rs;
    const int s0 = A.bptr[i], deg = A.bptr[i + 1] - s0;
    // lower slots in elimination order (colour, then node id)
    int low[ILU_MAXDEG]; int nl = 0; int diag = 0;
    for (int j = 0; j < deg; j++) {
        const int b = A.bcol[s0 + j];
        if (b == i) diag = j;
        if (P.node_color[b] < ci) {
            const long key = (long)P.node_color[b] * (1L << 32) + b;
            int q = nl++;
            while (q > 0) {
                const int pb = A.bcol[s0 + low[q - 1]];
                const long pk = (long)P.node_color[pb] * (1L << 32) + pb;
                if (pk <= key) break;
                low[q] = low[q - 1]; q--;
            }
            low[q] = j;
        }
    }
    for (int q = 0; q < nl; q++) {
        const int jk = low[q];
        const int k = A.bcol[s0 + jk];
        double Bik[9], Dk[9], L[9];
        ld_blk(LU, rs, len, jk, Bik);
#pragma unroll
        for (int x = 0; x < 9; x++) Dk[x] = dinv[9 * k + x];
        mm33(Bik, Dk, L);
        st_blk(LU, rs, len, jk, L);
        const int ck = P.node_color[k];
        const int rk = A.indptr[3 * k], lenk = A.indptr[3 * k + 1] - rk;
        const int sk0 = A.bptr[k], degk = A.bptr[k + 1] - sk0;
        for (int qq = 0; qq < degk; qq++) {
            const int jj = A.bcol[sk0 + qq];
            if (P.node_color[jj] <= ck) continue;   // only the upper part of row k
            int ji = -1;
            for (int x = 0; x < deg; x++) if (A.bcol[s0 + x] == jj) { ji = x; break; }
            if (ji < 0) continue;                   // outside the ILU(0) pattern
            double Ukj[9], Bij[9], LU_[9];
            ld_blk(LU, rk, lenk, qq, Ukj);
            ld_blk(LU, rs, len, ji, Bij);
            mm33(L, Ukj, LU_);
#pragma unroll
            for (int x = 0; x < 9; x++) Bij[x] -= LU_[x];
            st_blk(LU, rs, len, ji, Bij);
        }
    }
    double Bii[9], Di[9];
    ld_blk(LU, rs, len, diag, Bii);
    inv33(Bii, Di);
#pragma unroll
    for (int x = 0; x < 9; x++) dinv[9 * i + x] = Di[x];
}

// forward sweep of one colour: y_i = z_i - sum_{lower b} L_ib y_b  (in place)
template <class VT>
__global__ void __launch_bounds__(256) k_bilu_fwd(BlockCSR A, IluView P, int cbeg, int cend, const VT* __restrict__ LU,
                                                  VT* __restrict__ y) {
    if (P.skip && *P.skip) return;
    const int g8 = threadIdx.x & 7, sub = (threadIdx.x & 31) >> 3;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int cnt = cend - cbeg;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 4; base < cnt; base += nw * 4) {
        const int t = base + sub;
        const bool valid = t < cnt;
        const int i = valid ? P.color_nodes[cbeg + t] : 0;
        const int ci = valid ? P.node_color[i] : 0;
        double a0 = 0, a1 = 0, a2 = 0;
        const int rs = valid ? A.indptr[3 * i] : 0, len = valid ? A.indptr[3 * i + 1] - rs : 0;
        const int s0 = valid ? A.bptr[i] : 0, deg = valid ? A.bptr[i + 1] - s0 : 0;
        for (int j = g8; j < deg; j += 8) {
            const int b = A.bcol[s0 + j];
            if (P.node_color[b] >= ci) continue;
            const double y0 = y[3 * b], y1 = y[3 * b + 1], y2 = y[3 * b + 2];
            const VT* v0 = LU + rs + 3 * j;
            a0 += (double)v0[0] * y0 + (double)v0[1] * y1 + (double)v0[2] * y2;
            const VT* v1 = v0 + len;
            a1 += (double)v1[0] * y0 + (double)v1[1] * y1 + (double)v1[2] * y2;
            const VT* v2 = v1 + len;
            a2 += (double)v2[0] * y0 + (double)v2[1] * y1 + (double)v2[2] * y2;
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
        if (g8 == 0 && valid) {
            y[3 * i] = (VT)((double)y[3 * i] - a0);
            y[3 * i + 1] = (VT)((double)y[3 * i + 1] - a1);
            y[3 * i + 2] = (VT)((double)y[3 * i + 2] - a2);
        }
    }
}

// backward sweep of one colour: x_i = D_i^-1 (y_i - sum_{upper b} U_ib x_b)  (in place)
template <class VT>
__global__ void __launch_bounds__(256) k_bilu_bwd(BlockCSR A, IluView P, int cbeg, int cend, const VT* __restrict__ LU,
                                                  const VT* __restrict__ dinv, VT* __restrict__ y) {
    if (P.skip && *P.skip) return;
    const int g8 = threadIdx.x & 7, sub = (threadIdx.x & 31) >> 3;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int cnt = cend - cbeg;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 4; base < cnt; base += nw * 4) {
        const int t = base + sub;
        const bool valid = t < cnt;
        const int i = valid ? P.color_nodes[cbeg + t] : 0;
        const int ci = valid ? P.node_color[i] : 0;
        double a0 = 0, a1 = 0, a2 = 0;
        const int rs = valid ? A.indptr[3 * i] : 0, len = valid ? A.indptr[3 * i + 1] - rs : 0;
        const int s0 = valid ? A.bptr[i] : 0, deg = valid ? A.bptr[i + 1] - s0 : 0;
        for (int j = g8; j < deg; j += 8) {
            const int b = A.bcol[s0 + j];
            if (P.node_color[b] <= ci) continue;
            const double y0 = y[3 * b], y1 = y[3 * b + 1], y2 = y[3 * b + 2];
            const VT* v0 = LU + rs + 3 * j;
            a0 += (double)v0[0] * y0 + (double)v0[1] * y1 + (double)v0[2] * y2;
            const VT* v1 = v0 + len;
            a1 += (double)v1[0] * y0 + (double)v1[1] * y1 + (double)v1[2] * y2;
            const VT* v2 = v1 + len;
            a2 += (double)v2[0] * y0 + (double)v2[1] * y1 + (double)v2[2] * y2;
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
        if (g8 == 0 && valid) {
            const double r0 = (double)y[3 * i] - a0, r1 = (double)y[3 * i + 1] - a1, r2 = (double)y[3 * i + 2] - a2;
            const VT* D = dinv + 9 * i;
            y[3 * i] = (VT)((double)D[0] * r0 + (double)D[1] * r1 + (double)D[2] * r2);
            y[3 * i + 1] = (VT)((double)D[3] * r0 + (double)D[4] * r1 + (double)D[5] * r2);
            y[3 * i + 2] = (VT)((double)D[6] * r0 + (double)D[7] * r1 + (double)D[8] * r2);
        }
    }
}

void launch_bilu_factor(const BlockCSR& A, const IluHost& H, const double* vals, double* lu, double* dinv,
                        cudaStream_t st) {
    cudaMemcpyAsync(lu, vals, sizeof(double) * (size_t)A.nnz, cudaMemcpyDeviceToDevice, st);
    for (int c = 0; c < H.ncolors; c++) {
        const int b = H.color_ptr[c], e = H.color_ptr[c + 1];
        if (e > b) k_bilu_factor<<<(e - b + 127) / 128, 128, 0, st>>>(A, H.view, b, e, lu, dinv);
    }
}

template <class VT>
void launch_bilu_apply(const BlockCSR& A, const IluHost& H, const VT* lu, const VT* dinv, VT* y, cudaStream_t st) {
    for (int c = 0; c < H.ncolors; c++) {
        const int b = H.color_ptr[c], e = H.color_ptr[c + 1];
        if (e > b) k_bilu_fwd<VT><<<grid_for_nodes(e - b), 256, 0, st>>>(A, H.view, b, e, lu, y);
    }
    for (int c = H.ncolors - 1; c >= 0; c--) {
        const int b = H.color_ptr[c], e = H.color_ptr[c + 1];
        if (e > b) k_bilu_bwd<VT><<<grid_for_nodes(e - b), 256, 0, st>>>(A, H.view, b, e, lu, dinv, y);
    }
}
template void launch_bilu_apply<double>(const BlockCSR&, const IluHost&, const double*, const double*, double*, cudaStream_t);
template void launch_bilu_apply<float>(const BlockCSR&, const IluHost&, const float*, const float*, float*, cudaStream_t);

}  // namespace sw2
