// One cycle of right-preconditioned GMRES(m) on the scaled SW2 system, entirely
// on the device so that a cycle is one CUDA graph replay.
//
// Why next to the reference's BiCGStab: with an approximate multilevel
// preconditioner the preconditioned SW2 operator at large Courant numbers is far
// from normal, and BiCGStab's residual then swings by orders of magnitude (in
// FP32 it does not recover).  GMRES minimises the residual over the Krylov space,
// so it decreases monotonically; restarted from the true FP64 residual after each
// cycle it serves both the FP64 solve and the FP32 inner solve of the iterative
// refinement.
//
// A cycle from x = 0 on right-hand side r, minimising ||W (r - A M^-1 V y)||_2 for
// the row weights W = diag(rw):
//   beta = ||W r||_2, v_0 = W r / beta, g = beta e_0
//   for j < m:  w = W A M^-1 v_j ; h_{:,j} = V_j^T w (one multi-dot pass) ;
//               w -= V_j h_{:,j} ; h_{j+1,j} = ||w|| ; v_{j+1} = w / h_{j+1,j} ;
//               Givens rotation of column j ; stop when |g_{j+1}| <= rtol * beta
//   y = H^-1 g (k x k triangular), out = M^-1 (V_k y)
// Classical Gram-Schmidt keeps one pass over the basis per step; its dot products
// accumulate in FP64 whatever the basis precision.  The rotations and the
// triangular solve run in one thread (k <= kGmM).  Deterministic: fixed block
// order in every reduction, no atomics besides the last-block counter.
#include <cmath>
#include "sw2_launch.h"

namespace sw2 {

static int gm_grid(long n) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0; cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    long need = (n + 255) / 256, cap = 4L * sms;
    if (cap > kMaxBlocks) cap = kMaxBlocks;
    return (int)(need < cap ? (need < 1 ? 1 : need) : cap);
}

// last block of the grid (thread 0) after every block published its partials
__device__ __forceinline__ bool gm_last_block(const GmresDev& G) {
    __shared__ bool is_last;
    __threadfence();   // every thread's partial writes are visible device-wide before the count
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int total = gridDim.x * gridDim.y;
        unsigned int t = atomicInc(G.counter, total - 1);
        is_last = (t == total - 1);
    }
    __syncthreads();
    return is_last;
}

// 16-byte loads and stores of basis entries (4 floats or 2 doubles); the basis stride is a
// multiple of 4 entries, so every vector starts on a 16-byte boundary.
template <class VT> struct Quad { static constexpr int N = 16 / sizeof(VT); };
__device__ __forceinline__ void ld16(const float* p, float (&o)[4]) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
}
__device__ __forceinline__ void ld16(const double* p, double (&o)[2]) {
    const double2 t = __ldg(reinterpret_cast<const double2*>(p));
    o[0] = t.x; o[1] = t.y;
}
__device__ __forceinline__ void ld16_rw(const float* p, float (&o)[4]) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
}
__device__ __forceinline__ void ld16_rw(const double* p, double (&o)[2]) {
    const double2 t = *reinterpret_cast<const double2*>(p);
    o[0] = t.x; o[1] = t.y;
}
__device__ __forceinline__ void st16(float* p, const float (&o)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
}
__device__ __forceinline__ void st16(double* p, const double (&o)[2]) {
    *reinterpret_cast<double2*>(p) = make_double2(o[0], o[1]);
}

// In the last block, the sum of column col of the blocks' partials by all its threads
// (each thread a fixed stride of blocks, then the warp and block trees): the result in
// thread 0.  Every thread of the block calls it.
__device__ __forceinline__ double gm_sum_partials(const GmresDev& G, int col) {
    __shared__ double red[8];
    double t = 0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t += __ldcg(G.partial + b * (kGmM + 1) + col);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    double s = 0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += red[k];
    return s;
}

// beta = ||r||_2 ; g = beta e_0 ; target = rtol * beta ; columns = 0
template <class VT>
__global__ void __launch_bounds__(256) k_gm_start(int n, const VT* __restrict__ r, const double* __restrict__ rw,
                                                  GmresDev G) {
    __shared__ double sh[8];
    double ss = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = (double)r[i] * rw[i];
        ss += v * v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = ss;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int k = 0; k < 8; k++) t += sh[k];
        G.partial[blockIdx.x * (kGmM + 1)] = t;
    }
    if (!gm_last_block(G)) return;
    const double tsum = gm_sum_partials(G, 0);
    if (threadIdx.x == 0) {
        const double beta = sqrt(tsum);
        G.scal[0] = beta;
        G.scal[1] = G.scal[3] * beta;       // stopping target on |g_{j+1}|
        G.scal[2] = beta;
        for (int k = 0; k <= kGmM; k++) G.g[k] = 0.0;
        G.g[0] = beta;
        G.state[1] = 0;
        G.state[2] = isfinite(beta) ? 0 : 2;
        G.state[0] = (beta > 0.0 && isfinite(beta)) ? 0 : 1;
    }
}

template <class VT>
__global__ void k_gm_v0(int n, const VT* __restrict__ r, const double* __restrict__ rw, VT* __restrict__ v0, GmresDev G) {
    if (G.state[0]) return;
    const double inv = 1.0 / G.scal[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        v0[i] = (VT)((double)r[i] * rw[i] * inv);
}

// w <- rw o w (row weights of the minimised residual norm)
template <class VT>
__global__ void k_gm_rowweight(int n, VT* __restrict__ w, const double* __restrict__ rw, GmresDev G) {
    if (G.state[0]) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) w[i] = (VT)((double)w[i] * rw[i]);
}

// h_k = v_k . w for k < nv (w = v_nv before orthogonalisation), into column j of H.
// blockIdx.y picks a group of kDotGroup basis vectors: each thread keeps kDotGroup
// accumulators (about 40 registers instead of one per basis vector), so 6 blocks fit on
// an SM and every load of the group is issued at once.  A thread's elements and the
// reduction tree do not depend on the group, so every h_k is the same sum as with all
// accumulators in one thread.  w is read once per group.
constexpr int kDotGroup = 8;
template <class VT>
__global__ void __launch_bounds__(256) k_gm_dots(int n, int nv, const VT* __restrict__ Vb, size_t ld, double* dst,
                                                 GmresDev G) {
    if (G.state[0]) return;
    __shared__ double sh[8][kDotGroup];
    const int k0 = blockIdx.y * kDotGroup;
    const VT* w = Vb + (size_t)nv * ld;
    double acc[kDotGroup];
#pragma unroll
    for (int k = 0; k < kDotGroup; k++) acc[k] = 0.0;
    constexpr int NQ = Quad<VT>::N;
    const int nq = n / NQ;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        const size_t i = (size_t)q * NQ;
        VT wq[NQ];
        ld16_rw(w + i, wq);
        VT x[kDotGroup][NQ];
#pragma unroll
        for (int k = 0; k < kDotGroup; k++)
            if (k0 + k < nv) ld16(Vb + (size_t)(k0 + k) * ld + i, x[k]);
#pragma unroll
        for (int k = 0; k < kDotGroup; k++)
            if (k0 + k < nv) {
#pragma unroll
                for (int c = 0; c < NQ; c++) acc[k] += (double)x[k][c] * (double)wq[c];
            }
    }
    for (int i = nq * NQ + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double wi = w[i];
#pragma unroll
        for (int k = 0; k < kDotGroup; k++)
            if (k0 + k < nv) acc[k] += (double)Vb[(size_t)(k0 + k) * ld + i] * wi;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kDotGroup; k++) {
        if (k0 + k < nv) {
            double v = acc[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) sh[warp][k] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x < kDotGroup && k0 + (int)threadIdx.x < nv) {
        double t = 0;
        for (int w8 = 0; w8 < 8; w8++) t += sh[w8][threadIdx.x];
        G.partial[blockIdx.x * (kGmM + 1) + k0 + threadIdx.x] = t;
    }
    if (gm_last_block(G)) {   // warp w sums columns w, w + 8, ...; its lanes stride over the blocks
        for (int c = warp; c < nv; c += (int)(blockDim.x >> 5)) {
            double t = 0;
            for (int b = lane; b < (int)gridDim.x; b += 32) t += __ldcg(G.partial + b * (kGmM + 1) + c);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0) dst[c] = t;
        }
    }
}

// First pass of classical Gram-Schmidt with re-orthogonalisation (CGS2): w -= sum_k h_k v_k, no norm.
template <class VT>
__global__ void __launch_bounds__(256) k_gm_sub(int n, int j, VT* __restrict__ Vb, size_t ld, GmresDev G) {
    if (G.state[0]) return;
    __shared__ double h[kGmM + 1];
    for (int k = threadIdx.x; k <= j; k += blockDim.x) h[k] = __ldcg(G.H + j * (kGmM + 1) + k);
    __syncthreads();
    VT* w = Vb + (size_t)(j + 1) * ld;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double v = w[i];
        int k = 0;
        for (; k + 8 <= j + 1; k += 8) {
            double x[8];
#pragma unroll
            for (int u = 0; u < 8; u++) x[u] = (double)Vb[(size_t)(k + u) * ld + i];
#pragma unroll
            for (int u = 0; u < 8; u++) v -= h[k + u] * x[u];
        }
        for (; k <= j; k++) v -= h[k] * (double)Vb[(size_t)k * ld + i];
        w[i] = (VT)v;
    }
}

// w -= sum_k h_k v_k ; h_{j+1,j} = ||w|| ; Givens rotation of column j ; convergence test.
// SECOND: the coefficients come from the re-orthogonalisation pass (G.H2) and are added to
// those of the first pass (column j of G.H) before the rotations.
template <class VT, bool SECOND>
__global__ void __launch_bounds__(256) k_gm_orth(int n, int j, VT* __restrict__ Vb, size_t ld, GmresDev G) {
    if (G.state[0]) return;
    __shared__ double sh[8];
    __shared__ double h[kGmM + 1];
    for (int k = threadIdx.x; k <= j; k += blockDim.x)
        h[k] = SECOND ? __ldcg(G.H2 + k) : __ldcg(G.H + j * (kGmM + 1) + k);
    __syncthreads();
    VT* w = Vb + (size_t)(j + 1) * ld;
    double ss = 0;
    constexpr int NQ = Quad<VT>::N;
    const int nq = n / NQ;
    // NQ consecutive entries per thread, eight 16-byte basis loads in flight, then the
    // updates of each entry in basis order (the same arithmetic per entry as one at a time)
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        const size_t i = (size_t)q * NQ;
        VT wq[NQ];
        ld16_rw(w + i, wq);
        double v[NQ];
#pragma unroll
        for (int c = 0; c < NQ; c++) v[c] = wq[c];
        int k = 0;
        for (; k + 8 <= j + 1; k += 8) {
            VT x[8][NQ];
#pragma unroll
            for (int u = 0; u < 8; u++) ld16(Vb + (size_t)(k + u) * ld + i, x[u]);
#pragma unroll
            for (int u = 0; u < 8; u++)
#pragma unroll
                for (int c = 0; c < NQ; c++) v[c] -= h[k + u] * (double)x[u][c];
        }
        for (; k <= j; k++) {
            VT x[NQ];
            ld16(Vb + (size_t)k * ld + i, x);
#pragma unroll
            for (int c = 0; c < NQ; c++) v[c] -= h[k] * (double)x[c];
        }
        VT o[NQ];
#pragma unroll
        for (int c = 0; c < NQ; c++) {
            o[c] = (VT)v[c];
            ss += (double)o[c] * (double)o[c];
        }
        st16(w + i, o);
    }
    for (int i = nq * NQ + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double v = w[i];
        for (int k = 0; k <= j; k++) v -= h[k] * (double)Vb[(size_t)k * ld + i];
        const VT vv = (VT)v;
        w[i] = vv;
        ss += (double)vv * (double)vv;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = ss;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int k = 0; k < 8; k++) t += sh[k];
        G.partial[blockIdx.x * (kGmM + 1)] = t;
    }
    if (!gm_last_block(G)) return;
    const double tsum = gm_sum_partials(G, 0);
    if (threadIdx.x == 0) {
        const double hn = sqrt(tsum);
        double* col = G.H + j * (kGmM + 1);
        if (SECOND)
            for (int k = 0; k <= j; k++) col[k] += G.H2[k];
        for (int k = 0; k < j; k++) {                 // earlier rotations
            const double a = col[k], b = col[k + 1];
            col[k] = G.cs[k] * a + G.sn[k] * b;
            col[k + 1] = -G.sn[k] * a + G.cs[k] * b;
        }
        const double a = col[j], b = hn;
        const double rr = hypot(a, b);
        const double c = rr > 0.0 ? a / rr : 1.0, s = rr > 0.0 ? b / rr : 0.0;
        G.cs[j] = c; G.sn[j] = s;
        col[j] = rr; col[j + 1] = 0.0;
        G.g[j + 1] = -s * G.g[j];
        G.g[j] = c * G.g[j];
        G.scal[4] = hn;
        G.scal[2] = fabs(G.g[j + 1]);
        G.state[1] = j + 1;
        if (!isfinite(rr) || !isfinite(hn)) { G.state[2] = 2; G.state[0] = 1; G.state[1] = j; }
        else if (rr == 0.0) { G.state[2] = 1; G.state[0] = 1; G.state[1] = j; }   // breakdown: drop column j
        else if (!(fabs(G.g[j + 1]) > G.scal[1]) || hn == 0.0) G.state[0] = 1;
    }
}

template <class VT>
__global__ void k_gm_scale(int n, int j, VT* __restrict__ Vb, size_t ld, GmresDev G) {
    if (G.state[0]) return;
    const double inv = 1.0 / G.scal[4];
    VT* w = Vb + (size_t)(j + 1) * ld;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) w[i] = (VT)((double)w[i] * inv);
}

// y = H^-1 g on the k columns built (upper triangular after the rotations)
__global__ void k_gm_solve(GmresDev G) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int k = G.state[1];
    for (int i = k - 1; i >= 0; i--) {
        double s = G.g[i];
        for (int t = i + 1; t < k; t++) s -= G.H[t * (kGmM + 1) + i] * G.y[t];
        const double d = G.H[i * (kGmM + 1) + i];
        G.y[i] = d != 0.0 ? s / d : 0.0;
    }
    G.state[0] = 0;   // let the final preconditioner apply run
}

// out = V_k y
template <class VT>
__global__ void k_gm_combine(int n, const VT* __restrict__ Vb, size_t ld, VT* __restrict__ out, GmresDev G) {
    __shared__ double y[kGmM];
    const int k = G.state[1];
    for (int t = threadIdx.x; t < k; t += blockDim.x) y[t] = G.y[t];
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0;
        for (int t = 0; t < k; t++) s += y[t] * (double)Vb[(size_t)t * ld + i];
        out[i] = (VT)s;
    }
}

template <class VT>
void gmres_cycle(const BlockCSR& A, const PrecondOp<VT>& P, const VT* vals, VT* Vb, size_t ld, VT* z, const VT* rhs,
                 VT* out, const double* rw, const GmresDev& G, cudaStream_t st, int m, bool reorth) {
    const int n = A.n, g = gm_grid(n);
    const int* done = G.state;
    k_gm_start<VT><<<g, 256, 0, st>>>(n, rhs, rw, G);
    k_gm_v0<VT><<<g, 256, 0, st>>>(n, rhs, rw, Vb, G);
    if (m < 1 || m > kGmM) m = kGmM;
    for (int j = 0; j < m; j++) {
        VT* vj = Vb + (size_t)j * ld;
        VT* w = Vb + (size_t)(j + 1) * ld;
        copy_skip<VT>(n, vj, z, done, st);
        precond_apply<VT>(A, P, z, done, st);
        spmv_skip<VT>(A, vals, z, w, done, st);
        k_gm_rowweight<VT><<<g, 256, 0, st>>>(n, w, rw, G);
        const dim3 dg(g, (j + 1 + kDotGroup - 1) / kDotGroup);
        k_gm_dots<VT><<<dg, 256, 0, st>>>(n, j + 1, Vb, ld, G.H + (size_t)j * (kGmM + 1), G);
        if (reorth) {
            k_gm_sub<VT><<<g, 256, 0, st>>>(n, j, Vb, ld, G);
            k_gm_dots<VT><<<dg, 256, 0, st>>>(n, j + 1, Vb, ld, G.H2, G);
            k_gm_orth<VT, true><<<g, 256, 0, st>>>(n, j, Vb, ld, G);
        } else {
            k_gm_orth<VT, false><<<g, 256, 0, st>>>(n, j, Vb, ld, G);
        }
        k_gm_scale<VT><<<g, 256, 0, st>>>(n, j, Vb, ld, G);
    }
    k_gm_solve<<<1, 32, 0, st>>>(G);
    k_gm_combine<VT><<<g, 256, 0, st>>>(n, Vb, ld, out, G);
    precond_apply<VT>(A, P, out, nullptr, st);
}
template void gmres_cycle<double>(const BlockCSR&, const PrecondOp<double>&, const double*, double*, size_t, double*,
                                  const double*, double*, const double*, const GmresDev&, cudaStream_t, int, bool);
template void gmres_cycle<float>(const BlockCSR&, const PrecondOp<float>&, const float*, float*, size_t, float*,
                                 const float*, float*, const double*, const GmresDev&, cudaStream_t, int, bool);

}  // namespace sw2
