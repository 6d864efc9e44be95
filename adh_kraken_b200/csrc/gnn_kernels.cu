// Message-passing network over the mesh's node graph that predicts the next SW2
// time step (the Newton initial guess), with its training kernels.
//
// Per node i (H = 64 hidden features):
//   e0   = SiLU(W0 f_i + b0)                              f_i: 8 normalised inputs
//   for l = 1..3:
//     X_l = [e | mean_j e_j | sum_j wx_ij (e_j - e_i) | sum_j wy_ij (e_j - e_i)]   (4H)
//     e  <- e + SiLU(W_l X_l + b_l)
//   y    = S S (Wd e + bd)                                 3 outputs (normalised correction)
// where S is the neighbourhood mean (self included) that keeps the correction smooth.
// with wx_ij = (x_j - x_i) / (L deg_i) over the mesh edges (L = mean edge length):
// the mean and the two edge-weighted differences let a layer see values and
// first differences of its neighbourhood in both directions.
//
// Weights are stored in BF16 and converted to FP32 in shared memory; every sum
// accumulates in FP32.  The node graph is symmetric, so the backward pass of the
// aggregation is again a gather over each node's neighbours (the reverse slot of
// each edge is precomputed): no atomics, and training is deterministic.
// Weight gradients reduce per block into partial sums that a second kernel adds in
// block order.
//
// The dense layers run on CUDA cores: at 64 hidden features a layer is ~33 kFLOP
// per node against ~1.3 KB of gathered activations, so the pass is bound by the
// neighbour gathers, not by the arithmetic.
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace {

constexpr int H = 64;
constexpr int TILE = 64;        // nodes per block in the dense kernels
constexpr int MAXIN = 4 * H;

struct Graph {
    int n;
    const int* indptr;      // [n+1]
    const int* nbr;         // [nnz] neighbour node of each slot
    const int* rev;         // [nnz] slot of the reverse edge (in the neighbour's list)
    const float* wx;        // [nnz] (x_j - x_i) / (L deg_i)
    const float* wy;
    const float* inv_deg;   // [n]
    const float* swx;       // [n] sum_j wx_ij
    const float* swy;
};

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// X[i] = [E_i, mean E_j, sum wx (E_j - E_i), sum wy (E_j - E_i)]; one warp per node, 2 features per lane
__global__ void k_agg_fwd(Graph g, const float* __restrict__ E, float* __restrict__ X) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= g.n) return;
    const int i = warp;
    const float2 ei = reinterpret_cast<const float2*>(E + (size_t)i * H)[lane];
    float2 a = {0, 0}, gx = {0, 0}, gy = {0, 0};
    for (int s = g.indptr[i]; s < g.indptr[i + 1]; s++) {
        const int j = g.nbr[s];
        const float2 ej = reinterpret_cast<const float2*>(E + (size_t)j * H)[lane];
        const float wx = g.wx[s], wy = g.wy[s];
        a.x += ej.x; a.y += ej.y;
        gx.x += wx * (ej.x - ei.x); gx.y += wx * (ej.y - ei.y);
        gy.x += wy * (ej.x - ei.x); gy.y += wy * (ej.y - ei.y);
    }
    const float d = g.inv_deg[i];
    float2* xo = reinterpret_cast<float2*>(X + (size_t)i * MAXIN);
    xo[lane] = ei;
    xo[32 + lane] = make_float2(a.x * d, a.y * d);
    xo[64 + lane] = gx;
    xo[96 + lane] = gy;
}

// dE[j] += dX_e[j] + sum_{i in N(j)} (dA_i / deg_i + wx_ij dGx_i + wy_ij dGy_i) - swx_j dGx_j - swy_j dGy_j
__global__ void k_agg_bwd(Graph g, const float* __restrict__ dX, float* __restrict__ dE) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= g.n) return;
    const int j = warp;
    const float2* xj = reinterpret_cast<const float2*>(dX + (size_t)j * MAXIN);
    float2 acc = xj[lane];
    const float2 gxj = xj[64 + lane], gyj = xj[96 + lane];
    acc.x -= g.swx[j] * gxj.x + g.swy[j] * gyj.x;
    acc.y -= g.swx[j] * gxj.y + g.swy[j] * gyj.y;
    for (int s = g.indptr[j]; s < g.indptr[j + 1]; s++) {
        const int i = g.nbr[s], r = g.rev[s];        // slot r of node i points to j
        const float2* xi = reinterpret_cast<const float2*>(dX + (size_t)i * MAXIN);
        const float2 da = xi[32 + lane], dgx = xi[64 + lane], dgy = xi[96 + lane];
        const float di = g.inv_deg[i], wx = g.wx[r], wy = g.wy[r];
        acc.x += da.x * di + wx * dgx.x + wy * dgy.x;
        acc.y += da.y * di + wx * dgx.y + wy * dgy.y;
    }
    float2* o = reinterpret_cast<float2*>(dE + (size_t)j * H);
    float2 cur = o[lane];
    cur.x += acc.x; cur.y += acc.y;
    o[lane] = cur;
}

// Y = act(W X + b) (+ R): tile of TILE nodes per block, W [out][in] BF16 -> shared FP32 [in][out]
// 256 threads: thread t computes node t/4, outputs (t%4)*16 .. +16 (out <= 64)
__global__ void __launch_bounds__(256) k_dense_fwd(int n, int in, int out, const __nv_bfloat16* __restrict__ W,
                                                   const float* __restrict__ b, const float* __restrict__ X,
                                                   const float* __restrict__ R, int act, float* __restrict__ Z,
                                                   float* __restrict__ Y) {
    extern __shared__ float sm[];
    float* Ws = sm;                       // [in][64]
    const int ldx = in + 1;               // padded rows: the 8 nodes of a warp hit 8 banks
    float* Xs = sm + in * H;              // [TILE][ldx]
    const int base = blockIdx.x * TILE;
    for (int t = threadIdx.x; t < in * H; t += blockDim.x) {
        const int k = t / H, o = t % H;
        Ws[t] = o < out ? __bfloat162float(W[(size_t)o * in + k]) : 0.0f;
    }
    for (int t = threadIdx.x; t < TILE * in; t += blockDim.x) {
        const int r = t / in, k = t % in, node = base + r;
        Xs[r * ldx + k] = node < n ? X[(size_t)node * in + k] : 0.0f;
    }
    __syncthreads();
    const int r = threadIdx.x >> 2, o0 = (threadIdx.x & 3) * 16, node = base + r;
    float acc[16];
#pragma unroll
    for (int q = 0; q < 16; q++) acc[q] = 0.0f;
    const float* xr = Xs + r * ldx;
    for (int k = 0; k < in; k++) {
        const float xv = xr[k];
        const float4* w4 = reinterpret_cast<const float4*>(Ws + k * H + o0);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const float4 w = w4[q];
            acc[4 * q] += w.x * xv; acc[4 * q + 1] += w.y * xv; acc[4 * q + 2] += w.z * xv; acc[4 * q + 3] += w.w * xv;
        }
    }
    if (node >= n) return;
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int o = o0 + q;
        if (o >= out) break;
        const float z = acc[q] + b[o];
        if (Z) Z[(size_t)node * out + o] = z;
        float y = act ? silu(z) : z;
        if (R) y += R[(size_t)node * out + o];
        Y[(size_t)node * out + o] = y;
    }
}

// dZ = dY * act'(Z) (in place into dZ), then dX = W^T dZ (dX may be null)
// 256 threads, TILE nodes per block; thread t: node t/4, inputs (t%4) + 4q
__global__ void __launch_bounds__(256) k_dense_bwd_x(int n, int in, int out, const __nv_bfloat16* __restrict__ W,
                                                     const float* __restrict__ Z, const float* __restrict__ dY, int act,
                                                     float* __restrict__ dZ, float* __restrict__ dX) {
    extern __shared__ float sm[];
    float* Ws = sm;                       // [out][in]
    const int ldd = out + 1;
    float* Ds = sm + out * in;            // [TILE][ldd]
    const int base = blockIdx.x * TILE;
    for (int t = threadIdx.x; t < out * in; t += blockDim.x) Ws[t] = __bfloat162float(W[t]);
    for (int t = threadIdx.x; t < TILE * out; t += blockDim.x) {
        const int r = t / out, o = t % out, node = base + r;
        float d = 0.0f;
        if (node < n) {
            const size_t idx = (size_t)node * out + o;
            d = dY[idx];
            if (act) d *= dsilu(Z[idx]);
            dZ[idx] = d;
        }
        Ds[r * ldd + o] = d;
    }
    __syncthreads();
    if (!dX) return;
    const int r = threadIdx.x >> 2, node = base + r;
    if (node >= n) return;
    const float* dr = Ds + r * ldd;
    for (int k = threadIdx.x & 3; k < in; k += 4) {
        float s = 0.0f;
        for (int o = 0; o < out; o++) s += Ws[o * in + k] * dr[o];
        dX[(size_t)node * in + k] = s;
    }
}

// partial dW[o][k] and db[o] over a chunk of nodes per block: thread k (< in) keeps column k for all o
__global__ void __launch_bounds__(256) k_dense_bwd_w(int n, int in, int out, int nodes_per_block,
                                                     const float* __restrict__ X, const float* __restrict__ dZ,
                                                     float* __restrict__ part) {
    __shared__ float ds[H];
    const int k = threadIdx.x;
    float acc[H];
#pragma unroll
    for (int o = 0; o < H; o++) acc[o] = 0.0f;
    float bacc = 0.0f;
    const int n0 = blockIdx.x * nodes_per_block, n1 = min(n, n0 + nodes_per_block);
    for (int node = n0; node < n1; node++) {
        __syncthreads();
        if (threadIdx.x < out) ds[threadIdx.x] = dZ[(size_t)node * out + threadIdx.x];
        __syncthreads();
        const float xv = k < in ? X[(size_t)node * in + k] : 0.0f;
#pragma unroll
        for (int o = 0; o < H; o++)
            if (o < out) acc[o] += ds[o] * xv;
        if (k < out) bacc += ds[k];
    }
    float* p = part + (size_t)blockIdx.x * (out * in + out);
    if (k < in)
        for (int o = 0; o < out; o++) p[o * in + k] = acc[o];
    if (k < out) p[out * in + k] = bacc;
}

// g[c] = sum over blocks of part[blk][c] (fixed block order)
__global__ void k_reduce_parts(int nparts, int count, const float* __restrict__ part, float* __restrict__ g) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= count) return;
    float s = 0.0f;
    for (int p = 0; p < nparts; p++) s += part[(size_t)p * count + c];
    g[c] = s;
}

// Adam on the FP32 master weights, then their BF16 copy
__global__ void k_adam(int count, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, __nv_bfloat16* __restrict__ wb, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi; v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16(wi);
}

__global__ void k_to_bf16(int count, const float* __restrict__ w, __nv_bfloat16* __restrict__ wb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) wb[i] = __float2bfloat16(w[i]);
}

// Inputs f_i (8) from the FP64 state: [h, u, v, dh, du, dv, z, wet] normalised by (mu, sd)
__global__ void k_features(int n, const double* __restrict__ sol, const double* __restrict__ sol_prev,
                           const double* __restrict__ z, const float* __restrict__ mu, const float* __restrict__ sd,
                           float* __restrict__ F) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float f[8];
    for (int v = 0; v < 3; v++) {
        f[v] = (float)sol[3 * i + v];
        f[3 + v] = (float)(sol[3 * i + v] - sol_prev[3 * i + v]);
    }
    f[6] = (float)z[i];
    f[7] = sol[3 * i] > 0.0 ? 1.0f : 0.0f;
    for (int c = 0; c < 8; c++) F[(size_t)i * 8 + c] = (f[c] - mu[c]) / sd[c];
}

// targets: T = (sol_next - sol - (sol - sol_prev)) / scale  -- the correction to linear extrapolation;
// M = 1 where the guess will use the network (h > min_depth now and next), else 0
__global__ void k_targets(int n, const double* __restrict__ sol_next, const double* __restrict__ sol,
                          const double* __restrict__ sol_prev, const float* __restrict__ scale, double min_depth,
                          float* __restrict__ T, float* __restrict__ M) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int v = 0; v < 3; v++) {
        const int d = 3 * i + v;
        T[d] = (float)((sol_next[d] - 2.0 * sol[d] + sol_prev[d]) / (double)scale[v]);
    }
    M[i] = (sol[3 * i] > min_depth && sol_next[3 * i] > min_depth) ? 1.0f : 0.0f;
}

// 3-channel neighbourhood mean (self included): Ys_i = (Y_i + sum_j Y_j) / (deg_i + 1).  Smooths the
// network's correction so that its errors stay smooth: the SW2 residual differentiates the guess, and
// node-to-node noise in it costs more residual than the same error spread smoothly.
__global__ void k_smooth3(Graph g, const float* __restrict__ Y, float* __restrict__ Ys) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    float a = Y[3 * i], b = Y[3 * i + 1], c = Y[3 * i + 2];
    for (int s = g.indptr[i]; s < g.indptr[i + 1]; s++) {
        const int j = g.nbr[s];
        a += Y[3 * j]; b += Y[3 * j + 1]; c += Y[3 * j + 2];
    }
    const float w = 1.0f / (float)(g.indptr[i + 1] - g.indptr[i] + 1);
    Ys[3 * i] = a * w; Ys[3 * i + 1] = b * w; Ys[3 * i + 2] = c * w;
}
// adjoint: dY_j = dYs_j / (deg_j + 1) + sum_{i in N(j)} dYs_i / (deg_i + 1)
__global__ void k_smooth3_adj(Graph g, const float* __restrict__ dYs, float* __restrict__ dY) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= g.n) return;
    const float wj = 1.0f / (float)(g.indptr[j + 1] - g.indptr[j] + 1);
    float a = dYs[3 * j] * wj, b = dYs[3 * j + 1] * wj, c = dYs[3 * j + 2] * wj;
    for (int s = g.indptr[j]; s < g.indptr[j + 1]; s++) {
        const int i = g.nbr[s];
        const float wi = 1.0f / (float)(g.indptr[i + 1] - g.indptr[i] + 1);
        a += dYs[3 * i] * wi; b += dYs[3 * i + 1] * wi; c += dYs[3 * i + 2] * wi;
    }
    dY[3 * j] = a; dY[3 * j + 1] = b; dY[3 * j + 2] = c;
}

// loss partials and dY = 2 M (Y - T) / count over the node mask M (1: the node counts)
__global__ void __launch_bounds__(256) k_mse(int n3, const float* __restrict__ Y, const float* __restrict__ T,
                                             const float* __restrict__ M, float inv_count, float* __restrict__ dY,
                                             float* __restrict__ part) {
    __shared__ float sh[8];
    float s = 0.0f;
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n3; d += gridDim.x * blockDim.x) {
        const float e = (Y[d] - T[d]) * M[d / 3];
        s += e * e;
        dY[d] = 2.0f * e * inv_count;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < 8; w++) t += sh[w];
        part[blockIdx.x] = t * inv_count;
    }
}

// guess = sol + (sol - sol_prev) + scale * Y   (FP64 out), per node; a node that is
// shallow now or would be shallow in the guess (h <= min_depth) keeps sol: the
// guess must not move the wet/dry front, which the residual punishes hardest
__global__ void k_apply_guess(int n, const double* __restrict__ sol, const double* __restrict__ sol_prev,
                              const float* __restrict__ Y, const float* __restrict__ scale, double min_depth,
                              double* __restrict__ guess) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double g[3];
    for (int v = 0; v < 3; v++)
        g[v] = 2.0 * sol[3 * i + v] - sol_prev[3 * i + v] + (double)scale[v] * (double)Y[3 * i + v];
    const bool keep = !(sol[3 * i] > min_depth) || !(g[0] > min_depth);
    for (int v = 0; v < 3; v++) guess[3 * i + v] = keep ? sol[3 * i + v] : g[v];
}

inline int nb(long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

// ------------------------------------------------------------------ C ABI (include/adh_sw2_gnn.h)
extern "C" {

static Graph mk(int n, const int* indptr, const int* nbr, const int* rev, const float* wx, const float* wy,
                const float* inv_deg, const float* swx, const float* swy) {
    return Graph{n, indptr, nbr, rev, wx, wy, inv_deg, swx, swy};
}

int sw2n_agg_fwd(int n, const int* indptr, const int* nbr, const int* rev, const float* wx, const float* wy,
                 const float* inv_deg, const float* swx, const float* swy, const float* E, float* X, void* stream) {
    if (n <= 0 || !E || !X) return -1;
    k_agg_fwd<<<nb(32L * n, 256), 256, 0, (cudaStream_t)stream>>>(mk(n, indptr, nbr, rev, wx, wy, inv_deg, swx, swy), E, X);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int sw2n_agg_bwd(int n, const int* indptr, const int* nbr, const int* rev, const float* wx, const float* wy,
                 const float* inv_deg, const float* swx, const float* swy, const float* dX, float* dE, void* stream) {
    if (n <= 0 || !dX || !dE) return -1;
    k_agg_bwd<<<nb(32L * n, 256), 256, 0, (cudaStream_t)stream>>>(mk(n, indptr, nbr, rev, wx, wy, inv_deg, swx, swy), dX, dE);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

static bool dense_smem(int in, int out, size_t* fwd, size_t* bwd) {
    if (in <= 0 || in > MAXIN || out <= 0 || out > H || (in % 4) != 0) return false;
    *fwd = sizeof(float) * ((size_t)in * H + (size_t)TILE * (in + 1));
    *bwd = sizeof(float) * ((size_t)out * in + (size_t)TILE * (out + 1));
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_dense_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
        cudaFuncSetAttribute(k_dense_bwd_x, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
        attr = true;
    }
    return true;
}

int sw2n_dense_fwd(int n, int in, int out, const void* W_bf16, const float* b, const float* X, const float* R, int act,
                   float* Z, float* Y, void* stream) {
    size_t f, g;
    if (n <= 0 || !dense_smem(in, out, &f, &g) || !W_bf16 || !b || !X || !Y) return -1;
    k_dense_fwd<<<nb(n, TILE), 256, f, (cudaStream_t)stream>>>(n, in, out, (const __nv_bfloat16*)W_bf16, b, X, R, act, Z, Y);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// backward of a dense layer: dZ (out) = dY * act'(Z); dX = W^T dZ (if dX); gW [out*in + out] = (dW, db)
// summed over nodes; part must hold nparts * (out*in + out) floats with nparts = ceil(n / nodes_per_block)
int sw2n_dense_bwd(int n, int in, int out, const void* W_bf16, const float* X, const float* Z, const float* dY, int act,
                   float* dZ, float* dX, int nodes_per_block, float* part, float* gW, void* stream) {
    size_t f, g;
    if (n <= 0 || !dense_smem(in, out, &f, &g) || nodes_per_block <= 0 || !dZ || !part || !gW) return -1;
    cudaStream_t st = (cudaStream_t)stream;
    k_dense_bwd_x<<<nb(n, TILE), 256, g, st>>>(n, in, out, (const __nv_bfloat16*)W_bf16, Z, dY, act, dZ, dX);
    const int nparts = nb(n, nodes_per_block);
    k_dense_bwd_w<<<nparts, 256, 0, st>>>(n, in, out, nodes_per_block, X, dZ, part);
    const int count = out * in + out;
    k_reduce_parts<<<nb(count, 256), 256, 0, st>>>(nparts, count, part, gW);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int sw2n_adam(int count, float* w, const float* g, float* m, float* v, void* w_bf16, float lr, float b1, float b2,
              float eps, int t, void* stream) {
    if (count <= 0 || t <= 0) return -1;
    float c1 = 1.0f, c2 = 1.0f, p1 = 1.0f, p2 = 1.0f;
    for (int k = 0; k < t && k < 100000; k++) { p1 *= b1; p2 *= b2; }
    c1 = 1.0f - p1; c2 = 1.0f - p2;
    k_adam<<<nb(count, 256), 256, 0, (cudaStream_t)stream>>>(count, w, g, m, v, (__nv_bfloat16*)w_bf16, lr, b1, b2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int sw2n_to_bf16(int count, const float* w, void* w_bf16, void* stream) {
    if (count <= 0) return -1;
    k_to_bf16<<<nb(count, 256), 256, 0, (cudaStream_t)stream>>>(count, w, (__nv_bfloat16*)w_bf16);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int sw2n_features(int n, const double* sol, const double* sol_prev, const double* z, const float* mu, const float* sd,
                  float* F, void* stream) {
    if (n <= 0) return -1;
    k_features<<<nb(n, 256), 256, 0, (cudaStream_t)stream>>>(n, sol, sol_prev, z, mu, sd, F);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int sw2n_targets(int n, const double* sol_next, const double* sol, const double* sol_prev, const float* scale,
                 double min_depth, float* T, float* M, void* stream) {
    if (n <= 0) return -1;
    k_targets<<<nb(n, 256), 256, 0, (cudaStream_t)stream>>>(n, sol_next, sol, sol_prev, scale, min_depth, T, M);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// part must hold 148*4 floats; the loss is the sum of part[0 .. returned count)
int sw2n_mse(int n, const float* Y, const float* T, const float* M, float* dY, float* part, void* stream) {
    if (n <= 0) return -1;
    const int blocks = 148 * 4;
    k_mse<<<blocks, 256, 0, (cudaStream_t)stream>>>(3 * n, Y, T, M, 1.0f / (3.0f * n), dY, part);
    return cudaGetLastError() == cudaSuccess ? blocks : -2;
}

int sw2n_smooth3(int n, const int* indptr, const int* nbr, const float* Y, float* Ys, void* stream) {
    if (n <= 0 || !Y || !Ys || Y == Ys) return -1;
    Graph g{}; g.n = n; g.indptr = indptr; g.nbr = nbr;
    k_smooth3<<<nb(n, 256), 256, 0, (cudaStream_t)stream>>>(g, Y, Ys);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int sw2n_smooth3_adj(int n, const int* indptr, const int* nbr, const float* dYs, float* dY, void* stream) {
    if (n <= 0 || !dYs || !dY || dYs == dY) return -1;
    Graph g{}; g.n = n; g.indptr = indptr; g.nbr = nbr;
    k_smooth3_adj<<<nb(n, 256), 256, 0, (cudaStream_t)stream>>>(g, dYs, dY);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int sw2n_apply_guess(int n, const double* sol, const double* sol_prev, const float* Y, const float* scale,
                     double min_depth, double* guess, void* stream) {
    if (n <= 0) return -1;
    k_apply_guess<<<nb(n, 256), 256, 0, (cudaStream_t)stream>>>(n, sol, sol_prev, Y, scale, min_depth, guess);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // extern "C"
