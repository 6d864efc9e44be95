// SW2 element kernels: wet/dry flags, element residuals, the central-difference
// element Jacobian, and the deterministic gathers that assemble them into the
// global residual and the reference's CSR matrix.
//
// Compiled with --fmad=false: element residuals and Jacobian entries are
// bit-identical to the reference CPU build.
//
// Work decomposition (B200, 148 SMs):
//  * residual: one thread per element, 72 contiguous bytes out per thread;
//  * FD Jacobian: one thread per (element, perturbed column).  The grid's y
//    dimension is the column, so a warp covers 32 consecutive elements of one
//    column: its element loads are coalesced SoA reads, it runs one branch of the
//    reference's PRESSURE_FLAG logic, and it writes one contiguous 2304-byte run
//    of the column plane EJ[col][E][9];
//  * gathers: one thread per node (residual) or node-pair block (Jacobian) sums
//    its contributions in the reference's element order -- no atomics, so the
//    assembled values are run-to-run deterministic and equal to the CPU build's.
#include "sw2_element.cuh"
#include "sw2_device.h"
#include "sw2_launch.h"

namespace sw2 {

__device__ __forceinline__ void load_tri(const MeshView& M, const double* __restrict__ sol,
                                         const double* __restrict__ sol_old, const double* __restrict__ sol_older,
                                         const int* __restrict__ wd_flag, int e, TriData& T) {
    const int T_ = M.ntri;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        T.x[a].x = M.ex[a * T_ + e]; T.x[a].y = M.ey[a * T_ + e]; T.z[a] = M.ez[a * T_ + e];
        T.g[a].x = M.gx[a * T_ + e]; T.g[a].y = M.gy[a * T_ + e];
        const int n = M.tri[3 * e + a];
        T.h[a] = sol[3 * n]; T.vel[a].x = sol[3 * n + 1]; T.vel[a].y = sol[3 * n + 2];
        T.ho[a] = sol_old[3 * n]; T.velo[a].x = sol_old[3 * n + 1]; T.velo[a].y = sol_old[3 * n + 2];
        T.hoo[a] = sol_older[3 * n]; T.veloo[a].x = sol_older[3 * n + 1]; T.veloo[a].y = sol_older[3 * n + 2];
    }
    T.djac = M.djac[e];
    T.wd_flag = wd_flag[e];
}

__device__ __forceinline__ SegBC seg_bc(const StepParams& P) {
    return SegBC{P.bc_depth, P.bc_vx, P.bc_vy, P.bc_qs, P.bc_convey, P.bc_rough, P.bc_tail, P.bc_flux};
}

__device__ __forceinline__ void load_seg(const MeshView& M, const double* __restrict__ sol, int s, SegData& S) {
    S.n.x = M.snx[s]; S.n.y = M.sny[s]; S.djac = M.sdjac[s]; S.kind = M.skind[s]; S.z0 = M.sz0[s];
#pragma unroll
    for (int a = 0; a < 2; a++) {
        const int n = M.seg[2 * s + a];
        S.h[a] = sol[3 * n]; S.vel[a].x = sol[3 * n + 1]; S.vel[a].y = sol[3 * n + 2];
    }
}

// ---------------------------------------------------------------- wet/dry flags
// fe_sw2_wdflag_legacy (src/models/sw2/sw2_wdflag_legacy.c:34-95) in two passes:
// nodes touching a not-fully-wet element, then the element flag.
__global__ void k_wd_nodes(MeshView M, const double* __restrict__ sol, int* __restrict__ node_tmp) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M.ntri) return;
    int wet = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) if (sol[3 * M.tri[3 * e + a]] > 0.0) wet++;
    if (wet != 3) {
#pragma unroll
        for (int a = 0; a < 3; a++) node_tmp[M.tri[3 * e + a]] = 1;   // same value from every writer
    }
}
__global__ void k_wd_elems(MeshView M, const double* __restrict__ sol, const double* __restrict__ sol_old,
                           const int* __restrict__ node_tmp, int* __restrict__ wd_flag) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M.ntri) return;
    int n0 = M.tri[3 * e], n1 = M.tri[3 * e + 1], n2 = M.tri[3 * e + 2];
    int f = (node_tmp[n0] != 0 || node_tmp[n1] != 0 || node_tmp[n2] != 0) ? 1 : 0;
    if (sol[3 * n0] < 0 && sol[3 * n1] < 0 && sol[3 * n2] < 0 &&
        sol_old[3 * n0] < 0 && sol_old[3 * n1] < 0 && sol_old[3 * n2] < 0) f = 2;
    wd_flag[e] = f;
}
// fe_sw2_init (src/models/sw2/fe_sw2_init.c:38-49): a node dry at t^n gets its
// velocities into the (permanent) Dirichlet mask.
__global__ void k_dry_mask(int nnodes, const double* __restrict__ sol_old, int* __restrict__ bc_mask) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nnodes) return;
    if (sol_old[3 * n] <= 0.) { bc_mask[3 * n + 1] = 1; bc_mask[3 * n + 2] = 1; }
}

// ---------------------------------------------------------------- residuals
__global__ void __launch_bounds__(128) k_resid_tri(MeshView M, StepParams P, const double* __restrict__ sol,
                                                   const double* __restrict__ sol_old, const double* __restrict__ sol_older,
                                                   const int* __restrict__ wd_flag, double* __restrict__ ER) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M.ntri) return;
    TriData T;
    load_tri(M, sol, sol_old, sol_older, wd_flag, e, T);
    double r[9];
    body_resid<true>(T, P.dt, P.alpha, P.grav, r);
    double* out = ER + 9 * (size_t)e;
#pragma unroll
    for (int i = 0; i < 9; i++) out[i] = r[i];
}

__global__ void k_resid_seg(MeshView M, StepParams P, const double* __restrict__ sol, double* __restrict__ ER) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= M.nseg) return;
    SegData S;
    load_seg(M, sol, s, S);
    double r[6];
    seg_resid<true>(S, P.dt, P.grav, seg_bc(P), r);
    double* out = ER + 9 * ((size_t)M.ntri + s);
#pragma unroll
    for (int i = 0; i < 6; i++) out[i] = r[i];
}

// residual[3n+v] = sum over the node's element entries of (0 + (-1)*entry), in
// element order (load_pdes + load_global_resid, src/residual/assemble_residual.c:4-60,160-174)
__global__ void k_gather_resid(int nnodes, AssemblyMaps A, const double* __restrict__ ER, double* __restrict__ residual) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nnodes) return;
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
    for (int k = A.rptr[n]; k < A.rptr[n + 1]; k++) {
        const uint32_t c = A.rmap[k];
        const double* src = ER + 9 * (size_t)(c / 3) + 3 * (c % 3);
        acc0 += 0.0 + -1.0 * src[0];
        acc1 += 0.0 + -1.0 * src[1];
        acc2 += 0.0 + -1.0 * src[2];
    }
    residual[3 * n] = acc0; residual[3 * n + 1] = acc1; residual[3 * n + 2] = acc2;
}

// ---------------------------------------------------------------- FD Jacobian
// perturb_var + elem_matrix_deriv (src/jacobian/assemble_jacobian.c:304-397):
// column (node i, var k) = (R(u + eps e) - R(u - eps e)) / (2 eps).
// Template VAR: 0 perturbs h (pressure terms evaluated), 1/2 perturb u/v
// (pressure terms skipped, as the reference's PRESSURE_FLAG does).
template <int VAR>
__global__ void __launch_bounds__(128) k_fd_tri(MeshView M, StepParams P, const double* __restrict__ sol,
                                                const double* __restrict__ sol_old, const double* __restrict__ sol_older,
                                                const int* __restrict__ wd_flag, double* __restrict__ EJ, int Etot) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;          // perturbed node 0..2
    if (e >= M.ntri) return;
    TriData T;
    load_tri(M, sol, sol_old, sol_older, wd_flag, e, T);
    double u0 = VAR == 0 ? (i == 0 ? T.h[0] : i == 1 ? T.h[1] : T.h[2])
              : VAR == 1 ? (i == 0 ? T.vel[0].x : i == 1 ? T.vel[1].x : T.vel[2].x)
                         : (i == 0 ? T.vel[0].y : i == 1 ? T.vel[1].y : T.vel[2].y);
    const double eps = fd_eps(u0);
    const double eps2 = 2.0 * eps;
    double Rp[9], Rm[9];
#pragma unroll
    for (int sgn = 0; sgn < 2; sgn++) {
        TriData Q = T;
        const double d = (sgn == 0 ? 1 : -1) * eps;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            if (a != i) continue;
            if (VAR == 0) Q.h[a] += d;
            else if (VAR == 1) Q.vel[a].x += d;
            else Q.vel[a].y += d;
        }
        body_resid<VAR == 0>(Q, P.dt, P.alpha, P.grav, sgn == 0 ? Rp : Rm);
    }
    const int col = i * 3 + VAR;
    double* out = EJ + ((size_t)col * Etot + e) * 9;
#pragma unroll
    for (int r = 0; r < 9; r++) out[r] = (Rp[r] - Rm[r]) / eps2;
}

__global__ void k_fd_seg(MeshView M, StepParams P, const double* __restrict__ sol, double* __restrict__ EJ, int Etot) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int col = blockIdx.y;       // 0..5 = node*3 + var
    if (s >= M.nseg) return;
    const int i = col / 3, k = col % 3;
    SegData S;
    load_seg(M, sol, s, S);
    double u0 = k == 0 ? S.h[i] : (k == 1 ? S.vel[i].x : S.vel[i].y);
    const double eps = fd_eps(u0);
    const double eps2 = 2.0 * eps;
    const SegBC B = seg_bc(P);
    double Rp[6], Rm[6];
    for (int sgn = 0; sgn < 2; sgn++) {
        SegData Q = S;
        const double d = (sgn == 0 ? 1 : -1) * eps;
        if (k == 0) Q.h[i] += d; else if (k == 1) Q.vel[i].x += d; else Q.vel[i].y += d;
        if (k == 0) seg_resid<true>(Q, P.dt, P.grav, B, sgn == 0 ? Rp : Rm);
        else seg_resid<false>(Q, P.dt, P.grav, B, sgn == 0 ? Rp : Rm);
    }
    double* out = EJ + ((size_t)col * Etot + M.ntri + s) * 9;
    for (int r = 0; r < 6; r++) out[r] = (Rp[r] - Rm[r]) / eps2;
}

// CSR values: each node-pair block sums its element blocks in element order
// (load_global_mat_split_CSR, src/jacobian/assemble_jacobian.c:164-215, adds
// into vals zeroed at :60).  Thread = (block, row v); it reads three column
// planes (24 contiguous bytes each) per contribution and writes 24 contiguous bytes.
__global__ void k_gather_jac(AssemblyMaps A, const double* __restrict__ EJ, int Etot, double* __restrict__ vals) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = t / 3, v = t % 3;
    if (k >= A.nblocks) return;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int q = A.jptr[k]; q < A.jptr[k + 1]; q++) {
        const uint32_t c = A.jmap[q];
        const size_t E = c / 9;
        const int ia = (c % 9) / 3, ib = c % 3;
        const size_t base = E * 9 + ia * 3 + v;
        a0 += EJ[(size_t)(ib * 3 + 0) * Etot * 9 + base];
        a1 += EJ[(size_t)(ib * 3 + 1) * Etot * 9 + base];
        a2 += EJ[(size_t)(ib * 3 + 2) * Etot * 9 + base];
    }
    double* out = vals + A.boff[k] + v * A.blen[k];
    out[0] = a0; out[1] = a1; out[2] = a2;
}

// ---------------------------------------------------------------- mass balance
// tl_find_grid_mass_elem2d (src/tools/tl_grid_mass.c:198-275) per triangle, with
// the dry-vertex rule of fe_3m2d_dry_wet_factornew (:442-515): a vertex is dry when
// its depth is strictly negative; one dry vertex adds the wet part plus the dry
// corner's negative depth counted as positive mass, two dry vertices integrate the
// clipped depths times the wet fraction.
__device__ __forceinline__ double tri_mass_term(const MeshView& M, const double* __restrict__ sol, int e) {
    const int T_ = M.ntri;
    V2 x[3];
    double h[3], hneg[3] = {0.0, 0.0, 0.0};
    int passcode = 0, total = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        x[a].x = M.ex[a * T_ + e]; x[a].y = M.ey[a * T_ + e];
        h[a] = sol[3 * M.tri[3 * e + a]];
        const int d = (h[a] < 0.0) ? 1 : 0;
        total += d; passcode += (d << a);
    }
    const double djac = M.djac[e];
    double factor = 1.0;
    int num_dry = total;
    if (total == 3) factor = 0.0;
    else if (total != 0) {
        if (total != 1) passcode = 7 - passcode;
        const int o = passcode / 2;
        const double ho = sel3(h, o);
        const V2 xo = sel3(x, o);
        V2 nx[3];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            if (i != o) {
                const double xsi = h[i] / (h[i] - ho);
                nx[i].x = x[i].x + xsi * (xo.x - x[i].x);   // FIXED_POS, macro.h:756
                nx[i].y = x[i].y + xsi * (xo.y - x[i].y);
            } else {
                nx[i] = x[i];
            }
        }
        const double ax = nx[1].x - nx[0].x, ay = nx[1].y - nx[0].y;   // TRI_AREA, macro.h:771
        const double bx = nx[2].x - nx[0].x, by = nx[2].y - nx[0].y;
        const double area = (ax * by - ay * bx) / 2.0;
        if (area / djac < SW2_SMALL) {               // a sliver of dry (one vertex) or wet (two) area
            num_dry = (total % 2 == 1) ? 0 : 3;
            factor = (double)(total % 2);
        } else {
            factor = (total >> 1) - (total % 2);
            factor *= area / djac;
            factor = factor + ((factor < 0) ? 1.0 : 0.0);
        }
    }
    double f1 = factor, f2 = 0.0;
    if (num_dry == 1) {
#pragma unroll
        for (int a = 0; a < 3; a++) if (h[a] < 0.0) hneg[a] = h[a];
        f1 = 1.0; f2 = -1.0 * (1.0 - factor);
    } else if (num_dry == 2) {
#pragma unroll
        for (int a = 0; a < 3; a++) if (h[a] < 0.0) { hneg[a] = h[a]; h[a] = 0.0; }
    }
    // integrate_triangle_f, src/fe/fe_integrals_2d.c:25
    return (f1 * djac * (h[0] + h[1] + h[2]) / 3.0) + (f2 * djac * (hneg[0] + hneg[1] + hneg[2]) / 3.0);
}

// One boundary segment's mass inflow over a step (tl_grid_mass.c:310-320 with
// integrate_line_h_f, src/fe/fe_integrals_1d.c:42): -c len/6 ((2 vn0 + vn1) h0 + (vn0 + 2 vn1) h1),
// c = density dt, vn = v . n at the two nodes.
__device__ __forceinline__ double seg_mass_flux(const MeshView& M, const double* __restrict__ sol, int k, double c) {
    double vn[2], h[2];
#pragma unroll
    for (int a = 0; a < 2; a++) {
        const int nd = M.seg[2 * k + a];
        vn[a] = sol[3 * nd + 1] * M.snx[k] + sol[3 * nd + 2] * M.sny[k];
        h[a] = sol[3 * nd];
    }
    const double t1 = M.sdjac[k] * SW2_ONE_6 * c;
    return -(t1 * ((2 * vn[0] + vn[1]) * h[0] + (vn[0] + 2 * vn[1]) * h[1]));
}

// Grid-stride over triangles then segments; per-block sums in a fixed order and a
// last-block pass over the block partials in block order (run-to-run deterministic).
// out[0] = density * mass, out[1] = boundary inflow; elem_mass (optional) = per-triangle terms.
__global__ void __launch_bounds__(256) k_mass_balance(MeshView M, const double* __restrict__ sol, double density,
                                                      double c, double* __restrict__ elem_mass,
                                                      double* __restrict__ partial, unsigned int* __restrict__ counter,
                                                      double* __restrict__ out) {
    __shared__ double sh[2][8];
    __shared__ bool is_last;
    double mass = 0.0, flux = 0.0;
    const int stride = gridDim.x * blockDim.x;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < M.ntri; e += stride) {
        const double t = tri_mass_term(M, sol, e);
        if (elem_mass) elem_mass[e] = t;
        mass += t;
    }
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < M.nseg; k += stride) flux += seg_mass_flux(M, sol, k, c);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mass += __shfl_xor_sync(0xffffffffu, mass, o);
        flux += __shfl_xor_sync(0xffffffffu, flux, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { sh[0][w] = mass; sh[1][w] = flux; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int i = 0; i < 8; i++) { a += sh[0][i]; b += sh[1][i]; }
        partial[4 * blockIdx.x] = a; partial[4 * blockIdx.x + 1] = b;
        __threadfence();
        const unsigned int t = atomicInc(counter, gridDim.x - 1);   // the last block wraps it back to 0
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last && threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < (int)gridDim.x; k++) { a += __ldcg(partial + 4 * k); b += __ldcg(partial + 4 * k + 1); }
        out[0] = a * density;
        out[1] = b;
    }
}

// ---------------------------------------------------------------- launchers
static inline int blocks(long n, int b) { return (int)((n + b - 1) / b); }

void launch_wd_flags(const MeshView& M, const double* sol, const double* sol_old, int* node_tmp, int* wd_flag,
                     cudaStream_t st) {
    cudaMemsetAsync(node_tmp, 0, sizeof(int) * (size_t)M.nnodes, st);
    if (M.ntri == 0) return;
    k_wd_nodes<<<blocks(M.ntri, 256), 256, 0, st>>>(M, sol, node_tmp);
    k_wd_elems<<<blocks(M.ntri, 256), 256, 0, st>>>(M, sol, sol_old, node_tmp, wd_flag);
}

void launch_dry_mask(int nnodes, const double* sol_old, int* bc_mask, cudaStream_t st) {
    k_dry_mask<<<blocks(nnodes, 256), 256, 0, st>>>(nnodes, sol_old, bc_mask);
}

void launch_elem_resid(const MeshView& M, const StepParams& P, const double* sol, const double* sol_old,
                       const double* sol_older, const int* wd_flag, double* ER, cudaStream_t st) {
    if (M.ntri) k_resid_tri<<<blocks(M.ntri, 128), 128, 0, st>>>(M, P, sol, sol_old, sol_older, wd_flag, ER);
    if (M.nseg) k_resid_seg<<<blocks(M.nseg, 128), 128, 0, st>>>(M, P, sol, ER);
}

void launch_gather_resid(int nnodes, const AssemblyMaps& A, const double* ER, double* residual, cudaStream_t st) {
    k_gather_resid<<<blocks(nnodes, 256), 256, 0, st>>>(nnodes, A, ER, residual);
}

void launch_elem_jac(const MeshView& M, const StepParams& P, const double* sol, const double* sol_old,
                     const double* sol_older, const int* wd_flag, double* EJ, cudaStream_t st) {
    const int Etot = M.ntri + M.nseg;
    if (M.ntri) {
        dim3 g(blocks(M.ntri, 128), 3);
        k_fd_tri<0><<<g, 128, 0, st>>>(M, P, sol, sol_old, sol_older, wd_flag, EJ, Etot);
        k_fd_tri<1><<<g, 128, 0, st>>>(M, P, sol, sol_old, sol_older, wd_flag, EJ, Etot);
        k_fd_tri<2><<<g, 128, 0, st>>>(M, P, sol, sol_old, sol_older, wd_flag, EJ, Etot);
    }
    if (M.nseg) {
        dim3 g(blocks(M.nseg, 128), 6);
        k_fd_seg<<<g, 128, 0, st>>>(M, P, sol, EJ, Etot);
    }
}

void launch_gather_jac(const AssemblyMaps& A, const double* EJ, int Etot, double* vals, cudaStream_t st) {
    if (A.nblocks) k_gather_jac<<<blocks(3L * A.nblocks, 256), 256, 0, st>>>(A, EJ, Etot, vals);
}

void launch_mass_balance(const MeshView& M, const double* sol, double density, double density_dt, double* elem_mass,
                         Reduce R, cudaStream_t st) {
    long work = M.ntri > M.nseg ? M.ntri : M.nseg;
    int g = blocks(work, 256);
    if (g > kMaxBlocks) g = kMaxBlocks;
    if (g < 1) g = 1;
    k_mass_balance<<<g, 256, 0, st>>>(M, sol, density, density_dt, elem_mass, R.partial, R.counter, R.out);
}

}  // namespace sw2
