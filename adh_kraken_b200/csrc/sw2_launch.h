// Host-side launchers of the SW2 and linear-algebra kernels.
#pragma once
#include <cuda_runtime.h>
#include "sw2_device.h"

namespace sw2 {

// ---- element kernels (sw2_kernels.cu)
void launch_wd_flags(const MeshView& M, const double* sol, const double* sol_old, int* node_tmp, int* wd_flag,
                     cudaStream_t st);
void launch_dry_mask(int nnodes, const double* sol_old, int* bc_mask, cudaStream_t st);
void launch_elem_resid(const MeshView& M, const StepParams& P, const double* sol, const double* sol_old,
                       const double* sol_older, const int* wd_flag, double* ER, cudaStream_t st);
void launch_gather_resid(int nnodes, const AssemblyMaps& A, const double* ER, double* residual, cudaStream_t st);
void launch_elem_jac(const MeshView& M, const StepParams& P, const double* sol, const double* sol_old,
                     const double* sol_older, const int* wd_flag, double* EJ, cudaStream_t st);
void launch_gather_jac(const AssemblyMaps& A, const double* EJ, int Etot, double* vals, cudaStream_t st);

// ---- linear algebra (la_kernels.cu)
// Node-blocked view of the reference CSR: every node's three rows share one
// column pattern (3 consecutive columns per neighbour node), so row 3a+v of
// neighbour slot j starts at indptr[3a] + v*rowlen(a) + 3j.
struct BlockCSR {
    int nnodes, n, nnz;
    const int* indptr;    // [n+1] reference CSR
    const int* cols;      // [nnz]
    const int* bptr;      // [nnodes+1] neighbour-slot ranges
    const int* bcol;      // [nslots] neighbour node of each slot
    const int* diag;      // [n] position of the diagonal entry of each row
};

struct Reduce {           // reduction workspace (device)
    double* partial;      // [kMaxBlocks * 4]
    unsigned int* counter;
    double* out;          // [8] results written by the last block
};
constexpr int kMaxBlocks = 1184;   // 8 x 148 SMs

// Newton norms over non-Dirichlet dofs: out[0] = max|res|, out[1] = sum res^2,
// out[2] = max|dsol| (get_residual_norms, src/newton/newton_tools.c:303-373)
void launch_norms(int n, const double* res, const double* dsol, const int* bc_mask, Reduce R, cudaStream_t st);

void launch_check_diag(const BlockCSR& A, const double* vals, int* bc_mask, cudaStream_t st);
void launch_dirichlet_rowscale(const BlockCSR& A, const int* bc_mask, double* vals, double* b, double* x,
                               double* scale, cudaStream_t st);
void launch_scale_vals(const BlockCSR& A, const double* scale, double* vals, cudaStream_t st);
void launch_bj_setup(const BlockCSR& A, const double* vals, double* inv, cudaStream_t st);

// BiCGStab state living on the device
struct KrylovScalars {
    double rho, rhop, alpha, omega, beta, gamma;
    double rnorm, bnorm, tol, rtol;   // stop when rnorm <= tol + bnorm * rtol
    int it, max_it, done, status;   // status: 0 ok, 1 breakdown, 2 non-finite
};

template <class VT>
struct KrylovVecs {       // VT: double (FP64 path) or float (FP32 path)
    VT *x, *r, *p, *Ap, *q, *s, *As, *b;
    const VT* vals;       // matrix values in the reference CSR order
    const VT* inv;        // [nnodes*9] block-Jacobi inverses, or the inverted ILU diagonal blocks
    const VT* vals_pc;    // block-ILU factor in the CSR layout (unused by block-Jacobi)
};

template <class VT>
void launch_bicg_init(const BlockCSR& A, KrylovVecs<VT> V, KrylovScalars* S, Reduce R, cudaStream_t st);
template <class VT>
void launch_bicg_iteration(const BlockCSR& A, KrylovVecs<VT> V, KrylovScalars* S, Reduce R, cudaStream_t st);

// t = b - A x (FP64) and out[0] = max |M^-1 t| over all dofs
void launch_resid_pnorm(const BlockCSR& A, const double* vals, const double* inv, const double* x, const double* b,
                        double* t, Reduce R, cudaStream_t st);

void launch_masked_copy(int n, const int* mask, const double* src, double* dst, cudaStream_t st);
// ---- multicolour block ILU(0) (ilu_kernels.cu)
struct IluView {            // device
    const int* color_nodes; // nodes sorted by (colour, id)
    const int* node_color;  // [nnodes]
    const int* skip;        // optional device flag: non-zero makes the sweeps no-ops (a finished solve)
};
struct IluHost {
    int ncolors;
    const int* color_ptr;   // host [ncolors+1] ranges into color_nodes
    IluView view;
};
void launch_bilu_factor(const BlockCSR& A, const IluHost& H, const double* vals, double* lu, double* dinv,
                        cudaStream_t st);
template <class VT>
void launch_bilu_apply(const BlockCSR& A, const IluHost& H, const VT* lu, const VT* dinv, VT* y, cudaStream_t st);
int grid_for_nodes(long nodes);   // grid for 8-lanes-per-node kernels

// BiCGStab with an explicit preconditioner apply (block ILU): same scalars and
// stopping rule as the fused block-Jacobi kernels above.
template <class VT>
void launch_bicg_init_pc(const BlockCSR& A, const IluHost& H, KrylovVecs<VT> V, KrylovScalars* S, Reduce R,
                         cudaStream_t st);
template <class VT>
void launch_bicg_iteration_pc(const BlockCSR& A, const IluHost& H, KrylovVecs<VT> V, KrylovScalars* S, Reduce R,
                              cudaStream_t st);

// FP64 refinement helpers: t = b - A x ; z <- M^-1 z (block-Jacobi) ; out[0] = max |z|
void launch_spmv_sub(const BlockCSR& A, const double* vals, const double* x, const double* b, double* t, cudaStream_t st);
void launch_bj_apply(int nnodes, const double* inv, double* z, cudaStream_t st);
void launch_maxabs(int n, const double* z, Reduce R, cudaStream_t st);

void launch_unscale(int n, const double* x0, const double* scale, double* x, cudaStream_t st);
void launch_axpy(int n, double a, const double* x, double* y, cudaStream_t st);   // y += a x
void launch_scal(int n, double a, double* x, cudaStream_t st);                    // x *= a
void launch_to_float(int n, const double* src, float* dst, cudaStream_t st);
void launch_to_double(int n, const float* src, double* dst, cudaStream_t st);

}  // namespace sw2
