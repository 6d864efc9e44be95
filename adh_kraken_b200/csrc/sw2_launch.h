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

// Mass balance of a state: out[0] = density * grid mass (tl_find_grid_mass_elem2d,
// src/tools/tl_grid_mass.c:198), out[1] = the step's boundary mass inflow with
// density_dt = density * dt (tl_grid_mass.c:310-320); elem_mass (optional) [ntri].
void launch_mass_balance(const MeshView& M, const double* sol, double density, double density_dt, double* elem_mass,
                         Reduce R, cudaStream_t st);

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
    VT* z;                // work vector of the right-preconditioned form (M^-1 p, M^-1 s)
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
// The node-blocked matrix kernels (level-0 and coarse AMG sweeps, SpMV) are grid-stride
// loops of 256-thread blocks held to 40 registers by __launch_bounds__(256, kSweepBlocksPerSM):
// 65536 / (40 x 256) = 6 blocks fit on an SM.  Their grid is exactly the blocks that are
// resident at once, so every block runs in the first wave; a larger grid leaves a second,
// partial wave of blocks that start only when the first ones finish.
constexpr int kSweepBlocksPerSM = 6;
int grid_resident(long work_items, int blocks_per_sm);   // 256-thread blocks, at most blocks_per_sm x SMs

// ---- aggregation AMG over the node blocks (amg_kernels.cu)
constexpr int kAmgMaxLevels = 10;
constexpr int kAmgNu = 2;               // block-Jacobi sweeps before and after each coarse correction
constexpr double kAmgOmega = 0.67;      // damping of the sweeps
constexpr double kAmgL1Theta = 0.1;     // l1 fix-up of a row: |a_vv| < theta * off-block row sum
constexpr double kAmgGainMax = 20.0;    // l1 fix-up of a block: ||D^-1|| * off-block row sum above this
constexpr int kAmgCoarseSweeps = 30;    // sweeps on the coarsest level
constexpr int kAmgCoarsest = 256;       // stop coarsening at this many nodes
struct AmgLevel {                       // device pointers; level 0 uses only the vector buffers
    int n = 0, nb = 0;                  // rows (nodes) and 3x3 blocks
    const int* bptr = nullptr;          // [n+1] block CSR
    const int* bcol = nullptr;          // [nb]
    const int* dpos = nullptr;          // [n] position of the diagonal block
    double* val64 = nullptr; double* dinv64 = nullptr;   // [9*nb], [9*n]
    float* val32 = nullptr; float* dinv32 = nullptr;
    double *b64 = nullptr, *x64 = nullptr, *t64 = nullptr, *r64 = nullptr;   // [3n] each
    float *b32 = nullptr, *x32 = nullptr, *t32 = nullptr, *r32 = nullptr;
};
struct AmgLink {                        // level l -> level l+1
    const int* agg = nullptr;           // [n_l] aggregate of each node
    const int* mptr = nullptr;          // [n_{l+1}+1] members of each aggregate, increasing node order
    const int* mem = nullptr;
    const int* gptr = nullptr;          // [nb_{l+1}+1] fine blocks summed into each coarse block
    const int* gsrc = nullptr;          // level 0: slot ids of the node graph; else block ids
};
// Chunked exact solves on the level-0 nodes where the l1 fix-up leaves block-Jacobi
// smoothing nearly inert (shallow nodes along the wet/dry front): the flagged nodes and
// their neighbours are cut into chunks of at most kPatchMaxNodes nodes (own nodes plus one
// ring of overlap), each chunk's dense block of the scaled matrix is inverted once per
// Newton iteration, and after every level-0 V-cycle each chunk corrects its own nodes
// with its rows of that inverse (restricted additive Schwarz).
constexpr int kPatchMaxNodes = 53;          // 159 dofs: the dense chunk matrix fits in shared memory
constexpr double kPatchFlagRatio = 0.5;     // flag: sum |l1 block inverse| < ratio * sum |plain block inverse|
struct PatchDev {                           // device pointers (capacities kept by the host driver)
    int* flag = nullptr;                    // [nnodes] written by the level-0 smoother set-up
    int* counts = nullptr;                  // [2] chunks, ext entries of the current build
    int* chunk_ptr = nullptr;               // [chunks+1] offsets into ext_node
    int* own_cnt = nullptr;                 // [chunks] own nodes (listed first in the chunk's ext nodes)
    long long* rofs = nullptr;              // [chunks] offset of the chunk's inverse rows
    int* ext_node = nullptr;                // [entries] chunk nodes, own first then the ring
    double* r64 = nullptr; float* r32 = nullptr;   // own-dof rows of each chunk inverse, row-major
    double* e64 = nullptr; float* e32 = nullptr;   // [3*entries] residual at the chunk nodes
    int* failed = nullptr;                  // [1] chunks whose inversion met a zero pivot (left uncorrected)
    int grid = 0;                           // CTAs of the correction kernels (grid-stride over chunks)
    int mode = 0;                           // 0 off, 1 after each V-cycle, 2 inside it (after the level-0
                                            // pre-smoothing and after the post-smoothing)
};
struct AmgHost {
    int nlev = 0;                       // levels including level 0
    AmgLevel lev[kAmgMaxLevels];
    AmgLink link[kAmgMaxLevels];
    double* dinv0_64 = nullptr; float* dinv0_32 = nullptr;   // [9*nnodes] level-0 smoother blocks
    PatchDev patch;                     // level-0 chunk corrections (inactive while patch.flag is null)
};
template <class VT> struct AmgBuf;
template <> struct AmgBuf<double> {
    static const double* val(const AmgLevel& L) { return L.val64; }
    static const double* dinv(const AmgLevel& L) { return L.dinv64; }
    static const double* dinv0(const AmgHost& H) { return H.dinv0_64; }
    static double* b(const AmgLevel& L) { return L.b64; }
    static double* x(const AmgLevel& L) { return L.x64; }
    static double* t(const AmgLevel& L) { return L.t64; }
    static double* r(const AmgLevel& L) { return L.r64; }
};
template <> struct AmgBuf<float> {
    static const float* val(const AmgLevel& L) { return L.val32; }
    static const float* dinv(const AmgLevel& L) { return L.dinv32; }
    static const float* dinv0(const AmgHost& H) { return H.dinv0_32; }
    static float* b(const AmgLevel& L) { return L.b32; }
    static float* x(const AmgLevel& L) { return L.x32; }
    static float* t(const AmgLevel& L) { return L.t32; }
    static float* r(const AmgLevel& L) { return L.r32; }
};
// numeric set-up from the scaled level-0 matrix (FP64, plus FP32 copies); writes H.patch.flag
void amg_setup(const BlockCSR& A, const AmgHost& H, const AssemblyMaps& maps, const double* vals, cudaStream_t st);
// inverts the chunk blocks of the current patch build (nchunks from the host build)
void patch_invert(const BlockCSR& A, const PatchDev& P, const double* vals, int nchunks, cudaStream_t st);
// one level-0 smoothing sweep y = x + w Dinv (b - A x) (FP64; kernel timing)
void amg_smooth0_once(const BlockCSR& A, const AmgHost& H, const double* vals, const double* b, const double* x, double* y,
                      cudaStream_t st);
void amg_smooth0_once32(const BlockCSR& A, const AmgHost& H, const float* vals, const float* b, const float* x, float* y,
                        cudaStream_t st);
// y <- V-cycle(y) followed by the chunk corrections; vals0 = the level-0 values in the Krylov precision
template <class VT>
void amg_apply(const BlockCSR& A, const AmgHost& H, const VT* vals0, VT* y, const int* skip, cudaStream_t st);
// y += the chunk corrections of the residual b - A y (the last stage of amg_apply)
template <class VT>
void amg_patch_correct(const BlockCSR& A, const AmgHost& H, const VT* vals0, const VT* b, VT* y, const int* skip,
                       cudaStream_t st);

// ---- preconditioner dispatch for the BiCGStab "_pc" path
template <class VT>
struct PrecondOp {
    int kind = 0;                       // 1: block ILU(0), 2: aggregation AMG
    bool right = false;                 // right preconditioning: BiCGStab on A M^-1 (true residuals)
    const IluHost* ilu = nullptr; const VT* lu = nullptr; const VT* dinv = nullptr;
    const AmgHost* amg = nullptr; const VT* vals = nullptr;
    // mixed precision (VT = double only): apply the preconditioner in FP32 on a
    // rounded copy of the vector, from the FP32 matrix / factor / AMG values
    bool mixed = false;
    const float* vals32 = nullptr; const float* lu32 = nullptr; const float* dinv32 = nullptr;
    float* tmp32 = nullptr;             // [n] work vector
};
template <class VT>
void precond_apply(const BlockCSR& A, const PrecondOp<VT>& P, VT* y, const int* skip, cudaStream_t st);

// ---- restarted GMRES(m) cycle (gmres_kernels.cu)
constexpr int kGmM = 200;               // largest Krylov dimension of one cycle (Hessenberg and partial buffers)
constexpr int kGmDefault = 30;          // default restart length
struct GmresDev {                       // device buffers of one cycle
    double* H = nullptr;                // [kGmM][kGmM+1] Hessenberg columns (rotated in place)
    double* H2 = nullptr;               // [kGmM+1] coefficients of the re-orthogonalisation pass
    double* cs = nullptr; double* sn = nullptr;   // [kGmM] Givens rotations
    double* g = nullptr;                // [kGmM+1] rotated right-hand side
    double* y = nullptr;                // [kGmM] least-squares solution
    double* partial = nullptr;          // [kMaxBlocks*(kGmM+1)] block partials
    unsigned int* counter = nullptr;    // last-block counter (wraps to 0)
    int* state = nullptr;               // [0] done, [1] columns built, [2] status (0 ok, 1 breakdown, 2 non-finite)
    double* scal = nullptr;             // [0] beta, [1] target, [2] residual estimate, [3] rtol (host-set), [4] h_{j+1,j}
};
// out = M^-1 V_k y from one cycle on rhs (x0 = 0), minimising the rw-weighted
// residual 2-norm; Vb holds kGmM+1 vectors of stride ld
template <class VT>
void gmres_cycle(const BlockCSR& A, const PrecondOp<VT>& P, const VT* vals, VT* Vb, size_t ld, VT* z, const VT* rhs,
                 VT* out, const double* rw, const GmresDev& G, cudaStream_t st, int m, bool reorth);
// rw_i = 1 / s_i (weights that make a scaled system's residual the unscaled one)
void launch_inv_scale(int n, const double* scale, double* rw, cudaStream_t st);
template <class VT>
void copy_skip(int n, const VT* a, VT* b, const int* skip, cudaStream_t st);
// max_i |t_i / s_i|: the unscaled residual of a scaled system (out[0] of R)
void launch_maxabs_unscaled(int n, const double* t, const double* scale, Reduce R, cudaStream_t st);
template <class VT>
void spmv_skip(const BlockCSR& A, const VT* vals, const VT* x, VT* y, const int* skip, cudaStream_t st);

// BiCGStab with an explicit preconditioner apply: same scalars and stopping rule
// as the fused block-Jacobi kernels above.
template <class VT>
void launch_bicg_init_pc(const BlockCSR& A, const PrecondOp<VT>& P, KrylovVecs<VT> V, KrylovScalars* S, Reduce R,
                         cudaStream_t st);
template <class VT>
void launch_bicg_iteration_pc(const BlockCSR& A, const PrecondOp<VT>& P, KrylovVecs<VT> V, KrylovScalars* S, Reduce R,
                              cudaStream_t st);

void launch_spmv64(const BlockCSR& A, const double* vals, const double* x, double* y, cudaStream_t st);   // y = A x
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
