// C ABI and host driver of the B200 SW2 time step (declared in include/adh_sw2_gpu.h).
//
// The driver mirrors fe_newton (src/newton/fe_newton.c:44-915) and advance_time
// (src/timeloop/time_loop.c:56-89) step for step, but every array lives in HBM:
// the host only reads back the handful of scalars that steer the Newton loop
// (residual norms, the BiCGStab stop flag).  BiCGStab iterations are replayed
// from a captured CUDA graph in chunks, with the stop test evaluated on the
// device, so a converged solve wastes at most one chunk of early-exit launches.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <mutex>
#include <vector>
#include <algorithm>
#include <string>
#include "../../include/adh_sw2_gpu.h"
#include "sw2_launch.h"

using namespace sw2;

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;
extern "C" const char* sw2g_last_error(void) { return g_err.c_str(); }

#define CK(call)                                                                             \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            g_err = std::string(#call) + ": " + cudaGetErrorString(e_);                      \
            return SW2G_ERR_CUDA;                                                            \
        }                                                                                    \
    } while (0)
#define CKL()                                                                                \
    do {                                                                                     \
        cudaError_t e_ = cudaGetLastError();                                                 \
        if (e_ != cudaSuccess) {                                                             \
            g_err = std::string("kernel launch: ") + cudaGetErrorString(e_);                 \
            return SW2G_ERR_CUDA;                                                            \
        }                                                                                    \
    } while (0)
#define TRY(x) do { int r_ = (x); if (r_ != SW2G_OK) return r_; } while (0)

static const int kChunk = 8;   // BiCGStab iterations per graph replay
static const double kPatchTileEdges = 7.0;   // tile side of the AMG chunk corrections, in mean edge lengths

struct ProfRec { int cls; cudaEvent_t a, b; };

struct sw2g_model {
    int V = 0, T = 0, S = 0, Etot = 0, n = 0, nnz = 0, nslots = 0;
    int device = 0;   // the device current at sw2g_create: every buffer and the stream live there
    cudaStream_t st = nullptr; bool own_stream = false;
    std::vector<int> h_indptr, h_cols;
    std::vector<void*> allocs;
    // mesh
    int *d_tri = nullptr, *d_seg = nullptr, *d_skind = nullptr;
    double *d_ex = nullptr, *d_ey = nullptr, *d_ez = nullptr, *d_gx = nullptr, *d_gy = nullptr, *d_djac = nullptr;
    double *d_snx = nullptr, *d_sny = nullptr, *d_sdjac = nullptr, *d_sz0 = nullptr;
    // CSR and node blocks
    int *d_indptr = nullptr, *d_cols = nullptr, *d_bptr = nullptr, *d_bcol = nullptr, *d_diag = nullptr;
    // assembly maps
    int *d_rptr = nullptr, *d_jptr = nullptr, *d_boff = nullptr, *d_blen = nullptr;
    uint32_t *d_rmap = nullptr, *d_jmap = nullptr;
    // resident state
    double *d_sol = nullptr, *d_sol_old = nullptr, *d_sol_older = nullptr, *d_dirichlet = nullptr, *d_guess = nullptr;
    int *d_bc_mask = nullptr, *d_mask_save = nullptr;
    bool guess_set = false;
    bool can_undo = false;   // the levels were rotated by the last sw2g_step
    // work
    int *d_wd = nullptr, *d_node_tmp = nullptr;
    double *d_ER = nullptr, *d_EJ = nullptr, *d_res = nullptr, *d_vals = nullptr, *d_dsol = nullptr;
    double *d_scale = nullptr, *d_inv = nullptr, *d_x0 = nullptr, *d_b64 = nullptr, *d_t64 = nullptr;
    double *k_r = nullptr, *k_p = nullptr, *k_Ap = nullptr, *k_q = nullptr, *k_s = nullptr, *k_As = nullptr, *k_z = nullptr;
    double *k_xi = nullptr;   // correction of one restarted pass
    float *f_vals = nullptr, *f_inv = nullptr, *f_x = nullptr, *f_r = nullptr, *f_p = nullptr, *f_Ap = nullptr;
    float *f_q = nullptr, *f_s = nullptr, *f_As = nullptr, *f_b = nullptr, *f_z = nullptr;
    // reductions / scalars
    double *d_partial = nullptr, *d_rout = nullptr; unsigned int* d_counter = nullptr;
    KrylovScalars* d_ks = nullptr;
    double* h_rout = nullptr; KrylovScalars* h_ks = nullptr;
    cudaGraphExec_t graph64[3] = {nullptr, nullptr, nullptr}, graph32[3] = {nullptr, nullptr, nullptr};   // [precond]
    // multicolour block ILU(0)
    std::vector<int> h_color_ptr;
    int *d_color_nodes = nullptr, *d_node_color = nullptr;
    double* d_lu = nullptr; float* f_lu = nullptr;
    IluHost ilu{};
    // aggregation AMG (hierarchy built on first use)
    AmgHost amg{};
    bool amg_ready = false;
    // restarted GMRES (allocated on first use)
    GmresDev gm{};
    double* gm_V64 = nullptr;            // [cap+1][gm_ld(n)] Krylov basis
    float* gm_V32 = nullptr;             // [cap+1][gm_ld(n)] FP32 Krylov basis (krylov_basis_precision 32)
    int gm_cap64 = 0, gm_cap32 = 0;      // restart length the bases were allocated for
    cudaGraphExec_t gm_graph_b32 = nullptr;
    int gm_m64 = 0, gm_m32 = 0, gm_mb32 = 0;   // restart length each cycle graph was built for
    double* gm_rw = nullptr;             // [n] row weights 1/s: GMRES minimises the unscaled residual
    cudaGraphExec_t gm_graph64 = nullptr, gm_graph32 = nullptr;
    std::vector<int> h_bptr, h_bcol;   // node graph, kept for the AMG set-up
    // chunk corrections of the AMG (built every Newton iteration from the flagged nodes)
    std::vector<long long> h_tile;     // [V] tile of each node (squares of kPatchTileEdges mean edge lengths)
    int* h_pflag = nullptr;            // pinned [V] flags read back
    int *h_cptr = nullptr, *h_cown = nullptr, *h_cnode = nullptr;   // pinned staging of the chunk build
    long long* h_crofs = nullptr;
    int pcap_chunks = 0, pcap_entries = 0; long long pcap_r = 0;
    int p_nchunks = 0, p_nentries = 0, p_nflag = 0;
    long long p_rtot = 0;
    StepParams P{};
    MeshView M{}; AssemblyMaps A{}; BlockCSR B{};
    // profiling
    bool prof = false;
    std::vector<ProfRec> prof_pending;
    std::vector<cudaEvent_t> ev_pool;
    double prof_ms[SW2G_NCLASSES] = {0};
    long long prof_launch[SW2G_NCLASSES] = {0};
};

template <class T>
static int dalloc(sw2g_model* m, T** p, size_t count) {
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * count);
    if (e != cudaSuccess) { g_err = std::string("cudaMalloc: ") + cudaGetErrorString(e); *p = nullptr; return SW2G_ERR_NOMEM; }
    m->allocs.push_back((void*)*p);
    return SW2G_OK;
}
// frees one allocation made by dalloc
template <class T>
static void dfree(sw2g_model* m, T** p) {
    if (!*p) return;
    auto it = std::find(m->allocs.begin(), m->allocs.end(), (void*)*p);
    if (it != m->allocs.end()) m->allocs.erase(it);
    cudaFree(*p);
    *p = nullptr;
}
template <class T>
static int upload(sw2g_model* m, T** p, const T* h, size_t count) {
    TRY(dalloc(m, p, count));
    if (count) CK(cudaMemcpyAsync(*p, h, sizeof(T) * count, cudaMemcpyHostToDevice, m->st));
    return SW2G_OK;
}

// ------------------------------------------------------------------ profiling
static cudaEvent_t ev_get(sw2g_model* m) {
    if (!m->ev_pool.empty()) { cudaEvent_t e = m->ev_pool.back(); m->ev_pool.pop_back(); return e; }
    cudaEvent_t e; cudaEventCreate(&e); return e;
}
struct ProfScope {
    sw2g_model* m; int cls; cudaEvent_t a = nullptr;
    ProfScope(sw2g_model* m_, int c, int launches) : m(m_), cls(c) {
        m->prof_launch[c] += launches;
        if (m->prof) { a = ev_get(m); cudaEventRecord(a, m->st); }
    }
    ~ProfScope() {
        if (m->prof) { cudaEvent_t b = ev_get(m); cudaEventRecord(b, m->st); m->prof_pending.push_back({cls, a, b}); }
    }
};
static void prof_collect(sw2g_model* m) {
    if (m->prof_pending.empty()) return;
    cudaStreamSynchronize(m->st);
    for (auto& r : m->prof_pending) {
        float ms = 0; cudaEventElapsedTime(&ms, r.a, r.b);
        m->prof_ms[r.cls] += ms;
        m->ev_pool.push_back(r.a); m->ev_pool.push_back(r.b);
    }
    m->prof_pending.clear();
}

// ------------------------------------------------------------------ setup helpers
// Serial CSR of slin_sys_init_sparsity_mono (slin_sys_init_sparsity_mono.c:335-436)
// for an all-SW2 mesh: row 3a+v lists 3b+w for every node b sharing an element with
// a (a itself included), sorted.
static void build_csr(int V, int T, int S, const int* tri, const int* seg, std::vector<int>& indptr,
                      std::vector<int>& cols) {
    std::vector<int> cnt(V + 1, 0);
    for (int e = 0; e < T; e++) for (int a = 0; a < 3; a++) cnt[tri[3 * e + a]] += 3;
    for (int e = 0; e < S; e++) for (int a = 0; a < 2; a++) cnt[seg[2 * e + a]] += 2;
    std::vector<long> ptr(V + 1, 0);
    for (int i = 0; i < V; i++) ptr[i + 1] = ptr[i] + cnt[i];
    std::vector<int> buf(ptr[V]);
    std::fill(cnt.begin(), cnt.end(), 0);
    for (int e = 0; e < T; e++) for (int a = 0; a < 3; a++) { int i = tri[3 * e + a]; for (int b = 0; b < 3; b++) buf[ptr[i] + cnt[i]++] = tri[3 * e + b]; }
    for (int e = 0; e < S; e++) for (int a = 0; a < 2; a++) { int i = seg[2 * e + a]; for (int b = 0; b < 2; b++) buf[ptr[i] + cnt[i]++] = seg[2 * e + b]; }
    indptr.assign(3 * (size_t)V + 1, 0);
    cols.clear();
    cols.reserve((size_t)ptr[V] * 3);
    std::vector<int> uniq;
    for (int i = 0; i < V; i++) {
        uniq.assign(buf.begin() + ptr[i], buf.begin() + ptr[i + 1]);
        std::sort(uniq.begin(), uniq.end());
        uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
        for (int v = 0; v < 3; v++) {
            for (int b : uniq) for (int w = 0; w < 3; w++) cols.push_back(3 * b + w);
            indptr[3 * i + v + 1] = (int)cols.size();
        }
    }
}

extern "C" void sw2g_default_opts(sw2g_newton_opts* o) {
    o->tol_nonlin = 1e-8; o->inc_nonlin = 1e-6; o->max_nonlin_it = 10; o->max_linesearch_cuts = 5;
    o->krylov_max_it = 4000; o->krylov_tol = 1e-11; o->krylov_precision = 64;
    o->refine_tol = 1e-4; o->max_refine = 8; o->use_guess = 0; o->precond = SW2G_PC_AMG;
    o->krylov_method = SW2G_KRYLOV_GMRES;
    o->tol_nonlin_rel = 0.0;
    o->krylov_basis_precision = 64;
    o->krylov_restart = 30;
    o->amg_chunks = 0;
    o->tol_nonlin_min = 0.0;
}

extern "C" int sw2g_create(const sw2g_mesh* mesh, void* cuda_stream, sw2g_model** out) {
    if (!mesh || !out || mesh->nnodes <= 0 || mesh->ntri <= 0 || mesh->nseg < 0 || !mesh->xyz || !mesh->tri ||
        (mesh->nseg > 0 && (!mesh->seg || !mesh->seg_kind))) {
        g_err = "sw2g_create: bad mesh description";
        return SW2G_ERR_ARG;
    }
    const int V = mesh->nnodes, T = mesh->ntri, S = mesh->nseg;
    if ((long)(T + S) * 9 >= (1L << 31) || 3L * V >= (1L << 31)) { g_err = "sw2g_create: mesh too large for 32-bit maps"; return SW2G_ERR_ARG; }
    for (long i = 0; i < 3L * T; i++) if (mesh->tri[i] < 0 || mesh->tri[i] >= V) { g_err = "sw2g_create: triangle node id out of range"; return SW2G_ERR_MESH; }
    for (long i = 0; i < 2L * S; i++) if (mesh->seg[i] < 0 || mesh->seg[i] >= V) { g_err = "sw2g_create: segment node id out of range"; return SW2G_ERR_MESH; }
    for (int i = 0; i < S; i++) if (mesh->seg_kind[i] < 0 || mesh->seg_kind[i] > 5) { g_err = "sw2g_create: segment kind not in 0..5"; return SW2G_ERR_ARG; }
    sw2g_model* m = new sw2g_model();
    m->V = V; m->T = T; m->S = S; m->Etot = T + S; m->n = 3 * V;
    if (cudaGetDevice(&m->device) != cudaSuccess) { g_err = "sw2g_create: no current CUDA device"; delete m; return SW2G_ERR_CUDA; }
    if (cuda_stream) m->st = (cudaStream_t)cuda_stream;
    else {
        cudaError_t e = cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking);
        if (e != cudaSuccess) { g_err = std::string("cudaStreamCreate: ") + cudaGetErrorString(e); delete m; return SW2G_ERR_CUDA; }
        m->own_stream = true;
    }
    int rc = SW2G_OK;
    auto fail = [&](int r) { sw2g_destroy(m); return r; };

    // --- geometry: selem2d_get_triangle_linear_djac_nrml_gradPhi (src/structs/selem/selem_2d.c:270-350)
    //     and selem1d_load (src/structs/selem/selem_1d.c:27-58), evaluated in that order of operations
    std::vector<double> ex(3 * (size_t)T), ey(3 * (size_t)T), ez(3 * (size_t)T), gx(3 * (size_t)T), gy(3 * (size_t)T), dj(T);
    for (int e = 0; e < T; e++) {
        const double* p[3];
        for (int a = 0; a < 3; a++) p[a] = mesh->xyz + 3 * (size_t)mesh->tri[3 * e + a];
        double s1x = p[1][0] - p[0][0], s1y = p[1][1] - p[0][1];
        double s2x = p[2][0] - p[0][0], s2y = p[2][1] - p[0][1];
        double djac = (s1x * s2y) - (s2x * s1y);
        if (!(fabs(djac) > 2.220446049250313080847e-16)) { g_err = "sw2g_create: degenerate triangle"; return fail(SW2G_ERR_MESH); }
        double inv = 1. / djac;
        double g[6] = {(s1y - s2y) * inv, (s2x - s1x) * inv, s2y * inv, -s2x * inv, -s1y * inv, s1x * inv};
        for (int a = 0; a < 3; a++) {
            ex[(size_t)a * T + e] = p[a][0]; ey[(size_t)a * T + e] = p[a][1]; ez[(size_t)a * T + e] = p[a][2];
            gx[(size_t)a * T + e] = g[2 * a]; gy[(size_t)a * T + e] = g[2 * a + 1];
        }
        dj[e] = djac * (1.0 / 2.0);
        if (!(dj[e] > 1e-6)) { g_err = "sw2g_create: triangle not counter-clockwise (selem2d_load rejects it)"; return fail(SW2G_ERR_MESH); }
    }
    std::vector<double> snx(S + 1), sny(S + 1), sdj(S + 1), sz0(S + 1, 0.0);
    for (int k = 0; k < S; k++) {
        const double* a = mesh->xyz + 3 * (size_t)mesh->seg[2 * k];
        const double* b = mesh->xyz + 3 * (size_t)mesh->seg[2 * k + 1];
        sz0[k] = a[2];
        double d = sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]));
        if (!(d > 1e-6)) { g_err = "sw2g_create: zero-length boundary segment"; return fail(SW2G_ERR_MESH); }
        sdj[k] = d; snx[k] = (b[1] - a[1]) / d; sny[k] = -(b[0] - a[0]) / d;
    }

    // --- tiles of the AMG chunk corrections: squares of kPatchTileEdges mean edge lengths
    {
        double area = 0.0, xmin = 1e300, ymin = 1e300;
        for (int e = 0; e < T; e++) area += dj[e];
        for (int i = 0; i < V; i++) { xmin = std::min(xmin, mesh->xyz[3 * (size_t)i]); ymin = std::min(ymin, mesh->xyz[3 * (size_t)i + 1]); }
        const double edge = sqrt(2.0 * area / T), side = kPatchTileEdges * edge;
        m->h_tile.resize(V);
        for (int i = 0; i < V; i++) {
            const long long tx = (long long)floor((mesh->xyz[3 * (size_t)i] - xmin) / side);
            const long long ty = (long long)floor((mesh->xyz[3 * (size_t)i + 1] - ymin) / side);
            m->h_tile[i] = tx * 4000000LL + ty;
        }
    }

    // --- CSR (bit-exact with the reference) and its node-block view
    build_csr(V, T, S, mesh->tri, S ? mesh->seg : nullptr, m->h_indptr, m->h_cols);
    const std::vector<int>& ip = m->h_indptr; const std::vector<int>& cl = m->h_cols;
    m->nnz = (int)cl.size();
    if (mesh->indptr && mesh->cols) {
        for (int i = 0; i <= m->n; i++) if (mesh->indptr[i] != ip[i]) { g_err = "sw2g_create: caller CSR row pointers differ from the reference sparsity"; return fail(SW2G_ERR_MESH); }
        for (int k = 0; k < m->nnz; k++) if (mesh->cols[k] != cl[k]) { g_err = "sw2g_create: caller CSR columns differ from the reference sparsity"; return fail(SW2G_ERR_MESH); }
    }
    std::vector<int> bptr(V + 1, 0), bcol, diag(m->n);
    for (int a = 0; a < V; a++) {
        int len = ip[3 * a + 1] - ip[3 * a];
        bptr[a + 1] = bptr[a] + len / 3;
        for (int j = 0; j < len / 3; j++) bcol.push_back(cl[ip[3 * a] + 3 * j] / 3);
    }
    m->nslots = bptr[V];
    m->h_bptr = bptr; m->h_bcol = bcol;
    for (int r = 0; r < m->n; r++) {
        int a = r / 3, j = (int)(std::lower_bound(bcol.begin() + bptr[a], bcol.begin() + bptr[a + 1], a) - bcol.begin()) - bptr[a];
        diag[r] = ip[r] + 3 * j + r % 3;
    }

    // --- deterministic assembly maps, in element order (triangles, then segments)
    std::vector<int> rptr(V + 1, 0);
    for (int e = 0; e < T; e++) for (int a = 0; a < 3; a++) rptr[mesh->tri[3 * e + a] + 1]++;
    for (int s = 0; s < S; s++) for (int a = 0; a < 2; a++) rptr[mesh->seg[2 * s + a] + 1]++;
    for (int i = 0; i < V; i++) rptr[i + 1] += rptr[i];
    std::vector<uint32_t> rmap(rptr[V]);
    {
        std::vector<int> fill(rptr.begin(), rptr.end() - 1);
        for (int e = 0; e < T; e++) for (int a = 0; a < 3; a++) rmap[fill[mesh->tri[3 * e + a]]++] = (uint32_t)(3 * e + a);
        for (int s = 0; s < S; s++) for (int a = 0; a < 2; a++) rmap[fill[mesh->seg[2 * s + a]]++] = (uint32_t)(3 * (T + s) + a);
    }
    auto slot = [&](int a, int b) -> int {
        auto it = std::lower_bound(bcol.begin() + bptr[a], bcol.begin() + bptr[a + 1], b);
        return (int)(it - bcol.begin());
    };
    std::vector<int> jptr(m->nslots + 1, 0);
    std::vector<int> eslot(9 * (size_t)T + 4 * (size_t)S);
    for (int e = 0; e < T; e++) for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) {
        int k = slot(mesh->tri[3 * e + a], mesh->tri[3 * e + b]);
        eslot[9 * (size_t)e + 3 * a + b] = k; jptr[k + 1]++;
    }
    for (int s = 0; s < S; s++) for (int a = 0; a < 2; a++) for (int b = 0; b < 2; b++) {
        int k = slot(mesh->seg[2 * s + a], mesh->seg[2 * s + b]);
        eslot[9 * (size_t)T + 4 * (size_t)s + 2 * a + b] = k; jptr[k + 1]++;
    }
    for (int k = 0; k < m->nslots; k++) jptr[k + 1] += jptr[k];
    std::vector<uint32_t> jmap(jptr[m->nslots]);
    {
        std::vector<int> fill(jptr.begin(), jptr.end() - 1);
        for (int e = 0; e < T; e++) for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++)
            jmap[fill[eslot[9 * (size_t)e + 3 * a + b]]++] = (uint32_t)(9 * e + 3 * a + b);
        for (int s = 0; s < S; s++) for (int a = 0; a < 2; a++) for (int b = 0; b < 2; b++)
            jmap[fill[eslot[9 * (size_t)T + 4 * (size_t)s + 2 * a + b]]++] = (uint32_t)(9 * (T + s) + 3 * a + b);
    }
    std::vector<int> boff(m->nslots), blen(m->nslots);
    for (int a = 0; a < V; a++) for (int k = bptr[a]; k < bptr[a + 1]; k++) {
        boff[k] = ip[3 * a] + 3 * (k - bptr[a]);
        blen[k] = ip[3 * a + 1] - ip[3 * a];
    }

    // --- greedy colouring of the node graph for the block-ILU sweeps
    std::vector<int> color(V, -1);
    int ncolors = 0;
    {
        std::vector<int> seen(64, -1);
        for (int a = 0; a < V; a++) {
            if (bptr[a + 1] - bptr[a] > 32) { g_err = "sw2g_create: a node has more than 31 neighbours"; return fail(SW2G_ERR_MESH); }
            for (int k = bptr[a]; k < bptr[a + 1]; k++) if (color[bcol[k]] >= 0) seen[color[bcol[k]]] = a;
            int c = 0;
            while (seen[c] == a) c++;
            color[a] = c;
            ncolors = std::max(ncolors, c + 1);
        }
    }
    std::vector<int> color_nodes(V);
    m->h_color_ptr.assign(ncolors + 1, 0);
    for (int a = 0; a < V; a++) m->h_color_ptr[color[a] + 1]++;
    for (int c = 0; c < ncolors; c++) m->h_color_ptr[c + 1] += m->h_color_ptr[c];
    {
        std::vector<int> fill(m->h_color_ptr.begin(), m->h_color_ptr.end() - 1);
        for (int a = 0; a < V; a++) color_nodes[fill[color[a]]++] = a;
    }

    // --- device copies
    if ((rc = upload(m, &m->d_tri, mesh->tri, 3 * (size_t)T))) return fail(rc);
    std::vector<int> segv(2 * (size_t)S + 2, 0), kindv(S + 1, 0);
    for (long i = 0; i < 2L * S; i++) segv[i] = mesh->seg[i];
    for (int i = 0; i < S; i++) kindv[i] = mesh->seg_kind[i];
    if ((rc = upload(m, &m->d_seg, segv.data(), segv.size()))) return fail(rc);
    if ((rc = upload(m, &m->d_skind, kindv.data(), kindv.size()))) return fail(rc);
    if ((rc = upload(m, &m->d_ex, ex.data(), ex.size())) || (rc = upload(m, &m->d_ey, ey.data(), ey.size())) ||
        (rc = upload(m, &m->d_ez, ez.data(), ez.size())) || (rc = upload(m, &m->d_gx, gx.data(), gx.size())) ||
        (rc = upload(m, &m->d_gy, gy.data(), gy.size())) || (rc = upload(m, &m->d_djac, dj.data(), dj.size())) ||
        (rc = upload(m, &m->d_snx, snx.data(), snx.size())) || (rc = upload(m, &m->d_sny, sny.data(), sny.size())) ||
        (rc = upload(m, &m->d_sdjac, sdj.data(), sdj.size())) || (rc = upload(m, &m->d_sz0, sz0.data(), sz0.size())))
        return fail(rc);
    if ((rc = upload(m, &m->d_indptr, ip.data(), ip.size())) || (rc = upload(m, &m->d_cols, cl.data(), cl.size())) ||
        (rc = upload(m, &m->d_bptr, bptr.data(), bptr.size())) || (rc = upload(m, &m->d_bcol, bcol.data(), bcol.size())) ||
        (rc = upload(m, &m->d_diag, diag.data(), diag.size())) || (rc = upload(m, &m->d_rptr, rptr.data(), rptr.size())) ||
        (rc = upload(m, &m->d_rmap, rmap.data(), rmap.size())) || (rc = upload(m, &m->d_jptr, jptr.data(), jptr.size())) ||
        (rc = upload(m, &m->d_jmap, jmap.data(), jmap.size())) || (rc = upload(m, &m->d_boff, boff.data(), boff.size())) ||
        (rc = upload(m, &m->d_blen, blen.data(), blen.size())) ||
        (rc = upload(m, &m->d_color_nodes, color_nodes.data(), color_nodes.size())) ||
        (rc = upload(m, &m->d_node_color, color.data(), color.size())) || (rc = dalloc(m, &m->d_lu, (size_t)m->nnz)))
        return fail(rc);
    m->ilu = IluHost{ncolors, m->h_color_ptr.data(), IluView{m->d_color_nodes, m->d_node_color, nullptr}};
    const size_t n = m->n;
    if ((rc = dalloc(m, &m->d_sol, n)) || (rc = dalloc(m, &m->d_sol_old, n)) || (rc = dalloc(m, &m->d_sol_older, n)) ||
        (rc = dalloc(m, &m->d_dirichlet, n)) || (rc = dalloc(m, &m->d_guess, n)) || (rc = dalloc(m, &m->d_bc_mask, n)) ||
        (rc = dalloc(m, &m->d_wd, T)) || (rc = dalloc(m, &m->d_node_tmp, V)) ||
        (rc = dalloc(m, &m->d_ER, 9 * (size_t)m->Etot)) || (rc = dalloc(m, &m->d_EJ, 81 * (size_t)m->Etot)) ||
        (rc = dalloc(m, &m->d_res, n)) || (rc = dalloc(m, &m->d_vals, (size_t)m->nnz)) || (rc = dalloc(m, &m->d_dsol, n)) ||
        (rc = dalloc(m, &m->d_scale, n)) || (rc = dalloc(m, &m->d_inv, 9 * (size_t)V)) || (rc = dalloc(m, &m->d_x0, n)) ||
        (rc = dalloc(m, &m->d_b64, n)) || (rc = dalloc(m, &m->d_t64, 2 * (size_t)n)) ||
        (rc = dalloc(m, &m->k_r, n)) || (rc = dalloc(m, &m->k_p, n)) || (rc = dalloc(m, &m->k_Ap, n)) ||
        (rc = dalloc(m, &m->k_q, n)) || (rc = dalloc(m, &m->k_s, n)) || (rc = dalloc(m, &m->k_As, n)) ||
        (rc = dalloc(m, &m->k_z, n)) || (rc = dalloc(m, &m->k_xi, n)) ||
        (rc = dalloc(m, &m->d_partial, 4 * (size_t)kMaxBlocks)) || (rc = dalloc(m, &m->d_rout, 8)) ||
        (rc = dalloc(m, &m->d_counter, 1)) || (rc = dalloc(m, &m->d_ks, 1)))
        return fail(rc);
    CK(cudaMemsetAsync(m->d_counter, 0, sizeof(unsigned int), m->st));
    CK(cudaMemsetAsync(m->d_bc_mask, 0, sizeof(int) * n, m->st));
    CK(cudaMemsetAsync(m->d_dirichlet, 0, sizeof(double) * n, m->st));
    CK(cudaMemsetAsync(m->d_EJ, 0, sizeof(double) * 81 * (size_t)m->Etot, m->st));
    CK(cudaMemsetAsync(m->d_ER, 0, sizeof(double) * 9 * (size_t)m->Etot, m->st));
    if (cudaMallocHost((void**)&m->h_rout, 8 * sizeof(double)) != cudaSuccess ||
        cudaMallocHost((void**)&m->h_ks, sizeof(KrylovScalars)) != cudaSuccess) {
        g_err = "cudaMallocHost failed"; return fail(SW2G_ERR_NOMEM);
    }
    m->M = MeshView{V, T, S, m->d_tri, m->d_ex, m->d_ey, m->d_ez, m->d_gx, m->d_gy, m->d_djac,
                    m->d_seg, m->d_snx, m->d_sny, m->d_sdjac, m->d_skind, m->d_sz0};
    m->A = AssemblyMaps{m->nslots, m->d_rptr, m->d_rmap, m->d_jptr, m->d_jmap, m->d_boff, m->d_blen};
    m->B = BlockCSR{V, m->n, m->nnz, m->d_indptr, m->d_cols, m->d_bptr, m->d_bcol, m->d_diag};
    m->P = StepParams{1.0, 0.0, mesh->gravity, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0};
    CK(cudaStreamSynchronize(m->st));
    *out = m;
    return SW2G_OK;
}

static int alloc_fp32(sw2g_model* m) {
    if (m->f_vals) return SW2G_OK;
    const size_t n = m->n;
    TRY(dalloc(m, &m->f_vals, (size_t)m->nnz)); TRY(dalloc(m, &m->f_inv, 9 * (size_t)m->V));
    TRY(dalloc(m, &m->f_x, n)); TRY(dalloc(m, &m->f_r, n)); TRY(dalloc(m, &m->f_p, n)); TRY(dalloc(m, &m->f_Ap, n));
    TRY(dalloc(m, &m->f_q, n)); TRY(dalloc(m, &m->f_s, n)); TRY(dalloc(m, &m->f_As, n)); TRY(dalloc(m, &m->f_b, n));
    TRY(dalloc(m, &m->f_z, n));
    TRY(dalloc(m, &m->f_lu, (size_t)m->nnz));
    return SW2G_OK;
}

extern "C" void sw2g_destroy(sw2g_model* m) {
    if (!m) return;
    if (m->st) cudaStreamSynchronize(m->st);
    for (int k = 0; k < 3; k++) {
        if (m->graph64[k]) cudaGraphExecDestroy(m->graph64[k]);
        if (m->graph32[k]) cudaGraphExecDestroy(m->graph32[k]);
    }
    if (m->gm_graph64) cudaGraphExecDestroy(m->gm_graph64);
    if (m->gm_graph32) cudaGraphExecDestroy(m->gm_graph32);
    if (m->gm_graph_b32) cudaGraphExecDestroy(m->gm_graph_b32);
    for (void* p : m->allocs) cudaFree(p);
    if (m->h_rout) cudaFreeHost(m->h_rout);
    if (m->h_ks) cudaFreeHost(m->h_ks);
    if (m->h_pflag) cudaFreeHost(m->h_pflag);
    if (m->h_cptr) cudaFreeHost(m->h_cptr);
    if (m->h_cown) cudaFreeHost(m->h_cown);
    if (m->h_cnode) cudaFreeHost(m->h_cnode);
    if (m->h_crofs) cudaFreeHost(m->h_crofs);
    for (auto& r : m->prof_pending) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (auto e : m->ev_pool) cudaEventDestroy(e);
    if (m->own_stream) cudaStreamDestroy(m->st);
    delete m;
}

extern "C" int sw2g_sizes(const sw2g_model* m, int* ndofs, int* nnz) {
    if (!m) { g_err = "null model"; return SW2G_ERR_ARG; }
    if (ndofs) *ndofs = m->n;
    if (nnz) *nnz = m->nnz;
    return SW2G_OK;
}
extern "C" int sw2g_get_sparsity(const sw2g_model* m, int* indptr, int* cols) {
    if (!m || !indptr || !cols) { g_err = "sw2g_get_sparsity: null argument"; return SW2G_ERR_ARG; }
    memcpy(indptr, m->h_indptr.data(), sizeof(int) * m->h_indptr.size());
    memcpy(cols, m->h_cols.data(), sizeof(int) * m->h_cols.size());
    return SW2G_OK;
}
extern "C" int sw2g_set_step(sw2g_model* m, double dt, double tau, double bc_depth, double bc_vx, double bc_vy) {
    if (!m || !(dt > 0)) { g_err = "sw2g_set_step: bad model or dt"; return SW2G_ERR_ARG; }
    m->P.dt = dt; m->P.alpha = tau; m->P.bc_depth = bc_depth; m->P.bc_vx = bc_vx; m->P.bc_vy = bc_vy;
    return SW2G_OK;
}
extern "C" int sw2g_set_bc_structures(sw2g_model* m, double q_series, double conveyance, double rough_height,
                                      double tail_elev) {
    if (!m) { g_err = "sw2g_set_bc_structures: null model"; return SW2G_ERR_ARG; }
    if (!std::isfinite(q_series) || !std::isfinite(conveyance) || !std::isfinite(rough_height) || !std::isfinite(tail_elev)) {
        g_err = "sw2g_set_bc_structures: non-finite value"; return SW2G_ERR_ARG;
    }
    if (conveyance == 0.0) { g_err = "sw2g_set_bc_structures: zero conveyance"; return SW2G_ERR_ARG; }
    m->P.bc_qs = q_series; m->P.bc_convey = conveyance; m->P.bc_rough = rough_height; m->P.bc_tail = tail_elev;
    return SW2G_OK;
}
extern "C" int sw2g_set_bc_flux(sw2g_model* m, double flux_series) {
    if (!m) { g_err = "sw2g_set_bc_flux: null model"; return SW2G_ERR_ARG; }
    if (!std::isfinite(flux_series)) { g_err = "sw2g_set_bc_flux: non-finite value"; return SW2G_ERR_ARG; }
    m->P.bc_flux = flux_series;
    return SW2G_OK;
}
extern "C" void* sw2g_stream(sw2g_model* m) { return m ? (void*)m->st : nullptr; }
extern "C" int sw2g_device_state(sw2g_model* m, double** sol, double** sol_old, double** sol_older) {
    if (!m) { g_err = "null model"; return SW2G_ERR_ARG; }
    if (sol) *sol = m->d_sol; if (sol_old) *sol_old = m->d_sol_old; if (sol_older) *sol_older = m->d_sol_older;
    return SW2G_OK;
}

// ------------------------------------------------------------------ building blocks
static int do_wd(sw2g_model* m, const double* sol, const double* sol_old) {
    ProfScope ps(m, 5, 3);
    launch_wd_flags(m->M, sol, sol_old, m->d_node_tmp, m->d_wd, m->st);
    CKL();
    return SW2G_OK;
}
static int do_residual(sw2g_model* m, const double* sol, const double* sol_old, const double* sol_older, double* res) {
    ProfScope ps(m, 0, 3);
    launch_elem_resid(m->M, m->P, sol, sol_old, sol_older, m->d_wd, m->d_ER, m->st);
    launch_gather_resid(m->V, m->A, m->d_ER, res, m->st);
    CKL();
    return SW2G_OK;
}
static int do_jacobian(sw2g_model* m, const double* sol, const double* sol_old, const double* sol_older, double* vals) {
    {
        ProfScope ps(m, 1, 4);
        launch_elem_jac(m->M, m->P, sol, sol_old, sol_older, m->d_wd, m->d_EJ, m->st);
        CKL();
    }
    ProfScope ps(m, 2, 1);
    launch_gather_jac(m->A, m->d_EJ, m->Etot, vals, m->st);
    CKL();
    return SW2G_OK;
}
static int do_norms(sw2g_model* m, const double* res, const double* dsol, double* rmax, double* rl2, double* imax) {
    {
        ProfScope ps(m, 5, 1);
        Reduce R{m->d_partial, m->d_counter, m->d_rout};
        launch_norms(m->n, res, dsol, m->d_bc_mask, R, m->st);
        CKL();
    }
    CK(cudaMemcpyAsync(m->h_rout, m->d_rout, 3 * sizeof(double), cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    *rmax = m->h_rout[0]; *rl2 = sqrt(m->h_rout[1]) / m->n; *imax = m->h_rout[2];
    return SW2G_OK;
}
// check_diag + apply_Dirichlet_BC + scale_linear_system on device arrays
static int do_prepare(sw2g_model* m, double* vals, double* res, double* x) {
    ProfScope ps(m, 3, 3);
    launch_check_diag(m->B, vals, m->d_bc_mask, m->st);
    launch_dirichlet_rowscale(m->B, m->d_bc_mask, vals, res, x, m->d_scale, m->st);
    launch_scale_vals(m->B, m->d_scale, vals, m->st);
    CKL();
    return SW2G_OK;
}
static int build_amg(sw2g_model* m);
// preconditioner set-up on the scaled matrix (replaces prep_umfpack, bcgstab_solver.c:371)
static int build_patches(sw2g_model* m, const double* vals);
static void invalidate_graphs(sw2g_model* m);
static int do_precond_setup(sw2g_model* m, const double* vals, int precond, int chunks = 0) {
    if (precond == SW2G_PC_AMG) {
        if (!m->amg_ready) TRY(build_amg(m));
        if (m->amg.patch.mode != chunks) {   // the placement is baked into the captured solver graphs
            invalidate_graphs(m);
            m->amg.patch.mode = chunks;
        }
        {
            ProfScope ps(m, 3, 1 + 4 * (m->amg.nlev - 1));
            amg_setup(m->B, m->amg, m->A, vals, m->st);
            CKL();
        }
        return build_patches(m, vals);
    }
    if (precond == SW2G_PC_BILU0) {
        ProfScope ps(m, 3, 1 + m->ilu.ncolors);
        launch_bilu_factor(m->B, m->ilu, vals, m->d_lu, m->d_inv, m->st);
    } else {
        ProfScope ps(m, 3, 1);
        launch_bj_setup(m->B, vals, m->d_inv, m->st);
    }
    CKL();
    return SW2G_OK;
}

// ------------------------------------------------------------------ AMG hierarchy
// Structure of the aggregation hierarchy, built once per mesh on the host; the
// values are recomputed on the device every Newton iteration by amg_setup.
// Aggregation (greedy, node order): a node whose neighbours are all unassigned
// starts an aggregate with its whole neighbourhood; the leftovers join the
// aggregate of their first assigned neighbour.  Level 0 aggregates the node graph
// of the reference CSR; each coarser level aggregates the previous level's
// block graph, until at most kAmgCoarsest nodes remain.
static int aggregate_nodes(int n, const std::vector<int>& gp, const std::vector<int>& gc, std::vector<int>& agg) {
    agg.assign(n, -1);
    int na = 0;
    for (int i = 0; i < n; i++) {
        if (agg[i] >= 0) continue;
        bool free_ = true;
        for (int q = gp[i]; q < gp[i + 1]; q++) if (agg[gc[q]] >= 0) { free_ = false; break; }
        if (!free_) continue;
        for (int q = gp[i]; q < gp[i + 1]; q++) agg[gc[q]] = na;
        agg[i] = na++;
    }
    for (int i = 0; i < n; i++) {
        if (agg[i] >= 0) continue;
        for (int q = gp[i]; q < gp[i + 1]; q++) if (agg[gc[q]] >= 0) { agg[i] = agg[gc[q]]; break; }
        if (agg[i] < 0) agg[i] = na++;
    }
    return na;
}

static int build_amg(sw2g_model* m) {
    struct HostLev { int n; std::vector<int> bptr, bcol, dpos; };
    struct HostLink { std::vector<int> agg, mptr, mem, gptr, gsrc; };
    std::vector<HostLev> L(1);
    std::vector<HostLink> K;
    L[0].n = m->V; L[0].bptr = m->h_bptr; L[0].bcol = m->h_bcol;
    while ((L.back().n > kAmgCoarsest || L.size() == 1) && (int)L.size() < kAmgMaxLevels) {
        const HostLev& F = L.back();
        HostLink lk;
        const int nc = aggregate_nodes(F.n, F.bptr, F.bcol, lk.agg);
        if (nc >= F.n) break;   // nothing left to coarsen
        lk.mptr.assign(nc + 1, 0);
        for (int i = 0; i < F.n; i++) lk.mptr[lk.agg[i] + 1]++;
        for (int I = 0; I < nc; I++) lk.mptr[I + 1] += lk.mptr[I];
        lk.mem.assign(F.n, 0);
        {
            std::vector<int> fill(lk.mptr.begin(), lk.mptr.end() - 1);
            for (int i = 0; i < F.n; i++) lk.mem[fill[lk.agg[i]]++] = i;
        }
        HostLev C; C.n = nc; C.bptr.assign(nc + 1, 0);
        std::vector<int> row;
        for (int I = 0; I < nc; I++) {
            row.clear();
            for (int t = lk.mptr[I]; t < lk.mptr[I + 1]; t++) {
                const int i = lk.mem[t];
                for (int q = F.bptr[i]; q < F.bptr[i + 1]; q++) row.push_back(lk.agg[F.bcol[q]]);
            }
            std::sort(row.begin(), row.end());
            row.erase(std::unique(row.begin(), row.end()), row.end());
            C.bcol.insert(C.bcol.end(), row.begin(), row.end());
            C.bptr[I + 1] = (int)C.bcol.size();
        }
        // Galerkin gather lists: fine block q (row i, column j) adds into coarse block (agg i, agg j)
        const int nbf = F.bptr[F.n], nbc = (int)C.bcol.size();
        std::vector<int> target(nbf);
        lk.gptr.assign(nbc + 1, 0);
        for (int i = 0; i < F.n; i++) {
            const int I = lk.agg[i];
            for (int q = F.bptr[i]; q < F.bptr[i + 1]; q++) {
                const int J = lk.agg[F.bcol[q]];
                const int t = (int)(std::lower_bound(C.bcol.begin() + C.bptr[I], C.bcol.begin() + C.bptr[I + 1], J) -
                                    C.bcol.begin());
                target[q] = t; lk.gptr[t + 1]++;
            }
        }
        for (int t = 0; t < nbc; t++) lk.gptr[t + 1] += lk.gptr[t];
        lk.gsrc.assign(nbf, 0);
        {
            std::vector<int> fill(lk.gptr.begin(), lk.gptr.end() - 1);
            for (int q = 0; q < nbf; q++) lk.gsrc[fill[target[q]]++] = q;
        }
        K.push_back(std::move(lk));
        L.push_back(std::move(C));
    }
    if (L.size() < 2) { g_err = "amg: the node graph cannot be coarsened"; return SW2G_ERR_MESH; }
    for (size_t l = 1; l < L.size(); l++) {
        HostLev& H = L[l];
        H.dpos.assign(H.n, 0);
        for (int i = 0; i < H.n; i++)
            H.dpos[i] = (int)(std::lower_bound(H.bcol.begin() + H.bptr[i], H.bcol.begin() + H.bptr[i + 1], i) - H.bcol.begin());
    }
    auto up = [&](const int** dst, const std::vector<int>& v) {
        int* d = nullptr;
        int r = upload(m, &d, v.data(), v.size());
        *dst = d;
        return r;
    };
    AmgHost& A = m->amg;
    A.nlev = (int)L.size();
    for (int l = 0; l < A.nlev; l++) {
        AmgLevel& D = A.lev[l];
        const HostLev& H = L[l];
        D.n = H.n;
        const size_t n3 = 3 * (size_t)H.n;
        TRY(dalloc(m, &D.b64, n3)); TRY(dalloc(m, &D.x64, n3)); TRY(dalloc(m, &D.t64, n3)); TRY(dalloc(m, &D.r64, n3));
        TRY(dalloc(m, &D.b32, n3)); TRY(dalloc(m, &D.x32, n3)); TRY(dalloc(m, &D.t32, n3)); TRY(dalloc(m, &D.r32, n3));
        if (l == 0) continue;   // level 0 is the reference CSR itself
        D.nb = (int)H.bcol.size();
        TRY(up(&D.bptr, H.bptr)); TRY(up(&D.bcol, H.bcol)); TRY(up(&D.dpos, H.dpos));
        TRY(dalloc(m, &D.val64, 9 * (size_t)D.nb)); TRY(dalloc(m, &D.val32, 9 * (size_t)D.nb));
        TRY(dalloc(m, &D.dinv64, 9 * (size_t)D.n)); TRY(dalloc(m, &D.dinv32, 9 * (size_t)D.n));
    }
    for (int l = 0; l + 1 < A.nlev; l++) {
        AmgLink& D = A.link[l];
        TRY(up(&D.agg, K[l].agg)); TRY(up(&D.mptr, K[l].mptr)); TRY(up(&D.mem, K[l].mem));
        TRY(up(&D.gptr, K[l].gptr)); TRY(up(&D.gsrc, K[l].gsrc));
    }
    TRY(dalloc(m, &A.dinv0_64, 9 * (size_t)m->V)); TRY(dalloc(m, &A.dinv0_32, 9 * (size_t)m->V));
    {   // chunk corrections: flags and counters now, the chunk buffers on the first build
        PatchDev& P = A.patch;
        TRY(dalloc(m, &P.flag, (size_t)m->V)); TRY(dalloc(m, &P.counts, 2)); TRY(dalloc(m, &P.failed, 1));
        CK(cudaMemsetAsync(P.counts, 0, 2 * sizeof(int), m->st));
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device);
        P.grid = 4 * (sms > 0 ? sms : 148);
        P.mode = 0;   // set per solve from sw2g_newton_opts.amg_chunks
        if (cudaMallocHost((void**)&m->h_pflag, sizeof(int) * (size_t)m->V) != cudaSuccess) {
            g_err = "cudaMallocHost failed"; return SW2G_ERR_NOMEM;
        }
    }
    m->amg_ready = true;
    static const bool trace = getenv("SW2G_TRACE_KRYLOV") != nullptr;
    if (trace) {
        fprintf(stderr, "amg levels:");
        for (auto& h : L) fprintf(stderr, " %d(%zu)", h.n, h.bcol.size());
        fprintf(stderr, "\n");
    }
    return SW2G_OK;
}

// Drops every captured solver graph (their kernels hold buffer addresses that are about to change).
static void invalidate_graphs(sw2g_model* m) {
    cudaStreamSynchronize(m->st);
    for (int k = 0; k < 3; k++) {
        if (m->graph64[k]) { cudaGraphExecDestroy(m->graph64[k]); m->graph64[k] = nullptr; }
        if (m->graph32[k]) { cudaGraphExecDestroy(m->graph32[k]); m->graph32[k] = nullptr; }
    }
    if (m->gm_graph64) { cudaGraphExecDestroy(m->gm_graph64); m->gm_graph64 = nullptr; }
    if (m->gm_graph32) { cudaGraphExecDestroy(m->gm_graph32); m->gm_graph32 = nullptr; }
    if (m->gm_graph_b32) { cudaGraphExecDestroy(m->gm_graph_b32); m->gm_graph_b32 = nullptr; }
    m->gm_m64 = m->gm_m32 = m->gm_mb32 = -1;
}

// Chunks of the flagged nodes for the AMG's level-0 corrections (amg_kernels.cu).  The
// patch set is every node whose smoother block the l1 fix-up weakened (flags written by
// amg_setup) plus its neighbours.  Its nodes are taken tile by tile (tiles of
// kPatchTileEdges mean edge lengths), in node order within a tile; a chunk owns a run of
// them and extends over their neighbours in the patch set, closed before it would pass
// kPatchMaxNodes nodes.  Own nodes are listed first.  Deterministic: the same flags give
// the same chunks.  The chunk blocks are then inverted on the device.
static int build_patches(sw2g_model* m, const double* vals) {
    PatchDev& P = m->amg.patch;
    const int V = m->V;
    if (P.mode == 0) return SW2G_OK;
    ProfScope ps(m, 3, 1);
    CK(cudaMemcpyAsync(m->h_pflag, P.flag, sizeof(int) * (size_t)V, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    const std::vector<int>& bp = m->h_bptr;
    const std::vector<int>& bc = m->h_bcol;
    std::vector<char> inp(V, 0);
    int nflag = 0;
    for (int i = 0; i < V; i++)
        if (m->h_pflag[i]) {
            nflag++;
            for (int q = bp[i]; q < bp[i + 1]; q++) inp[bc[q]] = 1;
        }
    std::vector<std::pair<long long, int>> pn;
    for (int i = 0; i < V; i++) if (inp[i]) pn.emplace_back(m->h_tile[i], i);
    std::sort(pn.begin(), pn.end());
    std::vector<int> cptr(1, 0), cown, cnode;
    std::vector<long long> crofs;
    std::vector<int> stamp(V, -1);
    std::vector<char> role(V, 0);   // 1 own, 0 ring
    std::vector<int> own, members;
    long long rtot = 0;
    int piece = 0;
    auto finalize = [&]() {
        if (own.empty()) return;
        for (int a : own) cnode.push_back(a);
        for (int a : members) if (!role[a]) cnode.push_back(a);
        const int ne = (int)cnode.size() - cptr.back();
        crofs.push_back(rtot);
        rtot += 9LL * (long long)own.size() * ne;
        cown.push_back((int)own.size());
        cptr.push_back((int)cnode.size());
        own.clear(); members.clear();
        piece++;
    };
    for (size_t k = 0; k < pn.size(); k++) {
        if (k > 0 && pn[k].first != pn[k - 1].first) finalize();
        const int a = pn[k].second;
        int add = (stamp[a] != piece) ? 1 : 0;
        for (int q = bp[a]; q < bp[a + 1]; q++) { const int b = bc[q]; if (inp[b] && stamp[b] != piece && b != a) add++; }
        if ((int)members.size() + add > kPatchMaxNodes) finalize();
        if (stamp[a] != piece) { stamp[a] = piece; members.push_back(a); }
        role[a] = 1;
        own.push_back(a);
        for (int q = bp[a]; q < bp[a + 1]; q++) {
            const int b = bc[q];
            if (inp[b] && stamp[b] != piece) { stamp[b] = piece; role[b] = 0; members.push_back(b); }
        }
    }
    finalize();
    const int nch = (int)cown.size(), nent = (int)cnode.size();
    // capacities (grown with headroom; growing changes addresses the captured graphs hold)
    if (m->pcap_chunks == 0 || nch > m->pcap_chunks || nent > m->pcap_entries || rtot > m->pcap_r) {
        invalidate_graphs(m);
        const int cc = std::max(m->pcap_chunks, nch + nch / 4 + 64);
        const int ce = std::max(m->pcap_entries, nent + nent / 4 + 256);
        const long long cr = std::max(m->pcap_r, rtot + rtot / 4 + 4096);
        dfree(m, &P.chunk_ptr); dfree(m, &P.own_cnt); dfree(m, &P.rofs); dfree(m, &P.ext_node);
        dfree(m, &P.r64); dfree(m, &P.r32); dfree(m, &P.e64); dfree(m, &P.e32);
        TRY(dalloc(m, &P.chunk_ptr, (size_t)cc + 1)); TRY(dalloc(m, &P.own_cnt, (size_t)cc));
        TRY(dalloc(m, &P.rofs, (size_t)cc)); TRY(dalloc(m, &P.ext_node, (size_t)ce));
        TRY(dalloc(m, &P.r64, (size_t)cr)); TRY(dalloc(m, &P.r32, (size_t)cr));
        TRY(dalloc(m, &P.e64, 3 * (size_t)ce)); TRY(dalloc(m, &P.e32, 3 * (size_t)ce));
        if (m->h_cptr) { cudaFreeHost(m->h_cptr); cudaFreeHost(m->h_cown); cudaFreeHost(m->h_cnode); cudaFreeHost(m->h_crofs); }
        if (cudaMallocHost((void**)&m->h_cptr, sizeof(int) * ((size_t)cc + 3)) != cudaSuccess ||
            cudaMallocHost((void**)&m->h_cown, sizeof(int) * (size_t)cc) != cudaSuccess ||
            cudaMallocHost((void**)&m->h_cnode, sizeof(int) * (size_t)ce) != cudaSuccess ||
            cudaMallocHost((void**)&m->h_crofs, sizeof(long long) * (size_t)cc) != cudaSuccess) {
            g_err = "cudaMallocHost failed"; return SW2G_ERR_NOMEM;
        }
        m->pcap_chunks = cc; m->pcap_entries = ce; m->pcap_r = cr;
    }
    // staging: chunk_ptr [nch+1], then the two counts in the slots after it
    std::copy(cptr.begin(), cptr.end(), m->h_cptr);
    std::copy(cown.begin(), cown.end(), m->h_cown);
    std::copy(cnode.begin(), cnode.end(), m->h_cnode);
    std::copy(crofs.begin(), crofs.end(), m->h_crofs);
    m->h_cptr[nch + 1] = nch; m->h_cptr[nch + 2] = nent;
    CK(cudaMemcpyAsync(P.chunk_ptr, m->h_cptr, sizeof(int) * ((size_t)nch + 1), cudaMemcpyHostToDevice, m->st));
    CK(cudaMemcpyAsync(P.counts, m->h_cptr + nch + 1, 2 * sizeof(int), cudaMemcpyHostToDevice, m->st));
    if (nch > 0) {
        CK(cudaMemcpyAsync(P.own_cnt, m->h_cown, sizeof(int) * (size_t)nch, cudaMemcpyHostToDevice, m->st));
        CK(cudaMemcpyAsync(P.rofs, m->h_crofs, sizeof(long long) * (size_t)nch, cudaMemcpyHostToDevice, m->st));
        CK(cudaMemcpyAsync(P.ext_node, m->h_cnode, sizeof(int) * (size_t)nent, cudaMemcpyHostToDevice, m->st));
    }
    CK(cudaMemsetAsync(P.failed, 0, sizeof(int), m->st));
    patch_invert(m->B, P, vals, nch, m->st);
    CKL();
    m->p_nchunks = nch; m->p_nentries = nent; m->p_nflag = nflag; m->p_rtot = rtot;
    static const bool trace = getenv("SW2G_TRACE_KRYLOV") != nullptr;
    if (trace) {
        int failed = 0;
        CK(cudaMemcpyAsync(&failed, P.failed, sizeof(int), cudaMemcpyDeviceToHost, m->st));
        CK(cudaStreamSynchronize(m->st));
        fprintf(stderr, "amg chunks: %d flagged nodes, %zu patch nodes, %d chunks, %d entries, %lld inverse entries, %d singular\n",
                nflag, pn.size(), nch, nent, rtot, failed);
    }
    return SW2G_OK;
}

// kernel launches of one preconditioner application (profiling counts)
static int precond_launches(const sw2g_model* m, int precond) {
    if (precond == SW2G_PC_BILU0) return 2 * m->ilu.ncolors;
    if (precond == SW2G_PC_AMG) return 1 + (m->amg.nlev - 1) * (2 * kAmgNu + 4) + 1 + 2;
    return 1;
}

template <class VT>
static int run_bicg(sw2g_model* m, KrylovVecs<VT> V, int precond, cudaGraphExec_t* graph, int max_it, double atol,
                    double rtol, int* iters, int* status) {
    KrylovScalars init{};
    init.tol = atol; init.rtol = rtol; init.max_it = max_it;
    Reduce R{m->d_partial, m->d_counter, m->d_rout};
    const bool pc = precond != SW2G_PC_BLOCK_JACOBI;
    PrecondOp<VT> op;
    op.kind = precond; op.ilu = &m->ilu; op.lu = V.vals_pc; op.dinv = V.inv; op.amg = &m->amg; op.vals = V.vals;
    op.right = precond == SW2G_PC_AMG;
    const int per_apply = precond == SW2G_PC_BILU0 ? 2 * m->ilu.ncolors : precond_launches(m, precond);
    {
        ProfScope ps(m, 4, pc ? 3 + 2 * per_apply : 2);
        CK(cudaMemcpyAsync(m->d_ks, &init, sizeof(KrylovScalars), cudaMemcpyHostToDevice, m->st));
        if (pc) launch_bicg_init_pc<VT>(m->B, op, V, m->d_ks, R, m->st);
        else launch_bicg_init<VT>(m->B, V, m->d_ks, R, m->st);
        CKL();
    }
    if (!*graph) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(m->st, cudaStreamCaptureModeThreadLocal));
        for (int c = 0; c < kChunk; c++) {
            if (pc) launch_bicg_iteration_pc<VT>(m->B, op, V, m->d_ks, R, m->st);
            else launch_bicg_iteration<VT>(m->B, V, m->d_ks, R, m->st);
        }
        cudaError_t e1 = cudaGetLastError();
        cudaError_t e2 = cudaStreamEndCapture(m->st, &g);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            g_err = std::string("graph capture: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2);
            return SW2G_ERR_CUDA;
        }
        CK(cudaGraphInstantiate(graph, g, 0));
        cudaGraphDestroy(g);
    }
    const int per_it = pc ? 6 + 2 * per_apply : 4;
    static const bool trace = getenv("SW2G_TRACE_KRYLOV") != nullptr;   // diagnostic: residual history on stderr
    while (true) {
        CK(cudaMemcpyAsync(m->h_ks, m->d_ks, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, m->st));
        CK(cudaStreamSynchronize(m->st));
        if (trace)
            fprintf(stderr, "krylov it %d rnorm %.3e bnorm %.3e rel %.3e\n", m->h_ks->it, m->h_ks->rnorm, m->h_ks->bnorm,
                    m->h_ks->rnorm / (m->h_ks->bnorm > 0 ? m->h_ks->bnorm : 1.0));
        if (m->h_ks->done) break;
        ProfScope ps(m, 4, per_it * kChunk);
        CK(cudaGraphLaunch(*graph, m->st));
    }
    if (op.right) {   // x holds y of A M^-1 y = b: x = M^-1 y
        ProfScope ps(m, 4, per_apply);
        precond_apply<VT>(m->B, op, V.x, nullptr, m->st);
        CKL();
    }
    *iters = m->h_ks->it;
    *status = m->h_ks->status;
    // status 3: the iteration cap ended the solve before its stopping test held
    if (*status == 0 && !(m->h_ks->rnorm <= m->h_ks->tol + m->h_ks->bnorm * m->h_ks->rtol)) *status = 3;
    return SW2G_OK;
}

// Left-preconditioned BiCGStab of bcgstab_solver.c:65-330 on the prepared (scaled)
// system in d_vals: x (= dsol) in/out with the reference's x0 shift and unscaling;
// b is overwritten with M^-1 b as in the reference.
static int solve64(sw2g_model* m, double* x, double* b, int precond, int max_it, double tol, int* iters, int* status) {
    CK(cudaMemcpyAsync(m->d_x0, x, sizeof(double) * m->n, cudaMemcpyDeviceToDevice, m->st));
    KrylovVecs<double> V{x, m->k_r, m->k_p, m->k_Ap, m->k_q, m->k_s, m->k_As, b, m->d_vals, m->d_inv, m->d_lu, m->k_z};
    TRY(run_bicg<double>(m, V, precond, &m->graph64[precond], max_it, tol, tol, iters, status));
    ProfScope ps(m, 5, 1);
    launch_unscale(m->n, m->d_x0, m->d_scale, x, m->st);
    CKL();
    return SW2G_OK;
}

// AMG path in FP64: right-preconditioned BiCGStab, restarted from the true FP64
// residual after a breakdown or when the iteration budget of a pass ends, until
// max|b - A x| <= tol + tol * max|b| on the scaled system.  A pass that does not
// lower the residual is taken back and ends the solve (status 4).
static int solve64_restarted(sw2g_model* m, double* x, double* b, int max_it, double tol, int max_restart, int* iters,
                             int* passes, int* status) {
    const int n = m->n;
    Reduce R{m->d_partial, m->d_counter, m->d_rout};
    CK(cudaMemcpyAsync(m->d_x0, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, m->st));
    CK(cudaMemcpyAsync(m->d_b64, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, m->st));
    CK(cudaMemsetAsync(x, 0, sizeof(double) * n, m->st));
    *iters = 0; *passes = 0; *status = 0;
    double bn = -1, prev = 0;
    for (int pass = 0;; pass++) {
        {
            ProfScope ps(m, 4, 2);
            launch_spmv_sub(m->B, m->d_vals, x, m->d_b64, m->d_t64, m->st);
            launch_maxabs(n, m->d_t64, R, m->st);
            CKL();
        }
        CK(cudaMemcpyAsync(m->h_rout, m->d_rout, sizeof(double), cudaMemcpyDeviceToHost, m->st));
        CK(cudaStreamSynchronize(m->st));
        const double rn = m->h_rout[0];
        if (bn < 0) bn = rn;
        if (!std::isfinite(rn)) { *status = 2; break; }
        const double target = tol + tol * bn;
        if (!(rn > target)) break;
        if (pass > 0 && !(rn < prev)) {
            ProfScope ps(m, 5, 1);
            launch_axpy(n, -1.0, m->k_xi, x, m->st);
            CKL();
            if (!*status) *status = 4;
            break;
        }
        if (pass > max_restart || *iters >= max_it) { *status = 3; break; }
        prev = rn;
        KrylovVecs<double> V{m->k_xi, m->k_r, m->k_p, m->k_Ap, m->k_q, m->k_s, m->k_As, m->d_t64, m->d_vals, m->d_inv,
                             m->d_lu, m->k_z};
        int it = 0, st = 0;
        TRY(run_bicg<double>(m, V, SW2G_PC_AMG, &m->graph64[SW2G_PC_AMG], max_it - *iters, target, 0.0, &it, &st));
        *iters += it; *passes += 1;
        if (st == 2) { *status = 2; break; }
        {
            ProfScope ps(m, 5, 1);
            launch_axpy(n, 1.0, m->k_xi, x, m->st);
            CKL();
        }
    }
    ProfScope ps(m, 5, 1);
    launch_unscale(n, m->d_x0, m->d_scale, x, m->st);
    CKL();
    return SW2G_OK;
}

// ------------------------------------------------------------------ restarted GMRES
static int alloc_gmres(sw2g_model* m) {
    if (!m->gm.H) {
        GmresDev& G = m->gm;
        TRY(dalloc(m, &G.H, (size_t)kGmM * (kGmM + 1))); TRY(dalloc(m, &G.cs, kGmM)); TRY(dalloc(m, &G.sn, kGmM));
        TRY(dalloc(m, &G.H2, kGmM + 1));
        TRY(dalloc(m, &G.g, kGmM + 1)); TRY(dalloc(m, &G.y, kGmM));
        TRY(dalloc(m, &G.partial, (size_t)kMaxBlocks * (kGmM + 1)));
        TRY(dalloc(m, &G.counter, 1)); TRY(dalloc(m, &G.state, 4)); TRY(dalloc(m, &G.scal, 8));
        CK(cudaMemsetAsync(G.counter, 0, sizeof(unsigned int), m->st));
    }
    if (!m->gm_rw) TRY(dalloc(m, &m->gm_rw, (size_t)m->n));
    return SW2G_OK;
}

// Stride of the Krylov basis: n rounded up to 4 entries, so that every basis vector
// starts on a 16-byte boundary (the Gram-Schmidt kernels read 16 bytes per load)
static size_t gm_ld(int n) { return ((size_t)n + 3) & ~(size_t)3; }

// Krylov basis of mres + 1 vectors, grown when a longer restart is asked for
template <class T>
static int gmres_basis(sw2g_model* m, T** V, int* cap, int mres) {
    if (*V && *cap >= mres) return SW2G_OK;
    CK(cudaStreamSynchronize(m->st));
    dfree(m, V);
    TRY(dalloc(m, V, (size_t)(mres + 1) * gm_ld(m->n)));
    *cap = mres;
    return SW2G_OK;
}

// classical Gram-Schmidt with one re-orthogonalisation pass (SW2G_GM_REORTH=1; diagnostic switch)
static bool gm_reorth() {
    static const bool on = getenv("SW2G_GM_REORTH") != nullptr && getenv("SW2G_GM_REORTH")[0] == '1';
    return on;
}

// FP32 cycle: FP32 basis, FP32 matrix and FP32 preconditioner on the FP32 right-hand side f_b; the
// correction lands in f_x (the FP64 residual and the update stay with the caller)
static int gmres_graph32(sw2g_model* m, cudaGraphExec_t* graph, int* built_m, int precond, int mres) {
    if (*graph && *built_m == mres) return SW2G_OK;
    if (*graph) { cudaGraphExecDestroy(*graph); *graph = nullptr; }
    *built_m = mres;
    PrecondOp<float> op;
    op.kind = precond; op.right = true; op.ilu = &m->ilu; op.lu = m->f_lu; op.dinv = m->f_inv; op.amg = &m->amg;
    op.vals = m->f_vals;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(m->st, cudaStreamCaptureModeThreadLocal));
    gmres_cycle<float>(m->B, op, m->f_vals, m->gm_V32, gm_ld(m->n), m->f_z, m->f_b, m->f_x, m->gm_rw, m->gm, m->st,
                       mres, gm_reorth());
    cudaError_t e1 = cudaGetLastError();
    cudaError_t e2 = cudaStreamEndCapture(m->st, &g);
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
        g_err = std::string("graph capture: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2);
        return SW2G_ERR_CUDA;
    }
    CK(cudaGraphInstantiate(graph, g, 0));
    cudaGraphDestroy(g);
    return SW2G_OK;
}

static int gmres_graph(sw2g_model* m, cudaGraphExec_t* graph, int* built_m, bool mixed, int precond, int mres) {
    if (*graph && *built_m == mres) return SW2G_OK;
    if (*graph) { cudaGraphExecDestroy(*graph); *graph = nullptr; }
    *built_m = mres;
    PrecondOp<double> op;
    op.kind = precond; op.right = true; op.ilu = &m->ilu; op.lu = m->d_lu; op.dinv = m->d_inv; op.amg = &m->amg;
    op.vals = m->d_vals;
    if (mixed) { op.mixed = true; op.vals32 = m->f_vals; op.lu32 = m->f_lu; op.dinv32 = m->f_inv; op.tmp32 = m->f_z; }
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(m->st, cudaStreamCaptureModeThreadLocal));
    gmres_cycle<double>(m->B, op, m->d_vals, m->gm_V64, gm_ld(m->n), m->k_z, m->d_t64, m->k_xi, m->gm_rw, m->gm,
                        m->st, mres, gm_reorth());
    cudaError_t e1 = cudaGetLastError();
    cudaError_t e2 = cudaStreamEndCapture(m->st, &g);
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
        g_err = std::string("graph capture: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2);
        return SW2G_ERR_CUDA;
    }
    CK(cudaGraphInstantiate(graph, g, 0));
    cudaGraphDestroy(g);
    return SW2G_OK;
}

// Restarted GMRES(kGmM) on the prepared (scaled) system, FP64 Krylov basis.  Each
// pass forms the FP64 residual t = b - A x, runs one right-preconditioned cycle
// on it and adds the correction.  The cycle minimises the 2-norm of the UNSCALED
// residual S^-1 t (row weights 1/s), the quantity the Newton test looks at; the
// symmetric scaling still conditions the operator and the AMG hierarchy.  With `mixed` the preconditioner runs in FP32
// (FP32 matrix values, block inverses and AMG hierarchy on a rounded copy of the
// vector): half the bytes of the dominant kernels, while the Krylov recurrence
// and the residuals stay FP64, so the attainable accuracy is the FP64 one.
// Stopping is inexact-Newton style on the UNSCALED linear residual r = S^-1 t:
// max|r| <= max(krylov_tol * fnorm, floor), floor = 0.1 tol_nonlin (0.01 under the absolute test), fnorm the current
// Newton residual max-norm, so the Newton loop can reach tol_nonlin on the
// reference's unscaled residual.  Also stops after krylov_max_it inner iterations
// or when three passes in a row lower max|r| by less than 1% (status 4).
static int solve_gmres(sw2g_model* m, double* x, double* b, const sw2g_newton_opts& o, bool mixed, double fnorm,
                       int* iters, int* passes, int* status) {
    const int n = m->n;
    const int mres = (o.krylov_restart >= 1 && o.krylov_restart <= kGmM) ? o.krylov_restart : kGmDefault;
    TRY(alloc_gmres(m));
    if (mixed) TRY(alloc_fp32(m));
    Reduce R{m->d_partial, m->d_counter, m->d_rout};
    CK(cudaMemcpyAsync(m->d_x0, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, m->st));
    CK(cudaMemcpyAsync(m->d_b64, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, m->st));
    CK(cudaMemsetAsync(x, 0, sizeof(double) * n, m->st));
    if (mixed) {
        ProfScope ps(m, 3, o.precond == SW2G_PC_BILU0 ? 3 : 2);
        launch_to_float(m->nnz, m->d_vals, m->f_vals, m->st);
        launch_to_float(9 * m->V, m->d_inv, m->f_inv, m->st);
        if (o.precond == SW2G_PC_BILU0) launch_to_float(m->nnz, m->d_lu, m->f_lu, m->st);
        CKL();
    }
    {
        ProfScope ps(m, 4, 1);
        launch_inv_scale(n, m->d_scale, m->gm_rw, m->st);
        CKL();
    }
    const bool basis32 = mixed && o.krylov_basis_precision == 32;
    if (basis32) {
        if (!m->gm_V32 || m->gm_cap32 < mres) {
            TRY(gmres_basis(m, &m->gm_V32, &m->gm_cap32, mres));
            m->gm_mb32 = -1;   // the cycle graph holds the old basis address
        }
        TRY(gmres_graph32(m, &m->gm_graph_b32, &m->gm_mb32, o.precond, mres));
    } else {
        if (!m->gm_V64 || m->gm_cap64 < mres) {
            TRY(gmres_basis(m, &m->gm_V64, &m->gm_cap64, mres));
            m->gm_m32 = m->gm_m64 = -1;
        }
        TRY(gmres_graph(m, mixed ? &m->gm_graph32 : &m->gm_graph64, mixed ? &m->gm_m32 : &m->gm_m64, mixed, o.precond,
                        mres));
    }
    const int pl = precond_launches(m, o.precond) + (mixed ? 2 : 0);
    const int per_cycle = mres * (6 + pl) + 4 + pl;
    // floor: a tenth of the Newton tolerance; a hundredth under the reference's absolute test, where the
    // converged state is compared with the reference's (exact-LU) one to 1e-8 relative
    const double target = std::max(o.krylov_tol * fnorm, (o.tol_nonlin_rel > 0.0 ? 0.1 : 0.01) * o.tol_nonlin);
    *iters = 0; *passes = 0; *status = 0;
    double prev = 0;
    int stall = 0, slow = 0;
    int hstate[4] = {0, 0, 0, 0};
    double hscal[3] = {0, 0, 0};
    static const bool trace = getenv("SW2G_TRACE_KRYLOV") != nullptr;   // diagnostic: pass history on stderr
    for (int pass = 0;; pass++) {
        {
            ProfScope ps(m, 4, 2);
            launch_spmv_sub(m->B, m->d_vals, x, m->d_b64, m->d_t64, m->st);
            launch_maxabs_unscaled(n, m->d_t64, m->d_scale, R, m->st);
            CKL();
        }
        CK(cudaMemcpyAsync(m->h_rout, m->d_rout, sizeof(double), cudaMemcpyDeviceToHost, m->st));
        if (pass > 0) CK(cudaMemcpyAsync(hstate, m->gm.state, sizeof(int) * 3, cudaMemcpyDeviceToHost, m->st));
        if (pass > 0 && trace) CK(cudaMemcpyAsync(hscal, m->gm.scal, sizeof(double) * 3, cudaMemcpyDeviceToHost, m->st));
        CK(cudaStreamSynchronize(m->st));
        if (pass > 0) {
            *iters += hstate[1];
            if (hstate[2] == 2) { *status = 2; break; }
        }
        const double rn = m->h_rout[0];
        if (trace)
            fprintf(stderr, "gmres pass %d max|r| %.3e target %.3e inner %d status %d cycle-reduction %.3e\n", pass, rn,
                    target, pass > 0 ? hstate[1] : 0, pass > 0 ? hstate[2] : 0,
                    (pass > 0 && hscal[0] > 0) ? hscal[2] / hscal[0] : 0.0);
        if (!std::isfinite(rn)) { *status = 2; break; }
        if (!(rn > target)) break;
        if (pass > 0) {
            // stalled: three passes in a row gaining less than 1%, or five gaining less than 10%
            stall = (rn > 0.99 * prev) ? stall + 1 : 0;
            slow = (rn > 0.9 * prev) ? slow + 1 : 0;
            if (stall >= 3 || slow >= 5) {
                *status = 4;
                if (trace) {   // where the stalled linear residual sits (largest unscaled entries)
                    std::vector<double> t(n), sc(n);
                    CK(cudaMemcpyAsync(t.data(), m->d_t64, sizeof(double) * n, cudaMemcpyDeviceToHost, m->st));
                    CK(cudaMemcpyAsync(sc.data(), m->d_scale, sizeof(double) * n, cudaMemcpyDeviceToHost, m->st));
                    CK(cudaStreamSynchronize(m->st));
                    std::vector<int> idx(n);
                    for (int i = 0; i < n; i++) { idx[i] = i; t[i] = fabs(t[i] / sc[i]); }
                    std::partial_sort(idx.begin(), idx.begin() + 8, idx.end(), [&](int a, int b) { return t[a] > t[b]; });
                    fprintf(stderr, "gmres stalled; largest |r|:");
                    for (int k = 0; k < 8; k++) fprintf(stderr, " %d:%.2e", idx[k], t[idx[k]]);
                    fprintf(stderr, "\n");
                }
                break;
            }
        }
        if (*iters >= o.krylov_max_it) { *status = 3; break; }
        prev = rn;
        double rtol = 0.5 * target / rn;         // the cycle's own 2-norm estimate of the reduction still needed
        if (rtol < (basis32 ? 1e-5 : 1e-12)) rtol = basis32 ? 1e-5 : 1e-12;   // FP32 resolves no more per cycle
        CK(cudaMemcpyAsync(m->gm.scal + 3, &rtol, sizeof(double), cudaMemcpyHostToDevice, m->st));
        {
            ProfScope ps(m, 4, per_cycle + 1);
            if (basis32) {   // FP32 Krylov cycle inside the FP64 refinement
                launch_to_float(n, m->d_t64, m->f_b, m->st);
                CK(cudaGraphLaunch(m->gm_graph_b32, m->st));
                launch_to_double(n, m->f_x, m->k_xi, m->st);
            } else {
                CK(cudaGraphLaunch(mixed ? m->gm_graph32 : m->gm_graph64, m->st));
            }
            launch_axpy(n, 1.0, m->k_xi, x, m->st);
            CKL();
        }
        *passes += 1;
    }
    ProfScope ps(m, 5, 1);
    launch_unscale(n, m->d_x0, m->d_scale, x, m->st);
    CKL();
    return SW2G_OK;
}

// FP32 BiCGStab inside FP64 iterative refinement, on the same scaled and
// preconditioned system.  x accumulates in FP64.  Each pass forms the FP64
// residual t = b - A x and applies the FP64 preconditioner (left-preconditioned
// kinds; the AMG path tests t itself); the reference's
// stopping test (max|M^-1 t| <= tol + tol * max|M^-1 b|) ends the refinement;
// otherwise A d = t is solved in FP32 (matrix, factor and vectors in FP32) to a
// relative reduction refine_tol and d is added to x in FP64.
static int solve32(sw2g_model* m, double* x, double* b, const sw2g_newton_opts& o, int* iters, int* passes, int* status) {
    TRY(alloc_fp32(m));
    const int n = m->n;
    const bool ilu = o.precond == SW2G_PC_BILU0;
    Reduce R{m->d_partial, m->d_counter, m->d_rout};
    CK(cudaMemcpyAsync(m->d_x0, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, m->st));
    CK(cudaMemcpyAsync(m->d_b64, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, m->st));
    CK(cudaMemsetAsync(x, 0, sizeof(double) * n, m->st));
    {
        ProfScope ps(m, 3, 3);
        launch_to_float(m->nnz, m->d_vals, m->f_vals, m->st);
        launch_to_float(9 * m->V, m->d_inv, m->f_inv, m->st);
        if (ilu) launch_to_float(m->nnz, m->d_lu, m->f_lu, m->st);
        CKL();
    }
    *iters = 0; *passes = 0; *status = 0;
    double bnorm = -1, prev_rn = 0;
    double* z = m->k_s;   // FP64 Krylov vectors are free in this mode
    for (int pass = 0; pass <= o.max_refine; pass++) {
        {
            ProfScope ps(m, 4, 3 + (ilu ? 2 * m->ilu.ncolors : 1));
            launch_spmv_sub(m->B, m->d_vals, x, m->d_b64, m->d_t64, m->st);
            CK(cudaMemcpyAsync(z, m->d_t64, sizeof(double) * n, cudaMemcpyDeviceToDevice, m->st));
            if (o.precond == SW2G_PC_BLOCK_JACOBI) launch_bj_apply(m->V, m->d_inv, z, m->st);
            else if (o.precond == SW2G_PC_AMG) {
                // right-preconditioned inner solves: the test is on the true residual
            } else {
                PrecondOp<double> op;
                op.kind = o.precond; op.ilu = &m->ilu; op.lu = m->d_lu; op.dinv = m->d_inv; op.amg = &m->amg;
                op.vals = m->d_vals;
                precond_apply<double>(m->B, op, z, nullptr, m->st);
            }
            launch_maxabs(n, z, R, m->st);
            CKL();
        }
        CK(cudaMemcpyAsync(m->h_rout, m->d_rout, sizeof(double), cudaMemcpyDeviceToHost, m->st));
        CK(cudaStreamSynchronize(m->st));
        const double rn = m->h_rout[0];
        if (bnorm < 0) bnorm = rn;                 // x = 0 on the first pass: M^-1 t = M^-1 b
        if (pass > 0 && !(rn < prev_rn)) {         // the last FP32 correction did not help: take it back, stop
            ProfScope ps(m, 5, 1);
            launch_axpy(n, -1.0, m->d_t64 + n, x, m->st);
            CKL();
            if (!*status) *status = 4;
            break;
        }
        if (!std::isfinite(rn)) { *status = 2; break; }
        if (!(rn > o.krylov_tol + bnorm * o.krylov_tol)) break;
        if (pass == o.max_refine) { if (!*status) *status = 3; break; }
        prev_rn = rn;
        {
            ProfScope ps(m, 4, 1);
            launch_to_float(n, m->d_t64, m->f_b, m->st);
            CKL();
        }
        KrylovVecs<float> V32{m->f_x, m->f_r, m->f_p, m->f_Ap, m->f_q, m->f_s, m->f_As, m->f_b, m->f_vals, m->f_inv, m->f_lu,
                              m->f_z};
        int it = 0, st = 0;
        TRY(run_bicg<float>(m, V32, o.precond, &m->graph32[o.precond], o.krylov_max_it, 0.0, o.refine_tol, &it, &st));
        *iters += it; *passes += 1;
        if (st == 1 || st == 2) *status = st;
        {
            ProfScope ps(m, 5, 2);
            launch_to_double(n, m->f_x, m->d_t64 + n, m->st);   // the correction, kept for a possible undo
            launch_axpy(n, 1.0, m->d_t64 + n, x, m->st);
            CKL();
        }
        if (st == 2) break;
    }
    ProfScope ps(m, 5, 1);
    launch_unscale(n, m->d_x0, m->d_scale, x, m->st);
    CKL();
    return SW2G_OK;
}

// ------------------------------------------------------------------ Newton step
// fe_newton (src/newton/fe_newton.c:44-915), serial non-PETSc branch, on the
// resident state d_sol / d_sol_old / d_sol_older / d_bc_mask / d_dirichlet.
// diagnostic (SW2G_TRACE_NEWTON): the first elements whose residual is not finite, with their nodal states
static void debug_nonfinite(sw2g_model* m) {
    std::vector<double> er(9 * (size_t)m->Etot), sol(m->n), old(m->n);
    std::vector<int> tri(3 * (size_t)m->T), wd(m->T);
    cudaMemcpyAsync(er.data(), m->d_ER, sizeof(double) * er.size(), cudaMemcpyDeviceToHost, m->st);
    cudaMemcpyAsync(sol.data(), m->d_sol, sizeof(double) * m->n, cudaMemcpyDeviceToHost, m->st);
    cudaMemcpyAsync(old.data(), m->d_sol_old, sizeof(double) * m->n, cudaMemcpyDeviceToHost, m->st);
    cudaMemcpyAsync(tri.data(), m->d_tri, sizeof(int) * tri.size(), cudaMemcpyDeviceToHost, m->st);
    cudaMemcpyAsync(wd.data(), m->d_wd, sizeof(int) * wd.size(), cudaMemcpyDeviceToHost, m->st);
    cudaStreamSynchronize(m->st);
    int shown = 0;
    for (int e = 0; e < m->Etot && shown < 5; e++) {
        bool bad = false;
        for (int k = 0; k < 9; k++) bad |= !std::isfinite(er[9 * (size_t)e + k]);
        if (!bad) continue;
        shown++;
        if (e < m->T) {
            fprintf(stderr, "non-finite residual: triangle %d wd_flag %d\n", e, wd[e]);
            for (int a = 0; a < 3; a++) {
                const int nd = tri[3 * (size_t)e + a];
                fprintf(stderr, "  node %d h %.6e u %.6e v %.6e | old h %.6e u %.6e v %.6e\n", nd, sol[3 * nd],
                        sol[3 * nd + 1], sol[3 * nd + 2], old[3 * nd], old[3 * nd + 1], old[3 * nd + 2]);
            }
        } else {
            fprintf(stderr, "non-finite residual: segment %d\n", e - m->T);
        }
    }
}

static bool valid_precond(int p) {
    return p == SW2G_PC_BLOCK_JACOBI || p == SW2G_PC_BILU0 || p == SW2G_PC_AMG;
}
static int newton_device(sw2g_model* m, const sw2g_newton_opts& o_in, sw2g_newton_stats* S) {
    if (!(valid_precond(o_in.precond) && (o_in.krylov_precision == 32 || o_in.krylov_precision == 64) && o_in.krylov_max_it >= 0 &&
          (o_in.krylov_method == SW2G_KRYLOV_BICGSTAB ||
           (o_in.krylov_method == SW2G_KRYLOV_GMRES && o_in.precond != SW2G_PC_BLOCK_JACOBI)) &&
          o_in.max_nonlin_it >= 0 && o_in.max_linesearch_cuts >= 0 && o_in.max_refine >= 0 &&
          o_in.amg_chunks >= 0 && o_in.amg_chunks <= 2)) {
        g_err = "sw2g newton: bad options";
        return SW2G_ERR_ARG;
    }
    const int n = m->n;
    sw2g_newton_stats st{};
    // initialize_system (newton_tools.c:21-53): sol <- sol_old, then fe_sw2_init:
    // wet/dry flags of (sol, sol_old) and the dry-node velocity masks
    CK(cudaMemcpyAsync(m->d_sol, m->d_sol_old, sizeof(double) * n, cudaMemcpyDeviceToDevice, m->st));
    TRY(do_wd(m, m->d_sol, m->d_sol_old));
    {
        ProfScope ps(m, 5, 1);
        launch_dry_mask(m->V, m->d_sol_old, m->d_bc_mask, m->st);
        CKL();
    }
    {   // initialize_dirichlet_bc (newton_tools.c:130)
        ProfScope ps(m, 5, 1);
        launch_masked_copy(n, m->d_bc_mask, m->d_dirichlet, m->d_sol, m->st);
        CKL();
    }
    CK(cudaMemsetAsync(m->d_dsol, 0, sizeof(double) * n, m->st));
    double rmax, rl2, imax;
    TRY(do_residual(m, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_res));
    TRY(do_norms(m, m->d_res, m->d_dsol, &rmax, &rl2, &imax));
    if (!std::isfinite(rl2)) { g_err = "non-finite residual at the initial guess"; return SW2G_ERR_NONFINITE; }
    st.prev_resid_max = rmax;
    // Initial-guess hook (after initialize_system): a supplied guess replaces the
    // previous-step state only if its residual L2 norm is smaller -- the Newton
    // residual judges the guess, the previous step is the fallback.  (L2, not the
    // max-norm: one node's spike must not veto a guess that is better everywhere else.)
    if (o_in.use_guess && m->guess_set) {
        CK(cudaMemcpyAsync(m->d_sol, m->d_guess, sizeof(double) * n, cudaMemcpyDeviceToDevice, m->st));
        {
            ProfScope ps(m, 5, 1);
            launch_masked_copy(n, m->d_bc_mask, m->d_dirichlet, m->d_sol, m->st);
            CKL();
        }
        double gmax, gl2, gi;
        TRY(do_residual(m, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_res));
        TRY(do_norms(m, m->d_res, m->d_dsol, &gmax, &gl2, &gi));
        static const bool trace = getenv("SW2G_TRACE_NEWTON") != nullptr;
        if (trace)
            fprintf(stderr, "guess judge: l2 %.6e (previous step %.6e), max %.6e (previous step %.6e)\n", gl2, rl2, gmax,
                    rmax);
        if (std::isfinite(gl2) && gl2 < rl2) {
            rmax = gmax; rl2 = gl2; imax = gi; st.guess_used = 1;
        } else {   // fall back to the previous-step state
            CK(cudaMemcpyAsync(m->d_sol, m->d_sol_old, sizeof(double) * n, cudaMemcpyDeviceToDevice, m->st));
            {
                ProfScope ps(m, 5, 1);
                launch_masked_copy(n, m->d_bc_mask, m->d_dirichlet, m->d_sol, m->st);
                CKL();
            }
            TRY(do_residual(m, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_res));
            TRY(do_norms(m, m->d_res, m->d_dsol, &rmax, &rl2, &imax));
        }
    }
    st.initial_resid_max = rmax;
    st.initial_resid_l2 = rl2;
    sw2g_newton_opts o = o_in;   // the step's effective options
    // relative test: against the previous-step state's residual, the same reference with or without a guess
    if (o_in.tol_nonlin_rel > 0.0) o.tol_nonlin = std::max(o_in.tol_nonlin_rel * st.prev_resid_max, o_in.tol_nonlin_min);
    int it = 0, stalled_its = 0; bool ok = true, keep, lin_ok = true;
    double rmax_prev = rmax;
    do {
        TRY(do_jacobian(m, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_vals));
        CK(cudaMemsetAsync(m->d_dsol, 0, sizeof(double) * n, m->st));
        TRY(do_prepare(m, m->d_vals, m->d_res, m->d_dsol));
        TRY(do_precond_setup(m, m->d_vals, o.precond, o.amg_chunks));
        int kit = 0, kst = 0, passes = 0;
        if (o.krylov_method == SW2G_KRYLOV_GMRES)
            TRY(solve_gmres(m, m->d_dsol, m->d_res, o, o.krylov_precision == 32, rmax, &kit, &passes, &kst));
        else if (o.krylov_precision == 32) TRY(solve32(m, m->d_dsol, m->d_res, o, &kit, &passes, &kst));
        else if (o.precond == SW2G_PC_AMG)
            TRY(solve64_restarted(m, m->d_dsol, m->d_res, o.krylov_max_it, o.krylov_tol, o.max_refine, &kit, &passes, &kst));
        else TRY(solve64(m, m->d_dsol, m->d_res, o.precond, o.krylov_max_it, o.krylov_tol, &kit, &kst));
        const int lin_status = kst;
        st.krylov_its += kit; st.refine_passes += passes;
        if (kst == 1 || kst == 2) st.krylov_breakdowns++;
        {   // increment_function (newton_tools.c:261) and dsol = -dsol (fe_newton.c:553-555)
            ProfScope ps(m, 5, 2);
            launch_axpy(n, 1.0, m->d_dsol, m->d_sol, m->st);
            launch_scal(n, -1.0, m->d_dsol, m->st);
            CKL();
        }
        const double old_l2 = rl2;
        TRY(do_residual(m, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_res));
        TRY(do_norms(m, m->d_res, m->d_dsol, &rmax, &rl2, &imax));
        int cuts = 0;   // line search, fe_newton.c:681-741
        // a step into a state whose residual is not finite is cut like a step that raised the residual
        // (the reference would stop with a NaN residual, newton_tools.c:344-349)
        while (rmax > o.tol_nonlin && (rl2 > old_l2 || !std::isfinite(rl2)) && cuts < o.max_linesearch_cuts) {
            {
                ProfScope ps(m, 5, 2);
                launch_scal(n, 0.5, m->d_dsol, m->st);
                launch_axpy(n, 1.0, m->d_dsol, m->d_sol, m->st);
                CKL();
            }
            TRY(do_residual(m, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_res));
            TRY(do_norms(m, m->d_res, m->d_dsol, &rmax, &rl2, &imax));
            cuts++;
        }
        if (std::isnan(rl2) || std::isinf(rl2)) {
            ok = false;
            static const bool trace_nf = getenv("SW2G_TRACE_NEWTON") != nullptr;
            if (trace_nf) debug_nonfinite(m);
        }
        // The increment test stands for convergence only when the linear solve reached its target: with
        // the reference's exact LU (bcgstab_solver.c:371-420) a small increment means Newton converged,
        // with an iterative solve that stopped early it may only mean the solve stalled.
        lin_ok = (lin_status == 0);
        if (!lin_ok) st.linear_unconverged++;
        // a stalled linear solve that does not halve max|R| twice in a row ends the solve as failed:
        // retrying the interval with a smaller dt is cheaper than the remaining stalled iterations
        stalled_its = (lin_status == 4 && !(rmax < 0.5 * rmax_prev)) ? stalled_its + 1 : 0;
        rmax_prev = rmax;
        st.linesearch_cuts += cuts;
        it++;
        static const bool trace = getenv("SW2G_TRACE_NEWTON") != nullptr;   // diagnostic: Newton history on stderr
        if (trace)
            fprintf(stderr, "newton it %d krylov %d status %d refine %d resid_max %.3e resid_l2 %.3e inc_max %.3e cuts %d\n",
                    it, kit, kst, passes, rmax, rl2, imax, cuts);
        keep = ok && it < o.max_nonlin_it && rmax < 1.0E+20 && rmax > o.tol_nonlin && (imax > o.inc_nonlin || !lin_ok) &&
               stalled_its < 2;
    } while (keep);
    st.newton_its = it;
    st.resid_max = rmax; st.resid_l2 = rl2; st.inc_max = imax;
    st.tol_used = o.tol_nonlin;
    // fe_newton.c:870-871 (success unless max|R| > tol and the increment > inc_nonlin), with the
    // increment test counted only after a linear solve that reached its target
    st.success = ok && rmax < 1.0E+20 && (!(rmax > o.tol_nonlin) || (!(imax > o.inc_nonlin) && lin_ok));
    if (!st.success) {   // fe_newton.c:887-890: reset to the old values
        CK(cudaMemcpyAsync(m->d_sol, m->d_sol_old, sizeof(double) * n, cudaMemcpyDeviceToDevice, m->st));
        launch_masked_copy(n, m->d_bc_mask, m->d_dirichlet, m->d_sol, m->st);
        CKL();
    }
    if (S) *S = st;
    if (!ok) { g_err = "non-finite residual norm during Newton"; return SW2G_ERR_NONFINITE; }
    return SW2G_OK;
}

// ------------------------------------------------------------------ C ABI
#define NEED(cond, msg) do { if (!(cond)) { g_err = msg; return SW2G_ERR_ARG; } } while (0)

static int put3(sw2g_model* m, const double* sol, const double* sol_old, const double* sol_older) {
    const size_t b = sizeof(double) * m->n;
    m->can_undo = false;
    CK(cudaMemcpyAsync(m->d_sol, sol, b, cudaMemcpyHostToDevice, m->st));
    CK(cudaMemcpyAsync(m->d_sol_old, sol_old, b, cudaMemcpyHostToDevice, m->st));
    CK(cudaMemcpyAsync(m->d_sol_older, sol_older, b, cudaMemcpyHostToDevice, m->st));
    return SW2G_OK;
}

extern "C" int sw2g_wd_flags(sw2g_model* m, const double* sol, const double* sol_old, int* wd_flag) {
    NEED(m && sol && sol_old && wd_flag, "sw2g_wd_flags: null argument");
    TRY(put3(m, sol, sol_old, sol_old));
    TRY(do_wd(m, m->d_sol, m->d_sol_old));
    CK(cudaMemcpyAsync(wd_flag, m->d_wd, sizeof(int) * m->T, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    return SW2G_OK;
}

extern "C" int sw2g_elem_resid(sw2g_model* m, const double* sol, const double* sol_old, const double* sol_older,
                               double* out_tri, double* out_seg) {
    NEED(m && sol && sol_old && sol_older && out_tri && (m->S == 0 || out_seg), "sw2g_elem_resid: null argument");
    TRY(put3(m, sol, sol_old, sol_older));
    TRY(do_wd(m, m->d_sol, m->d_sol_old));
    {
        ProfScope ps(m, 0, 2);
        launch_elem_resid(m->M, m->P, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_wd, m->d_ER, m->st);
        CKL();
    }
    std::vector<double> er(9 * (size_t)m->Etot);
    CK(cudaMemcpyAsync(er.data(), m->d_ER, sizeof(double) * er.size(), cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    memcpy(out_tri, er.data(), sizeof(double) * 9 * (size_t)m->T);
    for (int s = 0; s < m->S; s++) for (int i = 0; i < 6; i++) out_seg[6 * (size_t)s + i] = er[9 * ((size_t)m->T + s) + i];
    return SW2G_OK;
}

extern "C" int sw2g_elem_jac(sw2g_model* m, const double* sol, const double* sol_old, const double* sol_older,
                             double* out_tri, double* out_seg) {
    NEED(m && sol && sol_old && sol_older && out_tri && (m->S == 0 || out_seg), "sw2g_elem_jac: null argument");
    TRY(put3(m, sol, sol_old, sol_older));
    TRY(do_wd(m, m->d_sol, m->d_sol_old));
    {
        ProfScope ps(m, 1, 4);
        launch_elem_jac(m->M, m->P, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_wd, m->d_EJ, m->st);
        CKL();
    }
    std::vector<double> ej(81 * (size_t)m->Etot);
    CK(cudaMemcpyAsync(ej.data(), m->d_EJ, sizeof(double) * ej.size(), cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    const size_t Et = m->Etot;
    for (size_t e = 0; e < (size_t)m->T; e++)
        for (int c = 0; c < 9; c++) for (int r = 0; r < 9; r++) out_tri[e * 81 + r * 9 + c] = ej[(c * Et + e) * 9 + r];
    for (size_t s = 0; s < (size_t)m->S; s++)
        for (int c = 0; c < 6; c++) for (int r = 0; r < 6; r++) out_seg[s * 36 + r * 6 + c] = ej[(c * Et + m->T + s) * 9 + r];
    return SW2G_OK;
}

extern "C" int sw2g_assemble_residual(sw2g_model* m, const double* sol, const double* sol_old, const double* sol_older,
                                      double* residual) {
    NEED(m && sol && sol_old && sol_older && residual, "sw2g_assemble_residual: null argument");
    TRY(put3(m, sol, sol_old, sol_older));
    TRY(do_wd(m, m->d_sol, m->d_sol_old));
    TRY(do_residual(m, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_res));
    CK(cudaMemcpyAsync(residual, m->d_res, sizeof(double) * m->n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    return SW2G_OK;
}

extern "C" int sw2g_assemble_jacobian(sw2g_model* m, const double* sol, const double* sol_old, const double* sol_older,
                                      double* vals) {
    NEED(m && sol && sol_old && sol_older && vals, "sw2g_assemble_jacobian: null argument");
    TRY(put3(m, sol, sol_old, sol_older));
    TRY(do_wd(m, m->d_sol, m->d_sol_old));
    TRY(do_jacobian(m, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_vals));
    CK(cudaMemcpyAsync(vals, m->d_vals, sizeof(double) * m->nnz, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    return SW2G_OK;
}

// The same two assemblies with the caller's wet/dry flags: inside fe_newton the
// reference evaluates every residual and Jacobian of a Newton solve with the flags
// fe_sw2_init set at its start (initialize_system, newton_tools.c:21-53), not with
// flags of the current iterate.
static int put_wd(sw2g_model* m, const int* wd_flag) {
    for (int e = 0; e < m->T; e++)
        if (wd_flag[e] < 0 || wd_flag[e] > 2) { g_err = "wet/dry flags must be 0, 1 or 2"; return SW2G_ERR_ARG; }
    CK(cudaMemcpyAsync(m->d_wd, wd_flag, sizeof(int) * m->T, cudaMemcpyHostToDevice, m->st));
    return SW2G_OK;
}

extern "C" int sw2g_assemble_residual_wd(sw2g_model* m, const double* sol, const double* sol_old,
                                         const double* sol_older, const int* wd_flag, double* residual) {
    NEED(m && sol && sol_old && sol_older && wd_flag && residual, "sw2g_assemble_residual_wd: null argument");
    TRY(put_wd(m, wd_flag));
    TRY(put3(m, sol, sol_old, sol_older));
    TRY(do_residual(m, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_res));
    CK(cudaMemcpyAsync(residual, m->d_res, sizeof(double) * m->n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    return SW2G_OK;
}

extern "C" int sw2g_assemble_jacobian_wd(sw2g_model* m, const double* sol, const double* sol_old,
                                         const double* sol_older, const int* wd_flag, double* vals) {
    NEED(m && sol && sol_old && sol_older && wd_flag && vals, "sw2g_assemble_jacobian_wd: null argument");
    TRY(put_wd(m, wd_flag));
    TRY(put3(m, sol, sol_old, sol_older));
    TRY(do_jacobian(m, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_vals));
    CK(cudaMemcpyAsync(vals, m->d_vals, sizeof(double) * m->nnz, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    return SW2G_OK;
}

extern "C" int sw2g_prepare_system(sw2g_model* m, double* vals, double* residual, double* x, int* bc_mask, double* scale) {
    NEED(m && vals && residual && x && bc_mask && scale, "sw2g_prepare_system: null argument");
    const size_t n = m->n;
    CK(cudaMemcpyAsync(m->d_vals, vals, sizeof(double) * m->nnz, cudaMemcpyHostToDevice, m->st));
    CK(cudaMemcpyAsync(m->d_res, residual, sizeof(double) * n, cudaMemcpyHostToDevice, m->st));
    CK(cudaMemcpyAsync(m->d_dsol, x, sizeof(double) * n, cudaMemcpyHostToDevice, m->st));
    CK(cudaMemcpyAsync(m->d_bc_mask, bc_mask, sizeof(int) * n, cudaMemcpyHostToDevice, m->st));
    TRY(do_prepare(m, m->d_vals, m->d_res, m->d_dsol));
    CK(cudaMemcpyAsync(vals, m->d_vals, sizeof(double) * m->nnz, cudaMemcpyDeviceToHost, m->st));
    CK(cudaMemcpyAsync(residual, m->d_res, sizeof(double) * n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaMemcpyAsync(x, m->d_dsol, sizeof(double) * n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaMemcpyAsync(bc_mask, m->d_bc_mask, sizeof(int) * n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaMemcpyAsync(scale, m->d_scale, sizeof(double) * n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    return SW2G_OK;
}

extern "C" int sw2g_solve_linear_sys_bcgstab(sw2g_model* m, double* x, const double* vals, double* b,
                                             const double* scale_vect, int max_it, double tol, int precond, int* iters) {
    NEED(m && x && vals && b && scale_vect && max_it >= 0 && tol >= 0 &&
         valid_precond(precond), "sw2g_solve_linear_sys_bcgstab: bad argument");
    const size_t n = m->n;
    CK(cudaMemcpyAsync(m->d_vals, vals, sizeof(double) * m->nnz, cudaMemcpyHostToDevice, m->st));
    CK(cudaMemcpyAsync(m->d_res, b, sizeof(double) * n, cudaMemcpyHostToDevice, m->st));
    CK(cudaMemcpyAsync(m->d_dsol, x, sizeof(double) * n, cudaMemcpyHostToDevice, m->st));
    CK(cudaMemcpyAsync(m->d_scale, scale_vect, sizeof(double) * n, cudaMemcpyHostToDevice, m->st));
    TRY(do_precond_setup(m, m->d_vals, precond));
    int it = 0, status = 0;
    TRY(solve64(m, m->d_dsol, m->d_res, precond, max_it, tol, &it, &status));
    CK(cudaMemcpyAsync(x, m->d_dsol, sizeof(double) * n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaMemcpyAsync(b, m->d_res, sizeof(double) * n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    if (iters) *iters = (status == 1 || status == 2) ? -it - 1 : it;
    return SW2G_OK;
}

extern "C" int sw2g_load_state(sw2g_model* m, const double* sol, const double* sol_old, const double* sol_older,
                               const int* bc_mask, const double* dirichlet) {
    NEED(m && sol && sol_old && sol_older, "sw2g_load_state: null argument");
    TRY(put3(m, sol, sol_old, sol_older));
    if (bc_mask) CK(cudaMemcpyAsync(m->d_bc_mask, bc_mask, sizeof(int) * m->n, cudaMemcpyHostToDevice, m->st));
    else CK(cudaMemsetAsync(m->d_bc_mask, 0, sizeof(int) * m->n, m->st));
    if (dirichlet) CK(cudaMemcpyAsync(m->d_dirichlet, dirichlet, sizeof(double) * m->n, cudaMemcpyHostToDevice, m->st));
    else CK(cudaMemsetAsync(m->d_dirichlet, 0, sizeof(double) * m->n, m->st));
    CK(cudaStreamSynchronize(m->st));
    return SW2G_OK;
}

extern "C" int sw2g_store_state(sw2g_model* m, double* sol, double* sol_old, double* sol_older, int* bc_mask) {
    NEED(m, "sw2g_store_state: null model");
    const size_t b = sizeof(double) * m->n;
    if (sol) CK(cudaMemcpyAsync(sol, m->d_sol, b, cudaMemcpyDeviceToHost, m->st));
    if (sol_old) CK(cudaMemcpyAsync(sol_old, m->d_sol_old, b, cudaMemcpyDeviceToHost, m->st));
    if (sol_older) CK(cudaMemcpyAsync(sol_older, m->d_sol_older, b, cudaMemcpyDeviceToHost, m->st));
    if (bc_mask) CK(cudaMemcpyAsync(bc_mask, m->d_bc_mask, sizeof(int) * m->n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    return SW2G_OK;
}

extern "C" int sw2g_set_guess(sw2g_model* m, const double* guess, int on_device) {
    NEED(m, "sw2g_set_guess: null model");
    if (!guess) { m->guess_set = false; return SW2G_OK; }
    CK(cudaMemcpyAsync(m->d_guess, guess, sizeof(double) * m->n,
                       on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, m->st));
    m->guess_set = true;
    return SW2G_OK;
}

// Newton from a supplied guess that fails (no convergence, or a non-finite residual) is
// repeated from the previous-step state, the reference's start; the work of both
// attempts is counted.
static int newton_with_fallback(sw2g_model* m, const sw2g_newton_opts& o, sw2g_newton_stats* S) {
    const bool may_retry = o.use_guess && m->guess_set;
    if (may_retry) {   // the retry starts from the Dirichlet marks the step began with
        if (!m->d_mask_save) TRY(dalloc(m, &m->d_mask_save, (size_t)m->n));
        CK(cudaMemcpyAsync(m->d_mask_save, m->d_bc_mask, sizeof(int) * m->n, cudaMemcpyDeviceToDevice, m->st));
    }
    sw2g_newton_stats a{};
    int rc = newton_device(m, o, &a);
    const bool guessed = may_retry && a.guess_used;
    if (guessed && (rc == SW2G_ERR_NONFINITE || (rc == SW2G_OK && !a.success))) {
        CK(cudaMemcpyAsync(m->d_bc_mask, m->d_mask_save, sizeof(int) * m->n, cudaMemcpyDeviceToDevice, m->st));
        sw2g_newton_opts o2 = o;
        o2.use_guess = 0;
        sw2g_newton_stats b{};
        rc = newton_device(m, o2, &b);
        b.newton_its += a.newton_its; b.krylov_its += a.krylov_its; b.linesearch_cuts += a.linesearch_cuts;
        b.refine_passes += a.refine_passes; b.krylov_breakdowns += a.krylov_breakdowns;
        b.linear_unconverged += a.linear_unconverged;
        b.guess_fallback = 1;
        a = b;
    }
    if (S) *S = a;
    return rc;
}

extern "C" int sw2g_fe_newton(sw2g_model* m, double* sol, const double* sol_old, const double* sol_older, int* bc_mask,
                              const double* dirichlet, const sw2g_newton_opts* opts, sw2g_newton_stats* stats) {
    NEED(m && sol && sol_old && sol_older && bc_mask, "sw2g_fe_newton: null argument");
    sw2g_newton_opts o; if (opts) o = *opts; else sw2g_default_opts(&o);
    TRY(sw2g_load_state(m, sol_old, sol_old, sol_older, bc_mask, dirichlet));
    int rc = newton_with_fallback(m, o, stats);
    CK(cudaMemcpyAsync(sol, m->d_sol, sizeof(double) * m->n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaMemcpyAsync(bc_mask, m->d_bc_mask, sizeof(int) * m->n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    return rc;
}

extern "C" int sw2g_step(sw2g_model* m, const sw2g_newton_opts* opts, sw2g_newton_stats* stats) {
    NEED(m, "sw2g_step: null model");
    sw2g_newton_opts o; if (opts) o = *opts; else sw2g_default_opts(&o);
    // smodel_super_prep_sol: sol_older <- sol_old <- sol (a pointer rotation)
    double* t = m->d_sol_older; m->d_sol_older = m->d_sol_old; m->d_sol_old = m->d_sol; m->d_sol = t;
    m->can_undo = true;
    int rc = newton_with_fallback(m, o, stats);
    m->guess_set = false;
    return rc;
}

extern "C" int sw2g_undo_step(sw2g_model* m) {
    NEED(m, "sw2g_undo_step: null model");
    NEED(m->can_undo, "sw2g_undo_step: no sw2g_step to undo since the state was loaded or last undone");
    NEED(m->P.alpha == 0.0, "sw2g_undo_step: the three-level scheme (tau_temporal != 0) needs the sol_older level, "
                            "which the step overwrote");
    // the step's rotation was sol_older <- sol_old <- sol <- (sol_older's buffer); turn it back.  The
    // start state and its previous level were never written by the step; sol_older's buffer was.
    double* c = m->d_sol; m->d_sol = m->d_sol_old; m->d_sol_old = m->d_sol_older; m->d_sol_older = c;
    m->can_undo = false;
    return SW2G_OK;
}

extern "C" int sw2g_grid_mass(sw2g_model* m, const double* sol, double density, double dt, double* out,
                              double* elem_mass) {
    NEED(m && out, "sw2g_grid_mass: null argument");
    NEED(dt >= 0.0, "sw2g_grid_mass: negative dt");
    const double* d = m->d_sol;
    if (sol) {   // a host state goes to a work vector: the resident state stays as it is
        CK(cudaMemcpyAsync(m->d_t64, sol, sizeof(double) * m->n, cudaMemcpyHostToDevice, m->st));
        d = m->d_t64;
    }
    {
        ProfScope ps(m, 5, 1);
        Reduce R{m->d_partial, m->d_counter, m->d_rout};
        launch_mass_balance(m->M, d, density, density * dt, elem_mass ? m->d_ER : nullptr, R, m->st);
        CKL();
    }
    CK(cudaMemcpyAsync(m->h_rout, m->d_rout, 2 * sizeof(double), cudaMemcpyDeviceToHost, m->st));
    if (elem_mass && m->T)
        CK(cudaMemcpyAsync(elem_mass, m->d_ER, sizeof(double) * m->T, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    out[0] = m->h_rout[0]; out[1] = m->h_rout[1];
    return SW2G_OK;
}

extern "C" int sw2g_precond_info(sw2g_model* m, long long* info) {
    NEED(m && info, "sw2g_precond_info: null argument");
    int failed = 0;
    if (m->amg.patch.failed) {
        CK(cudaMemcpyAsync(&failed, m->amg.patch.failed, sizeof(int), cudaMemcpyDeviceToHost, m->st));
        CK(cudaStreamSynchronize(m->st));
    }
    info[0] = m->p_nflag; info[1] = m->p_nchunks; info[2] = m->p_nentries; info[3] = m->p_rtot; info[4] = failed;
    return SW2G_OK;
}

extern "C" int sw2g_set_profiling(sw2g_model* m, int on) {
    NEED(m, "null model");
    m->prof = on != 0;
    return SW2G_OK;
}
extern "C" int sw2g_get_profile(sw2g_model* m, double* ms, long long* launches) {
    NEED(m, "null model");
    prof_collect(m);
    for (int c = 0; c < SW2G_NCLASSES; c++) { if (ms) ms[c] = m->prof_ms[c]; if (launches) launches[c] = m->prof_launch[c]; }
    return SW2G_OK;
}
extern "C" int sw2g_reset_profile(sw2g_model* m) {
    NEED(m, "null model");
    prof_collect(m);
    for (int c = 0; c < SW2G_NCLASSES; c++) { m->prof_ms[c] = 0; m->prof_launch[c] = 0; }
    return SW2G_OK;
}

extern "C" int sw2g_time_kernel(sw2g_model* m, int which, int reps, double* avg_ms, double* bytes) {
    NEED(m && avg_ms && bytes && reps > 0 && which >= 0 && which <= 9, "sw2g_time_kernel: bad argument");
    NEED(which != 8 || m->gm_graph_b32, "sw2g_time_kernel: no FP32 GMRES cycle has run yet");
    const double nnz = m->nnz, n = m->n, T = m->T, S = m->S;
    if (which >= 4) {   // the AMG sweeps
        if (!m->amg_ready) TRY(build_amg(m));
        amg_setup(m->B, m->amg, m->A, m->d_vals, m->st);
    }
    if (which == 5 || which == 6 || which == 7 || which == 9) {
        TRY(alloc_fp32(m));
        launch_to_float(m->nnz, m->d_vals, m->f_vals, m->st);
    }
    const double zero = 0.0;
    auto launch = [&]() {
        switch (which) {
            case 0: launch_spmv64(m->B, m->d_vals, m->k_p, m->k_Ap, m->st); break;
            case 1: launch_elem_jac(m->M, m->P, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_wd, m->d_EJ, m->st); break;
            case 2: launch_elem_resid(m->M, m->P, m->d_sol, m->d_sol_old, m->d_sol_older, m->d_wd, m->d_ER, m->st); break;
            case 3: launch_gather_jac(m->A, m->d_EJ, m->Etot, m->d_vals, m->st); break;
            case 4: amg_smooth0_once(m->B, m->amg, m->d_vals, m->k_p, m->k_Ap, m->k_As, m->st); break;
            case 5: amg_smooth0_once32(m->B, m->amg, m->f_vals, m->f_p, m->f_Ap, m->f_As, m->st); break;
            case 6: amg_apply<float>(m->B, m->amg, m->f_vals, m->f_Ap, nullptr, m->st); break;
            case 7: spmv_skip<float>(m->B, m->f_vals, m->f_p, m->f_Ap, nullptr, m->st); break;
            case 8:   // a whole FP32 GMRES cycle with its stopping test off: every iteration runs
                cudaMemcpyAsync(m->gm.scal + 3, &zero, sizeof(double), cudaMemcpyHostToDevice, m->st);
                cudaGraphLaunch(m->gm_graph_b32, m->st);
                break;
            case 9: amg_patch_correct<float>(m->B, m->amg, m->f_vals, m->f_p, m->f_Ap, nullptr, m->st); break;

        }
    };
    launch();   // warm-up
    CKL();
    cudaEvent_t a = ev_get(m), b = ev_get(m);
    CK(cudaEventRecord(a, m->st));
    for (int r = 0; r < reps; r++) launch();
    CK(cudaEventRecord(b, m->st));
    CK(cudaEventSynchronize(b));
    CKL();
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, a, b));
    m->ev_pool.push_back(a); m->ev_pool.push_back(b);
    *avg_ms = ms / reps;
    switch (which) {   // algorithmic bytes of one launch
        case 0: *bytes = 12.0 * nnz + 20.0 * n; break;                      // CSR SpMV: vals+cols, rowptr+x+y
        case 1: *bytes = 1290.0 * T + 632.0 * S; break;                     // element inputs + slot ids + 81/36 writes
        case 2: *bytes = 316.0 * T + 200.0 * S + 8.0 * n; break;            // element inputs + residual out
        case 3: *bytes = 8.0 * 81.0 * T + 8.0 * 36.0 * S + 12.0 * nnz; break;   // element blocks in, CSR values + map out
        case 4: *bytes = 12.0 * nnz + 20.0 * n + 24.0 * n + 16.0 * n; break;    // SpMV + block-Jacobi apply
        case 6: *bytes = 4.0 * (8.0 * nnz + 32.0 * n); break;   // ~4 level-0 matrix passes (coarse levels extra)
        case 5: *bytes = 8.0 * nnz + 12.0 * n + 12.0 * n + 8.0 * n; break;   // FP32 SpMV + FP32 block apply
        case 7: *bytes = 8.0 * nnz + 12.0 * n; break;                        // FP32 values + cols, x and y
        case 8: *bytes = (double)m->gm_mb32; break;                          // iterations of the cycle (not bytes)
        case 9: *bytes = 4.0 * (double)m->p_rtot + 12.0 * m->p_nentries; break;   // FP32 inverse rows + residuals
    }
    return SW2G_OK;
}

// ------------------------------------------------------------------ residual without allocation
// For callers that cannot allocate device memory when they call in: an application
// that hands all free device memory to its own pool at start-up, or a time loop
// that must not allocate (or free) inside its steps.  sw2g_assemble_residual keeps
// its element-residual and wet/dry work buffers in memory that sw2g_create
// allocated; this variant keeps them in file-scope device arrays of a fixed size
// instead, so a call allocates nothing.  Every GPU that loads the library holds
// these arrays (about 10.5 MB) until the process exits.
constexpr int kNoAllocMaxElems = 1 << 17;   // triangles + boundary segments
constexpr int kNoAllocMaxNodes = 1 << 17;
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) double g_na_elem_resid[9 * (size_t)kNoAllocMaxElems];
static __device__ __align__(256) int g_na_wd_flags[kNoAllocMaxElems];
static __device__ __align__(256) int g_na_node_work[kNoAllocMaxNodes];
// device addresses of the arrays, looked up once per device (host code may not use
// the arrays' names as addresses: those are host-side stand-ins)
struct NoAllocScratch { double* er; int* wd; int* node; };
static NoAllocScratch g_na_ptr[kNoAllocMaxDevices];
static bool g_na_ready[kNoAllocMaxDevices];
static std::mutex g_na_mutex;

static int noalloc_scratch(const sw2g_model* m, NoAllocScratch* out) {
    // cudaGetSymbolAddress answers for the current device, so that must be the model's
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev != m->device) {
        g_err = "sw2g_assemble_residual_noalloc: the current device is not the model's (make the device that was "
                "current at sw2g_create current again)";
        return SW2G_ERR_ARG;
    }
    if (dev < 0 || dev >= kNoAllocMaxDevices) { g_err = "sw2g_assemble_residual_noalloc: device index too large"; return SW2G_ERR_ARG; }
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ready[dev]) {
        NoAllocScratch p{};
        CK(cudaGetSymbolAddress((void**)&p.er, g_na_elem_resid));
        CK(cudaGetSymbolAddress((void**)&p.wd, g_na_wd_flags));
        CK(cudaGetSymbolAddress((void**)&p.node, g_na_node_work));
        g_na_ptr[dev] = p;
        g_na_ready[dev] = true;
    }
    *out = g_na_ptr[dev];
    return SW2G_OK;
}

extern "C" int sw2g_assemble_residual_noalloc(sw2g_model* m, const double* d_sol, const double* d_sol_old,
                                              const double* d_sol_older, double* d_residual) {
    NEED(m && d_sol && d_sol_old && d_sol_older && d_residual, "sw2g_assemble_residual_noalloc: null argument");
    if (m->Etot > kNoAllocMaxElems || m->V > kNoAllocMaxNodes) {
        g_err = "sw2g_assemble_residual_noalloc: the mesh has more than 131072 elements or nodes (the size of its "
                "fixed work arrays); use sw2g_assemble_residual";
        return SW2G_ERR_ARG;
    }
    NoAllocScratch S{};
    TRY(noalloc_scratch(m, &S));
    // every entry of the three arrays that the gather reads is written first by this call
    // (wet/dry node marks, element flags, 9 (6) residual entries per triangle (segment)), so
    // nothing needs clearing between calls
    launch_wd_flags(m->M, d_sol, d_sol_old, S.node, S.wd, m->st);
    launch_elem_resid(m->M, m->P, d_sol, d_sol_old, d_sol_older, S.wd, S.er, m->st);
    launch_gather_resid(m->V, m->A, S.er, d_residual, m->st);
    CKL();
    CK(cudaStreamSynchronize(m->st));
    return SW2G_OK;
}
