// Host runtime and C ABI of the PD soft-body solver (see include/mgsb.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mgsb.h"
#include "kernels.cuh"
#include "kernels_diag.cuh"
#include "kernels_learned.cuh"
#include "kernels_twolevel.cuh"
#include "kernels_mg.cuh"
#include "kernels_mixed.cuh"
#include "kernels_contact.cuh"
#include "mesh.hpp"
#include "mlp.hpp"
#include "plan.hpp"
#include "setup.hpp"
#include "twolevel.hpp"

using namespace mgsb;

namespace {

constexpr int kBlock = 256;
inline int grid_for(int n) { return (n + kBlock - 1) / kBlock; }
// blocks of kBlock threads for a row-group kernel (32/S lanes per row, slices of S rows)
inline int grid_rows(int n, int S) { return ((n + S - 1) / S * 32 + kBlock - 1) / kBlock; }

// Device allocation owned by the solver.
struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
};

using BodyHost = PlanBody;

struct LevelDev {
    int n = 0;
    int S = 32;
    int nnz = 0;
    int nchild = 0;        // restriction entries (children of this level's vertices)
    int ell_entries = 0;   // stored sliced-ELL entries incl. padding
    // sliced ELL (off-diagonal)
    int32_t* slice_ptr = nullptr;
    int32_t* ell_col = nullptr;
    float* ell_val = nullptr;
    float* diag0 = nullptr;
    float* c = nullptr;
    float* dfull = nullptr;
    float* dinv = nullptr;
    float4* r = nullptr;
    float4* e = nullptr;
    float4* e2 = nullptr;
    float4* res = nullptr;
    // prolongation rows of the next finer level (this level = coarse side)
    int4* pid = nullptr;
    float4* pw = nullptr;
    // OP = Off(this level) * P(next coarser level), sliced ELL (this level's slice height)
    int32_t* op_slice_ptr = nullptr;
    int32_t* op_col = nullptr;
    float* op_val = nullptr;
    // restriction CSR (children in the finer level)
    int32_t* rptr = nullptr;
    int32_t* rcol = nullptr;
    float* rw = nullptr;
    // level 1: RO = R * Off(level 0), CSR (columns: level-0 vertices)
    int32_t* ro_ptr = nullptr;
    int32_t* ro_col = nullptr;
    float* ro_val = nullptr;
};

}  // namespace

struct mgsb_solver {
    mgsb_params p{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    std::vector<BodyHost> bodies;
    int N0 = 0, T = 0;
    bool dirty = true;          // derived data must be rebuilt before the next step
    bool graph_valid = false;
    cudaGraphExec_t graph_exec = nullptr;
    cudaGraph_t graph = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timed = false;
    bool capture_error = false;   // a graph-building step inside a capture failed
    mgsb_status enqueue_status = MGSB_OK;   // first failed launch of the frame being enqueued (message in err)
    int launches = 0;
    // per-launch CUDA events of a profiled (eager) frame
    bool profiling = false;
    // kernel replay (mgsb_time_kernel): while profiling with replay_name set,
    // only the launches of that kernel get events, and each is repeated
    // replay_reps times back to back between them
    std::string replay_name;
    int replay_reps = 1;
    std::vector<std::string> prof_names;
    std::vector<cudaEvent_t> prof_ev;
    std::vector<DevMem> state_mem, derived_mem;
    // host-side tool/body table (what the next step uploads) and a ring of
    // pinned staging slots, each reused only after its previous copy finished
    BodyDev* bodies_host = nullptr;
    SphereSet* spheres_host = nullptr;
    static constexpr int kStage = 4;
    char* stage[kStage] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t stage_ev[kStage] = {nullptr, nullptr, nullptr, nullptr};
    int stage_idx = 0;
    // pinned host buffer for readbacks (N0 x 16 bytes: positions, velocities, flags)
    char* readback = nullptr;
    float* xpack = nullptr;   // positions as packed xyz (mgsb_get_frame_view)
    // ---- state (kept across rebuilds)
    float4 *x = nullptr, *xb = nullptr, *v = nullptr, *s = nullptr, *last = nullptr, *prev = nullptr;
    int32_t* cflag = nullptr;
    float* cdepth = nullptr;
    float* cenergy = nullptr;    // reference kind: contact energy of the last iteration
    int32_t* nonfinite = nullptr;
    BodyDev* bodies_dev = nullptr;
    SphereSet* spheres_dev = nullptr;
    // ---- derived (rebuilt)
    int32_t* body_of = nullptr;
    float* fixf = nullptr;
    float* mass = nullptr;       // ref: density-1 mass; mg: m/h^2
    float* vdiag = nullptr;      // ref: volume diagonal; mg: L diagonal
    int4* tets = nullptr;
    float4 *tA = nullptr, *tB = nullptr;
    float2* tC = nullptr;
    int4* slot_of = nullptr;
    int32_t* slot_ptr = nullptr;
    float4* slots = nullptr;
    // multigrid
    float4 *b = nullptr, *b0 = nullptr, *target = nullptr, *d = nullptr, *d2 = nullptr;
    // mixed precision (FP64 master state and outer residual)
    double4 *x64 = nullptr, *v64 = nullptr, *s64 = nullptr, *last64 = nullptr, *dd64 = nullptr, *b64 = nullptr,
            *b0_64 = nullptr;
    float4 *d32 = nullptr, *r32 = nullptr;
    double *ell_val64 = nullptr, *diag64 = nullptr, *A0dense64 = nullptr, *B0dense64 = nullptr, *Ainv64 = nullptr;
    uint8_t* is_surf = nullptr;
    size_t factor_smem64 = 0;
    float* c0 = nullptr;
    int32_t* surf = nullptr;
    int nsurf = 0;
    // capsule against the surface triangles (multigrid kinds): per triangle its
    // vertices + the inner vertex of its tet, per vertex its triangles (CSR over
    // all vertices, ascending), per triangle this frame's push
    bool tri_contact = false;
    int ctri_n = 0;
    int4* ctri = nullptr;
    int32_t *vt_ptr = nullptr, *vt_idx = nullptr;
    double4* tri_push = nullptr;
    // uniform-grid broad phase of the tool contact (multigrid kinds)
    bool broad_phase = false;
    BpGrid* bp_grids = nullptr;
    int bp_ncells = 0;
    int32_t *bp_counts = nullptr, *bp_start = nullptr, *bp_sorted = nullptr, *bp_list = nullptr, *bp_nlist = nullptr;
    int2* bp_cellrank = nullptr;
    uint8_t* bp_cand = nullptr;
    float4* d_final = nullptr;   // displacement buffer that holds the last frame's d (FP32 multigrid)
    // surface normals: triangles (global vertex ids), surface vertices, and the
    // vertex->triangle CSR (triangle ids local to the body); per body the
    // triangle range [f_off, f_off+nf) and surface-vertex range [sv_off, sv_off+nsv)
    int4* nrm_tris = nullptr;
    int32_t *nrm_sv = nullptr, *nrm_ptr = nullptr, *nrm_fidx = nullptr;
    std::vector<int> nrm_f_off, nrm_nf, nrm_sv_off, nrm_nsv;
    std::vector<int32_t> nrm_sv_host;
    int nrm_max_f = 0, nrm_max_sv = 0;
    float4 *nrm_face = nullptr, *nrm_out = nullptr;   // scratch: triangle normals, vertex normals
    // energy reduction scratch: per-block partials and the five results
    double *energy_part = nullptr, *energy_out = nullptr;
    std::vector<LevelDev> lev;   // lev[0] = finest
    float *A0dense = nullptr, *B0dense = nullptr, *Lfac = nullptr, *Ldinv = nullptr, *c_prev = nullptr;
    int2* range = nullptr;
    int32_t* dense_off_d = nullptr;
    int cluster = 1;
    int fuse_l0 = 1;
    int coarse_block = 512;
    int split = 1;   // first level of the cluster kernel; levels 1..split-1 run grid-wide
    bool pdl = true;  // programmatic dependent launch between consecutive kernels
    bool fuse_prolong = true;   // prolongation + first post-sweep as one kernel (k_prolong_sweep)
    bool fuse_res0 = false;     // level-1 restriction straight from level 0 (k_lvl_restrict_res0)
    // autotuner overrides (0 / -1 = pick by size)
    int tune_cluster = 0, tune_fuse = -1, tune_split = 0;
    // dense coarse operator (one body): levels split..L-1 as M = their V-cycle's matrix,
    // formed once per frame (k_op_* kernels) and applied per V-cycle (k_coarse_apply)
    int tune_dense = 0;
    bool dense_op = false;
    int dop_cap = 0;                           // rows of the largest level the operator may start at
    float* dop_work = nullptr;                 // per level l: R, E, E2, RES blocks of n_l x dop_cap floats
    std::vector<size_t> dop_off;               // offset of level l's four blocks in dop_work (SIZE_MAX: none)
    const float* dop_result = nullptr;         // the frame's M (n_F x n_F, row-major): in dop_work, or the coarsest inverse
    std::vector<int> maxv;   // largest body's rows on each level
    std::vector<int2> range_host;
    int max_smem_optin = 0;
    int32_t* fac_valid = nullptr;
    size_t factor_smem = 0;
    int max_coarsest = 0;
    // host copies of precompute for export
    std::vector<float> h_inv, h_ac, h_vol, h_mass, h_diag;
    // learned smoother (multigrid kinds): network, guard ratio and level-0 buffers
    const mgsb_mlp* ls_net = nullptr;
    cudaStream_t aux_stream = nullptr;   // captures the bodies of conditional graph nodes
    float ls_gamma = 0.5f;
    int ls_ntiles = 0, ls_nblk = 0, sm_count = 148;
    uint8_t* ls_tiles = nullptr;
    float* ls_scale = nullptr;
    float4 *ls_r = nullptr, *ls_save = nullptr, *ls_dpost = nullptr;
    float4* ls_rc = nullptr;    // per-frame row constants of the sweep's features (k_ls_row_consts)
    int2* ls_win = nullptr;     // per 128-row tile: the residual rows the sweep stages in shared memory
    float *ls_part0 = nullptr, *ls_part1 = nullptr;
    // ls_gate: the last frame's decision (1: a learned V-cycle failed its check and the
    // frame's solve was repeated with plain V-cycles); ls_part0 / ls_part1: block sums of
    // |r|^2 before / after each of the frame's ls_cycles learned V-cycles (ls_nblk each)
    int32_t *ls_gate = nullptr, *ls_werr = nullptr;
    int ls_cycles = 1;
    unsigned int* ls_ticket = nullptr;   // last-block ticket of the guard kernel (self-resetting)
    unsigned long long* ls_stats = nullptr;
    // training-pair generation (allocated on first use)
    float *ls_xf = nullptr, *ls_t = nullptr, *ls_s = nullptr;
    uint8_t* ls_mask = nullptr;
    float4 *ls_e1 = nullptr, *ls_e2 = nullptr, *ls_ec = nullptr;
    std::vector<DevMem> pair_mem;
    ~mgsb_solver();
};

mgsb_solver::~mgsb_solver() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto& m : derived_mem) cudaFree(m.p);
    for (auto& m : state_mem) cudaFree(m.p);
    for (auto& m : pair_mem) cudaFree(m.p);
    delete[] bodies_host;
    delete spheres_host;
    for (int k = 0; k < kStage; ++k) {
        if (stage[k]) cudaFreeHost(stage[k]);
        if (stage_ev[k]) cudaEventDestroy(stage_ev[k]);
    }
    if (readback) cudaFreeHost(readback);
    if (aux_stream) cudaStreamDestroy(aux_stream);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (cudaEvent_t e : prof_ev) cudaEventDestroy(e);
    if (own_stream && stream) cudaStreamDestroy(stream);
}

namespace {

mgsb_status set_err(mgsb_solver* h, mgsb_status s, const char* fmt, ...) {
    if (h) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        h->err = buf;
    }
    return s;
}

#define CUDA_TRY(h, call)                                                                                  \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess)                                                                             \
            return set_err(h, MGSB_CUDA_ERROR, "%s failed: %s", #call, cudaGetErrorString(e_));            \
    } while (0)

template <typename T>
mgsb_status dalloc(mgsb_solver* h, std::vector<DevMem>& pool, T** out, size_t count) {
    *out = nullptr;
    if (count == 0) count = 1;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) return set_err(h, MGSB_OUT_OF_MEMORY, "cudaMalloc(%zu) failed: %s", count * sizeof(T), cudaGetErrorString(e));
    pool.push_back({p, count * sizeof(T)});
    *out = static_cast<T*>(p);
    return MGSB_OK;
}

template <typename T>
mgsb_status dupload(mgsb_solver* h, std::vector<DevMem>& pool, T** out, const std::vector<T>& src) {
    mgsb_status s = dalloc(h, pool, out, src.size());
    if (s != MGSB_OK) return s;
    if (!src.empty()) CUDA_TRY(h, cudaMemcpy(*out, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    return MGSB_OK;
}

void free_pool(std::vector<DevMem>& pool) {
    for (auto& m : pool) cudaFree(m.p);
    pool.clear();
}

#define TRY(expr)                          \
    do {                                   \
        mgsb_status s_ = (expr);           \
        if (s_ != MGSB_OK) return s_;      \
    } while (0)

bool is_mg(const mgsb_solver* h) { return h->p.solver == MGSB_SOLVER_MULTIGRID; }

// Level-0 Jacobi sweeps (before and after the coarse correction) of a learned
// solver's plain fallback at least: the configured plain multigrid's 2+2.
constexpr int kFallbackL0Sweeps = 2;

// Shape of the coarse V-cycle kernel: explicit tuning if set, else by size
// (level-0 work fused for bodies up to 40k vertices; ~2.5k rows per CTA).
size_t coarse_smem_bytes(const mgsb_solver* h, int cs, int split);

// Largest body's rows on a coarse level below which it stays in the cluster
// kernel by default; larger levels run as grid-wide kernels over all SMs.
constexpr int kClusterLevelRows = 1024;

// The dense coarse operator can start at level `split`: one body, at most
// dop_cap rows there, and the apply kernel's shared memory (the split level's
// rows and this CTA's share of them) within the device's limit.
bool dense_eligible(const mgsb_solver* h, int split) {
    return h->bodies.size() == 1 && split >= 1 && h->dop_work != nullptr && h->maxv[split] <= h->dop_cap &&
           coarse_apply_smem_bytes(h->maxv[split]) <= (size_t)h->max_smem_optin;
}

void apply_tuning(mgsb_solver* h) {
    // Default: the distributed-shared-memory kernel for the levels up to
    // kClusterLevelRows rows; larger coarse levels run grid-wide.
    const int L = h->p.levels;
    if ((int)h->maxv.size() < L) return;   // before set-up
    h->fuse_l0 = h->tune_fuse >= 0 ? h->tune_fuse : 0;
    if (h->p.precision == MGSB_PRECISION_MIXED || h->ls_net) h->fuse_l0 = 0;   // these run the DSM kernel
    if (h->fuse_l0) {
        h->split = 1;
    } else if (h->tune_split > 0) {
        h->split = std::min(h->tune_split, L - 1);
    } else {
        h->split = 1;
        while (h->split < L - 1 && h->maxv[h->split] > kClusterLevelRows) ++h->split;
    }
    h->dense_op = h->tune_dense && !h->fuse_l0 && dense_eligible(h, h->split);
    if (h->tune_cluster > 0) {
        h->cluster = h->tune_cluster;
    } else if (h->fuse_l0) {
        h->cluster = std::min(16, std::max(1, (h->maxv[0] + 2559) / 2560));
    } else {
        // ~64 rows of the first owned level per CTA (one body: latency bound, so
        // more CTAs shorten every phase); at most 2 CTAs per body in a batch
        const int cap = h->bodies.size() > 1 ? 2 : 16;
        h->cluster = std::min(cap, std::max(1, (h->maxv[h->split] + 63) / 64));
        while (h->cluster < 16 && coarse_smem_bytes(h, h->cluster, h->split) > (size_t)h->max_smem_optin) ++h->cluster;
    }
}

void invalidate_graph(mgsb_solver* h) {
    if (h->graph_exec) {
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    if (h->graph) {
        cudaGraphDestroy(h->graph);
        h->graph = nullptr;
    }
    h->graph_valid = false;
}

// Uniform grids of the broad phase: per body, cells of about twice the
// surface vertex spacing (sqrt(bbox area / surface vertices)), at most 128
// per axis, over the rest bounding box of its surface plus one cell.
mgsb_status setup_broad_phase(mgsb_solver* h, std::vector<DevMem>& pool) {
    std::vector<BpGrid> grids;
    int cells = 0, sorted = 0;
    for (const BodyHost& B : h->bodies) {
        double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        for (size_t k = 0; k < B.surface.size(); ++k)
            for (int a = 0; a < 3; ++a) {
                const double x = B.rest[3 * (size_t)B.surface[k] + a];
                lo[a] = k ? std::min(lo[a], x) : x;
                hi[a] = k ? std::max(hi[a], x) : x;
            }
        const double ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
        const double area = 2.0 * (ext[0] * ext[1] + ext[1] * ext[2] + ext[0] * ext[2]);
        double hc = 2.0 * std::sqrt(area / (double)std::max<size_t>(B.surface.size(), 1));
        for (int a = 0; a < 3; ++a) hc = std::max(hc, ext[a] / 128.0);
        if (!(hc > 0.0)) hc = 1.0;
        BpGrid g;
        g.ox = (float)(lo[0] - hc);
        g.oy = (float)(lo[1] - hc);
        g.oz = (float)(lo[2] - hc);
        g.inv_h = (float)(1.0 / hc);
        g.nx = (int)std::floor(ext[0] / hc) + 3;
        g.ny = (int)std::floor(ext[1] / hc) + 3;
        g.nz = (int)std::floor(ext[2] / hc) + 3;
        g.cell_off = cells;
        g.start_off = cells + (int)grids.size();
        g.sorted_off = sorted;
        cells += g.nx * g.ny * g.nz;
        sorted += (int)B.surface.size();
        grids.push_back(g);
    }
    if (sorted != h->nsurf) return set_err(h, MGSB_NOT_SUPPORTED, "surface lists disagree (%d vs %d)", sorted, h->nsurf);
    h->bp_ncells = cells;
    TRY(dupload(h, pool, &h->bp_grids, grids));
    TRY(dalloc(h, pool, &h->bp_counts, (size_t)cells));
    TRY(dalloc(h, pool, &h->bp_start, (size_t)cells + grids.size()));
    TRY(dalloc(h, pool, &h->bp_sorted, (size_t)h->nsurf));
    TRY(dalloc(h, pool, &h->bp_list, (size_t)h->nsurf));
    TRY(dalloc(h, pool, &h->bp_nlist, 1));
    TRY(dalloc(h, pool, &h->bp_cellrank, (size_t)h->nsurf));
    TRY(dalloc(h, pool, &h->bp_cand, (size_t)h->N0));
    CUDA_TRY(h, cudaMemset(h->bp_nlist, 0, sizeof(int32_t)));
    CUDA_TRY(h, cudaMemset(h->bp_cand, 0, (size_t)h->N0));
    return MGSB_OK;
}

// Surface triangles of every body (extract_surface order), the surface
// vertices in ascending order and, per surface vertex, its triangles in
// ascending order; plus the two scratch arrays the normals pass writes.
mgsb_status upload_normals_data(mgsb_solver* h, std::vector<DevMem>& pool) {
    std::vector<int4> tris_all, ctri_all;
    std::vector<int32_t> sv_all, ptr_all{0}, fidx_all;
    std::vector<int32_t> vt_cnt(h->N0 + 1, 0), vt_idx_all;
    h->nrm_f_off.clear();
    h->nrm_nf.clear();
    h->nrm_sv_off.clear();
    h->nrm_nsv.clear();
    h->nrm_max_f = h->nrm_max_sv = 0;
    for (const BodyHost& B : h->bodies) {
        std::vector<int32_t> tris, opp;
        extract_surface(B.tets.data(), B.T, tris, opp);
        const int nf = (int)(tris.size() / 3);
        h->nrm_f_off.push_back((int)tris_all.size());
        h->nrm_nf.push_back(nf);
        std::vector<int32_t> cnt(B.V + 1, 0);
        for (int f = 0; f < nf; ++f) {
            tris_all.push_back(int4{tris[3 * f] + B.v_off, tris[3 * f + 1] + B.v_off, tris[3 * f + 2] + B.v_off, 0});
            ctri_all.push_back(
                int4{tris[3 * f] + B.v_off, tris[3 * f + 1] + B.v_off, tris[3 * f + 2] + B.v_off, opp[f] + B.v_off});
            for (int q = 0; q < 3; ++q) ++cnt[tris[3 * f + q] + 1];
        }
        std::vector<int32_t> start(B.V + 1, 0);
        for (int i = 0; i < B.V; ++i) start[i + 1] = start[i] + cnt[i + 1];
        std::vector<int32_t> list(start[B.V]);
        std::vector<int32_t> fill(start.begin(), start.end() - 1);
        for (int f = 0; f < nf; ++f)
            for (int q = 0; q < 3; ++q) list[fill[tris[3 * f + q]]++] = f;   // ascending f per vertex
        h->nrm_sv_off.push_back((int)sv_all.size());
        int nsv = 0;
        for (int i = 0; i < B.V; ++i) {
            if (start[i + 1] == start[i]) continue;
            sv_all.push_back(i + B.v_off);
            for (int e = start[i]; e < start[i + 1]; ++e) fidx_all.push_back(list[e]);
            ptr_all.push_back((int32_t)fidx_all.size());
            ++nsv;
        }
        h->nrm_nsv.push_back(nsv);
        h->nrm_max_f = std::max(h->nrm_max_f, nf);
        h->nrm_max_sv = std::max(h->nrm_max_sv, nsv);
    }
    // vertex -> surface triangles over all vertices (global triangle ids, ascending)
    for (const int4& t : ctri_all) {
        ++vt_cnt[t.x + 1];
        ++vt_cnt[t.y + 1];
        ++vt_cnt[t.z + 1];
    }
    for (int i = 0; i < h->N0; ++i) vt_cnt[i + 1] += vt_cnt[i];
    vt_idx_all.resize(vt_cnt[h->N0]);
    {
        std::vector<int32_t> fill(vt_cnt.begin(), vt_cnt.end() - 1);
        for (int g = 0; g < (int)ctri_all.size(); ++g) {
            vt_idx_all[fill[ctri_all[g].x]++] = g;
            vt_idx_all[fill[ctri_all[g].y]++] = g;
            vt_idx_all[fill[ctri_all[g].z]++] = g;
        }
    }
    h->ctri_n = (int)ctri_all.size();
    TRY(dupload(h, pool, &h->ctri, ctri_all));
    TRY(dupload(h, pool, &h->vt_ptr, vt_cnt));
    TRY(dupload(h, pool, &h->vt_idx, vt_idx_all));
    TRY(dalloc(h, pool, &h->tri_push, (size_t)std::max(1, h->ctri_n)));
    CUDA_TRY(h, cudaMemset(h->tri_push, 0, (size_t)std::max(1, h->ctri_n) * sizeof(double4)));
    h->nrm_sv_host = sv_all;
    TRY(dupload(h, pool, &h->nrm_tris, tris_all));
    TRY(dupload(h, pool, &h->nrm_sv, sv_all));
    TRY(dupload(h, pool, &h->nrm_ptr, ptr_all));
    TRY(dupload(h, pool, &h->nrm_fidx, fidx_all));
    TRY(dalloc(h, pool, &h->nrm_face, (size_t)std::max(1, h->nrm_max_f)));
    TRY(dalloc(h, pool, &h->nrm_out, (size_t)std::max(1, h->nrm_max_sv)));
    return MGSB_OK;
}

// ---------------------------------------------------------------------------
// Derived data (rebuilt when fixed set / material / params change)
// ---------------------------------------------------------------------------
mgsb_status rebuild(mgsb_solver* h) {
    CUDA_TRY(h, cudaSetDevice(h->device));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (h->graph_exec) {
        cudaGraphExecDestroy(h->graph_exec);
        h->graph_exec = nullptr;
    }
    if (h->graph) {
        cudaGraphDestroy(h->graph);
        h->graph = nullptr;
    }
    h->graph_valid = false;
    free_pool(h->derived_mem);
    h->lev.clear();
    auto& pool = h->derived_mem;
    const bool mg = is_mg(h);
    Plan P;
    std::string perr;
    if (!build_plan(h->bodies, h->p, P, perr)) return set_err(h, MGSB_INVALID_ARG, "%s", perr.c_str());
    const int N0 = P.N0, T = P.T;
    TRY(dupload(h, pool, &h->body_of, P.body_of));
    TRY(dupload(h, pool, &h->fixf, P.fixf));
    TRY(dupload(h, pool, &h->mass, P.mass));
    TRY(dupload(h, pool, &h->vdiag, P.diag));
    TRY(dupload(h, pool, &h->tets, P.tets));
    TRY(dupload(h, pool, &h->slot_of, P.slot_of));
    TRY(dupload(h, pool, &h->tA, P.tA));
    TRY(dupload(h, pool, &h->tB, P.tB));
    TRY(dupload(h, pool, &h->tC, P.tC));
    TRY(dupload(h, pool, &h->slot_ptr, P.slot_ptr));
    TRY(dalloc(h, pool, &h->slots, 4 * (size_t)T));
    CUDA_TRY(h, cudaMemset(h->slots, 0, 4 * (size_t)T * sizeof(float4)));
    h->h_inv = P.h_inv;
    h->h_ac = P.h_ac;
    h->h_vol = P.h_vol;
    h->h_mass = P.h_mass;
    h->h_diag = P.h_diag;
    if (mg) {
        const int L = h->p.levels;
        for (int l = 0; l < L; ++l) {
            const PlanLevel& pl = P.levels[l];
            LevelDev ld;
            ld.n = pl.n;
            ld.S = pl.S;
            ld.nnz = pl.nnz;
            ld.nchild = pl.rptr.empty() ? 0 : pl.rptr.back();
            ld.ell_entries = (int)pl.ell_col.size();
            TRY(dupload(h, pool, &ld.slice_ptr, pl.slice_ptr));
            TRY(dupload(h, pool, &ld.ell_col, pl.ell_col));
            TRY(dupload(h, pool, &ld.ell_val, pl.ell_val));
            if (!pl.op_slice_ptr.empty()) {
                TRY(dupload(h, pool, &ld.op_slice_ptr, pl.op_slice_ptr));
                TRY(dupload(h, pool, &ld.op_col, pl.op_col));
                TRY(dupload(h, pool, &ld.op_val, pl.op_val));
            }
            if (!pl.ro_ptr.empty() && !pl.ro_col.empty()) {
                TRY(dupload(h, pool, &ld.ro_ptr, pl.ro_ptr));
                TRY(dupload(h, pool, &ld.ro_col, pl.ro_col));
                TRY(dupload(h, pool, &ld.ro_val, pl.ro_val));
            }
            TRY(dalloc(h, pool, &ld.dfull, pl.n));
            TRY(dalloc(h, pool, &ld.dinv, pl.n));
            TRY(dalloc(h, pool, &ld.res, pl.n));
            if (l == 0) {
                ld.diag0 = h->vdiag;
                TRY(dalloc(h, pool, &h->c0, N0));
                CUDA_TRY(h, cudaMemset(h->c0, 0, N0 * sizeof(float)));
                ld.c = h->c0;
            } else {
                TRY(dupload(h, pool, &ld.diag0, pl.diag0));
                TRY(dupload(h, pool, &ld.pid, pl.pid));
                TRY(dupload(h, pool, &ld.pw, pl.pw));
                TRY(dupload(h, pool, &ld.rptr, pl.rptr));
                TRY(dupload(h, pool, &ld.rcol, pl.rcol));
                TRY(dupload(h, pool, &ld.rw, pl.rw));
                TRY(dalloc(h, pool, &ld.c, pl.n));
                TRY(dalloc(h, pool, &ld.r, pl.n));
                TRY(dalloc(h, pool, &ld.e, pl.n));
                TRY(dalloc(h, pool, &ld.e2, pl.n));
                CUDA_TRY(h, cudaMemset(ld.e, 0, pl.n * sizeof(float4)));
                CUDA_TRY(h, cudaMemset(ld.e2, 0, pl.n * sizeof(float4)));
            }
            h->lev.push_back(ld);
        }
        TRY(dalloc(h, pool, &h->b, N0));
        TRY(dalloc(h, pool, &h->b0, N0));
        TRY(dalloc(h, pool, &h->d, N0));
        TRY(dalloc(h, pool, &h->d2, N0));
        CUDA_TRY(h, cudaMemset(h->d, 0, N0 * sizeof(float4)));
        CUDA_TRY(h, cudaMemset(h->d2, 0, N0 * sizeof(float4)));
        TRY(dalloc(h, pool, &h->target, N0));
        CUDA_TRY(h, cudaMemset(h->target, 0, N0 * sizeof(float4)));
        for (size_t bi = 0; bi < h->bodies.size(); ++bi) {
            BodyDev& BD = h->bodies_host[bi];
            BD.cl_off = P.cl_off[bi];
            BD.cl_n = P.cl_n[bi];
            BD.dense_off = P.dense_off[bi];
        }
        h->max_coarsest = P.max_coarsest;
        h->factor_smem = coarsest_smem_elems(P.max_coarsest) * sizeof(float);
        int dev_smem = 0;
        CUDA_TRY(h, cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
        if (h->factor_smem > (size_t)dev_smem)
            return set_err(h, MGSB_NOT_SUPPORTED,
                           "coarsest level has %d vertices; its dense factor needs %zu B of shared memory (max %d): add a level",
                           P.max_coarsest, h->factor_smem, dev_smem);
        CUDA_TRY(h, cudaFuncSetAttribute(k_coarsest_update<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)h->factor_smem));
        TRY(dupload(h, pool, &h->A0dense, P.dense));
        TRY(dupload(h, pool, &h->B0dense, P.dense_inv));
        TRY(dalloc(h, pool, &h->Lfac, P.dense.size()));   // explicit inverse of the coarsest matrix
        TRY(dupload(h, pool, &h->range, P.range));
        h->range_host = P.range;
        if (L > kMaxLevels) return set_err(h, MGSB_NOT_SUPPORTED, "at most %d levels", kMaxLevels);
        CUDA_TRY(h, cudaFuncSetAttribute(k_coarse_vcycle_dsm, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        CUDA_TRY(h, cudaDeviceGetAttribute(&h->max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
        CUDA_TRY(h, cudaFuncSetAttribute(k_coarse_vcycle_dsm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         h->max_smem_optin));
        CUDA_TRY(h, cudaFuncSetAttribute(k_coarse_vcycle_cta, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         h->max_smem_optin));
        CUDA_TRY(h, cudaFuncSetAttribute(k_coarse_apply, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         h->max_smem_optin));
        TRY(dupload(h, pool, &h->dense_off_d, P.dense_off));
        // cluster size of the coarse V-cycle kernel: sized by the rows one body
        // brings to it (level 0 when fused, else level 1)
        h->maxv.assign(L, 0);
        for (size_t bi = 0; bi < h->bodies.size(); ++bi)
            for (int l = 0; l < L; ++l) h->maxv[l] = std::max(h->maxv[l], P.range[bi * L + l].y);
        // the dense coarse operator's matrix, for the largest coarse level it may start at (one body)
        h->dop_cap = 0;
        h->dop_work = nullptr;
        h->dop_result = nullptr;
        h->dop_off.assign(L, SIZE_MAX);
        if (h->bodies.size() == 1)
            for (int l = 1; l < L; ++l)
                if (h->maxv[l] <= kDenseOpMaxRows) h->dop_cap = std::max(h->dop_cap, h->maxv[l]);
        if (h->dop_cap > 0) {   // the levels the operator can span: from the first eligible one down
            size_t tot = 0;
            for (int l = 1; l < L; ++l)
                if (h->maxv[l] <= h->dop_cap) {   // levels shrink with l: every level from the first eligible one
                    h->dop_off[l] = tot;
                    tot += 4 * (size_t)h->maxv[l] * h->dop_cap;
                }
            TRY(dalloc(h, pool, &h->dop_work, tot));
        }
        for (int l = 1; l < L; ++l)
            if (h->lev[l].S != 32 / kLanesC)
                return set_err(h, MGSB_NOT_SUPPORTED, "coarse level %d has slice height %d", l, h->lev[l].S);
        apply_tuning(h);
        CUDA_TRY(h, cudaFuncSetAttribute(k_coarse_vcycle, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        TRY(dalloc(h, pool, &h->c_prev, (size_t)h->lev[L - 1].n));
        TRY(dalloc(h, pool, &h->fac_valid, h->bodies.size()));
        CUDA_TRY(h, cudaMemset(h->fac_valid, 0, h->bodies.size() * sizeof(int32_t)));
        if (h->p.precision == MGSB_PRECISION_MIXED) {
            TRY(dalloc(h, pool, &h->s64, N0));
            TRY(dalloc(h, pool, &h->last64, N0));
            TRY(dalloc(h, pool, &h->dd64, N0));
            TRY(dalloc(h, pool, &h->b64, N0));
            TRY(dalloc(h, pool, &h->b0_64, N0));
            TRY(dalloc(h, pool, &h->d32, N0));
            TRY(dalloc(h, pool, &h->r32, N0));
            TRY(dupload(h, pool, &h->ell_val64, P.levels[0].ell_val64));
            TRY(dupload(h, pool, &h->diag64, P.diag64));
            TRY(dupload(h, pool, &h->A0dense64, P.dense64));
            TRY(dupload(h, pool, &h->B0dense64, P.dense_inv64));
            TRY(dalloc(h, pool, &h->Ainv64, P.dense64.size()));
            TRY(dupload(h, pool, &h->is_surf, P.is_surf));
            h->factor_smem64 = coarsest_smem_elems(P.max_coarsest) * sizeof(double);
            if (h->factor_smem64 > (size_t)h->max_smem_optin)
                return set_err(h, MGSB_NOT_SUPPORTED, "coarsest level has %d vertices; its FP64 factor needs %zu B of shared memory",
                               P.max_coarsest, h->factor_smem64);
            CUDA_TRY(h, cudaFuncSetAttribute(k_coarsest_update<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)h->factor_smem64));
        }
        h->nsurf = (int)P.surf.size();
        TRY(dupload(h, pool, &h->surf, P.surf));
        TRY(setup_broad_phase(h, pool));
    }
    for (size_t bi = 0; bi < h->bodies.size(); ++bi) {
        BodyDev& BD = h->bodies_host[bi];
        BD.v0_off = h->bodies[bi].v_off;
        BD.v0_n = h->bodies[bi].V;
    }
    TRY(upload_normals_data(h, pool));
    if (mg) {
        // learned-smoother level-0 buffers (used when a network is attached)
        h->ls_ntiles = (N0 + kMlpTile - 1) / kMlpTile;
        h->ls_nblk = grid_rows(N0, h->lev[0].S);
        TRY(dalloc(h, pool, &h->ls_tiles, (size_t)h->ls_ntiles * kTileBytes));
        TRY(dalloc(h, pool, &h->ls_scale, (size_t)N0));
        TRY(dalloc(h, pool, &h->ls_r, (size_t)N0));
        TRY(dalloc(h, pool, &h->ls_dpost, (size_t)N0));
        TRY(dalloc(h, pool, &h->ls_rc, (size_t)N0));
        {   // residual window per tile: the tile's rows and every column its rows' ELL entries name
            const PlanLevel& pl = P.levels[0];
            std::vector<int2> win(h->ls_ntiles);
            for (int t = 0; t < h->ls_ntiles; ++t) {
                const int r0 = t * kMlpTile, r1 = std::min(N0, r0 + kMlpTile);
                int lo = r0, hi = r1;
                for (int row = r0; row < r1; ++row) {
                    const int slice = row / pl.S;
                    for (int e = pl.slice_ptr[slice] + (row - slice * pl.S); e < pl.slice_ptr[slice + 1]; e += pl.S) {
                        lo = std::min(lo, pl.ell_col[e]);
                        hi = std::max(hi, pl.ell_col[e] + 1);
                    }
                }
                win[t] = (hi - lo <= kLsWinRows) ? int2{lo, hi} : int2{0, 0};
            }
            TRY(dupload(h, pool, &h->ls_win, win));
        }
        TRY(dalloc(h, pool, &h->ls_save, (size_t)N0));
        h->ls_cycles = std::max(1, h->p.iterations * std::max(1, h->p.refinement_passes));
        TRY(dalloc(h, pool, &h->ls_part0, (size_t)h->ls_cycles * h->ls_nblk));
        TRY(dalloc(h, pool, &h->ls_part1, (size_t)h->ls_cycles * h->ls_nblk));
        TRY(dalloc(h, pool, &h->ls_gate, 1));
        TRY(dalloc(h, pool, &h->ls_werr, 1));
        TRY(dalloc(h, pool, &h->ls_stats, 2));
        TRY(dalloc(h, pool, &h->ls_ticket, 1));
        CUDA_TRY(h, cudaMemset(h->ls_ticket, 0, sizeof(unsigned int)));
        CUDA_TRY(h, cudaMemset(h->ls_stats, 0, 2 * sizeof(unsigned long long)));
        CUDA_TRY(h, cudaMemset(h->ls_gate, 0, sizeof(int32_t)));
        CUDA_TRY(h, cudaMemset(h->ls_werr, 0, sizeof(int32_t)));
        CUDA_TRY(h, cudaFuncSetAttribute(k_ls_sweep_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)ls_sweep_smem_bytes()));
        CUDA_TRY(h, cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device));
    }
    TRY(dalloc(h, pool, &h->energy_part, (size_t)kEnergyBlocks * kEnergyTerms));
    TRY(dalloc(h, pool, &h->energy_out, kEnergyTerms));
    h->dirty = false;
    return MGSB_OK;
}

// ---------------------------------------------------------------------------
// Frame enqueue
// ---------------------------------------------------------------------------
void prof_mark(mgsb_solver* h, const char* name) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    // External: inside stream capture this becomes a real event-record node.
    cudaEventRecordWithFlags(e, h->stream, cudaEventRecordExternal);
    h->prof_ev.push_back(e);
    if (name) h->prof_names.push_back(name);
}

// Number of back-to-back launches of one kernel launch site in the frame
// being enqueued (replay_reps for the kernel mgsb_time_kernel measures, else
// 1), with an event-record node before them when profiling.
int prof_begin(mgsb_solver* h, const char* name) {
    if (!h->profiling) return 1;
    if (!h->replay_name.empty() && h->replay_name != name) return 1;
    prof_mark(h, name);
    return h->replay_name.empty() ? 1 : h->replay_reps;
}

void prof_end(mgsb_solver* h, const char* name) {
    if (h->profiling && (h->replay_name.empty() || h->replay_name == name)) prof_mark(h, nullptr);
}

// Kernel launch on the solver's stream.  With h->pdl the launch carries the
// programmatic-serialization attribute: its blocks may be scheduled while the
// previous kernel finishes, and wait in pdl_enter() until that kernel has
// completed (every kernel launched here calls it first).  Arguments are
// converted to the kernel's parameter types, so every parameter is passed.
template <typename... KArgs, typename... Args>
void launch_kernel(mgsb_solver* h, void (*kernel)(KArgs...), dim3 grid, int block, size_t smem, Args&&... args) {
    static_assert(sizeof...(KArgs) == sizeof...(Args), "pass every kernel parameter");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = h->pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

#define LAUNCH(h, kernel, grid, block, smem, ...)                                  \
    do {                                                                             \
        const int reps_ = prof_begin((h), #kernel);                                  \
        for (int r_ = 0; r_ < reps_; ++r_)                                           \
            launch_kernel((h), kernel, (grid), (block), (smem), __VA_ARGS__);       \
        prof_end((h), #kernel);                                                      \
        ++(h)->launches;                                                             \
    } while (0)

void enqueue_ref_frame(mgsb_solver* h) {
    const int n = h->N0, T = h->T;
    const mgsb_params& p = h->p;
    const BodyHost& B = h->bodies[0];
    LAUNCH(h, k_ref_predict, grid_for(n), kBlock, 0, n, h->x, h->v, h->s, h->prev, h->last, h->fixf, B.damping, p.dt,
           B.gravity[0], B.gravity[1], B.gravity[2]);
    float omega = 1.0f;
    for (int it = 0; it < p.iterations; ++it) {
        LAUNCH(h, k_ref_local, grid_for(T), kBlock, 0, T, h->tets, h->tA, h->tB, h->tC, h->x, h->slot_of, h->slots,
               p.volume_stiffness, 1);
        omega = 4 / (4 - p.cheb_rho * p.cheb_rho * omega);
        LAUNCH(h, k_ref_vertex, grid_for(n), kBlock, 0, n, h->x, h->prev, h->s, h->last, h->v, h->fixf, h->mass,
               h->vdiag, h->slot_ptr, h->slots, h->spheres_dev, p.collision_stiffness, p.dt, omega,
               (double)p.relaxation, it == p.iterations - 1 ? 3 : 0, h->cflag, h->cdepth, h->cenergy,
               h->nonfinite, nullptr, nullptr, nullptr);
    }
    if (p.iterations == 0) {
        // velocity only
        LAUNCH(h, k_velocity, grid_for(n), kBlock, 0, n, h->x, h->last, h->v, p.dt, h->nonfinite);
    }
}

// Dynamic shared memory of the distributed-shared-memory coarse kernel: the
// largest body's rows per CTA on every level it owns (4 vectors) + the whole
// coarsest right-hand side.
// With a cluster of one CTA the one-CTA kernel runs instead: 4 vectors of
// every level it owns.
size_t coarse_smem_bytes(const mgsb_solver* h, int cs, int split) {
    const int L = h->p.levels;
    int best = 0;
    for (size_t bi = 0; bi < h->bodies.size(); ++bi) {
        int nl[kMaxLevels] = {0};
        for (int l = 0; l < L; ++l) nl[l] = h->range_host[bi * L + l].y;
        best = std::max(best, cs == 1 ? coarse_cta_smem_float4(nl, L, split)
                                      : coarse_smem_float4(nl, L, split, cs, nl[L - 1]));
    }
    return (size_t)best * sizeof(float4);
}

// Can the device co-schedule one cluster of this shape?
bool coarse_shape_feasible(mgsb_solver* h, int cs, int block, int fused, int split) {
    const size_t smem = fused ? 0 : coarse_smem_bytes(h, cs, split);
    if (smem > (size_t)h->max_smem_optin) return false;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cs);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (!fused && cs == 1) {   // the one-CTA kernel: an ordinary launch
        int nblk = 0;
        const cudaError_t e1 = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nblk, k_coarse_vcycle_cta, block, smem);
        if (e1 != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return nblk > 0;
    }
    const cudaError_t e = fused ? cudaOccupancyMaxActiveClusters(&nclusters, k_coarse_vcycle, &cfg)
                                : cudaOccupancyMaxActiveClusters(&nclusters, k_coarse_vcycle_dsm, &cfg);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return nclusters > 0;
}

mgsb_status launch_coarse_cluster(mgsb_solver* h, const CoarseArgs& args);

// Coarse part of one V-cycle: from the level-0 residual lv[0].res to the
// level-1 correction lv[1].e.  Levels 1..split-1 run as grid-wide kernels
// (restrict + first sweep, further pre-sweeps, residual going down;
// prolongation and post-sweeps coming back up), the rest in one cluster
// kernel per body.  The post-sweeps of a grid-wide level start in the buffer
// that makes the last one land in lv[l].e.
mgsb_status launch_coarse(mgsb_solver* h, const CoarseArgs& args_in) {
    CoarseArgs args = args_in;
    const int F = h->fuse_l0 ? 1 : h->split;
    args.first = F;
    args.fuse_prolong = h->fuse_prolong ? 1 : 0;
    const int32_t* gate = args.gate;
    float4* cur[kMaxLevels] = {};
    for (int l = 1; l < F; ++l) {
        const LevelView& C = args.lv[l];
        const int g = grid_rows(C.n, 32 / kLanesC);
        if (l == 1 && args.res0_b)
            LAUNCH(h, k_lvl_restrict_res0, g, kBlock, 0, C.n, C.rptr, C.rcol, C.rw, args.ro_ptr, args.ro_col,
                   args.ro_val, args.res0_b, args.lv[0].dfull, (const float4*)args.d, args.pre > 0 ? C.dinv : nullptr,
                   C.r, C.e, gate);
        else
            LAUNCH(h, k_lvl_restrict, g, kBlock, 0, C.n, C.rptr, C.rcol, C.rw, args.lv[l - 1].res,
                   args.pre > 0 ? C.dinv : nullptr, C.r, C.e, gate);
        float4 *a = C.e, *b = C.e2;
        for (int k = 1; k < args.pre; ++k) {
            LAUNCH(h, k_lvl_sweep, g, kBlock, 0, C.n, C.slice_ptr, C.col, C.val, C.dfull, C.dinv, C.r, a, b, gate);
            std::swap(a, b);
        }
        LAUNCH(h, k_lvl_residual, g, kBlock, 0, C.n, C.slice_ptr, C.col, C.val, C.dfull, C.r, a, C.res, gate);
        cur[l] = a;
    }
    if (h->dense_op) {   // levels F..L-1: the restriction to level F and the dense operator, one launch
        const LevelView& C = args.lv[F];
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)coarse_apply_ctas(C.n));
        cfg.blockDim = dim3((unsigned)kDenseApplyThreads);
        cfg.dynamicSmemBytes = coarse_apply_smem_bytes(C.n);
        cfg.stream = h->stream;
        cudaLaunchAttribute attr[2];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)kApplyCluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = h->pdl ? 2 : 1;
        const int reps = prof_begin(h, "k_coarse_apply");
        cudaError_t e = cudaSuccess;
        for (int r = 0; r < reps && e == cudaSuccess; ++r)
            e = cudaLaunchKernelEx(&cfg, k_coarse_apply, C.n, (const int32_t*)C.rptr, (const int32_t*)C.rcol,
                                   (const float*)C.rw, (const float4*)args.lv[F - 1].res,
                                   (const float*)h->dop_result, C.e, gate);
        prof_end(h, "k_coarse_apply");
        ++h->launches;
        if (e != cudaSuccess)
            return h->enqueue_status = set_err(h, MGSB_CUDA_ERROR, "dense coarse apply launch failed: %s",
                                               cudaGetErrorString(e));
    } else {
        TRY(launch_coarse_cluster(h, args));
    }
    for (int l = F - 1; l >= 1; --l) {
        const LevelView& C = args.lv[l];
        const LevelView& Cc = args.lv[l + 1];
        const int g = grid_rows(C.n, 32 / kLanesC);
        if (h->fuse_prolong && args.post > 0) {
            // prolongation + first post-sweep in one launch (from the residual C.res of the descent)
            float4* a = ((args.post - 1) % 2 == 0) ? C.e : C.e2;
            float4* b = (a == C.e) ? C.e2 : C.e;
            LAUNCH(h, k_prolong_sweep<kLanesC>, g, kBlock, 0, C.n, Cc.pid, Cc.pw, Cc.e, C.op_slice_ptr, C.op_col,
                   C.op_val, C.dfull, C.dinv, C.res, cur[l], a, nullptr, nullptr, gate, nullptr, nullptr, nullptr,
                   nullptr);
            for (int k = 1; k < args.post; ++k) {
                LAUNCH(h, k_lvl_sweep, g, kBlock, 0, C.n, C.slice_ptr, C.col, C.val, C.dfull, C.dinv, C.r, a, b, gate);
                std::swap(a, b);
            }
            continue;
        }
        float4* a = (args.post % 2 == 0) ? C.e : C.e2;
        float4* b = (a == C.e) ? C.e2 : C.e;
        LAUNCH(h, k_lvl_prolong, grid_for(C.n), kBlock, 0, C.n, Cc.pid, Cc.pw, Cc.e, cur[l], a, gate);
        for (int k = 0; k < args.post; ++k) {
            LAUNCH(h, k_lvl_sweep, g, kBlock, 0, C.n, C.slice_ptr, C.col, C.val, C.dfull, C.dinv, C.r, a, b, gate);
            std::swap(a, b);
        }
    }
    return MGSB_OK;
}

mgsb_status launch_coarse_cluster(mgsb_solver* h, const CoarseArgs& args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(h->bodies.size() * h->cluster));
    cfg.blockDim = dim3((unsigned)h->coarse_block);
    cfg.dynamicSmemBytes = h->fuse_l0 ? 0 : coarse_smem_bytes(h, h->cluster, args.first);
    if (cfg.dynamicSmemBytes > (size_t)h->max_smem_optin) {
        h->enqueue_status = set_err(h, MGSB_NOT_SUPPORTED,
                                    "coarse kernel shape (cluster %d, split %d) needs %zu B of shared memory per CTA (max %d)",
                                    h->cluster, args.first, cfg.dynamicSmemBytes, h->max_smem_optin);
        return h->enqueue_status;
    }
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)h->cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = h->pdl ? 2 : 1;
    const bool one_cta = !h->fuse_l0 && h->cluster == 1;
    if (one_cta) {   // no cluster attribute: one CTA per body
        cfg.attrs = attr + 1;
        cfg.numAttrs = h->pdl ? 1 : 0;
    }
    // fused: global-memory kernel that also owns the level-0 residual and prolongation;
    // one CTA: every owned level in one CTA's shared memory; else the
    // distributed-shared-memory kernel over the cluster
    const int reps = prof_begin(h, "k_coarse_vcycle");
    cudaError_t e = cudaSuccess;
    for (int r = 0; r < reps && e == cudaSuccess; ++r)
        e = h->fuse_l0 ? cudaLaunchKernelEx(&cfg, k_coarse_vcycle, args)
            : one_cta  ? cudaLaunchKernelEx(&cfg, k_coarse_vcycle_cta, args)
                       : cudaLaunchKernelEx(&cfg, k_coarse_vcycle_dsm, args);
    prof_end(h, "k_coarse_vcycle");
    ++h->launches;
    if (e != cudaSuccess) {
        h->enqueue_status = set_err(h, MGSB_CUDA_ERROR, "coarse V-cycle launch failed: %s", cudaGetErrorString(e));
        return h->enqueue_status;
    }
    return MGSB_OK;
}

// Level 1's restriction forms R (b - D d) - RO d from level 0 directly
// (k_lvl_restrict_res0) when level 1 runs grid-wide (split >= 2), the fused
// prolongation forms the level-0 residual rows it needs, and RO exists; the
// level-0 residual launch is then left out of the V-cycle.
bool res0_fused(const mgsb_solver* h) {
    return h->fuse_res0 && h->fuse_prolong && !h->fuse_l0 && h->split >= 2 && h->lev.size() > 1 &&
           h->lev[1].ro_ptr != nullptr;
}

// Level-0 prolongation d += P e1 and the post-smoothing sweeps (ping-pong
// xa -> xb; on return xa holds the result): the first sweep fused with the
// prolongation (k_prolong_sweep, from the level-0 residual lv[0].res of the
// descent) unless disabled.  b: the right-hand side of the sweeps.
void enqueue_l0_post(mgsb_solver* h, float4*& xa, float4*& xb, float4* b, const int32_t* gate, int post = -1,
                     bool form_res = false) {
    const mgsb_params& p = h->p;
    if (post < 0) post = p.post_sweeps;
    const int n0 = h->N0;
    const LevelDev& l0 = h->lev[0];
    const LevelDev& l1 = h->lev[1];
    const int g0 = grid_rows(n0, l0.S);
    int k0 = 0;
    if (h->fuse_prolong && post > 0) {
        LAUNCH(h, k_prolong_sweep<kLanesL0>, g0, kBlock, 0, n0, l1.pid, l1.pw, l1.e, l0.op_slice_ptr, l0.op_col,
               l0.op_val, l0.dfull, l0.dinv, form_res ? nullptr : l0.res, xa, xb, nullptr, nullptr, gate,
               form_res ? b : nullptr, l0.slice_ptr, l0.ell_col, l0.ell_val);
        std::swap(xa, xb);
        k0 = 1;
    } else {
        LAUNCH(h, k_l0_prolong, grid_for(n0), kBlock, 0, n0, l1.pid, l1.pw, l1.e, xa, gate);
    }
    for (int k = k0; k < post; ++k) {
        LAUNCH(h, k_l0_sweep_rg, g0, kBlock, 0, n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, l0.dinv, xa, xb, b,
               h->b0, h->slot_ptr, h->slots, 0, gate);
        std::swap(xa, xb);
    }
}

// One learned V-cycle on level 0 for A d = b: d is the warm start, or zero
// when from_zero.  Pre-smoothing: residual -> features -> tensor-core MLP
// (d += scale * y).  Coarse correction as in the plain cycle.  Post-smoothing:
// the same learned sweep.  The residual check that judges the cycle is the
// caller's next launch (enqueue_learned_guard); cycle: the cycle's index in
// the frame (its starting residual's block sums go to ls_part0 there).
void enqueue_learned_vcycle(mgsb_solver* h, float4* d, const float4* b, bool from_zero, CoarseArgs ca, int cycle,
                            bool gather_b = false, bool start_residual_ready = false, double4* dd64 = nullptr,
                            float4* d32 = nullptr) {
    const int n0 = h->N0;
    std::vector<LevelDev>& lv = h->lev;
    const LevelDev& l0 = lv[0];
    const int g0 = h->ls_nblk;
    const uint8_t* img = mlp_device_image(h->ls_net);
    const int mgrid = std::min(h->ls_ntiles, 2 * h->sm_count);
    const size_t msmem = ls_sweep_smem_bytes();
    float4* bw = const_cast<float4*>(b);
    (void)from_zero;
    // pre-smoothing (with gather_b the right-hand side b = b0 + slots is assembled here first;
    // start_residual_ready: the previous kernel left ls_r and its block sums, d = 0)
    if (!start_residual_ready)
        LAUNCH(h, k_ls_residual, g0, kLsThreads, 0, n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, h->fixf, d, b,
               h->ls_r, nullptr, h->ls_part0 + (size_t)cycle * g0, gather_b ? h->b0 : nullptr, gather_b ? h->slot_ptr : nullptr,
               gather_b ? h->slots : nullptr, gather_b ? bw : nullptr);
    LAUNCH(h, k_ls_sweep_tc, mgrid, kMlpThreads, msmem, n0, h->ls_ntiles, l0.slice_ptr, l0.ell_col, l0.ell_val,
           l0.dfull, (const float4*)h->ls_rc, (const int2*)h->ls_win, h->fixf, h->ls_r, img, d, h->ls_werr, nullptr,
           nullptr, nullptr);
    // coarse correction (with res0_fused the level-0 residual is not formed: level 1's restriction
    // takes b and d, the post-smoothing kernel forms its rows into ls_dpost's sweep)
    const bool fr = res0_fused(h);
    if (!fr)
        LAUNCH(h, k_l0_residual_rg, g0, kBlock, 0, n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, d, b, l0.res,
               nullptr);
    ca.d = d;
    ca.gate = nullptr;
    ca.res0_b = fr ? b : nullptr;
    launch_coarse(h, ca);
    // post-smoothing: d += P e1 and the residual the learned sweep starts from
    float4* dpost = fr ? h->ls_dpost : d;
    if (h->fuse_prolong) {
        LAUNCH(h, k_prolong_sweep<kLanesL0>, g0, kBlock, 0, n0, lv[1].pid, lv[1].pw, lv[1].e, l0.op_slice_ptr,
               l0.op_col, l0.op_val, l0.dfull, l0.dinv, fr ? nullptr : l0.res, d, dpost, h->fixf, h->ls_r, nullptr,
               fr ? b : nullptr, l0.slice_ptr, l0.ell_col, l0.ell_val);
    } else {
        LAUNCH(h, k_l0_prolong, grid_for(n0), kBlock, 0, n0, lv[1].pid, lv[1].pw, lv[1].e, d, nullptr);
        LAUNCH(h, k_ls_residual, g0, kLsThreads, 0, n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, h->fixf, d, b,
               h->ls_r, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    }
    // with dd64 (mixed kind, check taken by the next outer residual) the sweep also applies d to dd64
    LAUNCH(h, k_ls_sweep_tc, mgrid, kMlpThreads, msmem, n0, h->ls_ntiles, l0.slice_ptr, l0.ell_col, l0.ell_val,
           l0.dfull, (const float4*)h->ls_rc, (const int2*)h->ls_win, h->fixf, h->ls_r, img, d, h->ls_werr, dd64, d32,
           dpost != d ? (const float4*)dpost : nullptr);
}

// The learned sweep's per-frame row constants, once the frame's level-0
// diagonal (contacts included) is known.
void enqueue_ls_row_consts(mgsb_solver* h) {
    const LevelDev& l0 = h->lev[0];
    LAUNCH(h, k_ls_row_consts, h->ls_nblk, kLsThreads, 0, h->N0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull,
           h->vdiag, h->ls_rc);
}

// The residual check of the learned V-cycle `cycle` just enqueued (d, b as
// given to it).  final: the frame's last check, which takes the frame's
// decision (with fb.cond, into the IF node's condition).  dd64 / d32: the
// mixed kind's FP64 update, fused into the check.
struct LearnedFallback {
    bool cond = false;                      // inside a capture: the IF node's handle is valid
    cudaGraphConditionalHandle hnd = 0;
};

// The checks pair the block sums of k_mx_residual / k_ls_residual and of the
// guard block by block: the same 64 rows per block.
static_assert(kLsThreads == kBlock && kLsThreads / kLanesL0 == 64 && kMxThreads / kLanesMx == 64,
              "learned-cycle block sums are paired block by block");

void enqueue_learned_guard(mgsb_solver* h, const float4* d, const float4* b, int cycle, bool final,
                           const LearnedFallback& fb, double4* dd64 = nullptr, float4* d32 = nullptr) {
    const LevelDev& l0 = h->lev[0];
    if (final && fb.cond)
        LAUNCH(h, k_ls_guard_residual<true>, h->ls_nblk, kLsThreads, 0, h->N0, l0.slice_ptr, l0.ell_col, l0.ell_val,
               l0.dfull, h->fixf, d, b, cycle, 1, h->ls_part0, h->ls_part1, h->ls_gamma * h->ls_gamma, h->ls_gate,
               h->ls_stats, fb.hnd, 1, h->ls_ticket, dd64, d32);
    else
        LAUNCH(h, k_ls_guard_residual<false>, h->ls_nblk, kLsThreads, 0, h->N0, l0.slice_ptr, l0.ell_col, l0.ell_val,
               l0.dfull, h->fixf, d, b, cycle, final ? 1 : 0, h->ls_part0, h->ls_part1, h->ls_gamma * h->ls_gamma,
               h->ls_gate, h->ls_stats, fb.hnd, 0, h->ls_ticket, dd64, d32);
}

// Frame-level fallback of the learned smoother, before the frame's learned
// solve: inside a stream capture, the handle of the IF node that will hold
// the plain solve (reset to 0 at every launch of the graph).  A profiled
// frame gets no IF node (profilers do not see the kernels of a graph that
// holds conditional nodes): it is captured in two parts instead.
LearnedFallback begin_learned_fallback(mgsb_solver* h) {
    LearnedFallback fb;
    cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(h->stream, &cst);
    if (cst != cudaStreamCaptureStatusActive || h->profiling) return fb;
    cudaGraph_t g = nullptr;
    if (!h->aux_stream || cudaStreamGetCaptureInfo(h->stream, &cst, nullptr, &g, nullptr, nullptr) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&fb.hnd, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) {
        h->capture_error = true;
        return fb;
    }
    fb.cond = true;
    return fb;
}

// After the learned solve: the plain solve (body) runs when the frame's last
// check found a failed learned V-cycle.  In a capture it becomes the body of
// an IF node (captured on the auxiliary stream); eagerly the host reads the
// decision and enqueues it.  A profiled frame (capture, no IF node) ends its
// first part here, runs it, reads the decision and captures the rest of the
// frame (with the body when it is needed) as its second part on the same
// stream.
template <typename Body>
void end_learned_fallback(mgsb_solver* h, const LearnedFallback& fb, Body&& body) {
    cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(h->stream, &cst);
    if (!fb.cond) {
        if (cst != cudaStreamCaptureStatusNone && !h->profiling) {
            h->capture_error = true;
            return;
        }
        if (cst != cudaStreamCaptureStatusNone) {   // profiled frame: run the first part now
            cudaGraph_t g1 = nullptr;
            cudaGraphExec_t ge1 = nullptr;
            cudaError_t e = cudaStreamEndCapture(h->stream, &g1);
            if (e == cudaSuccess) e = cudaGraphInstantiate(&ge1, g1, 0);
            if (e == cudaSuccess) e = cudaGraphLaunch(ge1, h->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
            if (ge1) cudaGraphExecDestroy(ge1);
            if (g1) cudaGraphDestroy(g1);
            int32_t g = 0;
            if (e == cudaSuccess) e = cudaMemcpy(&g, h->ls_gate, sizeof g, cudaMemcpyDeviceToHost);
            const cudaError_t eb = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) e = eb;
            if (e != cudaSuccess) {
                h->enqueue_status = set_err(h, MGSB_CUDA_ERROR, "profiled frame, first part: %s", cudaGetErrorString(e));
                return;
            }
            if (g) body();
            return;
        }
        int32_t g = 0;
        cudaError_t e = cudaMemcpyAsync(&g, h->ls_gate, sizeof g, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) {
            h->enqueue_status = set_err(h, MGSB_CUDA_ERROR, "learned-smoother check: %s", cudaGetErrorString(e));
            return;
        }
        if (g) body();
        return;
    }
    cudaGraph_t cap_graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = fb.hnd;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    if (cudaStreamGetCaptureInfo(h->stream, &cst, nullptr, &cap_graph, &deps, &nd) != cudaSuccess ||
        cudaGraphAddNode(&node, cap_graph, deps, nd, &np) != cudaSuccess ||
        cudaStreamUpdateCaptureDependencies(h->stream, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess ||
        cudaStreamBeginCaptureToGraph(h->aux_stream, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        h->capture_error = true;
        return;
    }
    cudaStream_t main_stream = h->stream;
    const int launches = h->launches;
    h->stream = h->aux_stream;
    body();
    h->launches = launches;   // launches_per_frame counts the frame that runs when every check passes
    cudaGraph_t bg = nullptr;
    if (cudaStreamEndCapture(h->stream, &bg) != cudaSuccess) h->capture_error = true;
    h->stream = main_stream;
}

// Broad phase on the predicted positions spos: clear the previous
// candidates, bin, scan, scatter, query.  narrow: the query also runs the
// FP32 kind's narrow phase (contact flag, stiffness, target).
void enqueue_broad_phase(mgsb_solver* h, const float4* spos, bool narrow) {
    const int nb = (int)h->bodies.size();
    const int gclear = std::max(1, std::min(grid_for(std::max(h->bp_ncells, h->nsurf)), 4 * h->sm_count));
    LAUNCH(h, k_bp_clear, gclear, kBlock, 0, h->bp_ncells, h->bp_counts, h->bp_list, h->bp_nlist, h->bp_cand,
           narrow ? h->cflag : nullptr, narrow ? h->c0 : nullptr, narrow ? h->target : nullptr);
    LAUNCH(h, k_bp_bin, grid_for(h->nsurf), kBlock, 0, h->nsurf, h->surf, h->body_of, h->bp_grids, spos, h->bp_counts,
           h->bp_cellrank, h->bp_nlist);
    LAUNCH(h, k_bp_scan, nb, kBpScanThreads, 0, h->bp_grids, h->bp_counts, h->bp_start);
    LAUNCH(h, k_bp_scatter, grid_for(h->nsurf), kBlock, 0, h->nsurf, h->surf, h->bp_cellrank, h->bp_start,
           h->bp_sorted);
    LAUNCH(h, k_bp_query, nb, kBlock, 0, h->bp_grids, h->bodies_dev, h->bp_start, h->bp_sorted, spos, h->fixf,
           h->p.contact_stiffness, h->bp_cand, h->bp_list, h->bp_nlist, narrow ? h->cflag : nullptr,
           narrow ? h->c0 : nullptr, narrow ? h->target : nullptr);
}

// The frame's dense coarse operator M (levels split..L-1 of the one body), once
// the coarse diagonals and the coarsest inverse are refreshed: the V-cycle of
// those levels applied to the n_F x n_F identity, all columns at once (scalar
// blocks, a thread per column, one launch per phase: first sweep from zero, further pre-sweeps,
// residual, restriction going down; the dense coarsest product; prolongation
// and post-sweeps coming back up).  h->dop_result points at the block that
// holds M.
void enqueue_coarse_operator(mgsb_solver* h, const CoarseArgs& ca) {
    if (!h->dense_op) return;
    const mgsb_params& p = h->p;
    const int L = p.levels, F = h->split;
    const int m = ca.lv[F].n;
    auto blk = [&](int l, int v) { return h->dop_work + h->dop_off[l] + (size_t)v * ca.lv[l].n * h->dop_cap; };
    if (F == L - 1) {   // the operator is the coarsest inverse itself
        if (ca.Ainv64) {
            LAUNCH(h, k_op_round, grid_for(m * m), kBlock, 0, m * m, ca.Ainv64, blk(F, 0));
            h->dop_result = blk(F, 0);
        } else {
            h->dop_result = ca.Ainv;
        }
        return;
    }
    auto grid = [&](int n) { return dim3((unsigned)n, (unsigned)((m + kOpThreads - 1) / kOpThreads)); };
    constexpr int R = 0, E = 1, E2 = 2, RES = 3;
    float* cur[kMaxLevels] = {};
    LAUNCH(h, k_op_init, grid(m), kOpThreads, 0, m, m, (p.pre_sweeps > 0 && F < L - 1) ? ca.lv[F].dinv : nullptr,
           blk(F, R), blk(F, E));
    cur[F] = blk(F, E);
    for (int l = F; l < L - 1; ++l) {
        const LevelView& C = ca.lv[l];
        for (int k = 1; k < p.pre_sweeps; ++k) {
            float* dst = cur[l] == blk(l, E) ? blk(l, E2) : blk(l, E);
            LAUNCH(h, k_op_sweep, grid(C.n), kOpThreads, 0, C.n, m, C.slice_ptr, C.col, C.val, C.dfull, C.dinv,
                   (const float*)blk(l, R), (const float*)cur[l], dst, 0);
            cur[l] = dst;
        }
        LAUNCH(h, k_op_sweep, grid(C.n), kOpThreads, 0, C.n, m, C.slice_ptr, C.col, C.val, C.dfull, C.dinv,
               (const float*)blk(l, R), (const float*)cur[l], blk(l, RES), 1);
        const LevelView& Cc = ca.lv[l + 1];
        LAUNCH(h, k_op_restrict, grid(Cc.n), kOpThreads, 0, Cc.n, m, Cc.rptr, Cc.rcol, Cc.rw,
               (const float*)blk(l, RES), (p.pre_sweeps > 0 && l + 1 < L - 1) ? Cc.dinv : nullptr, blk(l + 1, R),
               blk(l + 1, E));
        cur[l + 1] = blk(l + 1, E);
    }
    const LevelView& Cl = ca.lv[L - 1];
    const dim3 gc((unsigned)((Cl.n + kOpcRows - 1) / kOpcRows), (unsigned)((m + kOpcCols - 1) / kOpcCols));
    if (ca.Ainv64)
        LAUNCH(h, k_op_coarsest<double>, gc, kOpcThreads, 0, Cl.n, m, ca.Ainv64, (const float*)blk(L - 1, R),
               blk(L - 1, E));
    else
        LAUNCH(h, k_op_coarsest<float>, gc, kOpcThreads, 0, Cl.n, m, ca.Ainv, (const float*)blk(L - 1, R),
               blk(L - 1, E));
    for (int l = L - 2; l >= F; --l) {
        const LevelView& C = ca.lv[l];
        const LevelView& Cc = ca.lv[l + 1];
        LAUNCH(h, k_op_prolong, grid(C.n), kOpThreads, 0, C.n, m, Cc.pid, Cc.pw, (const float*)cur[l + 1], cur[l]);
        for (int k = 0; k < p.post_sweeps; ++k) {
            float* dst = cur[l] == blk(l, E) ? blk(l, E2) : blk(l, E);
            LAUNCH(h, k_op_sweep, grid(C.n), kOpThreads, 0, C.n, m, C.slice_ptr, C.col, C.val, C.dfull, C.dinv,
                   (const float*)blk(l, R), (const float*)cur[l], dst, 0);
            cur[l] = dst;
        }
    }
    h->dop_result = cur[F];
}

void fill_coarse_args(mgsb_solver* h, CoarseArgs& ca) {
    const mgsb_params& p = h->p;
    const int L = p.levels;
    std::vector<LevelDev>& lv = h->lev;
    ca = CoarseArgs{};
    ca.L = L;
    ca.pre = p.pre_sweeps;
    ca.post = p.post_sweeps;
    ca.fuse_l0 = h->fuse_l0;
    ca.range = h->range;
    ca.dense_off = h->dense_off_d;
    ca.Ainv = h->Lfac;
    ca.Ainv64 = nullptr;
    ca.res0_b = nullptr;
    if (L > 1) {
        ca.ro_ptr = h->lev[1].ro_ptr;
        ca.ro_col = h->lev[1].ro_col;
        ca.ro_val = h->lev[1].ro_val;
    }
    ca.b = h->b;
    for (int l = 0; l < L; ++l) {
        LevelView& v = ca.lv[l];
        v.n = lv[l].n;
        v.slice_ptr = lv[l].slice_ptr;
        v.col = lv[l].ell_col;
        v.val = lv[l].ell_val;
        v.dfull = lv[l].dfull;
        v.dinv = lv[l].dinv;
        v.r = lv[l].r;
        v.e = lv[l].e;
        v.e2 = lv[l].e2;
        v.res = lv[l].res;
        v.pid = lv[l].pid;
        v.pw = lv[l].pw;
        v.rptr = lv[l].rptr;
        v.rcol = lv[l].rcol;
        v.rw = lv[l].rw;
        v.op_slice_ptr = lv[l].op_slice_ptr;
        v.op_col = lv[l].op_col;
        v.op_val = lv[l].op_val;
    }
}

// The FP32 multigrid kind's global solve of one frame, from the contact
// state: right-hand side and diagonals, coarse-level data and the coarsest
// inverse, then the PD iterations (local step, V-cycles).  Returns the
// buffer that holds the final displacement.  learned: learned V-cycles, each
// followed by its residual check.
float4* enqueue_mg_solve(mgsb_solver* h, bool learned, const LearnedFallback& fb) {
    const mgsb_params& p = h->p;
    const int n0 = h->N0, T = h->T, L = p.levels;
    const int nb = (int)h->bodies.size();
    const float om = p.jacobi_omega;
    std::vector<LevelDev>& lv = h->lev;
    float4* xa = h->d;    // displacement d = x - s (ping)
    float4* xb = h->d2;   // pong
    LAUNCH(h, k_l0_frame, grid_for(n0), kBlock, 0, n0, h->s, h->c0, h->target, h->vdiag, h->fixf, om, h->b0,
           lv[0].dfull, lv[0].dinv, xa);
    if (learned) enqueue_ls_row_consts(h);
    for (int l = 1; l < L; ++l)
        LAUNCH(h, k_coarse_frame, grid_for(lv[l].n), kBlock, 0, lv[l].n, lv[l].rptr, lv[l].rcol, lv[l].rw, lv[l - 1].c,
               lv[l].diag0, om, lv[l].c, lv[l].dfull, lv[l].dinv);
    LAUNCH(h, k_coarsest_update<float>, nb, 1024, h->factor_smem, h->range, L, h->dense_off_d, h->A0dense, h->B0dense,
           lv[L - 1].c, h->c_prev, h->Lfac, h->fac_valid);
    CoarseArgs ca;
    fill_coarse_args(h, ca);
    enqueue_coarse_operator(h, ca);
    const int g0 = grid_rows(n0, lv[0].S);
    // a learned solver's plain fallback smooths level 0 with at least the configured 2+2 Jacobi sweeps
    const bool fallback = !learned && h->ls_net != nullptr;
    const int l0_pre = fallback ? std::max(p.pre_sweeps, kFallbackL0Sweeps) : p.pre_sweeps;
    const int l0_post = fallback ? std::max(p.post_sweeps, kFallbackL0Sweeps) : p.post_sweeps;
    for (int it = 0; it < p.iterations; ++it) {
        LAUNCH(h, k_mg_local, grid_for(T), kBlock, 0, T, h->tets, h->tA, h->tB, h->tC, h->s, xa, h->slot_of, h->slots);
        if (learned) {
            for (int pass = 0; pass < p.refinement_passes; ++pass) {
                const int c = it * p.refinement_passes + pass;
                enqueue_learned_vcycle(h, xa, h->b, false, ca, c, pass == 0);
                enqueue_learned_guard(h, xa, h->b, c, c == h->ls_cycles - 1, fb);
            }
            continue;
        }
        for (int pass = 0; pass < p.refinement_passes; ++pass) {
            bool gathered = pass > 0;
            for (int k = 0; k < l0_pre; ++k) {
                LAUNCH(h, k_l0_sweep_rg, g0, kBlock, 0, n0, lv[0].slice_ptr, lv[0].ell_col, lv[0].ell_val, lv[0].dfull,
                       lv[0].dinv, xa, xb, h->b, h->b0, h->slot_ptr, h->slots, gathered ? 0 : 1, nullptr);
                gathered = true;
                std::swap(xa, xb);
            }
            if (!gathered) LAUNCH(h, k_gather_rhs, grid_for(n0), kBlock, 0, n0, h->b, h->b0, h->slot_ptr, h->slots);
            const bool fr = res0_fused(h);
            if (!h->fuse_l0 && !fr)
                LAUNCH(h, k_l0_residual_rg, g0, kBlock, 0, n0, lv[0].slice_ptr, lv[0].ell_col, lv[0].ell_val,
                       lv[0].dfull, xa, h->b, lv[0].res, nullptr);
            ca.d = xa;
            ca.res0_b = fr ? h->b : nullptr;
            launch_coarse(h, ca);
            if (!h->fuse_l0) {   // the shared-memory kernel leaves the level-1 correction in lv[1].e
                enqueue_l0_post(h, xa, xb, h->b, nullptr, l0_post, fr);
            } else {
                for (int k = 0; k < l0_post; ++k) {
                    LAUNCH(h, k_l0_sweep_rg, g0, kBlock, 0, n0, lv[0].slice_ptr, lv[0].ell_col, lv[0].ell_val,
                           lv[0].dfull, lv[0].dinv, xa, xb, h->b, h->b0, h->slot_ptr, h->slots, 0, nullptr);
                    std::swap(xa, xb);
                }
            }
        }
    }
    return xa;
}

void enqueue_mg_frame(mgsb_solver* h) {
    const mgsb_params& p = h->p;
    const int n0 = h->N0;
    LAUNCH(h, k_mg_predict, grid_for(n0), kBlock, 0, n0, h->x, h->v, h->s, h->last, h->fixf, h->body_of, h->bodies_dev, p.dt);
    if (h->nsurf > 0 && h->broad_phase)
        enqueue_broad_phase(h, h->s, true);
    else if (h->nsurf > 0) {
        const bool tri = h->tri_contact && h->ctri_n > 0;
        if (tri)
            LAUNCH(h, k_tri_capsule<float4>, grid_for(h->ctri_n), kBlock, 0, h->ctri_n, h->ctri, h->body_of,
                   h->bodies_dev, (const float4*)h->s, h->tri_push);
        LAUNCH(h, k_contact_all, grid_for(h->nsurf), kBlock, 0, h->nsurf, h->surf, h->body_of, h->bodies_dev, h->s,
               h->fixf, p.contact_stiffness, h->cflag, h->c0, h->target, tri ? h->vt_ptr : nullptr,
               tri ? h->vt_idx : nullptr, tri ? (const double4*)h->tri_push : nullptr);
    }
    const bool learned = h->ls_net != nullptr && h->p.iterations > 0 && h->p.refinement_passes > 0;
    const LearnedFallback fb = learned ? begin_learned_fallback(h) : LearnedFallback{};
    float4* d = enqueue_mg_solve(h, learned, fb);
    if (learned)   // a failed learned V-cycle: the frame's solve again with the plain V-cycle
        end_learned_fallback(h, fb, [&] {
            float4* dp = enqueue_mg_solve(h, false, fb);
            if (dp != d) LAUNCH(h, k_ls_copy, grid_for(n0), kBlock, 0, n0, dp, d);
        });
    LAUNCH(h, k_mg_finish, grid_for(n0), kBlock, 0, n0, h->s, d, h->x, h->v, 1.0f / p.dt, h->nonfinite);
    h->d_final = d;
}

// Mixed precision: FP64 state and outer residual, FP32 local step and
// correction V-cycles (refinement_passes per PD iteration).  The global
// solve of one frame, from the predicted FP64 positions: contact state,
// right-hand side and diagonals, coarse-level data and the coarsest FP64
// inverse, then the PD iterations; the displacement ends in dd64 / d32.
void enqueue_mixed_solve(mgsb_solver* h, bool learned, const LearnedFallback& fb) {
    const mgsb_params& p = h->p;
    const int n0 = h->N0, T = h->T, L = p.levels;
    const int nb = (int)h->bodies.size();
    const float om = p.jacobi_omega;
    std::vector<LevelDev>& lv = h->lev;
    const bool tri = h->tri_contact && h->ctri_n > 0 && !h->broad_phase;
    if (tri)
        LAUNCH(h, k_tri_capsule<double4>, grid_for(h->ctri_n), kBlock, 0, h->ctri_n, h->ctri, h->body_of, h->bodies_dev,
               (const double4*)h->s64, h->tri_push);
    LAUNCH(h, k_mx_contact_frame, grid_for(n0), kBlock, 0, n0, h->s64, h->fixf, h->body_of, h->bodies_dev, h->is_surf,
           h->broad_phase ? h->bp_cand : nullptr, p.contact_stiffness, h->vdiag, om, h->cflag, h->c0, h->b0_64, lv[0].dfull, lv[0].dinv, h->dd64, h->d32,
           h->target, tri ? h->vt_ptr : nullptr, tri ? h->vt_idx : nullptr, tri ? (const double4*)h->tri_push : nullptr);
    if (learned) enqueue_ls_row_consts(h);
    for (int l = 1; l < L; ++l)
        LAUNCH(h, k_coarse_frame, grid_for(lv[l].n), kBlock, 0, lv[l].n, lv[l].rptr, lv[l].rcol, lv[l].rw, lv[l - 1].c,
               lv[l].diag0, om, lv[l].c, lv[l].dfull, lv[l].dinv);
    LAUNCH(h, k_coarsest_update<double>, nb, 1024, h->factor_smem64, h->range, L, h->dense_off_d, h->A0dense64,
           h->B0dense64, lv[L - 1].c, h->c_prev, h->Ainv64, h->fac_valid);
    CoarseArgs ca;
    fill_coarse_args(h, ca);
    ca.Ainv64 = h->Ainv64;
    enqueue_coarse_operator(h, ca);
    const int g0 = grid_rows(n0, lv[0].S);
    // a learned solver's plain fallback smooths level 0 with at least the configured 2+2 Jacobi sweeps
    const bool fallback = !learned && h->ls_net != nullptr;
    const int l0_pre = fallback ? std::max(p.pre_sweeps, kFallbackL0Sweeps) : p.pre_sweeps;
    const int l0_post = fallback ? std::max(p.post_sweeps, kFallbackL0Sweeps) : p.post_sweeps;
    for (int it = 0; it < p.iterations; ++it) {
        LAUNCH(h, k_mg_local, grid_for(T), kBlock, 0, T, h->tets, h->tA, h->tB, h->tC, h->s, h->d32, h->slot_of, h->slots);
        for (int pass = 0; pass < p.refinement_passes; ++pass) {
            float4* ea = h->d;
            float4* eb = h->d2;
            // the first pass also assembles b = b0 + slots; with the learned smoother it
            // also leaves the learned cycle's starting residual (the cycle starts from e = 0)
            const bool gather = pass == 0;
            const int c = it * p.refinement_passes + pass;
            // learned: the residual check of the previous cycle (its correction already in dd64) rides on
            // this outer residual, against the right-hand side that cycle solved for
            LAUNCH(h, k_mx_residual, g0, kMxThreads, 0, n0, lv[0].slice_ptr, lv[0].ell_col, h->ell_val64, h->diag64, h->c0,
                   h->dd64, h->b64, lv[0].dinv, h->r32, ea, (l0_pre > 0 && !learned) ? 1 : 0,
                   gather ? h->b0_64 : nullptr, gather ? h->slot_ptr : nullptr, gather ? h->slots : nullptr, h->fixf,
                   learned ? h->ls_r : nullptr, learned ? h->ls_part0 + (size_t)c * h->ls_nblk : nullptr,
                   (learned && c > 0) ? h->ls_part1 + (size_t)(c - 1) * h->ls_nblk : nullptr);
            if (learned) {
                // every cycle but the frame's last applies its correction in its last sweep (dd64 += e) and
                // is checked by the next k_mx_residual; the last is checked (and applied) by the guard,
                // which takes the frame's decision
                const bool last = c == h->ls_cycles - 1;
                enqueue_learned_vcycle(h, ea, h->r32, true, ca, c, false, true, last ? nullptr : h->dd64,
                                       last ? nullptr : h->d32);
                if (last) enqueue_learned_guard(h, ea, h->r32, c, true, fb, h->dd64, h->d32);
                continue;
            }
            for (int k = 1; k < l0_pre; ++k) {
                LAUNCH(h, k_l0_sweep_rg, g0, kBlock, 0, n0, lv[0].slice_ptr, lv[0].ell_col, lv[0].ell_val, lv[0].dfull,
                       lv[0].dinv, ea, eb, h->r32, h->b0, h->slot_ptr, h->slots, 0, nullptr);
                std::swap(ea, eb);
            }
            const bool fr = res0_fused(h);
            if (!fr)
                LAUNCH(h, k_l0_residual_rg, g0, kBlock, 0, n0, lv[0].slice_ptr, lv[0].ell_col, lv[0].ell_val,
                       lv[0].dfull, ea, h->r32, lv[0].res, nullptr);
            ca.d = ea;
            ca.res0_b = fr ? h->r32 : nullptr;
            launch_coarse(h, ca);
            enqueue_l0_post(h, ea, eb, h->r32, nullptr, l0_post, fr);
            LAUNCH(h, k_mx_update, grid_for(n0), kBlock, 0, n0, ea, h->dd64, h->d32);
        }
    }
}

void enqueue_mixed_frame(mgsb_solver* h) {
    const mgsb_params& p = h->p;
    const int n0 = h->N0;
    LAUNCH(h, k_mx_predict, grid_for(n0), kBlock, 0, n0, h->x64, h->v64, h->s64, h->last64, h->s, h->x, h->fixf,
           h->body_of, h->bodies_dev, (double)p.dt);
    if (h->nsurf > 0 && h->broad_phase) enqueue_broad_phase(h, h->s, false);
    const bool learned = h->ls_net != nullptr && h->p.iterations > 0 && h->p.refinement_passes > 0;
    const LearnedFallback fb = learned ? begin_learned_fallback(h) : LearnedFallback{};
    enqueue_mixed_solve(h, learned, fb);
    if (learned)   // a failed learned V-cycle: the frame's solve again with the plain V-cycle
        end_learned_fallback(h, fb, [&] { enqueue_mixed_solve(h, false, fb); });
    LAUNCH(h, k_mx_finish, grid_for(n0), kBlock, 0, n0, h->s64, h->dd64, h->x64, h->v64, h->x, 1.0 / (double)p.dt,
           h->nonfinite);
}

void enqueue_frame(mgsb_solver* h) {
    h->launches = 0;
    if (is_mg(h) && h->p.precision == MGSB_PRECISION_MIXED)
        enqueue_mixed_frame(h);
    else if (is_mg(h))
        enqueue_mg_frame(h);
    else
        enqueue_ref_frame(h);
}

mgsb_status ensure_ready(mgsb_solver* h) {
    if (h->dirty) TRY(rebuild(h));
    return MGSB_OK;
}

mgsb_status push_tool(mgsb_solver* h) {
    const int k = h->stage_idx;
    h->stage_idx = (k + 1) % mgsb_solver::kStage;
    CUDA_TRY(h, cudaEventSynchronize(h->stage_ev[k]));
    const size_t nb = h->bodies.size() * sizeof(BodyDev);
    std::memcpy(h->stage[k], h->bodies_host, nb);
    std::memcpy(h->stage[k] + nb, h->spheres_host, sizeof(SphereSet));
    CUDA_TRY(h, cudaMemcpyAsync(h->bodies_dev, h->stage[k], nb, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->spheres_dev, h->stage[k] + nb, sizeof(SphereSet), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaEventRecord(h->stage_ev[k], h->stream));
    return MGSB_OK;
}

mgsb_status step_once(mgsb_solver* h) {
    TRY(ensure_ready(h));
    CUDA_TRY(h, cudaSetDevice(h->device));
    TRY(push_tool(h));
    CUDA_TRY(h, cudaEventRecord(h->ev0, h->stream));
    if (h->p.use_graph) {
        if (!h->graph_valid) {
            CUDA_TRY(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
            h->capture_error = false;
            h->enqueue_status = MGSB_OK;
            enqueue_frame(h);
            cudaError_t e = cudaStreamEndCapture(h->stream, &h->graph);
            if (h->enqueue_status != MGSB_OK) {
                if (e == cudaSuccess) cudaGraphDestroy(h->graph);
                h->graph = nullptr;
                return h->enqueue_status;
            }
            if (e == cudaSuccess && h->capture_error) {
                cudaGraphDestroy(h->graph);
                h->graph = nullptr;
                return set_err(h, MGSB_CUDA_ERROR, "graph capture failed: could not build a conditional node");
            }
            if (e != cudaSuccess) return set_err(h, MGSB_CUDA_ERROR, "graph capture failed: %s", cudaGetErrorString(e));
            CUDA_TRY(h, cudaGraphInstantiate(&h->graph_exec, h->graph, 0));
            h->graph_valid = true;
        }
        CUDA_TRY(h, cudaGraphLaunch(h->graph_exec, h->stream));
    } else {
        h->enqueue_status = MGSB_OK;
        enqueue_frame(h);
        if (h->enqueue_status != MGSB_OK) return h->enqueue_status;
        CUDA_TRY(h, cudaGetLastError());
    }
    CUDA_TRY(h, cudaEventRecord(h->ev1, h->stream));
    h->timed = true;
    return MGSB_OK;
}

mgsb_status sync_check(mgsb_solver* h) {
    CUDA_TRY(h, cudaSetDevice(h->device));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    int32_t nf = 0;
    CUDA_TRY(h, cudaMemcpy(&nf, h->nonfinite, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (nf) return set_err(h, MGSB_DIVERGED, "non-finite positions detected");
    return MGSB_OK;
}

mgsb_status check_body(mgsb_solver* h, int32_t body) {
    if (!h) return MGSB_INVALID_ARG;
    if (body < 0 || body >= (int32_t)h->bodies.size()) return set_err(h, MGSB_INVALID_ARG, "body %d out of range", body);
    return MGSB_OK;
}

void default_params(int32_t kind, mgsb_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->solver = kind;
    p->dt = 1.0f / 60.0f;
    p->damping = 0.95f;
    p->gravity[0] = 0.f;
    p->gravity[1] = -9.8f;
    p->gravity[2] = 0.f;
    p->volume_stiffness = 8000.f;
    p->collision_stiffness = 1000.f;
    p->cheb_rho = 0.9992f;
    p->relaxation = 0.6f;
    p->density = 1000.f;
    p->youngs_modulus = 1e5f;
    p->poisson_ratio = 0.3f;
    p->contact_stiffness = 1e6f;
    p->levels = 3;
    p->pre_sweeps = 2;
    p->post_sweeps = 2;
    p->jacobi_omega = 2.0f / 3.0f;
    p->precision = MGSB_PRECISION_FP32;
    p->refinement_passes = 1;
    p->use_graph = 1;
    p->device = 0;
    p->stream = nullptr;
    p->iterations = kind == MGSB_SOLVER_REFERENCE_JACOBI ? 20 : 10;
}

mgsb_status validate_params(mgsb_solver* h, const mgsb_params& p) {
    if (p.solver != MGSB_SOLVER_REFERENCE_JACOBI && p.solver != MGSB_SOLVER_MULTIGRID)
        return set_err(h, MGSB_INVALID_ARG, "unknown solver kind %d", p.solver);
    if (!(p.dt > 0) || p.iterations < 0 || p.iterations > 100000) return set_err(h, MGSB_INVALID_ARG, "bad dt/iterations");
    if (p.solver == MGSB_SOLVER_MULTIGRID) {
        if (p.levels < 2 || p.levels > 12) return set_err(h, MGSB_INVALID_ARG, "levels must be in [2,12]");
        if (p.pre_sweeps < 0 || p.post_sweeps < 0 || p.refinement_passes < 1)
            return set_err(h, MGSB_INVALID_ARG, "bad sweep/refinement counts");
        if (p.precision != MGSB_PRECISION_FP32 && p.precision != MGSB_PRECISION_MIXED)
            return set_err(h, MGSB_INVALID_ARG, "unknown precision %d", p.precision);
    }
    return MGSB_OK;
}

mgsb_status create_impl(int32_t nbodies, const mgsb_mesh* meshes, const mgsb_params* params, mgsb_solver** out) {
    if (!out) return MGSB_INVALID_ARG;
    *out = nullptr;
    if (nbodies <= 0 || !meshes || !params) return MGSB_INVALID_ARG;
    std::unique_ptr<mgsb_solver> h(new mgsb_solver());
    h->p = params[0];
    TRY(validate_params(h.get(), h->p));
    if (nbodies > 1 && h->p.solver != MGSB_SOLVER_MULTIGRID)
        return MGSB_NOT_SUPPORTED;
    h->device = h->p.device;
    h->bodies.resize(nbodies);
    int voff = 0, toff = 0;
    for (int bi = 0; bi < nbodies; ++bi) {
        BodyHost& B = h->bodies[bi];
        std::string e;
        mgsb_status st = make_body(meshes[bi], params[bi], h->p.solver == MGSB_SOLVER_MULTIGRID, B, e);
        if (st != MGSB_OK) return st;
        B.v_off = voff;
        B.t_off = toff;
        voff += B.V;
        toff += B.T;
    }
    h->N0 = voff;
    h->T = toff;
    mgsb_solver* hp = h.get();
    CUDA_TRY(hp, cudaSetDevice(h->device));
    if (h->p.stream) {
        h->stream = (cudaStream_t)h->p.stream;
    } else {
        CUDA_TRY(hp, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->own_stream = true;
    }
    CUDA_TRY(hp, cudaStreamCreateWithFlags(&h->aux_stream, cudaStreamNonBlocking));
    CUDA_TRY(hp, cudaEventCreate(&h->ev0));
    CUDA_TRY(hp, cudaEventCreate(&h->ev1));
    h->bodies_host = new BodyDev[nbodies];
    h->spheres_host = new SphereSet;
    for (int k = 0; k < mgsb_solver::kStage; ++k) {
        CUDA_TRY(hp, cudaMallocHost((void**)&h->stage[k], nbodies * sizeof(BodyDev) + sizeof(SphereSet)));
        CUDA_TRY(hp, cudaEventCreateWithFlags(&h->stage_ev[k], cudaEventDisableTiming));
    }
    std::memset(h->bodies_host, 0, nbodies * sizeof(BodyDev));
    std::memset(h->spheres_host, 0, sizeof(SphereSet));
    for (int bi = 0; bi < nbodies; ++bi) {
        BodyDev& BD = h->bodies_host[bi];
        const BodyHost& B = h->bodies[bi];
        for (int c = 0; c < 3; ++c) BD.gravity[c] = B.gravity[c];
        BD.damping = B.damping;
        BD.cap_r = 0.f;
    }
    auto& pool = h->state_mem;
    const int N0 = h->N0;
    // pinned readback: N0 float4 rows (or, for mgsb_get_frame_view, N0 packed xyz + N0 contact
    // flags), then the non-finite flag that every readback fetches with its data (at N0 x 16 B)
    CUDA_TRY(hp, cudaMallocHost((void**)&h->readback, (size_t)std::max(N0, 1) * sizeof(float4) + 16));
    TRY(dalloc(hp, pool, &h->x, N0));
    TRY(dalloc(hp, pool, &h->xpack, (size_t)3 * std::max(N0, 1)));
    TRY(dalloc(hp, pool, &h->xb, N0));
    TRY(dalloc(hp, pool, &h->v, N0));
    TRY(dalloc(hp, pool, &h->s, N0));
    TRY(dalloc(hp, pool, &h->last, N0));
    TRY(dalloc(hp, pool, &h->prev, N0));
    TRY(dalloc(hp, pool, &h->cflag, N0));
    TRY(dalloc(hp, pool, &h->cdepth, N0));
    TRY(dalloc(hp, pool, &h->cenergy, N0));
    TRY(dalloc(hp, pool, &h->nonfinite, 1));
    if (h->p.precision == MGSB_PRECISION_MIXED) {
        TRY(dalloc(hp, pool, &h->x64, N0));
        TRY(dalloc(hp, pool, &h->v64, N0));
        std::vector<double4> x(N0);
        for (const BodyHost& B : h->bodies)
            for (int i = 0; i < B.V; ++i) x[B.v_off + i] = make_double4(B.rest[3 * i], B.rest[3 * i + 1], B.rest[3 * i + 2], 0.0);
        CUDA_TRY(hp, cudaMemcpy(h->x64, x.data(), N0 * sizeof(double4), cudaMemcpyHostToDevice));
        CUDA_TRY(hp, cudaMemset(h->v64, 0, N0 * sizeof(double4)));
    }
    TRY(dalloc(hp, pool, &h->bodies_dev, nbodies));
    TRY(dalloc(hp, pool, &h->spheres_dev, 1));
    {
        std::vector<float4> x4(N0);
        for (const BodyHost& B : h->bodies)
            for (int i = 0; i < B.V; ++i)
                x4[B.v_off + i] = make_float4((float)B.rest[3 * i], (float)B.rest[3 * i + 1], (float)B.rest[3 * i + 2], 0.f);
        CUDA_TRY(hp, cudaMemcpy(h->x, x4.data(), N0 * sizeof(float4), cudaMemcpyHostToDevice));
        CUDA_TRY(hp, cudaMemcpy(h->xb, x4.data(), N0 * sizeof(float4), cudaMemcpyHostToDevice));
        CUDA_TRY(hp, cudaMemcpy(h->s, x4.data(), N0 * sizeof(float4), cudaMemcpyHostToDevice));
        CUDA_TRY(hp, cudaMemcpy(h->last, x4.data(), N0 * sizeof(float4), cudaMemcpyHostToDevice));
        CUDA_TRY(hp, cudaMemcpy(h->prev, x4.data(), N0 * sizeof(float4), cudaMemcpyHostToDevice));
    }
    CUDA_TRY(hp, cudaMemset(h->v, 0, N0 * sizeof(float4)));
    CUDA_TRY(hp, cudaMemset(h->cflag, 0, N0 * sizeof(int32_t)));
    CUDA_TRY(hp, cudaMemset(h->cdepth, 0, N0 * sizeof(float)));
    CUDA_TRY(hp, cudaMemset(h->cenergy, 0, N0 * sizeof(float)));
    CUDA_TRY(hp, cudaMemset(h->nonfinite, 0, sizeof(int32_t)));
    TRY(rebuild(hp));
    *out = h.release();
    return MGSB_OK;
}

// Device -> pinned readback buffer, together with the non-finite flag, in one
// stream synchronisation: MGSB_DIVERGED when the flag is set (the caller then
// writes nothing).
mgsb_status readback_checked(mgsb_solver* h, const void* src, size_t bytes) {
    CUDA_TRY(h, cudaSetDevice(h->device));
    int32_t* flag = reinterpret_cast<int32_t*>(h->readback + (size_t)std::max(h->N0, 1) * sizeof(float4));
    CUDA_TRY(h, cudaMemcpyAsync(flag, h->nonfinite, sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    if (bytes) CUDA_TRY(h, cudaMemcpyAsync(h->readback, src, bytes, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (*flag) return set_err(h, MGSB_DIVERGED, "non-finite positions detected");
    return MGSB_OK;
}

template <typename F>
mgsb_status copy_body_f4(mgsb_solver* h, int32_t body, const float4* src, F&& sink) {
    TRY(check_body(h, body));
    const BodyHost& B = h->bodies[body];
    TRY(readback_checked(h, src + B.v_off, B.V * sizeof(float4)));
    const float4* tmp = reinterpret_cast<const float4*>(h->readback);
    for (int i = 0; i < B.V; ++i) sink(i, tmp[i]);
    return MGSB_OK;
}

// Surface normals of one body from the current positions: triangle normals
// into fscratch (>= the body's triangle count), vertex normals of the
// surface vertices into vscratch (>= its surface-vertex count), then a copy
// to the host and a scatter into out[3V] (zero for interior vertices).  The
// copy lands in host_stage (>= the surface-vertex count of float4) when one is
// given, else in a temporary host vector.
mgsb_status run_normals(mgsb_solver* h, int32_t body, float4* fscratch, float4* vscratch, float4* host_stage,
                        float* out) {
    const BodyHost& B = h->bodies[body];
    const int nf = h->nrm_nf[body], nsv = h->nrm_nsv[body];
    const int f_off = h->nrm_f_off[body], sv_off = h->nrm_sv_off[body];
    CUDA_TRY(h, cudaSetDevice(h->device));
    if (nf > 0) {
        k_tri_normals<<<(nf + 255) / 256, 256, 0, h->stream>>>(nf, h->nrm_tris + f_off, h->x, fscratch);
        k_vert_normals<<<(nsv + 255) / 256, 256, 0, h->stream>>>(nsv, h->nrm_ptr + sv_off, h->nrm_fidx, fscratch, vscratch);
        CUDA_TRY(h, cudaGetLastError());
    }
    std::vector<float4> tmp;
    if (!host_stage) {
        tmp.resize(nsv);
        host_stage = tmp.data();
    }
    if (nsv > 0)
        CUDA_TRY(h, cudaMemcpyAsync(host_stage, vscratch, nsv * sizeof(float4), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    int32_t nf_flag = 0;
    CUDA_TRY(h, cudaMemcpy(&nf_flag, h->nonfinite, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (nf_flag) return set_err(h, MGSB_DIVERGED, "non-finite positions detected");
    std::fill(out, out + 3 * (size_t)B.V, 0.f);
    for (int j = 0; j < nsv; ++j) {
        const int i = h->nrm_sv_host[sv_off + j] - B.v_off;
        out[3 * i] = host_stage[j].x;
        out[3 * i + 1] = host_stage[j].y;
        out[3 * i + 2] = host_stage[j].z;
    }
    return MGSB_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

mgsb_status mgsb_default_params(int32_t solver_kind, mgsb_params* out) {
    if (!out) return MGSB_INVALID_ARG;
    if (solver_kind != MGSB_SOLVER_REFERENCE_JACOBI && solver_kind != MGSB_SOLVER_MULTIGRID) return MGSB_INVALID_ARG;
    default_params(solver_kind, out);
    return MGSB_OK;
}

mgsb_status mgsb_create(const mgsb_mesh* mesh, const mgsb_params* params, mgsb_solver** out) {
    return create_impl(1, mesh, params, out);
}

mgsb_status mgsb_batch_create(int32_t num_bodies, const mgsb_mesh* meshes, const mgsb_params* params, mgsb_solver** out) {
    return create_impl(num_bodies, meshes, params, out);
}

mgsb_status mgsb_destroy(mgsb_solver* h) {
    if (!h) return MGSB_INVALID_ARG;
    delete h;   // ~mgsb_solver releases every resource
    return MGSB_OK;
}

mgsb_status mgsb_num_bodies(const mgsb_solver* h, int32_t* n) {
    if (!h || !n) return MGSB_INVALID_ARG;
    *n = (int32_t)h->bodies.size();
    return MGSB_OK;
}

mgsb_status mgsb_num_verts(const mgsb_solver* h, int32_t body, int32_t* n) {
    if (!h || !n || body < 0 || body >= (int32_t)h->bodies.size()) return MGSB_INVALID_ARG;
    *n = h->bodies[body].V;
    return MGSB_OK;
}

mgsb_status mgsb_num_tets(const mgsb_solver* h, int32_t body, int32_t* n) {
    if (!h || !n || body < 0 || body >= (int32_t)h->bodies.size()) return MGSB_INVALID_ARG;
    *n = h->bodies[body].T;
    return MGSB_OK;
}

mgsb_status mgsb_set_material(mgsb_solver* h, int32_t body, const float* youngs, const float* poisson) {
    TRY(check_body(h, body));
    if (!youngs || !poisson) return set_err(h, MGSB_INVALID_ARG, "null material arrays");
    BodyHost& B = h->bodies[body];
    for (int t = 0; t < B.T; ++t) {
        if (!(youngs[t] > 0.f) || !(poisson[t] > -1.f && poisson[t] < 0.5f))
            return set_err(h, MGSB_INVALID_ARG, "tet %d: bad material (E=%g, nu=%g)", t, youngs[t], poisson[t]);
    }
    B.youngs.assign(youngs, youngs + B.T);
    B.poisson.assign(poisson, poisson + B.T);
    h->dirty = true;
    return MGSB_OK;
}

mgsb_status mgsb_get_params(const mgsb_solver* h, mgsb_params* out) {
    if (!h || !out) return MGSB_INVALID_ARG;
    *out = h->p;
    return MGSB_OK;
}

mgsb_status mgsb_set_params(mgsb_solver* h, const mgsb_params* params) {
    if (!h) return MGSB_INVALID_ARG;
    if (!params) return set_err(h, MGSB_INVALID_ARG, "null params");
    const mgsb_params& q = *params;
    TRY(validate_params(h, q));
    if (q.solver != h->p.solver)
        return set_err(h, MGSB_NOT_SUPPORTED, "the solver kind is fixed at create (%d, asked %d)", h->p.solver, q.solver);
    if (q.device != h->p.device || q.stream != h->p.stream)
        return set_err(h, MGSB_NOT_SUPPORTED, "device and stream are fixed at create");
    if (is_mg(h) && q.precision != h->p.precision)
        return set_err(h, MGSB_NOT_SUPPORTED, "the precision is fixed at create (its state buffers are allocated there)");
    if (!(q.density > 0.f) && is_mg(h)) return set_err(h, MGSB_INVALID_ARG, "density must be > 0");
    const bool material = q.youngs_modulus != h->p.youngs_modulus || q.poisson_ratio != h->p.poisson_ratio;
    if (material && is_mg(h) && (!(q.youngs_modulus > 0.f) || !(q.poisson_ratio > -1.f && q.poisson_ratio < 0.5f)))
        return set_err(h, MGSB_INVALID_ARG, "bad material (E=%g, nu=%g)", q.youngs_modulus, q.poisson_ratio);
    TRY(sync_check(h));
    h->p = q;
    for (size_t bi = 0; bi < h->bodies.size(); ++bi) {
        BodyHost& B = h->bodies[bi];
        BodyDev& BD = h->bodies_host[bi];
        for (int c = 0; c < 3; ++c) B.gravity[c] = BD.gravity[c] = q.gravity[c];
        B.damping = BD.damping = q.damping;
        if (material) {
            B.youngs.assign(B.T, q.youngs_modulus);
            B.poisson.assign(B.T, q.poisson_ratio);
        }
    }
    h->dirty = true;   // the next step rebuilds the plan, the hierarchy and the frame's graph
    return MGSB_OK;
}

mgsb_status mgsb_set_fixed(mgsb_solver* h, int32_t body, const uint8_t* mask) {
    TRY(check_body(h, body));
    if (!mask) return set_err(h, MGSB_INVALID_ARG, "null mask");
    BodyHost& B = h->bodies[body];
    B.fixed.assign(mask, mask + B.V);
    for (auto& f : B.fixed) f = f ? 1 : 0;
    h->dirty = true;
    return MGSB_OK;
}

mgsb_status mgsb_set_tool_capsule(mgsb_solver* h, int32_t body, const float a[3], const float b[3], float radius) {
    TRY(check_body(h, body));
    if (!a || !b) return set_err(h, MGSB_INVALID_ARG, "null capsule endpoints");
    BodyDev& BD = h->bodies_host[body];
    for (int c = 0; c < 3; ++c) {
        BD.cap_a[c] = a[c];
        BD.cap_b[c] = b[c];
    }
    BD.cap_r = radius > 0.f ? radius : 0.f;
    return MGSB_OK;
}

mgsb_status mgsb_set_tool_capsules(mgsb_solver* h, const float* a, const float* b, const float* radius) {
    if (!h || !a || !b || !radius) return MGSB_INVALID_ARG;
    for (size_t bi = 0; bi < h->bodies.size(); ++bi) {
        BodyDev& BD = h->bodies_host[bi];
        for (int c = 0; c < 3; ++c) {
            BD.cap_a[c] = a[3 * bi + c];
            BD.cap_b[c] = b[3 * bi + c];
        }
        BD.cap_r = radius[bi] > 0.f ? radius[bi] : 0.f;
    }
    return MGSB_OK;
}

mgsb_status mgsb_set_tool_spheres(mgsb_solver* h, int32_t count, const float* centers, const float* radii,
                                  const uint8_t* active) {
    if (!h) return MGSB_INVALID_ARG;
    if (count < 0 || count > 8 || (count > 0 && (!centers || !radii)))
        return set_err(h, MGSB_INVALID_ARG, "sphere count must be in [0,8]");
    SphereSet& S = *h->spheres_host;
    S.count = count;
    for (int q = 0; q < count; ++q) {
        S.cx[q] = centers[3 * q];
        S.cy[q] = centers[3 * q + 1];
        S.cz[q] = centers[3 * q + 2];
        S.r[q] = radii[q];
        S.active[q] = active ? (active[q] ? 1 : 0) : 1;
    }
    return MGSB_OK;
}

mgsb_status mgsb_step(mgsb_solver* h) {
    if (!h) return MGSB_INVALID_ARG;
    return step_once(h);
}

mgsb_status mgsb_step_n(mgsb_solver* h, int32_t n) {
    if (!h || n < 0) return MGSB_INVALID_ARG;
    for (int i = 0; i < n; ++i) TRY(step_once(h));
    return MGSB_OK;
}

mgsb_status mgsb_synchronize(mgsb_solver* h) {
    if (!h) return MGSB_INVALID_ARG;
    return sync_check(h);
}

mgsb_status mgsb_get_positions(mgsb_solver* h, int32_t body, float* out) {
    if (!out) return MGSB_INVALID_ARG;
    TRY(check_body(h, body));
    return copy_body_f4(h, body, h->x, [&](int i, float4 v) {
        out[3 * i] = v.x;
        out[3 * i + 1] = v.y;
        out[3 * i + 2] = v.z;
    });
}

mgsb_status mgsb_get_velocities(mgsb_solver* h, int32_t body, float* out) {
    if (!out) return MGSB_INVALID_ARG;
    TRY(check_body(h, body));
    TRY(sync_check(h));
    if (h->v64) {
        const BodyHost& B = h->bodies[body];
        std::vector<double4> tmp(B.V);
        CUDA_TRY(h, cudaMemcpy(tmp.data(), h->v64 + B.v_off, B.V * sizeof(double4), cudaMemcpyDeviceToHost));
        for (int i = 0; i < B.V; ++i) {
            out[3 * i] = (float)tmp[i].x;
            out[3 * i + 1] = (float)tmp[i].y;
            out[3 * i + 2] = (float)tmp[i].z;
        }
        return MGSB_OK;
    }
    return copy_body_f4(h, body, h->v, [&](int i, float4 v) {
        out[3 * i] = v.x;
        out[3 * i + 1] = v.y;
        out[3 * i + 2] = v.z;
    });
}

mgsb_status mgsb_get_all_positions(mgsb_solver* h, float* out) {
    if (!h || !out) return MGSB_INVALID_ARG;
    TRY(readback_checked(h, h->x, h->N0 * sizeof(float4)));
    const float4* tmp = reinterpret_cast<const float4*>(h->readback);
    for (int i = 0; i < h->N0; ++i) {
        out[3 * i] = tmp[i].x;
        out[3 * i + 1] = tmp[i].y;
        out[3 * i + 2] = tmp[i].z;
    }
    return MGSB_OK;
}

mgsb_status mgsb_get_positions_f64(mgsb_solver* h, int32_t body, double* out) {
    if (!out) return MGSB_INVALID_ARG;
    TRY(check_body(h, body));
    if (!h->x64) return set_err(h, MGSB_NOT_SUPPORTED, "FP64 positions exist only in mixed precision");
    TRY(sync_check(h));
    const BodyHost& B = h->bodies[body];
    std::vector<double4> tmp(B.V);
    CUDA_TRY(h, cudaMemcpy(tmp.data(), h->x64 + B.v_off, B.V * sizeof(double4), cudaMemcpyDeviceToHost));
    for (int i = 0; i < B.V; ++i) {
        out[3 * i] = tmp[i].x;
        out[3 * i + 1] = tmp[i].y;
        out[3 * i + 2] = tmp[i].z;
    }
    return MGSB_OK;
}

mgsb_status mgsb_get_contact_flags(mgsb_solver* h, int32_t body, int32_t* out) {
    if (!out) return MGSB_INVALID_ARG;
    TRY(check_body(h, body));
    const BodyHost& B = h->bodies[body];
    TRY(readback_checked(h, h->cflag + B.v_off, B.V * sizeof(int32_t)));
    std::memcpy(out, h->readback, B.V * sizeof(int32_t));
    return MGSB_OK;
}

mgsb_status mgsb_get_all_contact_flags(mgsb_solver* h, int32_t* out) {
    if (!h || !out) return MGSB_INVALID_ARG;
    TRY(readback_checked(h, h->cflag, h->N0 * sizeof(int32_t)));
    std::memcpy(out, h->readback, h->N0 * sizeof(int32_t));
    return MGSB_OK;
}

mgsb_status mgsb_get_frame(mgsb_solver* h, float* positions, int32_t* contact_flags) {
    if (!h || !positions || !contact_flags) return MGSB_INVALID_ARG;
    const float* pos = nullptr;
    const int32_t* flags = nullptr;
    TRY(mgsb_get_frame_view(h, &pos, &flags));
    const size_t n = (size_t)h->N0;
    std::memcpy(positions, pos, n * 3 * sizeof(float));
    std::memcpy(contact_flags, flags, n * sizeof(int32_t));
    return MGSB_OK;
}

mgsb_status mgsb_get_frame_view(mgsb_solver* h, const float** positions, const int32_t** contact_flags) {
    if (!h || !positions || !contact_flags) return MGSB_INVALID_ARG;
    const size_t n = (size_t)h->N0;
    float* pos = reinterpret_cast<float*>(h->readback);                           // [0, 12 N)
    int32_t* flags = reinterpret_cast<int32_t*>(h->readback + n * 3 * sizeof(float));   // [12 N, 16 N)
    CUDA_TRY(h, cudaSetDevice(h->device));
    if (n) {
        k_pack_xyz<<<grid_for((int)n), kBlock, 0, h->stream>>>((int)n, h->x, h->xpack);
        CUDA_TRY(h, cudaGetLastError());
        CUDA_TRY(h, cudaMemcpyAsync(pos, h->xpack, n * 3 * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaMemcpyAsync(flags, h->cflag, n * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    }
    TRY(readback_checked(h, nullptr, 0));   // the non-finite flag (at 16 N) and one synchronisation
    *positions = pos;
    *contact_flags = flags;
    return MGSB_OK;
}

mgsb_status mgsb_get_contacts(mgsb_solver* h, int32_t body, int32_t* idx, size_t cap, size_t* n) {
    if (!n) return MGSB_INVALID_ARG;
    TRY(check_body(h, body));
    const BodyHost& B = h->bodies[body];
    std::vector<int32_t> f(B.V);
    TRY(mgsb_get_contact_flags(h, body, f.data()));
    size_t cnt = 0;
    for (int i = 0; i < B.V; ++i)
        if (f[i]) {
            if (idx && cnt < cap) idx[cnt] = i;
            ++cnt;
        }
    *n = cnt;
    if (idx && cnt > cap) return set_err(h, MGSB_INVALID_ARG, "contact buffer too small (%zu < %zu)", cap, cnt);
    return MGSB_OK;
}

mgsb_status mgsb_get_collision_depth(mgsb_solver* h, int32_t body, float* out) {
    if (!out) return MGSB_INVALID_ARG;
    TRY(check_body(h, body));
    TRY(sync_check(h));
    const BodyHost& B = h->bodies[body];
    CUDA_TRY(h, cudaMemcpy(out, h->cdepth + B.v_off, B.V * sizeof(float), cudaMemcpyDeviceToHost));
    return MGSB_OK;
}

mgsb_status mgsb_get_device_positions(mgsb_solver* h, int32_t body, const float** dptr) {
    if (!dptr) return MGSB_INVALID_ARG;
    TRY(check_body(h, body));
    *dptr = reinterpret_cast<const float*>(h->x + h->bodies[body].v_off);
    return MGSB_OK;
}

mgsb_status mgsb_get_normals(mgsb_solver* h, int32_t body, float* out) {
    if (!out) return MGSB_INVALID_ARG;
    TRY(check_body(h, body));
    TRY(ensure_ready(h));
    return run_normals(h, body, h->nrm_face, h->nrm_out, nullptr, out);
}

mgsb_status mgsb_set_state(mgsb_solver* h, int32_t body, const float* positions, const float* velocities) {
    TRY(check_body(h, body));
    TRY(sync_check(h));
    const BodyHost& B = h->bodies[body];
    std::vector<float4> tmp(B.V);
    if (positions) {
        for (int i = 0; i < B.V; ++i) tmp[i] = make_float4(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2], 0.f);
        CUDA_TRY(h, cudaMemcpy(h->x + B.v_off, tmp.data(), B.V * sizeof(float4), cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(h->prev + B.v_off, tmp.data(), B.V * sizeof(float4), cudaMemcpyHostToDevice));
    }
    if (velocities) {
        for (int i = 0; i < B.V; ++i) tmp[i] = make_float4(velocities[3 * i], velocities[3 * i + 1], velocities[3 * i + 2], 0.f);
        CUDA_TRY(h, cudaMemcpy(h->v + B.v_off, tmp.data(), B.V * sizeof(float4), cudaMemcpyHostToDevice));
    }
    if (h->x64) {
        std::vector<double4> t64(B.V);
        if (positions) {
            for (int i = 0; i < B.V; ++i) t64[i] = make_double4(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2], 0.0);
            CUDA_TRY(h, cudaMemcpy(h->x64 + B.v_off, t64.data(), B.V * sizeof(double4), cudaMemcpyHostToDevice));
        }
        if (velocities) {
            for (int i = 0; i < B.V; ++i) t64[i] = make_double4(velocities[3 * i], velocities[3 * i + 1], velocities[3 * i + 2], 0.0);
            CUDA_TRY(h, cudaMemcpy(h->v64 + B.v_off, t64.data(), B.V * sizeof(double4), cudaMemcpyHostToDevice));
        }
    }
    CUDA_TRY(h, cudaMemset(h->nonfinite, 0, sizeof(int32_t)));
    return MGSB_OK;
}

mgsb_status mgsb_get_energy(mgsb_solver* h, int32_t body, double out[5]) {
    if (!out) return MGSB_INVALID_ARG;
    TRY(check_body(h, body));
    TRY(ensure_ready(h));
    TRY(sync_check(h));
    const BodyHost& B = h->bodies[body];
    const mgsb_params& p = h->p;
    EnergyArgs a{};
    a.kind = !is_mg(h) ? kEnergyReference : (p.precision == MGSB_PRECISION_MIXED ? kEnergyMixed : kEnergyMultigrid);
    a.v0 = B.v_off;
    a.nv = B.V;
    a.t0 = B.t_off;
    a.nt = B.T;
    a.inv_2h2 = 1.0 / (2.0 * (double)p.dt * (double)p.dt);
    a.kv = p.volume_stiffness;
    a.x = h->x;
    a.s = h->s;
    a.prev = h->prev;
    a.x64 = a.kind == kEnergyMixed ? h->x64 : nullptr;
    a.s64 = a.kind == kEnergyMixed ? h->s64 : nullptr;
    // the reference kind stores density-1 masses; the multigrid kinds m/h^2
    a.mass = h->mass;
    if (a.kind != kEnergyReference) a.inv_2h2 = 0.5;
    a.fixf = h->fixf;
    a.tets = h->tets;
    a.tA = h->tA;
    a.tB = h->tB;
    a.tC = h->tC;
    a.cflag = h->cflag;
    a.c0 = h->c0;
    a.cenergy = h->cenergy;
    a.target = h->target;
    if (a.kind != kEnergyReference) {
        // the residual exists once a frame has run
        a.residual = a.kind == kEnergyMixed ? (h->timed ? 1 : 0) : (h->d_final ? 1 : 0);
        a.S = h->lev[0].S;
        a.sp = h->lev[0].slice_ptr;
        a.col = h->lev[0].ell_col;
        a.val = h->lev[0].ell_val;
        a.dfull = h->lev[0].dfull;
        a.b = h->b;
        a.d = h->d_final;
        a.val64 = h->ell_val64;
        a.diag64 = h->diag64;
        a.b64 = h->b64;
        a.d64 = h->dd64;
    }
    const int work = std::max(B.V, B.T);
    const int nblk = std::max(1, std::min(kEnergyBlocks, (work + kEnergyThreads - 1) / kEnergyThreads));
    CUDA_TRY(h, cudaSetDevice(h->device));
    k_energy_partial<<<nblk, kEnergyThreads, 0, h->stream>>>(a, h->energy_part);
    k_energy_final<<<1, kEnergyThreads, 0, h->stream>>>(h->energy_part, nblk, h->energy_out);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaMemcpyAsync(out, h->energy_out, kEnergyTerms * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return MGSB_OK;
}

mgsb_status mgsb_last_frame_ms(mgsb_solver* h, float* ms) {
    if (!h || !ms) return MGSB_INVALID_ARG;
    if (!h->timed) return set_err(h, MGSB_INVALID_ARG, "no frame has run");
    CUDA_TRY(h, cudaEventSynchronize(h->ev1));
    CUDA_TRY(h, cudaEventElapsedTime(ms, h->ev0, h->ev1));
    return MGSB_OK;
}

// One frame captured into its own graph with an event-record node on both
// sides of every profiled launch (so the timings contain no host launch
// gaps), run to completion.  The events stay in prof_ev / prof_names.
cudaError_t run_profiled_frame(mgsb_solver* h) {
    h->profiling = true;
    h->prof_names.clear();
    h->prof_ev.clear();
    h->enqueue_status = MGSB_OK;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        enqueue_frame(h);
        e = cudaStreamEndCapture(h->stream, &g);
    }
    h->profiling = false;
    if (e == cudaSuccess && h->enqueue_status != MGSB_OK) e = cudaErrorInvalidConfiguration;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ge, g, 0);
    if (e == cudaSuccess) e = cudaGraphLaunch(ge, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    return e;
}

mgsb_status mgsb_profile_frame(mgsb_solver* h, int32_t cap, char* names, float* total_ms, int32_t* launches,
                               int32_t* count) {
    if (!h || !count || cap < 0 || (cap > 0 && (!names || !total_ms || !launches))) return MGSB_INVALID_ARG;
    TRY(ensure_ready(h));
    CUDA_TRY(h, cudaSetDevice(h->device));
    TRY(push_tool(h));
    h->replay_name.clear();
    const cudaError_t e = run_profiled_frame(h);
    std::vector<std::string> uniq;
    std::vector<float> tot;
    std::vector<int32_t> cnt;
    for (size_t k = 0; k < h->prof_names.size(); ++k) {
        float ms = 0.f;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, h->prof_ev[2 * k], h->prof_ev[2 * k + 1]);
        size_t u = 0;
        while (u < uniq.size() && uniq[u] != h->prof_names[k]) ++u;
        if (u == uniq.size()) {
            uniq.push_back(h->prof_names[k]);
            tot.push_back(0.f);
            cnt.push_back(0);
        }
        tot[u] += ms;
        cnt[u] += 1;
    }
    for (cudaEvent_t ev : h->prof_ev) cudaEventDestroy(ev);
    h->prof_ev.clear();
    if (h->enqueue_status != MGSB_OK) return h->enqueue_status;
    if (e != cudaSuccess) return set_err(h, MGSB_CUDA_ERROR, "profiled frame failed: %s", cudaGetErrorString(e));
    *count = (int32_t)uniq.size();
    for (size_t u = 0; u < uniq.size() && (int32_t)u < cap; ++u) {
        std::snprintf(names + 48 * u, 48, "%s", uniq[u].c_str());
        total_ms[u] = tot[u];
        launches[u] = cnt[u];
    }
    return MGSB_OK;
}

mgsb_status mgsb_time_kernel(mgsb_solver* h, const char* name, int32_t reps, float* us_per_launch,
                             int32_t* launches_per_frame) {
    if (!h || !name || !us_per_launch || !launches_per_frame || reps < 1 || reps > 1000) return MGSB_INVALID_ARG;
    if (std::strncmp(name, "k_bp_", 5) == 0)
        return set_err(h, MGSB_NOT_SUPPORTED, "%s appends to the broad phase's candidate lists; it is not repeated", name);
    TRY(ensure_ready(h));
    CUDA_TRY(h, cudaSetDevice(h->device));
    TRY(push_tool(h));
    // The repeated launches change the frame's result: the state (and the
    // guard's statistics) are saved before it and put back after it.
    std::vector<std::pair<void*, size_t>> keep;
    for (const DevMem& m : h->state_mem) keep.emplace_back(m.p, m.bytes);
    if (h->ls_stats) keep.emplace_back(h->ls_stats, 2 * sizeof(unsigned long long));
    size_t total = 0;
    for (auto& k : keep) total += (k.second + 255) / 256 * 256;
    char* save = nullptr;
    CUDA_TRY(h, cudaMalloc((void**)&save, std::max<size_t>(total, 256)));
    cudaError_t e = cudaSuccess;
    size_t off = 0;
    for (auto& k : keep) {
        if (e == cudaSuccess) e = cudaMemcpyAsync(save + off, k.first, k.second, cudaMemcpyDeviceToDevice, h->stream);
        off += (k.second + 255) / 256 * 256;
    }
    if (e == cudaSuccess) {
        h->replay_name = name;
        h->replay_reps = reps;
        e = run_profiled_frame(h);
        h->replay_name.clear();
        h->replay_reps = 1;
    }
    float ms = 0.f;
    const int k_launches = (int)h->prof_names.size();
    for (int k = 0; k < k_launches && e == cudaSuccess; ++k) {
        float t = 0.f;
        e = cudaEventElapsedTime(&t, h->prof_ev[2 * k], h->prof_ev[2 * k + 1]);
        ms += t;
    }
    for (cudaEvent_t ev : h->prof_ev) cudaEventDestroy(ev);
    h->prof_ev.clear();
    h->prof_names.clear();
    off = 0;
    cudaError_t er = cudaSuccess;
    for (auto& k : keep) {
        if (er == cudaSuccess) er = cudaMemcpyAsync(k.first, save + off, k.second, cudaMemcpyDeviceToDevice, h->stream);
        off += (k.second + 255) / 256 * 256;
    }
    if (er == cudaSuccess) er = cudaStreamSynchronize(h->stream);
    cudaFree(save);
    if (e == cudaSuccess) e = er;
    if (h->enqueue_status != MGSB_OK) return h->enqueue_status;
    if (e != cudaSuccess) return set_err(h, MGSB_CUDA_ERROR, "kernel replay failed: %s", cudaGetErrorString(e));
    if (k_launches == 0) return set_err(h, MGSB_INVALID_ARG, "no launch of %s in a frame", name);
    *us_per_launch = 1000.f * ms / (float)(reps * k_launches);
    *launches_per_frame = k_launches;
    return MGSB_OK;
}

mgsb_status mgsb_set_kernel_shape(mgsb_solver* h, int32_t cluster, int32_t block, int32_t fuse_level0) {
    if (!h) return MGSB_INVALID_ARG;
    if (cluster < 0 || cluster > 16 || (block != 0 && block != 256 && block != 512 && block != 1024) || fuse_level0 < -1 ||
        fuse_level0 > 1)
        return set_err(h, MGSB_INVALID_ARG, "bad kernel shape (cluster %d, block %d, fuse %d)", cluster, block, fuse_level0);
    h->tune_cluster = cluster;
    h->tune_fuse = fuse_level0;
    if (block) h->coarse_block = block;
    apply_tuning(h);
    invalidate_graph(h);
    return MGSB_OK;
}

mgsb_status mgsb_set_coarse_split(mgsb_solver* h, int32_t split) {
    if (!h) return MGSB_INVALID_ARG;
    if (!is_mg(h)) return set_err(h, MGSB_NOT_SUPPORTED, "the coarse split applies to the multigrid kind");
    if (split < 0 || split >= h->p.levels)
        return set_err(h, MGSB_INVALID_ARG, "split %d outside 0..%d", split, h->p.levels - 1);
    h->tune_split = split;
    apply_tuning(h);
    invalidate_graph(h);
    return MGSB_OK;
}

mgsb_status mgsb_set_surface_contact(mgsb_solver* h, int32_t mode) {
    if (!h || (mode != MGSB_CONTACT_VERTICES && mode != MGSB_CONTACT_VERTICES_AND_TRIANGLES)) return MGSB_INVALID_ARG;
    if (!is_mg(h)) return set_err(h, MGSB_NOT_SUPPORTED, "the capsule contact applies to the multigrid kinds");
    if (mode == MGSB_CONTACT_VERTICES_AND_TRIANGLES && h->broad_phase)
        return set_err(h, MGSB_NOT_SUPPORTED, "the triangle test runs over all surface triangles: turn the broad phase off");
    h->tri_contact = mode == MGSB_CONTACT_VERTICES_AND_TRIANGLES;
    invalidate_graph(h);
    return MGSB_OK;
}

mgsb_status mgsb_set_broad_phase(mgsb_solver* h, int32_t on) {
    if (!h || (on != 0 && on != 1)) return MGSB_INVALID_ARG;
    if (!is_mg(h)) return set_err(h, MGSB_NOT_SUPPORTED, "the broad phase applies to the multigrid kinds");
    if (on && h->tri_contact)
        return set_err(h, MGSB_NOT_SUPPORTED, "the broad phase bins vertices only: turn the triangle contact off first");
    TRY(ensure_ready(h));
    CUDA_TRY(h, cudaSetDevice(h->device));
    h->broad_phase = on != 0;
    invalidate_graph(h);
    // start from an empty contact state: the next frame recomputes it either way
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    CUDA_TRY(h, cudaMemset(h->cflag, 0, (size_t)h->N0 * sizeof(int32_t)));
    CUDA_TRY(h, cudaMemset(h->c0, 0, (size_t)h->N0 * sizeof(float)));
    CUDA_TRY(h, cudaMemset(h->target, 0, (size_t)h->N0 * sizeof(float4)));
    CUDA_TRY(h, cudaMemset(h->bp_cand, 0, (size_t)h->N0));
    CUDA_TRY(h, cudaMemset(h->bp_nlist, 0, sizeof(int32_t)));
    return MGSB_OK;
}

mgsb_status mgsb_set_fused_prolongation(mgsb_solver* h, int32_t on) {
    if (!h || (on != 0 && on != 1)) return MGSB_INVALID_ARG;
    h->fuse_prolong = on != 0;
    invalidate_graph(h);
    return MGSB_OK;
}

mgsb_status mgsb_set_fused_restriction(mgsb_solver* h, int32_t on) {
    if (!h || (on != 0 && on != 1)) return MGSB_INVALID_ARG;
    h->fuse_res0 = on != 0;
    invalidate_graph(h);
    return MGSB_OK;
}

mgsb_status mgsb_set_launch_overlap(mgsb_solver* h, int32_t on) {
    if (!h || (on != 0 && on != 1)) return MGSB_INVALID_ARG;
    h->pdl = on != 0;
    invalidate_graph(h);
    return MGSB_OK;
}

mgsb_status mgsb_set_coarse_dense(mgsb_solver* h, int32_t on) {
    if (!h || (on != 0 && on != 1)) return MGSB_INVALID_ARG;
    if (!is_mg(h)) return set_err(h, MGSB_NOT_SUPPORTED, "the coarse operator applies to the multigrid kind");
    TRY(ensure_ready(h));
    if (on && (h->fuse_l0 || !dense_eligible(h, h->split)))
        return set_err(h, MGSB_NOT_SUPPORTED,
                       "the dense coarse operator needs one body, at most %d rows on the coarse split's level "
                       "(split %d has %d) and that level's rows in shared memory",
                       kDenseOpMaxRows, h->split, h->maxv[h->split]);
    h->tune_dense = on;
    apply_tuning(h);
    invalidate_graph(h);
    return MGSB_OK;
}

mgsb_status mgsb_get_coarse_dense(mgsb_solver* h, int32_t* on) {
    if (!h || !on) return MGSB_INVALID_ARG;
    TRY(ensure_ready(h));
    *on = h->dense_op ? 1 : 0;
    return MGSB_OK;
}

mgsb_status mgsb_get_coarse_split(mgsb_solver* h, int32_t* split) {
    if (!h || !split) return MGSB_INVALID_ARG;
    if (!is_mg(h)) return set_err(h, MGSB_NOT_SUPPORTED, "the coarse split applies to the multigrid kind");
    TRY(ensure_ready(h));
    *split = h->fuse_l0 ? 1 : h->split;
    return MGSB_OK;
}

mgsb_status mgsb_autotune(mgsb_solver* h, int32_t frames, int32_t* chosen) {
    if (!h || frames < 1) return MGSB_INVALID_ARG;
    if (!is_mg(h)) return set_err(h, MGSB_NOT_SUPPORTED, "autotuning applies to the multigrid kind");
    TRY(ensure_ready(h));
    CUDA_TRY(h, cudaSetDevice(h->device));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    // Snapshot the state: every candidate starts from it and it is restored at the end.
    const size_t nbytes = (size_t)h->N0 * sizeof(float4);
    float4 *sx = nullptr, *sv = nullptr;
    CUDA_TRY(h, cudaMalloc(&sx, nbytes));
    CUDA_TRY(h, cudaMalloc(&sv, nbytes));
    cudaMemcpyAsync(sx, h->x, nbytes, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(sv, h->v, nbytes, cudaMemcpyDeviceToDevice, h->stream);
    double4 *sx64 = nullptr, *sv64 = nullptr;
    const size_t nbytes64 = (size_t)h->N0 * sizeof(double4);
    if (h->x64) {
        CUDA_TRY(h, cudaMalloc(&sx64, nbytes64));
        CUDA_TRY(h, cudaMalloc(&sv64, nbytes64));
        cudaMemcpyAsync(sx64, h->x64, nbytes64, cudaMemcpyDeviceToDevice, h->stream);
        cudaMemcpyAsync(sv64, h->v64, nbytes64, cudaMemcpyDeviceToDevice, h->stream);
    }
    auto restore = [&]() {
        cudaMemcpyAsync(h->x, sx, nbytes, cudaMemcpyDeviceToDevice, h->stream);
        cudaMemcpyAsync(h->v, sv, nbytes, cudaMemcpyDeviceToDevice, h->stream);
        if (h->x64) {
            cudaMemcpyAsync(h->x64, sx64, nbytes64, cudaMemcpyDeviceToDevice, h->stream);
            cudaMemcpyAsync(h->v64, sv64, nbytes64, cudaMemcpyDeviceToDevice, h->stream);
        }
    };
    struct Cand {
        int cluster, block, fuse, split, dense;
    };
    std::vector<Cand> cands;
    const int nb = (int)h->bodies.size();
    const int L = h->p.levels;
    const int cls[] = {1, 2, 4, 8, 12, 16};
    for (int c : cls) {
        if (nb > 1 && c > 2) continue;   // many bodies: small clusters, one per body
        for (int blk : {256, 512, 1024}) {
            // split: the cluster kernel's first level; skip clusters with < 32 of its rows per CTA
            for (int sp = 1; sp < L; ++sp)
                if ((c == 1 || h->maxv[sp] >= 32 * c) && coarse_shape_feasible(h, c, blk, 0, sp))
                    cands.push_back({c, blk, 0, sp, 0});
            if (blk >= 512 && c >= 2 && h->p.precision != MGSB_PRECISION_MIXED && !h->ls_net &&
                coarse_shape_feasible(h, c, blk, 1, 1))
                cands.push_back({c, blk, 1, 1, 0});
        }
    }
    // the dense coarse operator at every split it can start at (one body)
    if (nb == 1)
        for (int sp = 1; sp < L; ++sp)
            if (dense_eligible(h, sp)) cands.push_back({1, 256, 0, sp, 1});
    float best = 1e30f;
    Cand bestc = {h->cluster, h->coarse_block, h->fuse_l0, h->split, h->dense_op ? 1 : 0};
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    mgsb_status st = MGSB_OK;
    for (const Cand& c : cands) {
        h->tune_cluster = c.cluster;
        h->tune_fuse = c.fuse;
        h->tune_split = c.split;
        h->tune_dense = c.dense;
        h->coarse_block = c.block;
        apply_tuning(h);
        invalidate_graph(h);
        cudaMemsetAsync(h->fac_valid, 0, h->bodies.size() * sizeof(int32_t), h->stream);
        restore();
        st = step_once(h);   // warm-up: capture + coarsest factorisation
        if (st != MGSB_OK) {
            // a shape the device cannot launch: skip it (the capture already ended)
            cudaGetLastError();
            invalidate_graph(h);
            st = MGSB_OK;
            continue;
        }
        cudaEventRecord(a, h->stream);
        for (int f = 0; f < frames && st == MGSB_OK; ++f) st = step_once(h);
        cudaEventRecord(b, h->stream);
        if (st != MGSB_OK) break;
        if (cudaEventSynchronize(b) != cudaSuccess) {
            st = set_err(h, MGSB_CUDA_ERROR, "autotune candidate failed");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best) {
            best = ms;
            bestc = c;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    h->tune_cluster = bestc.cluster;
    h->tune_fuse = bestc.fuse;
    h->tune_split = bestc.split;
    h->tune_dense = bestc.dense;
    h->coarse_block = bestc.block;
    apply_tuning(h);
    invalidate_graph(h);
    const mgsb_status st2 = MGSB_OK;
    cudaMemsetAsync(h->fac_valid, 0, h->bodies.size() * sizeof(int32_t), h->stream);
    restore();
    cudaStreamSynchronize(h->stream);
    cudaFree(sx);
    cudaFree(sv);
    if (sx64) cudaFree(sx64);
    if (sv64) cudaFree(sv64);
    if (st != MGSB_OK) return st;
    if (st2 != MGSB_OK) return st2;
    if (chosen) {
        chosen[0] = bestc.cluster;
        chosen[1] = bestc.block;
        chosen[2] = bestc.fuse;
    }
    return MGSB_OK;
}

mgsb_status mgsb_inspect_level(const mgsb_mesh* mesh, const mgsb_params* params, const uint8_t* fixed, int32_t level,
                               int32_t* n, int32_t* nnz, int32_t* pid, float* pw, float* diag, int32_t* ptr, int32_t* col,
                               float* val) {
    if (!mesh || !params || !n || !nnz || params->solver != MGSB_SOLVER_MULTIGRID) return MGSB_INVALID_ARG;
    if (level < 0 || level >= params->levels || params->levels < 2) return MGSB_INVALID_ARG;
    std::vector<PlanBody> bodies(1);
    std::string e;
    mgsb_status st = make_body(*mesh, *params, true, bodies[0], e);
    if (st != MGSB_OK) return st;
    if (fixed)
        for (int i = 0; i < bodies[0].V; ++i) bodies[0].fixed[i] = fixed[i] ? 1 : 0;
    Plan P;
    if (!build_plan(bodies, *params, P, e)) return MGSB_INVALID_ARG;
    const PlanLevel& pl = P.levels[level];
    *n = pl.n;
    *nnz = pl.nnz;
    if (pid && pw && level > 0)
        for (size_t i = 0; i < pl.pid.size(); ++i) {
            pid[4 * i] = pl.pid[i].x; pid[4 * i + 1] = pl.pid[i].y; pid[4 * i + 2] = pl.pid[i].z; pid[4 * i + 3] = pl.pid[i].w;
            pw[4 * i] = pl.pw[i].x; pw[4 * i + 1] = pl.pw[i].y; pw[4 * i + 2] = pl.pw[i].z; pw[4 * i + 3] = pl.pw[i].w;
        }
    if (diag)
        for (int i = 0; i < pl.n; ++i) diag[i] = level == 0 ? P.diag[i] : pl.diag0[i];
    if (ptr && col && val) {
        // CSR from the sliced ELL; padding entries point at their own row.
        int z = 0;
        ptr[0] = 0;
        for (int r = 0; r < pl.n; ++r) {
            const int s0 = r / pl.S, lane = r % pl.S;
            for (int q = pl.slice_ptr[s0] + lane; q < pl.slice_ptr[s0 + 1]; q += pl.S)
                if (pl.ell_col[q] != r) {
                    col[z] = pl.ell_col[q];
                    val[z] = pl.ell_val[q];
                    ++z;
                }
            ptr[r + 1] = z;
        }
    }
    return MGSB_OK;
}

mgsb_status mgsb_launches_per_frame(const mgsb_solver* h, int32_t* n) {
    if (!h || !n) return MGSB_INVALID_ARG;
    *n = h->launches;
    return MGSB_OK;
}

mgsb_status mgsb_get_precompute(mgsb_solver* h, float* inv_dm, float* ac, float* volume, float* mass, float* diag) {
    if (!h) return MGSB_INVALID_ARG;
    TRY(ensure_ready(h));
    if (inv_dm) std::copy(h->h_inv.begin(), h->h_inv.end(), inv_dm);
    if (ac) std::copy(h->h_ac.begin(), h->h_ac.end(), ac);
    if (volume) std::copy(h->h_vol.begin(), h->h_vol.end(), volume);
    if (mass) std::copy(h->h_mass.begin(), h->h_mass.end(), mass);
    if (diag) std::copy(h->h_diag.begin(), h->h_diag.end(), diag);
    return MGSB_OK;
}

mgsb_status mgsb_level_size(mgsb_solver* h, int32_t level, int32_t* num_verts, int32_t* nnz_offdiag) {
    if (!h || !num_verts || !nnz_offdiag) return MGSB_INVALID_ARG;
    TRY(ensure_ready(h));
    if (level < 0 || level >= (int32_t)h->lev.size()) return set_err(h, MGSB_INVALID_ARG, "level %d out of range", level);
    *num_verts = h->lev[level].n;
    *nnz_offdiag = h->lev[level].nnz;
    return MGSB_OK;
}

mgsb_status mgsb_level_info(mgsb_solver* h, int32_t level, int32_t info[8]) {
    if (!h || !info) return MGSB_INVALID_ARG;
    TRY(ensure_ready(h));
    if (level < 0 || level >= (int32_t)h->lev.size()) return set_err(h, MGSB_INVALID_ARG, "level %d out of range", level);
    const LevelDev& l = h->lev[level];
    info[0] = l.n;
    info[1] = l.nnz;
    info[2] = l.nchild;
    info[3] = l.S;
    info[4] = l.ell_entries;
    info[5] = h->cluster;
    info[6] = h->coarse_block;
    info[7] = h->fuse_l0;
    return MGSB_OK;
}

mgsb_status mgsb_body_level_size(mgsb_solver* h, int32_t body, int32_t level, int32_t* n) {
    if (!h || !n) return MGSB_INVALID_ARG;
    TRY(check_body(h, body));
    TRY(ensure_ready(h));
    if (!is_mg(h)) return set_err(h, MGSB_NOT_SUPPORTED, "levels exist in the multigrid kinds only");
    if (level < 0 || level >= h->p.levels) return set_err(h, MGSB_INVALID_ARG, "level %d out of range", level);
    *n = h->range_host[(size_t)body * h->p.levels + level].y;
    return MGSB_OK;
}

const char* mgsb_last_error_string(const mgsb_solver* h) { return h ? h->err.c_str() : "null handle"; }

const char* mgsb_status_string(mgsb_status s) {
    switch (s) {
        case MGSB_OK: return "ok";
        case MGSB_INVALID_ARG: return "invalid argument";
        case MGSB_DEGENERATE_TET: return "degenerate tetrahedron";
        case MGSB_CUDA_ERROR: return "CUDA error";
        case MGSB_DIVERGED: return "diverged";
        case MGSB_TIMEOUT: return "timeout";
        case MGSB_NOT_SUPPORTED: return "not supported";
        case MGSB_OUT_OF_MEMORY: return "out of memory";
        case MGSB_IO_ERROR: return "I/O error";
    }
    return "unknown";
}

}  // extern "C"

// ===========================================================================
// Allocation-free normals readback
// ===========================================================================
// Some callers cannot allocate device memory while they run: a host that hands
// the library a fixed memory budget and forbids driver allocations inside its
// frame loop, or a real-time render/haptics thread that cannot take the
// implicit device synchronisation and latency of cudaMalloc/cudaFree.
// mgsb_get_normals may (re)allocate its scratch when a set-up is pending; this
// variant runs the same two kernels (k_tri_normals, k_vert_normals) on a fixed
// scratch array compiled into the library and allocates nothing.
namespace {

constexpr int kNoAllocMaxTris = 65536;        // triangle normals of one body
constexpr int kNoAllocMaxSurfVerts = 65536;   // surface-vertex normals of one body
constexpr int kNoAllocMaxDevices = 64;

// 131,072 float4 = 2 MiB: triangle normals in [0, kNoAllocMaxTris), vertex
// normals after them.  Every GPU that loads the library holds this array until
// the process exits.  Nothing in it needs to start at zero: each call writes
// every triangle slot it reads and every vertex slot it copies out.
static __device__ __align__(256) float4 g_noalloc_scratch[kNoAllocMaxTris + kNoAllocMaxSurfVerts];

// The driver's cuCtxGetCurrent, fetched through the runtime (no link against
// libcuda): the context a cached symbol address belongs to.
using CtxGetCurrentFn = int (*)(void**);

CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    return fn;
}

// Device address of the scratch on h's device (cudaGetSymbolAddress; no
// allocation), looked up with that device current once per device and context:
// if the device's context is destroyed and created again (cudaDeviceReset by
// the host or another library), the module may load at another address, so a
// new context repeats the look-up.  The first call on a device (and the first
// after such a reset) does this set-up, so make it outside any stream capture.
mgsb_status noalloc_scratch(mgsb_solver* h, float4** out) {
    static std::mutex mu;
    static float4* ptr[kNoAllocMaxDevices] = {};
    static void* ctx[kNoAllocMaxDevices] = {};
    if (h->device < 0 || h->device >= kNoAllocMaxDevices)
        return set_err(h, MGSB_NOT_SUPPORTED, "device %d: the allocation-free path supports devices 0..%d", h->device,
                       kNoAllocMaxDevices - 1);
    std::lock_guard<std::mutex> lock(mu);
    CUDA_TRY(h, cudaSetDevice(h->device));
    void* cur = nullptr;
    const CtxGetCurrentFn get = ctx_get_current();
    if (!get || get(&cur) != 0) cur = nullptr;   // unknown context: look the address up on every call
    if (!ptr[h->device] || !cur || cur != ctx[h->device]) {
        float4* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return set_err(h, MGSB_CUDA_ERROR, "cudaGetSymbolAddress of the normals scratch failed on device %d: %s",
                           h->device, cudaGetErrorString(e));
        ptr[h->device] = p;
        ctx[h->device] = cur;
    }
    *out = ptr[h->device];
    return MGSB_OK;
}

}  // namespace

extern "C" mgsb_status mgsb_get_normals_noalloc(mgsb_solver* h, int32_t body, float* out) {
    if (!out) return MGSB_INVALID_ARG;
    TRY(check_body(h, body));
    if (h->dirty)
        return set_err(h, MGSB_INVALID_ARG,
                       "set-up pending (fixed set, material or parameters changed): the allocation-free normals do not "
                       "rebuild; call mgsb_step or mgsb_get_normals once first");
    const int nf = h->nrm_nf[body], nsv = h->nrm_nsv[body];
    if (nf > kNoAllocMaxTris || nsv > kNoAllocMaxSurfVerts)
        return set_err(h, MGSB_NOT_SUPPORTED,
                       "body %d has %d surface triangles and %d surface vertices; the allocation-free normals hold at "
                       "most %d and %d (use mgsb_get_normals)",
                       body, nf, nsv, kNoAllocMaxTris, kNoAllocMaxSurfVerts);
    float4* scratch = nullptr;
    TRY(noalloc_scratch(h, &scratch));
    // the solver's pinned readback buffer (N0 float4, allocated at create) takes the copy
    return run_normals(h, body, scratch, scratch + kNoAllocMaxTris, reinterpret_cast<float4*>(h->readback), out);
}

// ===========================================================================
// Learned smoother: attach a network, counters, training pairs
// ===========================================================================
extern "C" mgsb_status mgsb_set_learned_smoother(mgsb_solver* h, const mgsb_mlp* net, float guard_ratio) {
    if (!h) return MGSB_INVALID_ARG;
    if (!is_mg(h)) return set_err(h, MGSB_NOT_SUPPORTED, "the learned smoother needs the multigrid solver kind");
    if (net && mlp_device(net) != h->device)
        return set_err(h, MGSB_INVALID_ARG, "network on device %d, solver on device %d", mlp_device(net), h->device);
    if (net && !(guard_ratio > 0.f && guard_ratio <= 10.f))
        return set_err(h, MGSB_INVALID_ARG, "guard ratio %g outside (0, 10]", (double)guard_ratio);
    TRY(sync_check(h));
    h->ls_net = net;
    if (net) h->ls_gamma = guard_ratio;
    if (!h->dirty) {
        apply_tuning(h);
        CUDA_TRY(h, cudaMemsetAsync(h->ls_stats, 0, 2 * sizeof(unsigned long long), h->stream));
    }
    invalidate_graph(h);
    return MGSB_OK;
}

extern "C" mgsb_status mgsb_learned_stats(mgsb_solver* h, uint64_t out[2]) {
    if (!h || !out) return MGSB_INVALID_ARG;
    out[0] = out[1] = 0;
    if (!is_mg(h) || h->dirty || !h->ls_stats) return MGSB_OK;
    TRY(sync_check(h));
    unsigned long long tmp[2] = {0, 0};
    CUDA_TRY(h, cudaMemcpy(tmp, h->ls_stats, sizeof tmp, cudaMemcpyDeviceToHost));
    out[0] = tmp[0];
    out[1] = tmp[1];
    return MGSB_OK;
}

extern "C" mgsb_status mgsb_learned_cycle_norms(mgsb_solver* h, double* before, double* after, int32_t cap,
                                                int32_t* n) {
    if (!h || !n || cap < 0 || (cap > 0 && (!before || !after))) return MGSB_INVALID_ARG;
    *n = 0;
    if (!is_mg(h) || h->dirty || !h->ls_part0) return MGSB_OK;
    TRY(sync_check(h));
    const size_t count = (size_t)h->ls_cycles * h->ls_nblk;
    std::vector<float> p0(count), p1(count);
    CUDA_TRY(h, cudaMemcpy(p0.data(), h->ls_part0, count * sizeof(float), cudaMemcpyDeviceToHost));
    CUDA_TRY(h, cudaMemcpy(p1.data(), h->ls_part1, count * sizeof(float), cudaMemcpyDeviceToHost));
    const int cycles = h->ls_cycles;
    for (int c = 0; c < cycles && c < cap; ++c) {
        double a = 0.0, q = 0.0;
        for (int i = 0; i < h->ls_nblk; ++i) {
            a += p0[(size_t)c * h->ls_nblk + i];
            q += p1[(size_t)c * h->ls_nblk + i];
        }
        before[c] = std::sqrt(a);
        after[c] = std::sqrt(q);
    }
    *n = cycles;
    return MGSB_OK;
}

extern "C" mgsb_status mgsb_smoother_pairs(mgsb_solver* h, int32_t sweeps, float* x, float* t, int64_t cap,
                                           int64_t* n) {
    if (!h || !n || sweeps < 1) return MGSB_INVALID_ARG;
    *n = 0;
    if (!is_mg(h) || h->p.precision != MGSB_PRECISION_FP32)
        return set_err(h, MGSB_NOT_SUPPORTED, "training pairs come from the plain FP32 multigrid solver");
    if (h->dirty || !h->d_final) return set_err(h, MGSB_INVALID_ARG, "run a frame before generating pairs");
    if (h->fuse_l0)
        return set_err(h, MGSB_NOT_SUPPORTED, "pair generation uses the shared-memory coarse kernel (fuse_level0 = 0)");
    TRY(sync_check(h));
    const int n0 = h->N0;
    auto& pool = h->pair_mem;
    if (!h->ls_xf) {
        TRY(dalloc(h, pool, &h->ls_xf, (size_t)n0 * kMlpIn));
        TRY(dalloc(h, pool, &h->ls_t, (size_t)n0 * kMlpOut));
        TRY(dalloc(h, pool, &h->ls_mask, (size_t)n0));
        TRY(dalloc(h, pool, &h->ls_e1, (size_t)n0));
        TRY(dalloc(h, pool, &h->ls_e2, (size_t)n0));
        TRY(dalloc(h, pool, &h->ls_ec, (size_t)n0));
        TRY(dalloc(h, pool, &h->ls_s, (size_t)n0));
    }
    std::vector<LevelDev>& lv = h->lev;
    const LevelDev& l0 = lv[0];
    const int g0 = h->ls_nblk;
    cudaStream_t st = h->stream;
    const mgsb_params& p = h->p;
    CUDA_TRY(h, cudaSetDevice(h->device));
    const int launches = h->launches;   // not part of a frame
    CoarseArgs ca;
    fill_coarse_args(h, ca);
    std::vector<float> hx((size_t)n0 * kMlpIn), ht((size_t)n0 * kMlpOut), hs(n0);
    std::vector<uint8_t> hm(n0);
    int64_t cnt = 0;
    // Jacobi sweeps from e = 0 on A e = rhs (ping-pong e1/e2); returns the result buffer
    auto sweeps_from_zero = [&](const float4* rhs, int k_sweeps) {
        float4* xa = h->ls_e1;
        float4* xb = h->ls_e2;
        cudaMemsetAsync(xa, 0, (size_t)n0 * sizeof(float4), st);
        for (int k = 0; k < k_sweeps; ++k) {
            k_l0_sweep_rg<<<g0, kBlock, 0, st>>>(n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, l0.dinv, xa, xb,
                                                 const_cast<float4*>(rhs), h->b0, h->slot_ptr, h->slots, 0, nullptr);
            std::swap(xa, xb);
        }
        return xa;
    };
    // one set of pairs for residual r: features of r against `sweeps` Jacobi sweeps
    auto collect = [&](const float4* r) -> mgsb_status {
        k_ls_features<<<g0, kLsThreads, 0, st>>>(n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, h->vdiag, h->fixf, r,
                                                 nullptr, h->ls_scale, h->ls_xf);
        const float4* ek = sweeps_from_zero(r, sweeps);
        CUDA_TRY(h, cudaMemsetAsync(h->ls_ec, 0, (size_t)n0 * sizeof(float4), st));   // no coarse part
        k_ls_targets<<<grid_for(n0), kBlock, 0, st>>>(n0, h->ls_scale, l0.dfull, ek, h->ls_ec, h->ls_t, h->ls_mask,
                                                      h->ls_s);
        CUDA_TRY(h, cudaGetLastError());
        CUDA_TRY(h, cudaMemcpyAsync(hx.data(), h->ls_xf, hx.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(h, cudaMemcpyAsync(ht.data(), h->ls_t, ht.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(h, cudaMemcpyAsync(hm.data(), h->ls_mask, hm.size(), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(h, cudaMemcpyAsync(hs.data(), h->ls_s, hs.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(h, cudaStreamSynchronize(st));
        // Rows whose residual is tiny next to the state's RMS carry no
        // information for the smoother: keep rows with s_i >= 1e-2 RMS(s).
        double ss = 0.0;
        int64_t nm = 0;
        for (int i = 0; i < n0; ++i)
            if (hm[i]) {
                ss += (double)hs[i] * hs[i];
                ++nm;
            }
        const double s_min = nm ? 1e-2 * std::sqrt(ss / (double)nm) : 0.0;
        for (int i = 0; i < n0; ++i) {
            if (!hm[i] || hs[i] < s_min) continue;
            if (x && t && cnt < cap) {
                std::copy(&hx[(size_t)i * kMlpIn], &hx[(size_t)i * kMlpIn] + kMlpIn, x + cnt * kMlpIn);
                std::copy(&ht[(size_t)i * kMlpOut], &ht[(size_t)i * kMlpOut] + kMlpOut, t + cnt * kMlpOut);
            }
            ++cnt;
        }
        return MGSB_OK;
    };
    // (1) the residual of the last global step, r = b - A d (a pre-smoothing input)
    k_ls_residual<<<g0, kLsThreads, 0, st>>>(n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, h->fixf, h->d_final,
                                             h->b, h->ls_r, nullptr, nullptr);
    TRY(collect(h->ls_r));
    // (2) the residual after plain pre-smoothing and the coarse correction (a
    //     post-smoothing input): e = sweeps(r) + P V_c(P^T (r - A e)), r2 = r - A e
    float4* e = sweeps_from_zero(h->ls_r, p.pre_sweeps);
    k_l0_residual_rg<<<g0, kBlock, 0, st>>>(n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, e, h->ls_r, l0.res, nullptr);
    ca.d = e;
    TRY(launch_coarse(h, ca));
    k_l0_prolong<<<grid_for(n0), kBlock, 0, st>>>(n0, lv[1].pid, lv[1].pw, lv[1].e, e, nullptr);
    k_ls_residual<<<g0, kLsThreads, 0, st>>>(n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, h->fixf, e, h->ls_r,
                                             h->ls_save, nullptr, nullptr);
    TRY(collect(h->ls_save));
    // (3) the residual a further PD iteration would start from: the local step
    //     at the current displacement gives b' = b0 + slots, r3 = b' - A d.
    //     (the slots are rebuilt by the next frame's first local step)
    k_mg_local<<<grid_for(h->T), kBlock, 0, st>>>(h->T, h->tets, h->tA, h->tB, h->tC, h->s, h->d_final, h->slot_of,
                                                   h->slots);
    k_gather_rhs<<<grid_for(n0), kBlock, 0, st>>>(n0, h->ls_ec, h->b0, h->slot_ptr, h->slots);
    k_ls_residual<<<g0, kLsThreads, 0, st>>>(n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, h->fixf, h->d_final,
                                             h->ls_ec, h->ls_save, nullptr, nullptr);
    TRY(collect(h->ls_save));
    h->launches = launches;
    *n = cnt;
    if (x && t && cnt > cap) return set_err(h, MGSB_INVALID_ARG, "pair buffer too small (%lld < %lld)", (long long)cap,
                                             (long long)cnt);
    return MGSB_OK;
}

// Convergence of V-cycles on the last global step's correction equation
// A e = r (r = b - A d, e from zero), for the smoother comparison: mode 0 =
// plain with the configured sweeps, 1 = plain with one sweep each side, 2 =
// learned (no fallback).  out[0] = |r|, out[k] = |r - A e| after k cycles.
extern "C" mgsb_status mgsb_vcycle_residuals(mgsb_solver* h, int32_t cycles, int32_t mode, double* out) {
    if (!h || !out || cycles < 1 || mode < 0 || mode > 2) return MGSB_INVALID_ARG;
    if (!is_mg(h) || h->p.precision != MGSB_PRECISION_FP32)
        return set_err(h, MGSB_NOT_SUPPORTED, "V-cycle residuals are measured on the plain FP32 multigrid solver");
    if (h->dirty || !h->d_final) return set_err(h, MGSB_INVALID_ARG, "run a frame first");
    if (mode == 2 && !h->ls_net) return set_err(h, MGSB_INVALID_ARG, "no learned smoother attached");
    if (h->fuse_l0) return set_err(h, MGSB_NOT_SUPPORTED, "needs the shared-memory coarse kernel (fuse_level0 = 0)");
    TRY(sync_check(h));
    const int n0 = h->N0;
    auto& pool = h->pair_mem;
    if (!h->ls_xf) {
        TRY(dalloc(h, pool, &h->ls_xf, (size_t)n0 * kMlpIn));
        TRY(dalloc(h, pool, &h->ls_t, (size_t)n0 * kMlpOut));
        TRY(dalloc(h, pool, &h->ls_mask, (size_t)n0));
        TRY(dalloc(h, pool, &h->ls_e1, (size_t)n0));
        TRY(dalloc(h, pool, &h->ls_e2, (size_t)n0));
        TRY(dalloc(h, pool, &h->ls_ec, (size_t)n0));
        TRY(dalloc(h, pool, &h->ls_s, (size_t)n0));
    }
    std::vector<LevelDev>& lv = h->lev;
    const LevelDev& l0 = lv[0];
    const int g0 = h->ls_nblk;
    cudaStream_t st = h->stream;
    CUDA_TRY(h, cudaSetDevice(h->device));
    float4* rhs = h->ls_ec;   // r, kept for the whole measurement
    k_ls_residual<<<g0, kLsThreads, 0, st>>>(n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, h->fixf, h->d_final,
                                             h->b, rhs, nullptr, nullptr);
    float4* e = h->ls_e1;
    float4* tmp = h->ls_e2;
    CUDA_TRY(h, cudaMemsetAsync(e, 0, (size_t)n0 * sizeof(float4), st));
    std::vector<float> part(g0);
    auto norm = [&](double* dst) -> mgsb_status {
        k_ls_residual<<<g0, kLsThreads, 0, st>>>(n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, h->fixf, e, rhs,
                                                 nullptr, nullptr, h->ls_part1);
        CUDA_TRY(h, cudaMemcpyAsync(part.data(), h->ls_part1, g0 * sizeof(float), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(h, cudaStreamSynchronize(st));
        double a = 0.0;
        for (float v : part) a += v;
        *dst = std::sqrt(a);
        return MGSB_OK;
    };
    TRY(norm(out));
    CoarseArgs ca;
    fill_coarse_args(h, ca);
    const mgsb_params& p = h->p;
    const int pre = mode == 1 ? 1 : p.pre_sweeps, post = mode == 1 ? 1 : p.post_sweeps;
    const bool prof = h->profiling;
    const int launches = h->launches;   // this measurement is not part of a frame
    h->profiling = false;
    if (mode == 2) enqueue_ls_row_consts(h);
    for (int c = 0; c < cycles; ++c) {
        if (mode == 2) {
            enqueue_learned_vcycle(h, e, rhs, c == 0, ca, 0);   // the learned cycle alone, no check
        } else {
            float4* xa = e;
            float4* xb = tmp;
            for (int k = 0; k < pre; ++k) {
                k_l0_sweep_rg<<<g0, kBlock, 0, st>>>(n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, l0.dinv, xa, xb,
                                                     rhs, h->b0, h->slot_ptr, h->slots, 0, nullptr);
                std::swap(xa, xb);
            }
            k_l0_residual_rg<<<g0, kBlock, 0, st>>>(n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, xa, rhs, l0.res,
                                                    nullptr);
            ca.d = xa;
            ca.gate = nullptr;
            TRY(launch_coarse(h, ca));
            k_l0_prolong<<<grid_for(n0), kBlock, 0, st>>>(n0, lv[1].pid, lv[1].pw, lv[1].e, xa, nullptr);
            for (int k = 0; k < post; ++k) {
                k_l0_sweep_rg<<<g0, kBlock, 0, st>>>(n0, l0.slice_ptr, l0.ell_col, l0.ell_val, l0.dfull, l0.dinv, xa, xb,
                                                     rhs, h->b0, h->slot_ptr, h->slots, 0, nullptr);
                std::swap(xa, xb);
            }
            if (xa != e) CUDA_TRY(h, cudaMemcpyAsync(e, xa, (size_t)n0 * sizeof(float4), cudaMemcpyDeviceToDevice, st));
        }
        CUDA_TRY(h, cudaGetLastError());
        TRY(norm(out + c + 1));
    }
    h->profiling = prof;
    h->launches = launches;
    return MGSB_OK;
}

// ===========================================================================
// The reference's two-level schedule (PDSolver_MG, PDSolver_MG.cpp:5-253)
// ===========================================================================
// Two reference-kind solvers share one stream: per frame both predict, the
// coarse level runs its Jacobi/Chebyshev iterations with sphere-vs-surface-
// triangle collision, the fine positions are interpolated from the coarse
// mesh, the fine level iterates with per-vertex sphere collision, the coarse
// positions are averaged back from the fine mesh, the fine-in-coarse weights are
// recomputed from the current shapes, and both velocities follow.
struct mgsb_two_level {
    mgsb_solver* coarse = nullptr;
    mgsb_solver* fine = nullptr;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    std::vector<DevMem> mem;
    int nf = 0, nc = 0, ntri = 0;
    int4* f_ids = nullptr;     // fine vertex -> coarse tet ids
    float4* f_w = nullptr;     //   and weights (recomputed every frame)
    int4* c_ids = nullptr;     // coarse vertex -> fine tet ids
    float4* c_w = nullptr;
    int4* tris = nullptr;      // coarse surface triangles
    int32_t *tri_ptr = nullptr, *tri_idx = nullptr;   // coarse vertex -> its triangles
    float4* push = nullptr;    // per-triangle push sum and contact count
    bool graph_valid = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~mgsb_two_level() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        delete coarse;
        delete fine;
        cudaSetDevice(device);
        for (auto& m : mem) cudaFree(m.p);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

namespace {

mgsb_status tl_err(mgsb_two_level* t, mgsb_status s, const char* msg) {
    if (t) t->err = msg;
    return s;
}

template <typename T>
mgsb_status tl_upload(mgsb_two_level* t, T** out, const T* src, size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return tl_err(t, MGSB_OUT_OF_MEMORY, "cudaMalloc failed");
    t->mem.push_back({p, n * sizeof(T)});
    *out = static_cast<T*>(p);
    if (n && cudaMemcpy(p, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        return tl_err(t, MGSB_CUDA_ERROR, "cudaMemcpy failed");
    return MGSB_OK;
}

void enqueue_two_level_frame(mgsb_two_level* t) {
    mgsb_solver* C = t->coarse;
    mgsb_solver* F = t->fine;
    const mgsb_params& pc = C->p;
    const mgsb_params& pf = F->p;
    C->launches = F->launches = 0;
    const BodyHost& BC = C->bodies[0];
    const BodyHost& BF = F->bodies[0];
    LAUNCH(C, k_ref_predict, grid_for(t->nc), kBlock, 0, t->nc, C->x, C->v, C->s, C->prev, C->last, C->fixf, BC.damping,
           pc.dt, BC.gravity[0], BC.gravity[1], BC.gravity[2]);
    LAUNCH(F, k_ref_predict, grid_for(t->nf), kBlock, 0, t->nf, F->x, F->v, F->s, F->prev, F->last, F->fixf, BF.damping,
           pf.dt, BF.gravity[0], BF.gravity[1], BF.gravity[2]);
    float omega = 1.0f;
    for (int it = 0; it < pc.iterations; ++it) {
        LAUNCH(C, k_ref_local, grid_for(C->T), kBlock, 0, C->T, C->tets, C->tA, C->tB, C->tC, C->x, C->slot_of, C->slots,
               pc.volume_stiffness, 0);
        LAUNCH(C, k_ref_tri_dcd, grid_for(t->ntri), kBlock, 0, t->ntri, t->tris, C->x, C->spheres_dev, t->push);
        omega = 4 / (4 - pc.cheb_rho * pc.cheb_rho * omega);
        LAUNCH(C, k_ref_vertex, grid_for(t->nc), kBlock, 0, t->nc, C->x, C->prev, C->s, C->last, C->v, C->fixf, C->mass,
               C->vdiag, C->slot_ptr, C->slots, C->spheres_dev, pc.collision_stiffness, pc.dt, omega,
               (double)pc.relaxation, it == pc.iterations - 1 ? 2 : 0, C->cflag, C->cdepth, C->cenergy, C->nonfinite,
               t->tri_ptr, t->tri_idx, t->push);
    }
    LAUNCH(F, k_tl_transfer, grid_for(t->nf), kBlock, 0, t->nf, t->f_ids, t->f_w, C->x, F->x, F->prev);
    omega = 1.0f;
    for (int it = 0; it < pf.iterations; ++it) {
        LAUNCH(F, k_ref_local, grid_for(F->T), kBlock, 0, F->T, F->tets, F->tA, F->tB, F->tC, F->x, F->slot_of, F->slots,
               pf.volume_stiffness, 0);
        omega = 4 / (4 - pf.cheb_rho * pf.cheb_rho * omega);
        LAUNCH(F, k_ref_vertex, grid_for(t->nf), kBlock, 0, t->nf, F->x, F->prev, F->s, F->last, F->v, F->fixf, F->mass,
               F->vdiag, F->slot_ptr, F->slots, F->spheres_dev, pf.collision_stiffness, pf.dt, omega,
               (double)pf.relaxation, it == pf.iterations - 1 ? 2 : 0, F->cflag, F->cdepth, F->cenergy, F->nonfinite,
               nullptr, nullptr, nullptr);
    }
    LAUNCH(C, k_tl_transfer, grid_for(t->nc), kBlock, 0, t->nc, t->c_ids, t->c_w, F->x, C->x, C->prev);
    LAUNCH(F, k_tl_update_mapping, grid_for(t->nf), kBlock, 0, t->nf, F->x, t->f_ids, C->x, t->f_w);
    LAUNCH(C, k_velocity, grid_for(t->nc), kBlock, 0, t->nc, C->x, C->last, C->v, pc.dt, C->nonfinite);
    LAUNCH(F, k_velocity, grid_for(t->nf), kBlock, 0, t->nf, F->x, F->last, F->v, pf.dt, F->nonfinite);
}

}  // namespace

extern "C" {

mgsb_status mgsb_mg2_create(const mgsb_mesh* coarse, const mgsb_mesh* fine, const mgsb_params* params,
                            mgsb_two_level** out) {
    if (!out) return MGSB_INVALID_ARG;
    *out = nullptr;
    if (!coarse || !fine || !params) return MGSB_INVALID_ARG;
    if (params->solver != MGSB_SOLVER_REFERENCE_JACOBI) return MGSB_NOT_SUPPORTED;
    std::unique_ptr<mgsb_two_level> t(new mgsb_two_level());
    t->device = params->device;
    if (cudaSetDevice(t->device) != cudaSuccess) return MGSB_CUDA_ERROR;
    mgsb_params p = *params;
    if (!p.stream) {
        cudaStream_t s = nullptr;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return MGSB_CUDA_ERROR;
        t->stream = s;
        t->own_stream = true;
        p.stream = s;
    } else {
        t->stream = (cudaStream_t)p.stream;
    }
    p.use_graph = 0;   // the two-level handle captures the whole frame itself
    mgsb_status st = create_impl(1, coarse, &p, &t->coarse);
    if (st != MGSB_OK) return st;
    st = create_impl(1, fine, &p, &t->fine);
    if (st != MGSB_OK) return st;
    t->nc = coarse->num_verts;
    t->nf = fine->num_verts;
    // bindings on the rest shapes (PDSolver_MG::Init)
    std::vector<int32_t> fid, cid;
    std::vector<float> fw, cw;
    std::string e;
    if (!tl_bind_fine_to_coarse(fine->positions, t->nf, coarse->positions, coarse->tets, coarse->num_tets, fid, fw, e) ||
        !tl_bind_coarse_to_fine(coarse->positions, t->nc, fine->positions, fine->tets, fine->num_tets, cid, cw, e)) {
        char buf[256];
        std::snprintf(buf, sizeof buf, "two-level binding: %s", e.c_str());
        t->err = buf;
        return MGSB_INVALID_ARG;
    }
    TRY(tl_upload(t.get(), &t->f_ids, reinterpret_cast<const int4*>(fid.data()), (size_t)t->nf));
    TRY(tl_upload(t.get(), &t->f_w, reinterpret_cast<const float4*>(fw.data()), (size_t)t->nf));
    TRY(tl_upload(t.get(), &t->c_ids, reinterpret_cast<const int4*>(cid.data()), (size_t)t->nc));
    TRY(tl_upload(t.get(), &t->c_w, reinterpret_cast<const float4*>(cw.data()), (size_t)t->nc));
    // coarse surface triangles (TetFaceExtraction order) and the vertex -> triangle CSR
    std::vector<int32_t> tris, opp;
    extract_surface(coarse->tets, coarse->num_tets, tris, opp);
    t->ntri = (int)(tris.size() / 3);
    std::vector<int4> t4(t->ntri);
    std::vector<int32_t> ptr(t->nc + 1, 0), idx;
    for (int f = 0; f < t->ntri; ++f) {
        t4[f] = int4{tris[3 * f], tris[3 * f + 1], tris[3 * f + 2], 0};
        for (int q = 0; q < 3; ++q) ++ptr[tris[3 * f + q] + 1];
    }
    for (int v = 0; v < t->nc; ++v) ptr[v + 1] += ptr[v];
    idx.resize(ptr[t->nc]);
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int f = 0; f < t->ntri; ++f)
        for (int q = 0; q < 3; ++q) idx[fill[tris[3 * f + q]]++] = f;
    TRY(tl_upload(t.get(), &t->tris, t4.data(), t4.size()));
    TRY(tl_upload(t.get(), &t->tri_ptr, ptr.data(), ptr.size()));
    TRY(tl_upload(t.get(), &t->tri_idx, idx.data(), idx.size()));
    std::vector<float4> zero(std::max(t->ntri, 1), float4{0, 0, 0, 0});
    TRY(tl_upload(t.get(), &t->push, zero.data(), (size_t)t->ntri));
    *out = t.release();
    return MGSB_OK;
}

mgsb_status mgsb_mg2_destroy(mgsb_two_level* t) {
    if (!t) return MGSB_INVALID_ARG;
    delete t;
    return MGSB_OK;
}

const char* mgsb_mg2_last_error(const mgsb_two_level* t) {
    if (!t) return "null handle";
    if (!t->err.empty()) return t->err.c_str();
    if (t->coarse && !t->coarse->err.empty()) return t->coarse->err.c_str();
    if (t->fine && !t->fine->err.empty()) return t->fine->err.c_str();
    return "";
}

mgsb_status mgsb_mg2_level(mgsb_two_level* t, int32_t level, mgsb_solver** out) {
    if (!t || !out || level < 0 || level > 1) return MGSB_INVALID_ARG;
    *out = level == 0 ? t->fine : t->coarse;
    return MGSB_OK;
}

mgsb_status mgsb_mg2_set_fixed(mgsb_two_level* t, const uint8_t* coarse_mask, const uint8_t* fine_mask) {
    if (!t) return MGSB_INVALID_ARG;
    if (coarse_mask) TRY(mgsb_set_fixed(t->coarse, 0, coarse_mask));
    if (fine_mask) TRY(mgsb_set_fixed(t->fine, 0, fine_mask));
    t->graph_valid = false;
    return MGSB_OK;
}

mgsb_status mgsb_mg2_set_tool_spheres(mgsb_two_level* t, int32_t count, const float* centers, const float* radii,
                                      const uint8_t* active) {
    if (!t) return MGSB_INVALID_ARG;
    TRY(mgsb_set_tool_spheres(t->coarse, count, centers, radii, active));
    TRY(mgsb_set_tool_spheres(t->fine, count, centers, radii, active));
    return MGSB_OK;
}

mgsb_status mgsb_mg2_step(mgsb_two_level* t) {
    if (!t) return MGSB_INVALID_ARG;
    mgsb_solver* C = t->coarse;
    mgsb_solver* F = t->fine;
    if (C->dirty || F->dirty) t->graph_valid = false;
    TRY(ensure_ready(C));
    TRY(ensure_ready(F));
    if (cudaSetDevice(t->device) != cudaSuccess) return tl_err(t, MGSB_CUDA_ERROR, "cudaSetDevice failed");
    TRY(push_tool(C));
    TRY(push_tool(F));
    if (!t->graph_valid) {
        if (t->exec) cudaGraphExecDestroy(t->exec);
        if (t->graph) cudaGraphDestroy(t->graph);
        t->exec = nullptr;
        t->graph = nullptr;
        if (cudaStreamBeginCapture(t->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return tl_err(t, MGSB_CUDA_ERROR, "graph capture could not start");
        enqueue_two_level_frame(t);
        if (cudaStreamEndCapture(t->stream, &t->graph) != cudaSuccess ||
            cudaGraphInstantiate(&t->exec, t->graph, 0) != cudaSuccess)
            return tl_err(t, MGSB_CUDA_ERROR, "graph capture of the two-level frame failed");
        t->graph_valid = true;
    }
    if (cudaGraphLaunch(t->exec, t->stream) != cudaSuccess) return tl_err(t, MGSB_CUDA_ERROR, "graph launch failed");
    C->timed = F->timed = false;
    return MGSB_OK;
}

mgsb_status mgsb_mg2_get_positions(mgsb_two_level* t, int32_t level, float* out) {
    if (!t || !out || level < 0 || level > 1) return MGSB_INVALID_ARG;
    return mgsb_get_positions(level == 0 ? t->fine : t->coarse, 0, out);
}

}  // extern "C"
