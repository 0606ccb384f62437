// Host runtime and C ABI of the PD soft-body solver (see include/mgsb.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/mgsb.h"
#include "kernels.cuh"
#include "mesh.hpp"
#include "setup.hpp"

using namespace mgsb;

namespace {

constexpr int kBlock = 256;
inline int grid_for(int n) { return (n + kBlock - 1) / kBlock; }

// Device allocation owned by the solver.
struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
};

struct BodyHost {
    int V = 0, T = 0;
    int v_off = 0, t_off = 0;
    std::vector<double> rest;        // 3V
    std::vector<int32_t> tets;       // 4T
    std::vector<float> youngs, poisson;
    std::vector<uint8_t> fixed;
    std::vector<int32_t> surface;    // surface vertex ids (local)
    int grid_dims[3] = {0, 0, 0};
    float gravity[3] = {0, 0, 0};
    float damping = 1.f;
    float cap_a[3] = {0, 0, 0}, cap_b[3] = {0, 0, 0};
    float cap_r = 0.f;
    std::vector<TetRest> tr;
    std::vector<CoarseLevel> levels;  // multigrid levels 1..L-1
};

struct LevelDev {
    int n = 0;
    int nnz = 0;
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
    // restriction CSR (children in the finer level)
    int32_t* rptr = nullptr;
    int32_t* rcol = nullptr;
    float* rw = nullptr;
    Ell ell() const { return Ell{slice_ptr, ell_col, ell_val}; }
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
    int launches = 0;
    // per-launch CUDA events of a profiled (eager) frame
    bool profiling = false;
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
    // ---- state (kept across rebuilds)
    float4 *x = nullptr, *xb = nullptr, *v = nullptr, *s = nullptr, *last = nullptr, *prev = nullptr;
    int32_t* cflag = nullptr;
    float* cdepth = nullptr;
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
    float4 *b = nullptr, *b0 = nullptr, *target = nullptr;
    float* c0 = nullptr;
    int32_t* surf = nullptr;
    int nsurf = 0;
    std::vector<LevelDev> lev;   // lev[0] = finest
    float *A0dense = nullptr, *Lfac = nullptr, *Ldinv = nullptr, *c_prev = nullptr;
    int32_t* fac_valid = nullptr;
    size_t factor_smem = 0;
    int max_coarsest = 0;
    // host copies of precompute for export
    std::vector<float> h_inv, h_ac, h_vol, h_mass, h_diag;
};

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

// Sliced ELL (32-row slices) from per-row sorted (col, val) lists.
void build_ell(const std::vector<int32_t>& ptr, const std::vector<int32_t>& col, const std::vector<double>& val, int n,
               std::vector<int32_t>& sptr, std::vector<int32_t>& ecol, std::vector<float>& eval) {
    const int ns = (n + 31) / 32;
    sptr.assign(ns + 1, 0);
    for (int s = 0; s < ns; ++s) {
        int w = 0;
        for (int r = s * 32; r < std::min(n, s * 32 + 32); ++r) w = std::max(w, ptr[r + 1] - ptr[r]);
        sptr[s + 1] = sptr[s] + 32 * w;
    }
    ecol.assign(sptr[ns], 0);
    eval.assign(sptr[ns], 0.f);
    for (int s = 0; s < ns; ++s) {
        const int w = (sptr[s + 1] - sptr[s]) / 32;
        for (int lane = 0; lane < 32; ++lane) {
            const int r = s * 32 + lane;
            for (int k = 0; k < w; ++k) {
                const int e = sptr[s] + k * 32 + lane;
                if (r < n && ptr[r] + k < ptr[r + 1]) {
                    ecol[e] = col[ptr[r] + k];
                    eval[e] = (float)val[ptr[r] + k];
                } else {
                    ecol[e] = r < n ? r : 0;
                    eval[e] = 0.f;
                }
            }
        }
    }
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
    const int N0 = h->N0, T = h->T;

    std::vector<int32_t> body_of(N0), tets4(4 * (size_t)T);
    std::vector<float> fixf(N0), massv(N0), diagv(N0);
    std::vector<float4> tA(T), tB(T);
    std::vector<float2> tC(T);
    std::vector<int32_t> slot_ptr(N0 + 1, 0);
    std::vector<int32_t> slot_of(4 * (size_t)T);
    h->h_inv.assign(9 * (size_t)h->bodies[0].T, 0.f);
    h->h_ac.assign(12 * (size_t)h->bodies[0].T, 0.f);
    h->h_vol.assign(h->bodies[0].T, 0.f);
    h->h_mass.assign(h->bodies[0].V, 0.f);
    h->h_diag.assign(h->bodies[0].V, 0.f);

    // multigrid host assembly per body
    const int L = mg ? h->p.levels : 1;
    std::vector<SparseSym> Lmat(h->bodies.size());
    for (size_t bi = 0; bi < h->bodies.size(); ++bi) {
        BodyHost& B = h->bodies[bi];
        const double dens = mg ? (double)h->p.density : 1.0;
        std::vector<double> m(B.V, 0.0), w(B.T, 0.0), vd(B.V, 0.0);
        for (int t = 0; t < B.T; ++t) {
            const TetRest& r = B.tr[t];
            for (int a = 0; a < 4; ++a) m[B.tets[4 * t + a]] += dens * r.volume / 4.0;
            if (mg) {
                const double mu = (double)B.youngs[t] / (2.0 * (1.0 + (double)B.poisson[t]));
                w[t] = 2.0 * mu * r.volume;
            } else {
                for (int a = 0; a < 4; ++a)
                    vd[B.tets[4 * t + a]] += (r.g[a][0] * r.g[a][0] + r.g[a][1] * r.g[a][1] + r.g[a][2] * r.g[a][2]) *
                                            r.volume * (double)h->p.volume_stiffness;
            }
        }
        if (mg) {
            assemble_pd_matrix(B.tr, B.tets.data(), B.V, w.data(), m.data(), h->p.dt, Lmat[bi]);
            int dims[3] = {B.grid_dims[0], B.grid_dims[1], B.grid_dims[2]};
            if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0)
                default_grid_dims(B.rest.data(), B.V, B.tets.data(), B.T, dims);
            build_hierarchy(B.rest.data(), B.V, Lmat[bi], B.fixed.data(), L, dims, B.levels);
        }
        const double ih2 = 1.0 / ((double)h->p.dt * h->p.dt);
        for (int i = 0; i < B.V; ++i) {
            const int gi = B.v_off + i;
            body_of[gi] = (int32_t)bi;
            fixf[gi] = B.fixed[i] ? 0.f : 1.f;
            massv[gi] = mg ? (float)(m[i] * ih2) : (float)m[i];
            diagv[gi] = mg ? (float)Lmat[bi].diag[i] : (float)vd[i];
        }
        for (int t = 0; t < B.T; ++t) {
            const TetRest& r = B.tr[t];
            const int gt = B.t_off + t;
            for (int a = 0; a < 4; ++a) tets4[4 * (size_t)gt + a] = B.tets[4 * t + a] + B.v_off;
            if (mg) {
                tA[gt] = make_float4((float)r.g[1][0], (float)r.g[1][1], (float)r.g[1][2], (float)r.g[2][0]);
                tB[gt] = make_float4((float)r.g[2][1], (float)r.g[2][2], (float)r.g[3][0], (float)r.g[3][1]);
                tC[gt] = make_float2((float)r.g[3][2], (float)w[t]);
            } else {
                tA[gt] = make_float4((float)r.inv[0], (float)r.inv[1], (float)r.inv[2], (float)r.inv[3]);
                tB[gt] = make_float4((float)r.inv[4], (float)r.inv[5], (float)r.inv[6], (float)r.inv[7]);
                tC[gt] = make_float2((float)r.inv[8], (float)r.volume);
            }
        }
        if (bi == 0) {
            for (int t = 0; t < B.T; ++t) {
                const TetRest& r = B.tr[t];
                for (int q = 0; q < 9; ++q) h->h_inv[9 * (size_t)t + q] = (float)r.inv[q];
                for (int rr = 0; rr < 3; ++rr)
                    for (int j = 0; j < 4; ++j) h->h_ac[12 * (size_t)t + rr * 4 + j] = (float)r.g[j][rr];
                h->h_vol[t] = (float)r.volume;
            }
            for (int i = 0; i < B.V; ++i) {
                h->h_mass[i] = (float)m[i];
                h->h_diag[i] = mg ? (float)Lmat[0].diag[i] : (float)vd[i];
            }
        }
    }
    // RHS slots: CSR by vertex, tets in ascending order within a vertex.
    for (int t = 0; t < T; ++t)
        for (int a = 0; a < 4; ++a) slot_ptr[tets4[4 * (size_t)t + a] + 1]++;
    for (int i = 0; i < N0; ++i) slot_ptr[i + 1] += slot_ptr[i];
    {
        std::vector<int32_t> fill(slot_ptr.begin(), slot_ptr.end() - 1);
        for (int t = 0; t < T; ++t)
            for (int a = 0; a < 4; ++a) slot_of[4 * (size_t)t + a] = fill[tets4[4 * (size_t)t + a]]++;
    }
    TRY(dupload(h, pool, &h->body_of, body_of));
    TRY(dupload(h, pool, &h->fixf, fixf));
    TRY(dupload(h, pool, &h->mass, massv));
    TRY(dupload(h, pool, &h->vdiag, diagv));
    {
        std::vector<int4> t4(T), s4(T);
        for (int t = 0; t < T; ++t) {
            t4[t] = make_int4(tets4[4 * (size_t)t], tets4[4 * (size_t)t + 1], tets4[4 * (size_t)t + 2], tets4[4 * (size_t)t + 3]);
            s4[t] = make_int4(slot_of[4 * (size_t)t], slot_of[4 * (size_t)t + 1], slot_of[4 * (size_t)t + 2], slot_of[4 * (size_t)t + 3]);
        }
        TRY(dupload(h, pool, &h->tets, t4));
        TRY(dupload(h, pool, &h->slot_of, s4));
    }
    TRY(dupload(h, pool, &h->tA, tA));
    TRY(dupload(h, pool, &h->tB, tB));
    TRY(dupload(h, pool, &h->tC, tC));
    TRY(dupload(h, pool, &h->slot_ptr, slot_ptr));
    TRY(dalloc(h, pool, &h->slots, 4 * (size_t)T));
    CUDA_TRY(h, cudaMemset(h->slots, 0, 4 * (size_t)T * sizeof(float4)));

    if (mg) {
        // ---- level 0
        LevelDev l0;
        l0.n = N0;
        {
            std::vector<int32_t> ptr(N0 + 1, 0), col;
            std::vector<double> val;
            for (size_t bi = 0; bi < h->bodies.size(); ++bi) {
                const BodyHost& B = h->bodies[bi];
                const SparseSym& A = Lmat[bi];
                for (int i = 0; i < B.V; ++i) {
                    for (int q = A.ptr[i]; q < A.ptr[i + 1]; ++q) {
                        col.push_back(A.col[q] + B.v_off);
                        val.push_back(A.val[q]);
                    }
                    ptr[B.v_off + i + 1] = (int32_t)col.size();
                }
            }
            std::vector<int32_t> sp, ec;
            std::vector<float> ev;
            build_ell(ptr, col, val, N0, sp, ec, ev);
            l0.nnz = (int)col.size();
            TRY(dupload(h, pool, &l0.slice_ptr, sp));
            TRY(dupload(h, pool, &l0.ell_col, ec));
            TRY(dupload(h, pool, &l0.ell_val, ev));
        }
        l0.diag0 = h->vdiag;
        TRY(dalloc(h, pool, &l0.dfull, N0));
        TRY(dalloc(h, pool, &l0.dinv, N0));
        TRY(dalloc(h, pool, &l0.res, N0));
        TRY(dalloc(h, pool, &h->c0, N0));
        CUDA_TRY(h, cudaMemset(h->c0, 0, N0 * sizeof(float)));
        l0.c = h->c0;
        TRY(dalloc(h, pool, &h->b, N0));
        TRY(dalloc(h, pool, &h->b0, N0));
        TRY(dalloc(h, pool, &h->target, N0));
        CUDA_TRY(h, cudaMemset(h->target, 0, N0 * sizeof(float4)));
        h->lev.push_back(l0);
        // ---- coarse levels
        std::vector<int> loff(h->bodies.size(), 0);
        for (int l = 1; l < L; ++l) {
            LevelDev ld;
            int n = 0;
            for (size_t bi = 0; bi < h->bodies.size(); ++bi) {
                loff[bi] = n;
                n += h->bodies[bi].levels[l - 1].n;
            }
            ld.n = n;
            const int nfin = h->lev[l - 1].n;
            std::vector<int32_t> ptr(n + 1, 0), col;
            std::vector<double> val;
            std::vector<float> diag0(n, 0.f);
            std::vector<int4> pid(nfin);
            std::vector<float4> pw(nfin);
            std::vector<int32_t> rptr(n + 1, 0), rcol;
            std::vector<float> rw;
            int fin_off = 0;
            for (size_t bi = 0; bi < h->bodies.size(); ++bi) {
                const CoarseLevel& C = h->bodies[bi].levels[l - 1];
                const int o = loff[bi];
                for (int J = 0; J < C.n; ++J) {
                    if (C.active[J]) {
                        diag0[o + J] = (float)C.A.diag[J];
                        for (int q = C.A.ptr[J]; q < C.A.ptr[J + 1]; ++q)
                            if (C.active[C.A.col[q]]) {
                                col.push_back(C.A.col[q] + o);
                                val.push_back(C.A.val[q]);
                            }
                    }
                    ptr[o + J + 1] = (int32_t)col.size();
                }
                const int nf = (int)(C.p_ids.size() / 4);
                for (int i = 0; i < nf; ++i) {
                    pid[fin_off + i] = make_int4(C.p_ids[4 * i] + o, C.p_ids[4 * i + 1] + o, C.p_ids[4 * i + 2] + o, C.p_ids[4 * i + 3] + o);
                    pw[fin_off + i] = make_float4((float)C.p_w[4 * i], (float)C.p_w[4 * i + 1], (float)C.p_w[4 * i + 2], (float)C.p_w[4 * i + 3]);
                }
                fin_off += nf;
            }
            // restriction CSR = transpose of the prolongation rows
            for (int i = 0; i < nfin; ++i) {
                const int ids[4] = {pid[i].x, pid[i].y, pid[i].z, pid[i].w};
                const float ws[4] = {pw[i].x, pw[i].y, pw[i].z, pw[i].w};
                for (int a = 0; a < 4; ++a)
                    if (ws[a] != 0.f) rptr[ids[a] + 1]++;
            }
            for (int J = 0; J < n; ++J) rptr[J + 1] += rptr[J];
            rcol.resize(rptr[n]);
            rw.resize(rptr[n]);
            {
                std::vector<int32_t> fill(rptr.begin(), rptr.end() - 1);
                for (int i = 0; i < nfin; ++i) {
                    const int ids[4] = {pid[i].x, pid[i].y, pid[i].z, pid[i].w};
                    const float ws[4] = {pw[i].x, pw[i].y, pw[i].z, pw[i].w};
                    for (int a = 0; a < 4; ++a)
                        if (ws[a] != 0.f) {
                            rcol[fill[ids[a]]] = i;
                            rw[fill[ids[a]]] = ws[a];
                            fill[ids[a]]++;
                        }
                }
            }
            std::vector<int32_t> sp, ec;
            std::vector<float> ev;
            build_ell(ptr, col, val, n, sp, ec, ev);
            ld.nnz = (int)col.size();
            TRY(dupload(h, pool, &ld.slice_ptr, sp));
            TRY(dupload(h, pool, &ld.ell_col, ec));
            TRY(dupload(h, pool, &ld.ell_val, ev));
            TRY(dupload(h, pool, &ld.diag0, diag0));
            TRY(dupload(h, pool, &ld.pid, pid));
            TRY(dupload(h, pool, &ld.pw, pw));
            TRY(dupload(h, pool, &ld.rptr, rptr));
            TRY(dupload(h, pool, &ld.rcol, rcol));
            TRY(dupload(h, pool, &ld.rw, rw));
            TRY(dalloc(h, pool, &ld.c, n));
            TRY(dalloc(h, pool, &ld.dfull, n));
            TRY(dalloc(h, pool, &ld.dinv, n));
            TRY(dalloc(h, pool, &ld.r, n));
            TRY(dalloc(h, pool, &ld.e, n));
            TRY(dalloc(h, pool, &ld.e2, n));
            TRY(dalloc(h, pool, &ld.res, n));
            CUDA_TRY(h, cudaMemset(ld.e, 0, n * sizeof(float4)));
            CUDA_TRY(h, cudaMemset(ld.e2, 0, n * sizeof(float4)));
            h->lev.push_back(ld);
        }
        // ---- coarsest dense blocks
        std::vector<float> dense;
        int maxn = 0;
        for (size_t bi = 0; bi < h->bodies.size(); ++bi) {
            const CoarseLevel& C = h->bodies[bi].levels[L - 2];
            std::vector<double> d;
            dense_from_sparse(C.A, C.active, d);
            BodyDev& BD = h->bodies_host[bi];
            BD.cl_off = loff[bi];
            BD.cl_n = C.n;
            BD.dense_off = (int)dense.size();
            for (double q : d) dense.push_back((float)q);
            maxn = std::max(maxn, C.n);
        }
        h->max_coarsest = maxn;
        h->factor_smem = ((size_t)maxn * maxn + maxn) * sizeof(float);
        int dev_smem = 0;
        CUDA_TRY(h, cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
        if (h->factor_smem > (size_t)dev_smem)
            return set_err(h, MGSB_NOT_SUPPORTED, "coarsest level has %d vertices; its dense factor needs %zu B of shared memory (max %d): add a level",
                           maxn, h->factor_smem, dev_smem);
        CUDA_TRY(h, cudaFuncSetAttribute(k_coarsest_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->factor_smem));
        TRY(dupload(h, pool, &h->A0dense, dense));
        TRY(dalloc(h, pool, &h->Lfac, dense.size()));
        TRY(dalloc(h, pool, &h->Ldinv, (size_t)h->lev[L - 1].n));
        TRY(dalloc(h, pool, &h->c_prev, (size_t)h->lev[L - 1].n));
        TRY(dalloc(h, pool, &h->fac_valid, h->bodies.size()));
        CUDA_TRY(h, cudaMemset(h->fac_valid, 0, h->bodies.size() * sizeof(int32_t)));
        // ---- surface vertices
        std::vector<int32_t> surf;
        for (const BodyHost& B : h->bodies)
            for (int i : B.surface) surf.push_back(i + B.v_off);
        h->nsurf = (int)surf.size();
        TRY(dupload(h, pool, &h->surf, surf));
    }
    for (size_t bi = 0; bi < h->bodies.size(); ++bi) {
        BodyDev& BD = h->bodies_host[bi];
        const BodyHost& B = h->bodies[bi];
        BD.v0_off = B.v_off;
        BD.v0_n = B.V;
    }
    h->dirty = false;
    return MGSB_OK;
}

// ---------------------------------------------------------------------------
// Frame enqueue
// ---------------------------------------------------------------------------
void prof_mark(mgsb_solver* h, const char* name) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, h->stream);
    h->prof_ev.push_back(e);
    if (name) h->prof_names.push_back(name);
}

#define LAUNCH(h, kernel, grid, block, smem, ...)                                  \
    do {                                                                             \
        if ((h)->profiling) prof_mark((h), #kernel);                                 \
        kernel<<<(grid), (block), (smem), (h)->stream>>>(__VA_ARGS__);              \
        if ((h)->profiling) prof_mark((h), nullptr);                                 \
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
               p.volume_stiffness);
        omega = 4 / (4 - p.cheb_rho * p.cheb_rho * omega);
        LAUNCH(h, k_ref_vertex, grid_for(n), kBlock, 0, n, h->x, h->prev, h->s, h->last, h->v, h->fixf, h->mass,
               h->vdiag, h->slot_ptr, h->slots, h->spheres_dev, p.collision_stiffness, p.dt, omega,
               (double)p.relaxation, it == p.iterations - 1 ? 1 : 0, h->cflag, h->cdepth, h->nonfinite);
    }
    if (p.iterations == 0) {
        // velocity only
        LAUNCH(h, k_velocity, grid_for(n), kBlock, 0, n, h->x, h->last, h->v, p.dt, h->nonfinite);
    }
}

void enqueue_mg_frame(mgsb_solver* h) {
    const mgsb_params& p = h->p;
    const int n0 = h->N0, T = h->T, L = p.levels;
    const int nb = (int)h->bodies.size();
    const float om = p.jacobi_omega;
    std::vector<LevelDev>& lv = h->lev;
    LAUNCH(h, k_mg_predict, grid_for(n0), kBlock, 0, n0, h->x, h->v, h->s, h->last, h->fixf, h->body_of, h->bodies_dev, p.dt);
    if (h->nsurf > 0)
        LAUNCH(h, k_contact_all, grid_for(h->nsurf), kBlock, 0, h->nsurf, h->surf, h->body_of, h->bodies_dev, h->s,
               h->fixf, p.contact_stiffness, h->cflag, h->c0, h->target);
    LAUNCH(h, k_l0_frame, grid_for(n0), kBlock, 0, n0, h->s, h->mass, h->c0, h->target, h->vdiag, h->fixf, om, h->b0,
           lv[0].dfull, lv[0].dinv);
    for (int l = 1; l < L; ++l)
        LAUNCH(h, k_coarse_frame, grid_for(lv[l].n), kBlock, 0, lv[l].n, lv[l].rptr, lv[l].rcol, lv[l].rw, lv[l - 1].c,
               lv[l].diag0, om, lv[l].c, lv[l].dfull, lv[l].dinv);
    LAUNCH(h, k_coarsest_factor, nb, 512, h->factor_smem, h->bodies_dev, h->A0dense, lv[L - 1].c, h->c_prev, h->Lfac,
           h->Ldinv, h->fac_valid);
    float4* xa = h->x;
    float4* xb = h->xb;
    for (int it = 0; it < p.iterations; ++it) {
        LAUNCH(h, k_mg_local, grid_for(T), kBlock, 0, T, h->tets, h->tA, h->tB, h->tC, xa, h->slot_of, h->slots);
        for (int pass = 0; pass < p.refinement_passes; ++pass) {
            // ---- level 0 pre-smoothing (the first sweep of the first pass assembles the RHS)
            bool gathered = pass > 0;
            for (int k = 0; k < p.pre_sweeps; ++k) {
                LAUNCH(h, k_l0_sweep, grid_for(n0), kBlock, 0, n0, lv[0].ell(), lv[0].dfull, lv[0].dinv, xa, xb, h->b,
                       h->b0, h->slot_ptr, h->slots, gathered ? 0 : 1);
                gathered = true;
                std::swap(xa, xb);
            }
            if (!gathered) LAUNCH(h, k_gather_rhs, grid_for(n0), kBlock, 0, n0, h->b, h->b0, h->slot_ptr, h->slots);
            LAUNCH(h, k_residual, grid_for(n0), kBlock, 0, n0, lv[0].ell(), lv[0].dfull, xa, h->b, lv[0].res);
            // ---- descend
            std::vector<float4*> ecur(L, nullptr), eoth(L, nullptr);
            for (int l = 1; l < L - 1; ++l) {
                LevelDev& C = lv[l];
                LAUNCH(h, k_restrict, grid_for(C.n), kBlock, 0, C.n, C.rptr, C.rcol, C.rw, lv[l - 1].res, C.dinv, C.r, C.e,
                       p.pre_sweeps > 0 ? 1 : 0);
                ecur[l] = C.e;
                eoth[l] = C.e2;
                for (int k = 1; k < p.pre_sweeps; ++k) {
                    LAUNCH(h, k_coarse_sweep, grid_for(C.n), kBlock, 0, C.n, C.ell(), C.dfull, C.dinv, C.r, ecur[l], eoth[l]);
                    std::swap(ecur[l], eoth[l]);
                }
                LAUNCH(h, k_residual, grid_for(C.n), kBlock, 0, C.n, C.ell(), C.dfull, ecur[l], C.r, C.res);
            }
            LAUNCH(h, k_coarsest_solve, nb, 256, (size_t)h->max_coarsest * sizeof(float4), h->bodies_dev, lv[L - 1].rptr,
                   lv[L - 1].rcol, lv[L - 1].rw, lv[L - 2].res, h->Lfac, h->Ldinv, lv[L - 1].e);
            ecur[L - 1] = lv[L - 1].e;
            // ---- ascend
            for (int l = L - 2; l >= 1; --l) {
                LevelDev& C = lv[l];
                LAUNCH(h, k_prolong, grid_for(C.n), kBlock, 0, C.n, lv[l + 1].pid, lv[l + 1].pw, ecur[l + 1], ecur[l]);
                for (int k = 0; k < p.post_sweeps; ++k) {
                    LAUNCH(h, k_coarse_sweep, grid_for(C.n), kBlock, 0, C.n, C.ell(), C.dfull, C.dinv, C.r, ecur[l], eoth[l]);
                    std::swap(ecur[l], eoth[l]);
                }
            }
            LAUNCH(h, k_prolong, grid_for(n0), kBlock, 0, n0, lv[1].pid, lv[1].pw, ecur[1], xa);
            for (int k = 0; k < p.post_sweeps; ++k) {
                LAUNCH(h, k_l0_sweep, grid_for(n0), kBlock, 0, n0, lv[0].ell(), lv[0].dfull, lv[0].dinv, xa, xb, h->b,
                       h->b0, h->slot_ptr, h->slots, 0);
                std::swap(xa, xb);
            }
        }
    }
    if (xa != h->x) {
        cudaMemcpyAsync(h->x, xa, n0 * sizeof(float4), cudaMemcpyDeviceToDevice, h->stream);
    }
    LAUNCH(h, k_velocity, grid_for(n0), kBlock, 0, n0, h->x, h->last, h->v, p.dt, h->nonfinite);
}

void enqueue_frame(mgsb_solver* h) {
    h->launches = 0;
    if (is_mg(h))
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
            enqueue_frame(h);
            cudaError_t e = cudaStreamEndCapture(h->stream, &h->graph);
            if (e != cudaSuccess) return set_err(h, MGSB_CUDA_ERROR, "graph capture failed: %s", cudaGetErrorString(e));
            CUDA_TRY(h, cudaGraphInstantiate(&h->graph_exec, h->graph, 0));
            h->graph_valid = true;
        }
        CUDA_TRY(h, cudaGraphLaunch(h->graph_exec, h->stream));
    } else {
        enqueue_frame(h);
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
        if (p.precision != MGSB_PRECISION_FP32)
            return set_err(h, MGSB_NOT_SUPPORTED, "precision %d not available in this build", p.precision);
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
        const mgsb_mesh& m = meshes[bi];
        if (m.num_verts <= 0 || m.num_tets <= 0 || !m.positions || !m.tets) return MGSB_INVALID_ARG;
        BodyHost& B = h->bodies[bi];
        B.V = m.num_verts;
        B.T = m.num_tets;
        B.v_off = voff;
        B.t_off = toff;
        voff += B.V;
        toff += B.T;
        B.rest.assign(3 * (size_t)B.V, 0.0);
        for (size_t q = 0; q < B.rest.size(); ++q) B.rest[q] = m.positions[q];
        B.tets.assign(m.tets, m.tets + 4 * (size_t)B.T);
        for (int32_t vv : B.tets)
            if (vv < 0 || vv >= B.V) return MGSB_INVALID_ARG;
        std::string e;
        if (!tet_rest(B.rest.data(), B.tets.data(), B.T, B.tr, e)) return MGSB_DEGENERATE_TET;
        const mgsb_params& pb = params[bi];
        B.youngs.assign(B.T, pb.youngs_modulus);
        B.poisson.assign(B.T, pb.poisson_ratio);
        B.fixed.assign(B.V, 0);
        for (int c = 0; c < 3; ++c) {
            B.grid_dims[c] = m.grid_dims[c];
            B.gravity[c] = pb.gravity[c];
        }
        B.damping = pb.damping;
        if (h->p.solver == MGSB_SOLVER_MULTIGRID) {
            std::vector<int32_t> tris, opp;
            extract_surface(B.tets.data(), B.T, tris, opp);
            std::vector<uint8_t> on(B.V, 0);
            for (int32_t q : tris) on[q] = 1;
            for (int i = 0; i < B.V; ++i)
                if (on[i]) B.surface.push_back(i);
        }
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
    TRY(dalloc(hp, pool, &h->x, N0));
    TRY(dalloc(hp, pool, &h->xb, N0));
    TRY(dalloc(hp, pool, &h->v, N0));
    TRY(dalloc(hp, pool, &h->s, N0));
    TRY(dalloc(hp, pool, &h->last, N0));
    TRY(dalloc(hp, pool, &h->prev, N0));
    TRY(dalloc(hp, pool, &h->cflag, N0));
    TRY(dalloc(hp, pool, &h->cdepth, N0));
    TRY(dalloc(hp, pool, &h->nonfinite, 1));
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
    CUDA_TRY(hp, cudaMemset(h->nonfinite, 0, sizeof(int32_t)));
    TRY(rebuild(hp));
    *out = h.release();
    return MGSB_OK;
}

template <typename F>
mgsb_status copy_body_f4(mgsb_solver* h, int32_t body, const float4* src, F&& sink) {
    TRY(check_body(h, body));
    const BodyHost& B = h->bodies[body];
    std::vector<float4> tmp(B.V);
    CUDA_TRY(h, cudaMemcpyAsync(tmp.data(), src + B.v_off, B.V * sizeof(float4), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    for (int i = 0; i < B.V; ++i) sink(i, tmp[i]);
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
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    free_pool(h->derived_mem);
    free_pool(h->state_mem);
    delete[] h->bodies_host;
    delete h->spheres_host;
    for (int k = 0; k < mgsb_solver::kStage; ++k) {
        if (h->stage[k]) cudaFreeHost(h->stage[k]);
        if (h->stage_ev[k]) cudaEventDestroy(h->stage_ev[k]);
    }
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->own_stream) cudaStreamDestroy(h->stream);
    delete h;
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
    TRY(sync_check(h));
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
    return copy_body_f4(h, body, h->v, [&](int i, float4 v) {
        out[3 * i] = v.x;
        out[3 * i + 1] = v.y;
        out[3 * i + 2] = v.z;
    });
}

mgsb_status mgsb_get_all_positions(mgsb_solver* h, float* out) {
    if (!h || !out) return MGSB_INVALID_ARG;
    TRY(sync_check(h));
    std::vector<float4> tmp(h->N0);
    CUDA_TRY(h, cudaMemcpy(tmp.data(), h->x, h->N0 * sizeof(float4), cudaMemcpyDeviceToHost));
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
    return set_err(h, MGSB_NOT_SUPPORTED, "FP64 positions exist only in mixed precision");
}

mgsb_status mgsb_get_contact_flags(mgsb_solver* h, int32_t body, int32_t* out) {
    if (!out) return MGSB_INVALID_ARG;
    TRY(check_body(h, body));
    TRY(sync_check(h));
    const BodyHost& B = h->bodies[body];
    CUDA_TRY(h, cudaMemcpy(out, h->cflag + B.v_off, B.V * sizeof(int32_t), cudaMemcpyDeviceToHost));
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
    // Surface normals from the current positions (host side for now).
    const BodyHost& B = h->bodies[body];
    std::vector<float> pos(3 * (size_t)B.V);
    TRY(mgsb_get_positions(h, body, pos.data()));
    std::vector<int32_t> tris, opp;
    extract_surface(B.tets.data(), B.T, tris, opp);
    std::vector<float> nrm(3 * (size_t)B.V, 0.f);
    for (size_t f = 0; f < tris.size() / 3; ++f) {
        const int a = tris[3 * f], b = tris[3 * f + 1], c = tris[3 * f + 2];
        const float ab[3] = {pos[3 * b] - pos[3 * a], pos[3 * b + 1] - pos[3 * a + 1], pos[3 * b + 2] - pos[3 * a + 2]};
        const float ac[3] = {pos[3 * c] - pos[3 * a], pos[3 * c + 1] - pos[3 * a + 1], pos[3 * c + 2] - pos[3 * a + 2]};
        float n[3] = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]};
        const float l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        for (int q = 0; q < 3; ++q) n[q] /= l;
        for (int v : {a, b, c})
            for (int q = 0; q < 3; ++q) nrm[3 * v + q] += n[q];
    }
    for (int i = 0; i < B.V; ++i) {
        const float l = std::sqrt(nrm[3 * i] * nrm[3 * i] + nrm[3 * i + 1] * nrm[3 * i + 1] + nrm[3 * i + 2] * nrm[3 * i + 2]);
        for (int q = 0; q < 3; ++q) out[3 * i + q] = l > 1.1920929e-07f ? nrm[3 * i + q] / l : nrm[3 * i + q];
    }
    return MGSB_OK;
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
    CUDA_TRY(h, cudaMemset(h->nonfinite, 0, sizeof(int32_t)));
    return MGSB_OK;
}

mgsb_status mgsb_get_energy(mgsb_solver* h, int32_t body, double out[5]) {
    if (!out) return MGSB_INVALID_ARG;
    TRY(check_body(h, body));
    return set_err(h, MGSB_NOT_SUPPORTED, "energy diagnostics not built yet");
}

mgsb_status mgsb_last_frame_ms(mgsb_solver* h, float* ms) {
    if (!h || !ms) return MGSB_INVALID_ARG;
    if (!h->timed) return set_err(h, MGSB_INVALID_ARG, "no frame has run");
    CUDA_TRY(h, cudaEventSynchronize(h->ev1));
    CUDA_TRY(h, cudaEventElapsedTime(ms, h->ev0, h->ev1));
    return MGSB_OK;
}

mgsb_status mgsb_profile_frame(mgsb_solver* h, int32_t cap, char* names, float* total_ms, int32_t* launches,
                               int32_t* count) {
    if (!h || !count || cap < 0 || (cap > 0 && (!names || !total_ms || !launches))) return MGSB_INVALID_ARG;
    TRY(ensure_ready(h));
    CUDA_TRY(h, cudaSetDevice(h->device));
    TRY(push_tool(h));
    h->profiling = true;
    h->prof_names.clear();
    h->prof_ev.clear();
    enqueue_frame(h);
    h->profiling = false;
    cudaError_t e = cudaStreamSynchronize(h->stream);
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
    if (e != cudaSuccess) return set_err(h, MGSB_CUDA_ERROR, "profiled frame failed: %s", cudaGetErrorString(e));
    *count = (int32_t)uniq.size();
    for (size_t u = 0; u < uniq.size() && (int32_t)u < cap; ++u) {
        std::snprintf(names + 48 * u, 48, "%s", uniq[u].c_str());
        total_ms[u] = tot[u];
        launches[u] = cnt[u];
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
