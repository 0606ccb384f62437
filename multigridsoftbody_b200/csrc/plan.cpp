// Host-side plan of the solver's device arrays (no CUDA calls).
#include "plan.hpp"

#include <algorithm>
#include <cmath>

#include "mesh.hpp"

namespace mgsb {

mgsb_status make_body(const mgsb_mesh& m, const mgsb_params& p, bool multigrid, PlanBody& B, std::string& err) {
    if (m.num_verts <= 0 || m.num_tets <= 0 || !m.positions || !m.tets) {
        err = "empty or null mesh";
        return MGSB_INVALID_ARG;
    }
    B.V = m.num_verts;
    B.T = m.num_tets;
    B.rest.assign(3 * (size_t)B.V, 0.0);
    for (size_t q = 0; q < B.rest.size(); ++q) B.rest[q] = m.positions[q];
    B.tets.assign(m.tets, m.tets + 4 * (size_t)B.T);
    for (int32_t v : B.tets)
        if (v < 0 || v >= B.V) {
            err = "tet index out of range";
            return MGSB_INVALID_ARG;
        }
    if (!tet_rest(B.rest.data(), B.tets.data(), B.T, B.tr, err)) return MGSB_DEGENERATE_TET;
    B.youngs.assign(B.T, p.youngs_modulus);
    B.poisson.assign(B.T, p.poisson_ratio);
    B.fixed.assign(B.V, 0);
    for (int c = 0; c < 3; ++c) {
        B.grid_dims[c] = m.grid_dims[c];
        B.gravity[c] = p.gravity[c];
    }
    B.damping = p.damping;
    B.surface.clear();
    if (multigrid) {
        std::vector<int32_t> tris, opp;
        extract_surface(B.tets.data(), B.T, tris, opp);
        std::vector<uint8_t> on(B.V, 0);
        for (int32_t q : tris) on[q] = 1;
        for (int i = 0; i < B.V; ++i)
            if (on[i]) B.surface.push_back(i);
    }
    return MGSB_OK;
}

void build_ell(const std::vector<int32_t>& ptr, const std::vector<int32_t>& col, const std::vector<double>& val, int n,
               int S, std::vector<int32_t>& sptr, std::vector<int32_t>& ecol, std::vector<float>& eval,
               const std::vector<int32_t>* pad_col) {
    const int ns = (n + S - 1) / S;
    sptr.assign(ns + 1, 0);
    for (int s = 0; s < ns; ++s) {
        int w = 0;
        for (int r = s * S; r < std::min(n, s * S + S); ++r) w = std::max(w, ptr[r + 1] - ptr[r]);
        sptr[s + 1] = sptr[s] + S * w;
    }
    ecol.assign(sptr[ns], 0);
    eval.assign(sptr[ns], 0.f);
    for (int s = 0; s < ns; ++s) {
        const int w = (sptr[s + 1] - sptr[s]) / S;
        for (int lane = 0; lane < S; ++lane) {
            const int r = s * S + lane;
            for (int k = 0; k < w; ++k) {
                const int e = sptr[s] + k * S + lane;
                if (r < n && ptr[r] + k < ptr[r + 1]) {
                    ecol[e] = col[ptr[r] + k];
                    eval[e] = (float)val[ptr[r] + k];
                } else {
                    // padding: a zero coefficient on a valid column (the row itself by default)
                    ecol[e] = r < n ? (pad_col ? (*pad_col)[r] : r) : (pad_col ? (*pad_col)[n - 1] : 0);
                    eval[e] = 0.f;
                }
            }
        }
    }
}

bool build_plan(std::vector<PlanBody>& bodies, const mgsb_params& p, Plan& P, std::string& err) {
    const bool mg = p.solver == MGSB_SOLVER_MULTIGRID;
    P = Plan();
    int N0 = 0, T = 0;
    for (const PlanBody& B : bodies) {
        N0 += B.V;
        T += B.T;
    }
    P.N0 = N0;
    P.T = T;
    P.body_of.assign(N0, 0);
    P.fixf.assign(N0, 1.f);
    P.mass.assign(N0, 0.f);
    P.diag.assign(N0, 0.f);
    P.tets.assign(T, int4{0, 0, 0, 0});
    P.slot_of.assign(T, int4{0, 0, 0, 0});
    P.tA.assign(T, float4{0, 0, 0, 0});
    P.tB.assign(T, float4{0, 0, 0, 0});
    P.tC.assign(T, float2{0, 0});
    P.slot_ptr.assign(N0 + 1, 0);
    P.h_inv.assign(9 * (size_t)bodies[0].T, 0.f);
    P.h_ac.assign(12 * (size_t)bodies[0].T, 0.f);
    P.h_vol.assign(bodies[0].T, 0.f);
    P.h_mass.assign(bodies[0].V, 0.f);
    P.h_diag.assign(bodies[0].V, 0.f);

    const int L = mg ? p.levels : 1;
    std::vector<SparseSym> Lmat(bodies.size());
    for (size_t bi = 0; bi < bodies.size(); ++bi) {
        PlanBody& B = bodies[bi];
        const double dens = mg ? (double)p.density : 1.0;
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
                                            r.volume * (double)p.volume_stiffness;
            }
        }
        if (mg) {
            assemble_pd_matrix(B.tr, B.tets.data(), B.V, w.data(), m.data(), p.dt, Lmat[bi]);
            int dims[3] = {B.grid_dims[0], B.grid_dims[1], B.grid_dims[2]};
            if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0)
                default_grid_dims(B.rest.data(), B.V, B.tets.data(), B.T, dims);
            build_hierarchy(B.rest.data(), B.V, Lmat[bi], B.fixed.data(), L, dims, B.levels);
            if ((int)B.levels.size() != L - 1) {
                err = "hierarchy construction failed";
                return false;
            }
        }
        const double ih2 = 1.0 / ((double)p.dt * p.dt);
        for (int i = 0; i < B.V; ++i) {
            const int gi = B.v_off + i;
            P.body_of[gi] = (int32_t)bi;
            P.fixf[gi] = B.fixed[i] ? 0.f : 1.f;
            P.mass[gi] = mg ? (float)(m[i] * ih2) : (float)m[i];
            P.diag[gi] = mg ? (float)Lmat[bi].diag[i] : (float)vd[i];
        }
        for (int t = 0; t < B.T; ++t) {
            const TetRest& r = B.tr[t];
            const int gt = B.t_off + t;
            P.tets[gt] = int4{B.tets[4 * t] + B.v_off, B.tets[4 * t + 1] + B.v_off, B.tets[4 * t + 2] + B.v_off,
                              B.tets[4 * t + 3] + B.v_off};
            if (mg) {
                P.tA[gt] = float4{(float)r.g[1][0], (float)r.g[1][1], (float)r.g[1][2], (float)r.g[2][0]};
                P.tB[gt] = float4{(float)r.g[2][1], (float)r.g[2][2], (float)r.g[3][0], (float)r.g[3][1]};
                P.tC[gt] = float2{(float)r.g[3][2], (float)w[t]};
            } else {
                P.tA[gt] = float4{(float)r.inv[0], (float)r.inv[1], (float)r.inv[2], (float)r.inv[3]};
                P.tB[gt] = float4{(float)r.inv[4], (float)r.inv[5], (float)r.inv[6], (float)r.inv[7]};
                P.tC[gt] = float2{(float)r.inv[8], (float)r.volume};
            }
        }
        if (bi == 0) {
            for (int t = 0; t < B.T; ++t) {
                const TetRest& r = B.tr[t];
                for (int q = 0; q < 9; ++q) P.h_inv[9 * (size_t)t + q] = (float)r.inv[q];
                for (int rr = 0; rr < 3; ++rr)
                    for (int j = 0; j < 4; ++j) P.h_ac[12 * (size_t)t + rr * 4 + j] = (float)r.g[j][rr];
                P.h_vol[t] = (float)r.volume;
            }
            for (int i = 0; i < B.V; ++i) {
                P.h_mass[i] = (float)m[i];
                P.h_diag[i] = mg ? (float)Lmat[0].diag[i] : (float)vd[i];
            }
        }
    }
    // RHS slots: CSR by vertex, tets ascending within a vertex.
    for (int t = 0; t < T; ++t) {
        const int4 v = P.tets[t];
        P.slot_ptr[v.x + 1]++;
        P.slot_ptr[v.y + 1]++;
        P.slot_ptr[v.z + 1]++;
        P.slot_ptr[v.w + 1]++;
    }
    for (int i = 0; i < N0; ++i) P.slot_ptr[i + 1] += P.slot_ptr[i];
    {
        std::vector<int32_t> fill(P.slot_ptr.begin(), P.slot_ptr.end() - 1);
        for (int t = 0; t < T; ++t) {
            const int4 v = P.tets[t];
            P.slot_of[t] = int4{fill[v.x]++, fill[v.y]++, fill[v.z]++, fill[v.w]++};
        }
    }
    if (!mg) return true;

    // CSR of the off-diagonal part of the level built last, and the first row
    // of each body on it (for OP = Off * P of that level)
    std::vector<int32_t> prev_ptr, prev_col, prev_body;
    std::vector<double> prev_val;
    // ---- level 0 matrix (off-diagonal, global ids)
    {
        PlanLevel l0;
        l0.n = N0;
        std::vector<int32_t> ptr(N0 + 1, 0), col;
        std::vector<double> val;
        for (size_t bi = 0; bi < bodies.size(); ++bi) {
            const PlanBody& B = bodies[bi];
            const SparseSym& A = Lmat[bi];
            for (int i = 0; i < B.V; ++i) {
                for (int q = A.ptr[i]; q < A.ptr[i + 1]; ++q) {
                    col.push_back(A.col[q] + B.v_off);
                    val.push_back(A.val[q]);
                }
                ptr[B.v_off + i + 1] = (int32_t)col.size();
            }
        }
        l0.S = kSliceL0;
        build_ell(ptr, col, val, N0, l0.S, l0.slice_ptr, l0.ell_col, l0.ell_val);
        {
            // FP64 values in the same sliced-ELL positions
            l0.ell_val64.assign(l0.ell_val.size(), 0.0);
            const int S = l0.S;
            for (int r = 0; r < N0; ++r) {
                const int sl = r / S, ln = r % S;
                for (int k = 0; k < ptr[r + 1] - ptr[r]; ++k) l0.ell_val64[l0.slice_ptr[sl] + k * S + ln] = val[ptr[r] + k];
            }
            P.diag64.assign(N0, 0.0);
            for (size_t bi = 0; bi < bodies.size(); ++bi)
                for (int i = 0; i < bodies[bi].V; ++i) P.diag64[bodies[bi].v_off + i] = Lmat[bi].diag[i];
        }
        l0.nnz = (int)col.size();
        l0.diag0 = P.diag;
        P.levels.push_back(std::move(l0));
        prev_ptr = std::move(ptr);
        prev_col = std::move(col);
        prev_val = std::move(val);
        prev_body = P.body_of;
    }
    // ---- coarse levels
    std::vector<int> loff(bodies.size(), 0);
    for (int l = 1; l < L; ++l) {
        PlanLevel ld;
        int n = 0;
        for (size_t bi = 0; bi < bodies.size(); ++bi) {
            loff[bi] = n;
            n += bodies[bi].levels[l - 1].n;
        }
        ld.n = n;
        const int nfin = P.levels[l - 1].n;
        std::vector<int32_t> ptr(n + 1, 0), col;
        std::vector<double> val;
        ld.diag0.assign(n, 0.f);
        ld.pid.assign(nfin, int4{0, 0, 0, 0});
        ld.pw.assign(nfin, float4{0, 0, 0, 0});
        int fin_off = 0;
        for (size_t bi = 0; bi < bodies.size(); ++bi) {
            const CoarseLevel& C = bodies[bi].levels[l - 1];
            const int o = loff[bi];
            for (int J = 0; J < C.n; ++J) {
                if (C.active[J]) {
                    ld.diag0[o + J] = (float)C.A.diag[J];
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
                ld.pid[fin_off + i] = int4{C.p_ids[4 * i] + o, C.p_ids[4 * i + 1] + o, C.p_ids[4 * i + 2] + o,
                                           C.p_ids[4 * i + 3] + o};
                ld.pw[fin_off + i] = float4{(float)C.p_w[4 * i], (float)C.p_w[4 * i + 1], (float)C.p_w[4 * i + 2],
                                            (float)C.p_w[4 * i + 3]};
            }
            fin_off += nf;
        }
        if (fin_off != nfin) {
            err = "prolongation row count mismatch";
            return false;
        }
        ld.rptr.assign(n + 1, 0);
        for (int i = 0; i < nfin; ++i) {
            const int ids[4] = {ld.pid[i].x, ld.pid[i].y, ld.pid[i].z, ld.pid[i].w};
            const float ws[4] = {ld.pw[i].x, ld.pw[i].y, ld.pw[i].z, ld.pw[i].w};
            for (int a = 0; a < 4; ++a)
                if (ws[a] != 0.f) ld.rptr[ids[a] + 1]++;
        }
        for (int J = 0; J < n; ++J) ld.rptr[J + 1] += ld.rptr[J];
        ld.rcol.assign(ld.rptr[n], 0);
        ld.rw.assign(ld.rptr[n], 0.f);
        {
            std::vector<int32_t> fill(ld.rptr.begin(), ld.rptr.end() - 1);
            for (int i = 0; i < nfin; ++i) {
                const int ids[4] = {ld.pid[i].x, ld.pid[i].y, ld.pid[i].z, ld.pid[i].w};
                const float ws[4] = {ld.pw[i].x, ld.pw[i].y, ld.pw[i].z, ld.pw[i].w};
                for (int a = 0; a < 4; ++a)
                    if (ws[a] != 0.f) {
                        ld.rcol[fill[ids[a]]] = i;
                        ld.rw[fill[ids[a]]] = ws[a];
                        fill[ids[a]]++;
                    }
            }
        }
        if (l == 1) {
            // RO = R * Off(level 0): row I = sum over its children i (weight w_Ii) of w_Ii * (row i of
            // the level-0 off-diagonal), accumulated in FP64, columns ascending
            ld.ro_ptr.assign(n + 1, 0);
            std::vector<double> acc(nfin, 0.0);
            std::vector<uint8_t> mark(nfin, 0);
            std::vector<int32_t> touched;
            for (int I = 0; I < n; ++I) {
                touched.clear();
                for (int q = ld.rptr[I]; q < ld.rptr[I + 1]; ++q) {
                    const int i = ld.rcol[q];
                    const double w = (double)ld.rw[q];
                    for (int e = prev_ptr[i]; e < prev_ptr[i + 1]; ++e) {
                        const int k = prev_col[e];
                        if (!mark[k]) {
                            mark[k] = 1;
                            touched.push_back(k);
                        }
                        acc[k] += w * prev_val[e];
                    }
                }
                std::sort(touched.begin(), touched.end());
                for (int k : touched) {
                    ld.ro_col.push_back(k);
                    ld.ro_val.push_back((float)acc[k]);
                    acc[k] = 0.0;
                    mark[k] = 0;
                }
                ld.ro_ptr[I + 1] = (int32_t)ld.ro_col.size();
            }
        }
        ld.S = kSliceCoarse;
        build_ell(ptr, col, val, n, ld.S, ld.slice_ptr, ld.ell_col, ld.ell_val);
        ld.nnz = (int)col.size();
        {
            // OP of the finer level: row i = sum over its neighbours j of a_ij * (prolongation row j),
            // accumulated in FP64 (weights as stored), columns ascending; padding on the body's
            // first row of this level; every column checked to lie in the row's body
            PlanLevel& fl = P.levels[l - 1];
            std::vector<int32_t> optr(nfin + 1, 0), ocol, pad(nfin, 0);
            std::vector<double> oval, acc(n, 0.0);
            std::vector<uint8_t> mark(n, 0);
            std::vector<int32_t> touched;
            for (int i = 0; i < nfin; ++i) {
                touched.clear();
                for (int q = prev_ptr[i]; q < prev_ptr[i + 1]; ++q) {
                    const int j = prev_col[q];
                    const int ids[4] = {ld.pid[j].x, ld.pid[j].y, ld.pid[j].z, ld.pid[j].w};
                    const float ws[4] = {ld.pw[j].x, ld.pw[j].y, ld.pw[j].z, ld.pw[j].w};
                    for (int a = 0; a < 4; ++a) {
                        if (ws[a] == 0.f) continue;
                        const int c = ids[a];
                        if (!mark[c]) {
                            mark[c] = 1;
                            touched.push_back(c);
                        }
                        acc[c] += prev_val[q] * (double)ws[a];
                    }
                }
                std::sort(touched.begin(), touched.end());
                for (int c : touched) {
                    ocol.push_back(c);
                    oval.push_back(acc[c]);
                    acc[c] = 0.0;
                    mark[c] = 0;
                }
                optr[i + 1] = (int32_t)ocol.size();
                pad[i] = loff[prev_body[i]];
            }
            build_ell(optr, ocol, oval, nfin, fl.S, fl.op_slice_ptr, fl.op_col, fl.op_val, &pad);
            std::vector<int32_t> body_of_level(n, 0);
            for (size_t bi = 0; bi < bodies.size(); ++bi)
                for (int J = loff[bi]; J < loff[bi] + bodies[bi].levels[l - 1].n; ++J) body_of_level[J] = (int32_t)bi;
            const int fS = fl.S;
            for (int sl = 0; sl + 1 < (int)fl.op_slice_ptr.size(); ++sl)
                for (int e = fl.op_slice_ptr[sl]; e < fl.op_slice_ptr[sl + 1]; ++e) {
                    const int i = sl * fS + (e - fl.op_slice_ptr[sl]) % fS;
                    if (i < nfin && body_of_level[fl.op_col[e]] != prev_body[i]) {
                        err = "prolonged operator column outside its body (level " + std::to_string(l - 1) + ")";
                        return false;
                    }
                }
            fl.op_nnz = (int)ocol.size();
            prev_body = body_of_level;
        }
        P.levels.push_back(std::move(ld));
        prev_ptr = std::move(ptr);
        prev_col = std::move(col);
        prev_val = std::move(val);
    }
    // ---- per-body row ranges on every level
    P.range.assign(bodies.size() * L, int2{0, 0});
    for (size_t bi = 0; bi < bodies.size(); ++bi) P.range[bi * L] = int2{bodies[bi].v_off, bodies[bi].V};
    for (int l = 1; l < L; ++l) {
        int o = 0;
        for (size_t bi = 0; bi < bodies.size(); ++bi) {
            P.range[bi * L + l] = int2{o, bodies[bi].levels[l - 1].n};
            o += bodies[bi].levels[l - 1].n;
        }
    }
    // ---- coarsest dense blocks
    P.cl_off = loff;
    P.cl_n.assign(bodies.size(), 0);
    P.dense_off.assign(bodies.size(), 0);
    for (size_t bi = 0; bi < bodies.size(); ++bi) {
        const CoarseLevel& C = bodies[bi].levels[L - 2];
        std::vector<double> d;
        dense_from_sparse(C.A, C.active, d);
        P.cl_n[bi] = C.n;
        P.dense_off[bi] = (int32_t)P.dense.size();
        for (double q : d) {
            P.dense.push_back((float)q);
            P.dense64.push_back(q);
        }
        std::vector<double> inv;
        if (!spd_inverse(d, C.n, inv)) {
            err = "coarsest-level matrix of body " + std::to_string(bi) + " is not positive definite";
            return false;
        }
        for (double q : inv) {
            P.dense_inv.push_back((float)q);
            P.dense_inv64.push_back(q);
        }
        P.max_coarsest = std::max(P.max_coarsest, C.n);
    }
    // ---- surface vertices
    P.is_surf.assign(N0, 0);
    for (const PlanBody& B : bodies)
        for (int i : B.surface) {
            P.surf.push_back(i + B.v_off);
            P.is_surf[i + B.v_off] = 1;
        }
    return true;
}

}  // namespace mgsb
