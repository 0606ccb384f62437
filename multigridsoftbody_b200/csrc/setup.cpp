// Host-side FP64 precompute and multigrid hierarchy construction.
#include "setup.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>

namespace mgsb {

double inverse3(const double A[9], double R[9]) {
    R[0] = A[4] * A[8] - A[7] * A[5];
    R[1] = A[7] * A[2] - A[1] * A[8];
    R[2] = A[1] * A[5] - A[4] * A[2];
    R[3] = A[5] * A[6] - A[3] * A[8];
    R[4] = A[0] * A[8] - A[2] * A[6];
    R[5] = A[2] * A[3] - A[0] * A[5];
    R[6] = A[3] * A[7] - A[4] * A[6];
    R[7] = A[1] * A[6] - A[0] * A[7];
    R[8] = A[0] * A[4] - A[1] * A[3];
    const double det = A[0] * R[0] + A[3] * R[1] + A[6] * R[2];
    const double inv_det = 1.0 / det;
    for (int i = 0; i < 9; ++i) R[i] *= inv_det;
    return det;
}

bool tet_rest(const double* pos, const int32_t* tets, int num_tets, std::vector<TetRest>& out, std::string& err) {
    out.resize(num_tets);
    for (int t = 0; t < num_tets; ++t) {
        const int32_t* v = tets + 4 * t;
        double D[9];
        double emax = 0.0;
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) {
                D[r * 3 + c] = pos[3 * v[c + 1] + r] - pos[3 * v[0] + r];
                emax = std::max(emax, std::fabs(D[r * 3 + c]));
            }
        TetRest& tr = out[t];
        tr.det = inverse3(D, tr.inv);
        if (!(std::fabs(tr.det) > 1e-12 * emax * emax * emax) || !std::isfinite(tr.det)) {
            char buf[128];
            std::snprintf(buf, sizeof buf, "degenerate tet %d (det %.3e)", t, tr.det);
            err = buf;
            return false;
        }
        tr.volume = std::fabs(tr.det) / 6.0;
        for (int k = 1; k < 4; ++k)
            for (int c = 0; c < 3; ++c) tr.g[k][c] = tr.inv[(k - 1) * 3 + c];
        for (int c = 0; c < 3; ++c) tr.g[0][c] = -(tr.g[1][c] + tr.g[2][c] + tr.g[3][c]);
    }
    return true;
}

static void vertex_adjacency(const int32_t* tets, int num_tets, int num_verts, std::vector<int32_t>& ptr,
                             std::vector<int32_t>& col) {
    std::vector<std::vector<int32_t>> nb(num_verts);
    for (int t = 0; t < num_tets; ++t)
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b)
                if (a != b) nb[tets[4 * t + a]].push_back(tets[4 * t + b]);
    ptr.assign(num_verts + 1, 0);
    col.clear();
    for (int i = 0; i < num_verts; ++i) {
        auto& v = nb[i];
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        col.insert(col.end(), v.begin(), v.end());
        ptr[i + 1] = (int32_t)col.size();
    }
}

void assemble_pd_matrix(const std::vector<TetRest>& rest, const int32_t* tets, int num_verts, const double* w,
                        const double* mass, double dt, SparseSym& L) {
    const int T = (int)rest.size();
    L.n = num_verts;
    vertex_adjacency(tets, T, num_verts, L.ptr, L.col);
    L.val.assign(L.col.size(), 0.0);
    L.diag.assign(num_verts, 0.0);
    const double inv_h2 = 1.0 / (dt * dt);
    for (int i = 0; i < num_verts; ++i) L.diag[i] = mass[i] * inv_h2;
    for (int t = 0; t < T; ++t) {
        const int32_t* v = tets + 4 * t;
        const TetRest& tr = rest[t];
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                const double gg = tr.g[a][0] * tr.g[b][0] + tr.g[a][1] * tr.g[b][1] + tr.g[a][2] * tr.g[b][2];
                const double c = w[t] * gg;
                if (a == b) {
                    L.diag[v[a]] += c;
                    continue;
                }
                const int32_t i = v[a], j = v[b];
                auto it = std::lower_bound(L.col.begin() + L.ptr[i], L.col.begin() + L.ptr[i + 1], j);
                L.val[it - L.col.begin()] += c;
            }
    }
}

void default_grid_dims(const double* pos, int num_verts, const int32_t* tets, int num_tets, int dims[3]) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < num_verts; ++i)
        for (int c = 0; c < 3; ++c) {
            lo[c] = std::min(lo[c], pos[3 * i + c]);
            hi[c] = std::max(hi[c], pos[3 * i + c]);
        }
    double sum = 0.0;
    long cnt = 0;
    static const int E[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    for (int t = 0; t < num_tets; ++t)
        for (auto& e : E) {
            const int a = tets[4 * t + e[0]], b = tets[4 * t + e[1]];
            double d2 = 0.0;
            for (int c = 0; c < 3; ++c) d2 += (pos[3 * a + c] - pos[3 * b + c]) * (pos[3 * a + c] - pos[3 * b + c]);
            sum += std::sqrt(d2);
            ++cnt;
        }
    const double h = cnt ? sum / cnt : 1.0;
    for (int c = 0; c < 3; ++c) dims[c] = std::max(1, (int)std::lround((hi[c] - lo[c]) / h));
}

void build_hierarchy(const double* pos, int num_verts, const SparseSym& A0, const uint8_t* fixed, int levels,
                     const int dims0[3], std::vector<CoarseLevel>& out) {
    out.clear();
    // prev_A points into `out`: reserve so emplace_back never reallocates.
    out.reserve(levels > 1 ? levels - 1 : 0);
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < num_verts; ++i)
        for (int c = 0; c < 3; ++c) {
            lo[c] = std::min(lo[c], pos[3 * i + c]);
            hi[c] = std::max(hi[c], pos[3 * i + c]);
        }
    std::vector<double> prev_pos(pos, pos + 3 * (size_t)num_verts);
    std::vector<uint8_t> prev_active(num_verts);
    for (int i = 0; i < num_verts; ++i) prev_active[i] = fixed ? (fixed[i] ? 0 : 1) : 1;
    const SparseSym* prev_A = &A0;
    int dims[3] = {dims0[0], dims0[1], dims0[2]};

    for (int lev = 1; lev < levels; ++lev) {
        out.emplace_back();
        CoarseLevel& L = out.back();
        for (int c = 0; c < 3; ++c) {
            dims[c] = std::max(1, (dims[c] + 1) / 2);
            L.dims[c] = dims[c];
        }
        double h[3];
        for (int c = 0; c < 3; ++c) h[c] = (hi[c] > lo[c]) ? (hi[c] - lo[c]) / dims[c] : 1.0;
        const int nprev = (int)(prev_pos.size() / 3);
        const int gx = dims[0] + 1, gz = dims[2] + 1;
        auto node = [&](int i, int j, int k) { return (size_t)i + (size_t)gx * ((size_t)k + (size_t)gz * j); };
        std::vector<uint8_t> kept((size_t)dims[0] * dims[1] * dims[2], 0);
        std::vector<int32_t> cell((size_t)3 * nprev);
        std::vector<double> u((size_t)3 * nprev);
        for (int i = 0; i < nprev; ++i) {
            int ci[3];
            for (int c = 0; c < 3; ++c) {
                const double s = (prev_pos[3 * i + c] - lo[c]) / h[c];
                int k = (int)std::floor(s);
                k = std::min(std::max(k, 0), dims[c] - 1);
                ci[c] = k;
                cell[3 * i + c] = k;
                u[3 * i + c] = std::min(1.0, std::max(0.0, s - k));
            }
            kept[(size_t)ci[0] + (size_t)dims[0] * ((size_t)ci[2] + (size_t)dims[2] * ci[1])] = 1;
        }
        std::vector<int32_t> remap((size_t)gx * (dims[1] + 1) * gz, -1);
        for (int j = 0; j < dims[1]; ++j)
            for (int k = 0; k < dims[2]; ++k)
                for (int i = 0; i < dims[0]; ++i) {
                    if (!kept[(size_t)i + (size_t)dims[0] * ((size_t)k + (size_t)dims[2] * j)]) continue;
                    for (int q = 0; q < 8; ++q) remap[node(i + (q & 1), j + ((q >> 1) & 1), k + ((q >> 2) & 1))] = 0;
                }
        int n = 0;
        for (int j = 0; j <= dims[1]; ++j)
            for (int k = 0; k <= dims[2]; ++k)
                for (int i = 0; i <= dims[0]; ++i) {
                    const size_t g = node(i, j, k);
                    if (remap[g] < 0) continue;
                    remap[g] = n++;
                    L.pos.push_back(lo[0] + h[0] * i);
                    L.pos.push_back(lo[1] + h[1] * j);
                    L.pos.push_back(lo[2] + h[2] * k);
                }
        L.n = n;
        // Prolongation rows (finer vertex -> 4 coarse corners of its Kuhn tet).
        L.p_ids.assign((size_t)4 * nprev, 0);
        L.p_w.assign((size_t)4 * nprev, 0.0);
        for (int i = 0; i < nprev; ++i) {
            const double* ui = &u[3 * i];
            int perm[3] = {0, 1, 2};
            // Axes by descending local coordinate; ties keep the lower axis first.
            std::stable_sort(perm, perm + 3, [&](int a, int b) { return ui[a] > ui[b]; });
            int c[3] = {0, 0, 0};
            int ids[4];
            const int* ci = &cell[3 * i];
            ids[0] = remap[node(ci[0], ci[1], ci[2])];
            for (int s = 0; s < 3; ++s) {
                c[perm[s]] = 1;
                ids[s + 1] = remap[node(ci[0] + c[0], ci[1] + c[1], ci[2] + c[2])];
            }
            double w[4] = {1.0 - ui[perm[0]], ui[perm[0]] - ui[perm[1]], ui[perm[1]] - ui[perm[2]], ui[perm[2]]};
            double sum = 0.0;
            for (int s = 0; s < 4; ++s) {
                if (w[s] < 1e-10) w[s] = 0.0;
                sum += w[s];
            }
            for (int s = 0; s < 4; ++s) {
                L.p_ids[4 * (size_t)i + s] = ids[s];
                L.p_w[4 * (size_t)i + s] = prev_active[i] ? w[s] / sum : 0.0;
            }
        }
        // Transpose of P (children of each coarse vertex).
        std::vector<int32_t> tptr(n + 1, 0), tcol;
        std::vector<double> tval;
        for (size_t e = 0; e < L.p_ids.size(); ++e)
            if (L.p_w[e] != 0.0) ++tptr[L.p_ids[e] + 1];
        for (int J = 0; J < n; ++J) tptr[J + 1] += tptr[J];
        tcol.resize(tptr[n]);
        tval.resize(tptr[n]);
        {
            std::vector<int32_t> fill(tptr.begin(), tptr.end() - 1);
            for (int i = 0; i < nprev; ++i)
                for (int s = 0; s < 4; ++s) {
                    const size_t e = 4 * (size_t)i + s;
                    if (L.p_w[e] == 0.0) continue;
                    const int J = L.p_ids[e];
                    tcol[fill[J]] = i;
                    tval[fill[J]] = L.p_w[e];
                    ++fill[J];
                }
        }
        L.active.assign(n, 0);
        for (int J = 0; J < n; ++J) L.active[J] = tptr[J + 1] > tptr[J] ? 1 : 0;
        // Galerkin product A_c = P^T A P, row by row with a dense accumulator.
        L.A.n = n;
        L.A.ptr.assign(n + 1, 0);
        L.A.diag.assign(n, 0.0);
        std::vector<double> acc(n, 0.0);
        std::vector<int32_t> mark(n, -1), touched;
        const SparseSym& A = *prev_A;
        for (int J = 0; J < n; ++J) {
            touched.clear();
            for (int e = tptr[J]; e < tptr[J + 1]; ++e) {
                const int i = tcol[e];
                const double pJ = tval[e];
                auto add_row = [&](int k, double a) {
                    for (int s = 0; s < 4; ++s) {
                        const double pK = L.p_w[4 * (size_t)k + s];
                        if (pK == 0.0) continue;
                        const int K = L.p_ids[4 * (size_t)k + s];
                        if (mark[K] != J) {
                            mark[K] = J;
                            acc[K] = 0.0;
                            touched.push_back(K);
                        }
                        acc[K] += pJ * a * pK;
                    }
                };
                add_row(i, A.diag[i]);
                for (int q = A.ptr[i]; q < A.ptr[i + 1]; ++q) add_row(A.col[q], A.val[q]);
            }
            std::sort(touched.begin(), touched.end());
            for (int K : touched) {
                if (K == J) {
                    L.A.diag[J] = acc[K];
                } else {
                    L.A.col.push_back(K);
                    L.A.val.push_back(acc[K]);
                }
            }
            L.A.ptr[J + 1] = (int32_t)L.A.col.size();
        }
        for (int J = 0; J < n; ++J)
            if (!(L.A.diag[J] > 0.0)) L.active[J] = 0;
        prev_pos = L.pos;
        prev_active = L.active;
        prev_A = &L.A;
    }
}

void dense_from_sparse(const SparseSym& A, const std::vector<uint8_t>& active, std::vector<double>& dense) {
    const int n = A.n;
    dense.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) {
        if (!active[i]) {
            dense[(size_t)i * n + i] = 1.0;
            continue;
        }
        dense[(size_t)i * n + i] = A.diag[i];
        for (int q = A.ptr[i]; q < A.ptr[i + 1]; ++q) {
            const int j = A.col[q];
            if (active[j]) dense[(size_t)i * n + j] = A.val[q];
        }
    }
}

bool spd_inverse(const std::vector<double>& A, int n, std::vector<double>& inv) {
    std::vector<double> Lm(A);   // lower triangle: L
    for (int j = 0; j < n; ++j) {
        double d = Lm[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) d -= Lm[(size_t)j * n + k] * Lm[(size_t)j * n + k];
        if (!(d > 0.0)) return false;
        d = std::sqrt(d);
        Lm[(size_t)j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double s = Lm[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) s -= Lm[(size_t)i * n + k] * Lm[(size_t)j * n + k];
            Lm[(size_t)i * n + j] = s / d;
        }
    }
    // X = L^-1 (lower), then A^-1 = X^T X
    std::vector<double> X((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        X[(size_t)j * n + j] = 1.0 / Lm[(size_t)j * n + j];
        for (int i = j + 1; i < n; ++i) {
            double s = 0.0;
            for (int k = j; k < i; ++k) s += Lm[(size_t)i * n + k] * X[(size_t)k * n + j];
            X[(size_t)i * n + j] = -s / Lm[(size_t)i * n + i];
        }
    }
    inv.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = 0.0;
            for (int k = i; k < n; ++k) s += X[(size_t)k * n + i] * X[(size_t)k * n + j];
            inv[(size_t)i * n + j] = inv[(size_t)j * n + i] = s;
        }
    return true;
}

}  // namespace mgsb
