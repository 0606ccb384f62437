// FP64 CPU oracle — TEST INFRASTRUCTURE ONLY (the checker for the CUDA path).
// See mgsb_oracle.h for the reference file:line each part restates.
#include "mgsb_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::array<double, 3> V3;

// ---------------------------------------------------------------------------
// 3x3 helpers
// ---------------------------------------------------------------------------

// Adjugate / determinant inverse, element layout of Matrix_Inverse_3
// (utils.cu:233-252).
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
    double det = A[0] * R[0] + A[3] * R[1] + A[6] * R[2];
    for (int i = 0; i < 9; ++i) R[i] /= det;
    return det;
}

// Polar rotation by the invariant / Cayley-Hamilton method of GetRotation_D
// (utils.cu:123-226), in FP64, with the same thresholds and failure branches
// (R = I on failure, F/sqrt(I_c/3) when the invariant k vanishes).
void ref_rotation(const double F[9], double R[9]) {
    for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
    double C[9] = {0}, C2[9] = {0};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) C[i * 3 + j] += F[k * 3 + i] * F[k * 3 + j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) C2[i * 3 + j] += C[i * 3 + k] * C[j * 3 + k];
    const double det = F[0] * F[4] * F[8] + F[1] * F[5] * F[6] + F[3] * F[7] * F[2] - F[2] * F[4] * F[6] -
                       F[1] * F[3] * F[8] - F[0] * F[5] * F[7];
    const double I_c = C[0] + C[4] + C[8];
    const double I_c2 = I_c * I_c;
    const double II_c = 0.5 * (I_c2 - C2[0] - C2[4] - C2[8]);
    const double III_c = det * det;
    const double k = I_c2 - 3 * II_c;
    double invU[9] = {0};
    if (k < 1e-6) {
        if (I_c < 1e-6) return;
        const double il = 1.0 / std::sqrt(I_c / 3.0);
        invU[0] = invU[4] = invU[8] = il;
    } else {
        const double l = I_c * (I_c * I_c - 4.5 * II_c) + 13.5 * III_c;
        const double kr = std::sqrt(k);
        double value = l / (k * kr);
        value = std::min(1.0, std::max(-1.0, value));
        const double phi = std::acos(value);
        const double lambda2 = (I_c + 2 * kr * std::cos(phi / 3)) / 3.0;
        const double lambda = std::sqrt(lambda2);
        const double III_u = det;  // sign(det) * sqrt(III_c)
        if (std::fabs(lambda) < 1e-6) return;
        if (-lambda2 + I_c + 2 * III_u / lambda < 1e-6) return;
        const double I_u = lambda + std::sqrt(-lambda2 + I_c + 2 * III_u / lambda);
        const double II_u = (I_u * I_u - I_c) * 0.5;
        if (std::fabs(I_u * II_u - III_u) < 1e-6) return;
        double inv_rate = 1.0 / (I_u * II_u - III_u);
        double U[9];
        const double f0 = I_u * III_u * inv_rate;
        const double f1 = (I_u * I_u - II_u) * inv_rate;
        for (int i = 0; i < 9; ++i) U[i] = f1 * C[i] - inv_rate * C2[i] + ((i % 4 == 0) ? f0 : 0.0);
        if (std::fabs(III_u) < 1e-6) return;
        inv_rate = 1.0 / III_u;
        const double g0 = II_u * inv_rate;
        const double g1 = -I_u * inv_rate;
        for (int i = 0; i < 9; ++i) invU[i] = g1 * U[i] + inv_rate * C[i] + ((i % 4 == 0) ? g0 : 0.0);
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k2 = 0; k2 < 3; ++k2) s += F[i * 3 + k2] * invU[k2 * 3 + j];
            R[i * 3 + j] = s;
        }
}

// Closest rotation via the rotation-variant SVD (U, V proper rotations):
// symmetric eigen-decomposition of F^T F by cyclic Jacobi iterated to
// convergence, eigenvalues sorted descending (column swaps keep det V = +1),
// u1 = F v1 / |F v1|, u2 = Gram-Schmidt(F v2), u3 = u1 x u2, R = U V^T.
void svd_rotation(const double F[9], double R[9]) {
    double S[9];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) S[a * 3 + b] = F[a] * F[b] + F[3 + a] * F[3 + b] + F[6 + a] * F[6 + b];
    double V[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    for (int sweep = 0; sweep < 50; ++sweep) {
        const double off = S[1] * S[1] + S[2] * S[2] + S[5] * S[5];
        const double dia = S[0] * S[0] + S[4] * S[4] + S[8] * S[8];
        if (off <= 1e-34 * dia || off == 0.0) break;
        for (auto& pq : pairs) {
            const int p = pq[0], q = pq[1], r = 3 - p - q;
            const double apq = S[p * 3 + q];
            if (apq == 0.0) continue;
            const double theta = (S[q * 3 + q] - S[p * 3 + p]) / (2 * apq);
            const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
            const double c = 1 / std::sqrt(t * t + 1), s = t * c;
            const double app = S[p * 3 + p], aqq = S[q * 3 + q], arp = S[r * 3 + p], arq = S[r * 3 + q];
            S[p * 3 + p] = app - t * apq;
            S[q * 3 + q] = aqq + t * apq;
            S[p * 3 + q] = S[q * 3 + p] = 0;
            S[r * 3 + p] = S[p * 3 + r] = c * arp - s * arq;
            S[r * 3 + q] = S[q * 3 + r] = s * arp + c * arq;
            for (int i = 0; i < 3; ++i) {
                const double vp = V[i * 3 + p], vq = V[i * 3 + q];
                V[i * 3 + p] = c * vp - s * vq;
                V[i * 3 + q] = s * vp + c * vq;
            }
        }
    }
    double lam[3] = {S[0], S[4], S[8]};
    auto swp = [&](int a, int b) {
        std::swap(lam[a], lam[b]);
        for (int i = 0; i < 3; ++i) {
            const double t = V[i * 3 + a];
            V[i * 3 + a] = V[i * 3 + b];
            V[i * 3 + b] = -t;
        }
    };
    if (lam[0] < lam[1]) swp(0, 1);
    if (lam[0] < lam[2]) swp(0, 2);
    if (lam[1] < lam[2]) swp(1, 2);
    double b1[3], b2[3];
    for (int i = 0; i < 3; ++i) {
        b1[i] = F[i * 3] * V[0] + F[i * 3 + 1] * V[3] + F[i * 3 + 2] * V[6];
        b2[i] = F[i * 3] * V[1] + F[i * 3 + 1] * V[4] + F[i * 3 + 2] * V[7];
    }
    const double n1 = b1[0] * b1[0] + b1[1] * b1[1] + b1[2] * b1[2];
    if (!(n1 > 1e-300)) {
        for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
        return;
    }
    const double r1 = 1 / std::sqrt(n1);
    double u1[3] = {b1[0] * r1, b1[1] * r1, b1[2] * r1};
    const double d = u1[0] * b2[0] + u1[1] * b2[1] + u1[2] * b2[2];
    double u2[3] = {b2[0] - d * u1[0], b2[1] - d * u1[1], b2[2] - d * u1[2]};
    double n2 = u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2];
    if (!(n2 > 1e-24 * n1)) {
        const double ax = std::fabs(u1[0]), ay = std::fabs(u1[1]), az = std::fabs(u1[2]);
        double e[3] = {0, 0, 0};
        if (ax <= ay && ax <= az) e[0] = 1; else if (ay <= az) e[1] = 1; else e[2] = 1;
        const double de = u1[0] * e[0] + u1[1] * e[1] + u1[2] * e[2];
        for (int i = 0; i < 3; ++i) u2[i] = e[i] - de * u1[i];
        n2 = u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2];
    }
    const double r2 = 1 / std::sqrt(n2);
    for (int i = 0; i < 3; ++i) u2[i] *= r2;
    const double u3[3] = {u1[1] * u2[2] - u1[2] * u2[1], u1[2] * u2[0] - u1[0] * u2[2], u1[0] * u2[1] - u1[1] * u2[0]};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[i * 3 + j] = u1[i] * V[j * 3] + u2[i] * V[j * 3 + 1] + u3[i] * V[j * 3 + 2];
}

// ---------------------------------------------------------------------------
// Multigrid level of the oracle (independent of the product's setup code).
// ---------------------------------------------------------------------------
struct Row {
    std::vector<int> col;
    std::vector<double> val;
};

struct OLevel {
    int n = 0;
    std::vector<double> diag;          // Galerkin diagonal (no contact)
    std::vector<Row> off;              // off-diagonal entries
    std::vector<char> active;
    std::vector<std::array<int, 4>> pid;     // prolongation rows, indexed by finer vertex
    std::vector<std::array<double, 4>> pw;
    std::vector<double> c;             // lumped contact weight this frame
    std::vector<double> chol;          // coarsest only: dense Cholesky factor (row-major lower)
};

struct Sphere {
    V3 c;
    double r;
    bool active;
};

struct Oracle {
    mgsb_params p;
    // coarse level of the two-level schedule: sphere collision against the
    // surface triangles (DCDByTriangle) instead of per vertex (DCDByPoint)
    bool tri_dcd = false;
    std::vector<int32_t> surf_tris;
    // local step of PDSolver::Step (getTetFRV2 + calTetIFV1) drops |c| < 1e-5;
    // calculateIF, used by the two-level schedule (PDSolver.cu:128-183), does not
    bool drop_small = true;
    int V = 0, T = 0;
    std::vector<double> rest;
    std::vector<int> tets;
    std::vector<double> youngs, poisson;
    std::vector<uint8_t> fixed;
    std::vector<int> grid_hint;
    // precompute
    std::vector<double> inv, ac, vol, mass, diag;   // diag = reference volDiag (ref mode)
    std::vector<double> w;                          // multigrid: 2 mu V
    // state
    std::vector<V3> x, v, s, last, prev, fext;
    std::vector<int> collided;
    std::vector<double> depth, cenergy;
    std::vector<Sphere> spheres;
    // multigrid
    bool have_capsule = false;
    V3 cap_a{}, cap_b{};
    double cap_r = 0;
    std::vector<int> surface_verts;
    // capsule against the surface triangles too (mgsb_set_surface_contact):
    // per surface triangle its three vertices and the fourth vertex of its tet
    bool tri_contact = false;
    std::vector<std::array<int, 4>> cap_tris;
    std::vector<double> c0;      // contact weight per vertex
    std::vector<V3> target;
    std::vector<double> Ldiag;   // L diagonal at level 0
    std::vector<Row> Loff;
    std::vector<OLevel> lev;     // lev[0] unused (level 0 handled via L)
    double last_residual = 0;
    bool hierarchy_dirty = true;
};

// ---------------------------------------------------------------------------
// Setup
// ---------------------------------------------------------------------------
bool precompute(Oracle& o, std::string& err) {
    const bool ref = o.p.solver == MGSB_SOLVER_REFERENCE_JACOBI;
    o.inv.assign(9 * (size_t)o.T, 0);
    o.ac.assign(12 * (size_t)o.T, 0);
    o.vol.assign(o.T, 0);
    o.mass.assign(o.V, 0);
    o.diag.assign(o.V, 0);
    for (int t = 0; t < o.T; ++t) {
        const int* id = &o.tets[4 * t];
        double D[9];
        // D[r*3+c] = (x_{c+1} - x_0)_r   (PDSolver.cpp:28-36)
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) D[r * 3 + c] = o.rest[3 * id[c + 1] + r] - o.rest[3 * id[0] + r];
        double* iv = &o.inv[9 * (size_t)t];
        const double det = inverse3(D, iv);
        if (!(std::fabs(det) > 0) || !std::isfinite(det)) {
            err = "degenerate tet " + std::to_string(t);
            return false;
        }
        o.vol[t] = std::fabs(det) / 6.0;
        const double dens = ref ? 1.0 : (double)o.p.density;
        for (int a = 0; a < 4; ++a) o.mass[id[a]] += dens * o.vol[t] / 4;
        double* A = &o.ac[12 * (size_t)t];
        // Ac rows r: [-sum_m inv[m][r], inv[0][r], inv[1][r], inv[2][r]]  (PDSolver.cpp:53-64)
        for (int r = 0; r < 3; ++r) {
            A[r * 4 + 0] = -iv[r] - iv[r + 3] - iv[r + 6];
            A[r * 4 + 1] = iv[r];
            A[r * 4 + 2] = iv[r + 3];
            A[r * 4 + 3] = iv[r + 6];
        }
        if (ref)
            for (int j = 0; j < 4; ++j)
                for (int r = 0; r < 3; ++r) o.diag[id[j]] += A[r * 4 + j] * A[r * 4 + j] * o.vol[t] * o.p.volume_stiffness;
    }
    return true;
}

void build_surface(Oracle& o) {
    std::map<std::array<int, 3>, int> cnt;
    std::map<std::array<int, 3>, std::array<int, 4>> face_of;   // a face and the tet vertex opposite it
    for (int t = 0; t < o.T; ++t) {
        const int* v = &o.tets[4 * t];
        const int f[4][4] = {{v[0], v[2], v[1], v[3]}, {v[0], v[1], v[3], v[2]}, {v[0], v[3], v[2], v[1]},
                             {v[1], v[2], v[3], v[0]}};
        for (auto& ff : f) {
            std::array<int, 3> k = {ff[0], ff[1], ff[2]};
            std::sort(k.begin(), k.end());
            cnt[k]++;
            face_of[k] = {ff[0], ff[1], ff[2], ff[3]};
        }
    }
    o.cap_tris.clear();
    for (auto& kv : cnt)
        if (kv.second == 1) o.cap_tris.push_back(face_of[kv.first]);
    std::vector<char> on(o.V, 0);
    o.surf_tris.clear();
    for (auto& kv : cnt)
        if (kv.second == 1) {
            for (int a : kv.first) on[a] = 1;
            for (int a : kv.first) o.surf_tris.push_back(a);
        }
    o.surface_verts.clear();
    for (int i = 0; i < o.V; ++i)
        if (on[i]) o.surface_verts.push_back(i);
}

void assemble_L(Oracle& o) {
    o.w.assign(o.T, 0);
    for (int t = 0; t < o.T; ++t) {
        const double mu = o.youngs[t] / (2.0 * (1.0 + o.poisson[t]));
        o.w[t] = 2.0 * mu * o.vol[t];
    }
    std::vector<std::map<int, double>> rows(o.V);
    const double ih2 = 1.0 / ((double)o.p.dt * (double)o.p.dt);
    o.Ldiag.assign(o.V, 0);
    for (int i = 0; i < o.V; ++i) o.Ldiag[i] = o.mass[i] * ih2;
    for (int t = 0; t < o.T; ++t) {
        const int* id = &o.tets[4 * t];
        const double* A = &o.ac[12 * (size_t)t];
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                const double gg = A[a] * A[b] + A[4 + a] * A[4 + b] + A[8 + a] * A[8 + b];
                if (a == b)
                    o.Ldiag[id[a]] += o.w[t] * gg;
                else
                    rows[id[a]][id[b]] += o.w[t] * gg;
            }
    }
    o.Loff.assign(o.V, Row());
    for (int i = 0; i < o.V; ++i)
        for (auto& kv : rows[i]) {
            o.Loff[i].col.push_back(kv.first);
            o.Loff[i].val.push_back(kv.second);
        }
}

// Coarse voxel grids by ceil-halving, Kuhn interpolation, Galerkin operators.
void build_levels(Oracle& o) {
    const int L = o.p.levels;
    o.lev.assign(L, OLevel());
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < o.V; ++i)
        for (int c = 0; c < 3; ++c) {
            lo[c] = std::min(lo[c], o.rest[3 * i + c]);
            hi[c] = std::max(hi[c], o.rest[3 * i + c]);
        }
    int dims[3] = {o.grid_hint[0], o.grid_hint[1], o.grid_hint[2]};
    std::vector<V3> fpos(o.V);
    for (int i = 0; i < o.V; ++i) fpos[i] = {o.rest[3 * i], o.rest[3 * i + 1], o.rest[3 * i + 2]};
    std::vector<char> factive(o.V);
    for (int i = 0; i < o.V; ++i) factive[i] = o.fixed[i] ? 0 : 1;
    o.lev[0].n = o.V;
    o.lev[0].active = factive;
    for (int l = 1; l < L; ++l) {
        OLevel& C = o.lev[l];
        double h[3];
        for (int c = 0; c < 3; ++c) {
            dims[c] = std::max(1, (dims[c] + 1) / 2);
            h[c] = hi[c] > lo[c] ? (hi[c] - lo[c]) / dims[c] : 1.0;
        }
        const int nf = (int)fpos.size();
        std::map<std::array<int, 3>, int> nodes;  // (j, k, i) ordering key -> id
        std::vector<std::array<int, 3>> fcell(nf);
        std::vector<V3> fu(nf);
        std::vector<char> kept((size_t)dims[0] * dims[1] * dims[2], 0);
        for (int i = 0; i < nf; ++i) {
            for (int c = 0; c < 3; ++c) {
                const double sc = (fpos[i][c] - lo[c]) / h[c];
                int k = (int)std::floor(sc);
                if (k < 0) k = 0;
                if (k > dims[c] - 1) k = dims[c] - 1;
                fcell[i][c] = k;
                double u = sc - k;
                fu[i][c] = u < 0 ? 0 : (u > 1 ? 1 : u);
            }
            kept[fcell[i][0] + (size_t)dims[0] * (fcell[i][2] + (size_t)dims[2] * fcell[i][1])] = 1;
        }
        for (int j = 0; j < dims[1]; ++j)
            for (int k = 0; k < dims[2]; ++k)
                for (int i = 0; i < dims[0]; ++i)
                    if (kept[i + (size_t)dims[0] * (k + (size_t)dims[2] * j)])
                        for (int q = 0; q < 8; ++q) nodes[{j + ((q >> 1) & 1), k + ((q >> 2) & 1), i + (q & 1)}] = 0;
        int n = 0;
        std::vector<V3> cpos;
        for (auto& kv : nodes) {
            kv.second = n++;
            cpos.push_back({lo[0] + h[0] * kv.first[2], lo[1] + h[1] * kv.first[0], lo[2] + h[2] * kv.first[1]});
        }
        C.n = n;
        C.pid.assign(nf, {0, 0, 0, 0});
        C.pw.assign(nf, {0, 0, 0, 0});
        for (int i = 0; i < nf; ++i) {
            const V3& u = fu[i];
            // order axes by descending local coordinate, ties -> lower axis first
            int ax[3] = {0, 1, 2};
            for (int a = 0; a < 3; ++a)
                for (int b = a + 1; b < 3; ++b)
                    if (u[ax[b]] > u[ax[a]] || (u[ax[b]] == u[ax[a]] && ax[b] < ax[a])) std::swap(ax[a], ax[b]);
            int off[3] = {0, 0, 0};
            const auto& ce = fcell[i];
            std::array<int, 4> ids;
            ids[0] = nodes[{ce[1], ce[2], ce[0]}];
            for (int s2 = 0; s2 < 3; ++s2) {
                off[ax[s2]] = 1;
                ids[s2 + 1] = nodes[{ce[1] + off[1], ce[2] + off[2], ce[0] + off[0]}];
            }
            double wv[4] = {1 - u[ax[0]], u[ax[0]] - u[ax[1]], u[ax[1]] - u[ax[2]], u[ax[2]]};
            double sum = 0;
            for (double& q : wv) {
                if (q < 1e-10) q = 0;
                sum += q;
            }
            C.pid[i] = ids;
            for (int s2 = 0; s2 < 4; ++s2) C.pw[i][s2] = factive[i] ? wv[s2] / sum : 0.0;
        }
        // Galerkin: A_c[J][K] = sum_i sum_k P[i][J] A_f[i][k] P[k][K]
        const OLevel& F = o.lev[l - 1];
        std::vector<std::map<int, double>> rows(n);
        for (int i = 0; i < nf; ++i) {
            for (int a = 0; a < 4; ++a) {
                const double pJ = C.pw[i][a];
                if (pJ == 0) continue;
                const int J = C.pid[i][a];
                auto add = [&](int k, double val) {
                    for (int b = 0; b < 4; ++b) {
                        const double pK = C.pw[k][b];
                        if (pK == 0) continue;
                        rows[J][C.pid[k][b]] += pJ * val * pK;
                    }
                };
                if (l == 1) {
                    add(i, o.Ldiag[i]);
                    for (size_t q = 0; q < o.Loff[i].col.size(); ++q) add(o.Loff[i].col[q], o.Loff[i].val[q]);
                } else {
                    add(i, F.diag[i]);
                    for (size_t q = 0; q < F.off[i].col.size(); ++q) add(F.off[i].col[q], F.off[i].val[q]);
                }
            }
        }
        C.diag.assign(n, 0);
        C.off.assign(n, Row());
        C.active.assign(n, 0);
        for (int J = 0; J < n; ++J)
            for (auto& kv : rows[J]) {
                if (kv.first == J)
                    C.diag[J] = kv.second;
                else {
                    C.off[J].col.push_back(kv.first);
                    C.off[J].val.push_back(kv.second);
                }
            }
        for (int i = 0; i < nf; ++i)
            for (int a = 0; a < 4; ++a)
                if (C.pw[i][a] != 0) C.active[C.pid[i][a]] = 1;
        for (int J = 0; J < n; ++J)
            if (!(C.diag[J] > 0)) C.active[J] = 0;
        fpos = cpos;
        factive = C.active;
    }
    o.hierarchy_dirty = false;
}

// ---------------------------------------------------------------------------
// Reference-faithful frame (PDSolver::Step, PDSolver.cpp:243-293)
// ---------------------------------------------------------------------------
void ref_predict(Oracle& o) {
    // calculateST, PDSolver.cu:72-116
    const double dt = o.p.dt;
    for (int i = 0; i < o.V; ++i) {
        const double fix = o.fixed[i] ? 0.0 : 1.0;
        o.last[i] = o.x[i];
        for (int c = 0; c < 3; ++c) {
            o.v[i][c] *= o.p.damping * fix;
            o.v[i][c] += o.p.gravity[c] * dt * fix;
            o.v[i][c] += o.fext[i][c] * dt * fix;
            o.x[i][c] += o.v[i][c] * dt * fix;
            o.fext[i][c] = 0;
        }
        o.s[i] = o.x[i];
        o.prev[i] = o.x[i];
    }
}

// Sphere vs surface triangles, every active sphere in order (UpdateTriNormal +
// DCDByTriangle_sphere_V2 + DCDByTriangle_sphere_response, PDSolver.cu:394-425,
// 462-501, 612-680): a contact of triangle (A, B, C) with a sphere adds k_c to
// every axis of the diagonal of A, B and C, k_c (centre - hit) to their force,
// and 1 to their contact count.
void ref_triangle_dcd(Oracle& o, std::vector<V3>& cdiag, std::vector<V3>& cforce) {
    auto sub = [](const V3& a, const V3& b) { return V3{a[0] - b[0], a[1] - b[1], a[2] - b[2]}; };
    auto dot = [](const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    auto cross = [](const V3& a, const V3& b) {
        return V3{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    };
    auto length = [&](const V3& a) { return std::sqrt(dot(a, a)); };
    const double k = o.p.collision_stiffness;
    const int F = (int)(o.surf_tris.size() / 3);
    for (const Sphere& sp : o.spheres) {
        if (!sp.active) continue;
        const V3 ctr = {sp.c[0], sp.c[1], sp.c[2]};
        const double r = sp.r;
        for (int f = 0; f < F; ++f) {
            const int ia = o.surf_tris[3 * f], ib = o.surf_tris[3 * f + 1], ic = o.surf_tris[3 * f + 2];
            const V3 A = o.x[ia], B = o.x[ib], C = o.x[ic];
            V3 n = cross(sub(B, A), sub(C, A));
            const double nl = length(n);
            for (int c = 0; c < 3; ++c) n[c] /= nl;
            const double sd = dot(n, sub(ctr, A));
            const double dist = std::fabs(sd);
            if (dist > r) continue;
            const V3 proj = {ctr[0] - n[0] * sd, ctr[1] - n[1] * sd, ctr[2] - n[2] * sd};
            V3 hit;
            bool found = false;
            {   // pointInTriangle, utils.cu:366-383
                const V3 v0 = sub(C, A), v1 = sub(B, A), v2 = sub(proj, A);
                const double d00 = dot(v0, v0), d01 = dot(v0, v1), d02 = dot(v0, v2), d11 = dot(v1, v1), d12 = dot(v1, v2);
                const double inv = 1.0 / (d00 * d11 - d01 * d01);
                const double u = (d11 * d02 - d01 * d12) * inv, v = (d00 * d12 - d01 * d02) * inv;
                if (u >= 0 && v >= 0 && u + v <= 1.0) {
                    const double sgn = sd < 0 ? -1.0 : 1.0;
                    for (int c = 0; c < 3; ++c) hit[c] = ctr[c] + n[c] * (r - dist) * sgn;
                    found = true;
                }
            }
            const V3 tv[3] = {A, B, C};
            for (int i = 0; i < 3 && !found; ++i) {
                const V3& Bg = tv[i];
                V3 ed = sub(tv[(i + 1) % 3], Bg);
                const double el = length(ed);
                for (int c = 0; c < 3; ++c) ed[c] /= el;
                const double t = dot(sub(ctr, Bg), ed);
                if (t < 0 || t > el) continue;
                const V3 cl = {Bg[0] + ed[0] * t, Bg[1] + ed[1] * t, Bg[2] + ed[2] * t};
                V3 rad = sub(ctr, cl);
                const double rl = length(rad);
                if (rl >= r) continue;
                if (dot(cross(ed, sub(tv[(i + 2) % 3], Bg)), cross(ed, sub(proj, Bg))) >= 0) continue;
                for (int c = 0; c < 3; ++c) hit[c] = cl[c] + rad[c] / rl * r;
                found = true;
            }
            for (int i = 0; i < 3 && !found; ++i) {
                const V3 vo = sub(ctr, tv[i]);
                const double vl = length(vo);
                if (vl > r) continue;
                for (int c = 0; c < 3; ++c) hit[c] = tv[i][c] + vo[c] / vl * r;
                found = true;
            }
            if (!found) continue;
            for (int vid : {ia, ib, ic}) {
                o.collided[vid] += 1;
                for (int c = 0; c < 3; ++c) {
                    cdiag[vid][c] += k;
                    cforce[vid][c] += k * (ctr[c] - hit[c]);
                }
            }
        }
    }
}

void ref_iteration(Oracle& o, double omega, std::vector<V3>& force, std::vector<V3>& cdiag, std::vector<V3>& cforce) {
    const int V = o.V;
    std::fill(force.begin(), force.end(), V3{0, 0, 0});
    std::fill(cdiag.begin(), cdiag.end(), V3{0, 0, 0});
    std::fill(cforce.begin(), cforce.end(), V3{0, 0, 0});
    std::fill(o.collided.begin(), o.collided.end(), 0);
    std::fill(o.depth.begin(), o.depth.end(), 0.0);
    std::fill(o.cenergy.begin(), o.cenergy.end(), 0.0);
    if (o.tri_dcd) {
        ref_triangle_dcd(o, cdiag, cforce);
    } else {
        // DCDByPoint_sphere, PDSolver.cu:277-331, every active sphere in order
        for (const Sphere& sp : o.spheres) {
            if (!sp.active) continue;
            const double k = o.p.collision_stiffness;
            for (int i = 0; i < V; ++i) {
                const V3 p = o.x[i];
                const V3 cp = {p[0] - sp.c[0], p[1] - sp.c[1], p[2] - sp.c[2]};
                const double dist = std::sqrt(cp[0] * cp[0] + cp[1] * cp[1] + cp[2] * cp[2]);
                const V3 dir = {cp[0] / dist, cp[1] / dist, cp[2] / dist};
                const double R = sp.r * 1.5;
                if (!(dist < R)) continue;
                const double b = 2 * (cp[0] * dir[0] + cp[1] * dir[1] + cp[2] * dir[2]);
                const double c = cp[0] * cp[0] + cp[1] * cp[1] + cp[2] * cp[2] - R * R;
                double t = (-b + std::sqrt(b * b - 4 * c)) / 2;
                if (t > 0.5 * sp.r) {
                    o.collided[i] = 1;
                    o.depth[i] = t - 0.5 * sp.r;
                }
                t = t / 2.0;
                const V3 colP = {p[0] + dir[0] * t, p[1] + dir[1] * t, p[2] + dir[2] * t};
                const V3 cc = {colP[0] - sp.c[0], colP[1] - sp.c[1], colP[2] - sp.c[2]};
                const double lc = std::sqrt(cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2]);
                const V3 n = {cc[0] / lc, cc[1] / lc, cc[2] / lc};
                const double nd = n[0] * dir[0] + n[1] * dir[1] + n[2] * dir[2];
                for (int a = 0; a < 3; ++a) {
                    cdiag[i][a] += k * n[a] * n[a];
                    cforce[i][a] += k * t * nd * n[a];
                }
                const double pe = (p[0] - colP[0]) * n[0] + (p[1] - colP[1]) * n[1] + (p[2] - colP[2]) * n[2];
                o.cenergy[i] += k * pe * pe;
            }
        }
    }
    // local step: getTetFRV2 + calTetIFV1 (PDSolverAc.cu:447-662)
    const double kv = o.p.volume_stiffness;
    std::vector<double> contrib(12 * (size_t)o.T);
#pragma omp parallel for schedule(static)
    for (int t = 0; t < o.T; ++t) {
        const int* id = &o.tets[4 * t];
        double D[9], F[9], R[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) D[r * 3 + c] = o.x[id[c + 1]][r] - o.x[id[0]][r];
        const double* iv = &o.inv[9 * (size_t)t];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) F[r * 3 + c] = D[r * 3] * iv[c] + D[r * 3 + 1] * iv[3 + c] + D[r * 3 + 2] * iv[6 + c];
        ref_rotation(F, R);
        const double* A = &o.ac[12 * (size_t)t];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 4; ++j) {
                double val = 0;
                for (int k = 0; k < 3; ++k) val += (R[i * 3 + k] - F[i * 3 + k]) * A[k * 4 + j];
                if (std::isnan(val)) val = 0;
                val = std::min(10.0, std::max(-10.0, val));
                double res = val * o.vol[t] * kv;
                if (o.drop_small && std::fabs(res) < 1e-5) res = 0;   // calTetIFV1; calculateIF keeps them
                contrib[12 * (size_t)t + j * 3 + i] = res;
            }
    }
    for (int t = 0; t < o.T; ++t)
        for (int j = 0; j < 4; ++j)
            for (int i = 0; i < 3; ++i) force[o.tets[4 * t + j]][i] += contrib[12 * (size_t)t + j * 3 + i];
    // calculatePOS, PDSolver.cu:192-235
    const double dt = o.p.dt;
    const double relax = o.p.relaxation;
    for (int i = 0; i < V; ++i) {
        const double fix = o.fixed[i] ? 0.0 : 1.0;
        const double dc = o.mass[i] / (dt * dt);
        V3 nx;
        for (int c = 0; c < 3; ++c) {
            const double el = force[i][c] + cforce[i][c];
            double nxt = (dc * (o.s[i][c] - o.x[i][c]) + el) / (o.diag[i] + cdiag[i][c] + dc) * fix + o.x[i][c];
            nxt = (nxt - o.x[i][c]) * relax + o.x[i][c];
            nxt = omega * (nxt - o.prev[i][c]) + o.prev[i][c];
            nx[c] = nxt;
        }
        o.prev[i] = o.x[i];
        o.x[i] = nx;
    }
}

void ref_frame(Oracle& o) {
    ref_predict(o);
    std::vector<V3> force(o.V), cdiag(o.V), cforce(o.V);
    // Chebyshev schedule omega <- 4/(4 - rho^2 omega), evaluated in float as
    // the host loop of PDSolver.cpp:261-271 does.
    float omega = 1.0f;
    for (int it = 0; it < o.p.iterations; ++it) {
        omega = 4 / (4 - o.p.cheb_rho * o.p.cheb_rho * omega);
        ref_iteration(o, (double)omega, force, cdiag, cforce);
    }
    for (int i = 0; i < o.V; ++i)
        for (int c = 0; c < 3; ++c) o.v[i][c] = (o.x[i][c] - o.last[i][c]) / o.p.dt;
}

// ---------------------------------------------------------------------------
// Multigrid frame
// ---------------------------------------------------------------------------
typedef std::vector<V3> Vec;

void spmv_level(const Oracle& o, int l, const Vec& xin, Vec& out) {
    const int n = (int)xin.size();
    out.assign(n, V3{0, 0, 0});
    const bool fine = (l == 0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const double d = fine ? (o.Ldiag[i] + o.c0[i]) : (o.lev[l].diag[i] + o.lev[l].c[i]);
        const Row& r = fine ? o.Loff[i] : o.lev[l].off[i];
        V3 acc = {d * xin[i][0], d * xin[i][1], d * xin[i][2]};
        if (!fine && !o.lev[l].active[i]) {
            out[i] = V3{0, 0, 0};
            continue;
        }
        for (size_t q = 0; q < r.col.size(); ++q)
            for (int c = 0; c < 3; ++c) acc[c] += r.val[q] * xin[r.col[q]][c];
        out[i] = acc;
    }
}

double dinv_level(const Oracle& o, int l, int i) {
    const double omega = o.p.jacobi_omega;
    if (l == 0) return o.fixed[i] ? 0.0 : omega / (o.Ldiag[i] + o.c0[i]);
    if (!o.lev[l].active[i]) return 0.0;
    return omega / (o.lev[l].diag[i] + o.lev[l].c[i]);
}

void coarsest_factor(Oracle& o) {
    OLevel& C = o.lev[o.p.levels - 1];
    const int n = C.n;
    std::vector<double> A((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) {
        if (!C.active[i]) {
            A[(size_t)i * n + i] = 1.0;
            continue;
        }
        A[(size_t)i * n + i] = C.diag[i] + C.c[i];
        for (size_t q = 0; q < C.off[i].col.size(); ++q) {
            const int j = C.off[i].col[q];
            if (C.active[j]) A[(size_t)i * n + j] = C.off[i].val[q];
        }
    }
    // Cholesky A = L L^T (lower, row-major)
    for (int j = 0; j < n; ++j) {
        double d = A[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) d -= A[(size_t)j * n + k] * A[(size_t)j * n + k];
        d = std::sqrt(d);
        A[(size_t)j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double s2 = A[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) s2 -= A[(size_t)i * n + k] * A[(size_t)j * n + k];
            A[(size_t)i * n + j] = s2 / d;
        }
    }
    C.chol.swap(A);
}

void coarsest_solve(const Oracle& o, const Vec& r, Vec& e) {
    const OLevel& C = o.lev[o.p.levels - 1];
    const int n = C.n;
    const std::vector<double>& Lm = C.chol;
    Vec y(n);
    for (int i = 0; i < n; ++i) {
        V3 s2 = C.active[i] ? r[i] : V3{0, 0, 0};
        for (int k = 0; k < i; ++k)
            for (int c = 0; c < 3; ++c) s2[c] -= Lm[(size_t)i * n + k] * y[k][c];
        for (int c = 0; c < 3; ++c) y[i][c] = s2[c] / Lm[(size_t)i * n + i];
    }
    e.assign(n, V3{0, 0, 0});
    for (int i = n - 1; i >= 0; --i) {
        V3 s2 = y[i];
        for (int k = i + 1; k < n; ++k)
            for (int c = 0; c < 3; ++c) s2[c] -= Lm[(size_t)k * n + i] * e[k][c];
        for (int c = 0; c < 3; ++c) e[i][c] = s2[c] / Lm[(size_t)i * n + i];
    }
    for (int i = 0; i < n; ++i)
        if (!C.active[i]) e[i] = V3{0, 0, 0};
}

// Correction-form V-cycle on level l: returns e ~= A_l^{-1} r.
void vcycle(const Oracle& o, int l, const Vec& r, Vec& e) {
    const int L = o.p.levels;
    if (l == L - 1) {
        coarsest_solve(o, r, e);
        return;
    }
    const int n = (int)r.size();
    e.assign(n, V3{0, 0, 0});
    Vec Ae;
    auto sweep = [&]() {
        spmv_level(o, l, e, Ae);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            const double di = dinv_level(o, l, i);
            for (int c = 0; c < 3; ++c) e[i][c] += di * (r[i][c] - Ae[i][c]);
        }
    };
    for (int k = 0; k < o.p.pre_sweeps; ++k) sweep();
    spmv_level(o, l, e, Ae);
    Vec res(n);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) res[i][c] = r[i][c] - Ae[i][c];
    const OLevel& C = o.lev[l + 1];
    Vec rc(C.n, V3{0, 0, 0});
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 4; ++a) {
            const double wgt = C.pw[i][a];
            if (wgt == 0) continue;
            for (int c = 0; c < 3; ++c) rc[C.pid[i][a]][c] += wgt * res[i][c];
        }
    Vec ec;
    vcycle(o, l + 1, rc, ec);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 4; ++a) {
            const double wgt = C.pw[i][a];
            if (wgt == 0) continue;
            for (int c = 0; c < 3; ++c) e[i][c] += wgt * ec[C.pid[i][a]][c];
        }
    for (int k = 0; k < o.p.post_sweeps; ++k) sweep();
}

// ---- capsule against the surface triangles --------------------------------
// Distance from point p to segment [a, b], with the closest point.
double point_segment(const V3& p, const V3& a, const V3& b, V3& cl) {
    const V3 ab = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const double l2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
    double t = 0;
    if (l2 > 0) t = std::min(1.0, std::max(0.0, ((p[0] - a[0]) * ab[0] + (p[1] - a[1]) * ab[1] + (p[2] - a[2]) * ab[2]) / l2));
    cl = {a[0] + t * ab[0], a[1] + t * ab[1], a[2] + t * ab[2]};
    return std::sqrt((p[0] - cl[0]) * (p[0] - cl[0]) + (p[1] - cl[1]) * (p[1] - cl[1]) + (p[2] - cl[2]) * (p[2] - cl[2]));
}

// Closest points of triangle (A, B, C) and segment [P0, P1]: the minimum over
// (i) each segment end point against the triangle -- its projection on the
// plane when that lies inside the triangle, else the nearest edge point --,
// (ii) each triangle edge against the segment -- the interior critical point
// of the two-parameter distance when it lies inside both, else the four end
// point / segment distances -- and (iii) the segment crossing the face.
// Returns the distance; h on the triangle, q on the segment.
double segment_triangle(const V3& P0, const V3& P1, const V3& A, const V3& B, const V3& C, V3& q, V3& h) {
    auto sub = [](const V3& a, const V3& b) { return V3{a[0] - b[0], a[1] - b[1], a[2] - b[2]}; };
    auto dot = [](const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    auto cross = [](const V3& a, const V3& b) {
        return V3{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    };
    auto dist = [&](const V3& a, const V3& b) { return std::sqrt(dot(sub(a, b), sub(a, b))); };
    const V3 n = cross(sub(B, A), sub(C, A));
    const double nn = dot(n, n);
    auto inside = [&](const V3& x) {
        return dot(cross(sub(B, A), sub(x, A)), n) >= 0 && dot(cross(sub(C, B), sub(x, B)), n) >= 0 &&
               dot(cross(sub(A, C), sub(x, C)), n) >= 0;
    };
    const V3 E[3][2] = {{A, B}, {B, C}, {C, A}};
    double best = 1e300;
    auto take = [&](double dd, const V3& qq, const V3& hh) {
        if (dd < best) {
            best = dd;
            q = qq;
            h = hh;
        }
    };
    for (const V3& P : {P0, P1}) {   // (i)
        if (nn > 0) {
            const double sd = dot(n, sub(P, A)) / nn;
            const V3 pr = {P[0] - sd * n[0], P[1] - sd * n[1], P[2] - sd * n[2]};
            if (inside(pr)) take(dist(P, pr), P, pr);
        }
        for (auto& e : E) {
            V3 cl;
            take(point_segment(P, e[0], e[1], cl), P, cl);
        }
    }
    for (auto& e : E) {   // (ii)
        const V3 u = sub(P1, P0), v = sub(e[1], e[0]), w = sub(P0, e[0]);
        const double a = dot(u, u), b = dot(u, v), c = dot(v, v), d = dot(u, w), ee = dot(v, w);
        const double den = a * c - b * b;
        if (den > 1e-300 * std::max(1.0, a * c)) {
            const double s = (b * ee - c * d) / den, t = (a * ee - b * d) / den;
            if (s > 0 && s < 1 && t > 0 && t < 1) {
                const V3 qs = {P0[0] + s * u[0], P0[1] + s * u[1], P0[2] + s * u[2]};
                const V3 ht = {e[0][0] + t * v[0], e[0][1] + t * v[1], e[0][2] + t * v[2]};
                take(dist(qs, ht), qs, ht);
            }
        }
        for (const V3& X : {e[0], e[1]}) {   // edge end points against the segment
            V3 cl;
            take(point_segment(X, P0, P1, cl), cl, X);
        }
    }
    if (nn > 0) {   // (iii)
        const double s0 = dot(n, sub(P0, A)), s1 = dot(n, sub(P1, A));
        if (((s0 <= 0 && s1 >= 0) || (s0 >= 0 && s1 <= 0)) && s0 != s1) {
            const double t = s0 / (s0 - s1);
            const V3 X = {P0[0] + t * (P1[0] - P0[0]), P0[1] + t * (P1[1] - P0[1]), P0[2] + t * (P1[2] - P0[2])};
            if (inside(X)) take(0.0, X, X);
        }
    }
    return best;
}

// Triangle contacts of the frame: every surface triangle closer to the
// capsule's segment than its radius pushes its vertices out by
// (h - q)/|h - q| (r - |h - q|) (r along the inward normal when the segment
// touches the face); a surface vertex not itself inside the capsule but on
// such triangles becomes a contact with target s + the mean of their pushes.
// The capsule form of the reference's sphere test DCDByTriangle_sphere_V2
// (PDSolver.cu:612-680) with its response (PDSolver.cu:462-501).
void capsule_triangles(Oracle& o) {
    const int F = (int)o.cap_tris.size();
    std::vector<V3> psum(o.V, V3{0, 0, 0});
    std::vector<int> pcnt(o.V, 0);
    const V3 P0 = o.cap_a, P1 = o.cap_b;
    const double r = o.cap_r;
    for (int f = 0; f < F; ++f) {
        const auto& t = o.cap_tris[f];
        const V3 A = o.s[t[0]], B = o.s[t[1]], C = o.s[t[2]], D = o.s[t[3]];
        V3 q, h;
        const double d = segment_triangle(P0, P1, A, B, C, q, h);
        if (!(d < r)) continue;
        V3 push;
        if (d > 1e-12) {
            for (int c = 0; c < 3; ++c) push[c] = (h[c] - q[c]) / d * (r - d);
        } else {
            const V3 ab = {B[0] - A[0], B[1] - A[1], B[2] - A[2]}, ac = {C[0] - A[0], C[1] - A[1], C[2] - A[2]};
            V3 n = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]};
            const double nl = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            const double toward_d = n[0] * (D[0] - A[0]) + n[1] * (D[1] - A[1]) + n[2] * (D[2] - A[2]);
            const double sg = toward_d > 0 ? 1.0 : -1.0;
            for (int c = 0; c < 3; ++c) push[c] = nl > 0 ? sg * r * n[c] / nl : 0.0;
        }
        for (int k = 0; k < 3; ++k) {
            for (int c = 0; c < 3; ++c) psum[t[k]][c] += push[c];
            ++pcnt[t[k]];
        }
    }
    for (int i : o.surface_verts) {
        if (o.collided[i] || pcnt[i] == 0) continue;
        o.collided[i] = 1;
        o.c0[i] = o.fixed[i] ? 0.0 : (double)o.p.contact_stiffness;
        for (int c = 0; c < 3; ++c) o.target[i][c] = o.s[i][c] + psum[i][c] / pcnt[i];
    }
}

void mg_frame(Oracle& o) {
    const int V = o.V;
    const double dt = o.p.dt, ih2 = 1.0 / (dt * dt);
    if (o.hierarchy_dirty) build_levels(o);
    // prediction (same form as calculateST, PDSolver.cu:72-116)
    for (int i = 0; i < V; ++i) {
        const double fix = o.fixed[i] ? 0.0 : 1.0;
        o.last[i] = o.x[i];
        for (int c = 0; c < 3; ++c) {
            o.v[i][c] *= o.p.damping * fix;
            o.v[i][c] += o.p.gravity[c] * dt * fix;
            o.x[i][c] += o.v[i][c] * dt * fix;
        }
        o.s[i] = o.x[i];
    }
    // contacts on the predicted positions (surface vertices vs the capsule)
    o.c0.assign(V, 0.0);
    o.target.assign(V, V3{0, 0, 0});
    std::fill(o.collided.begin(), o.collided.end(), 0);
    if (o.have_capsule && o.cap_r > 0) {
        const V3 ab = {o.cap_b[0] - o.cap_a[0], o.cap_b[1] - o.cap_a[1], o.cap_b[2] - o.cap_a[2]};
        const double l2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
        for (int i : o.surface_verts) {
            const V3& p = o.s[i];
            double t = 0;
            if (l2 > 0) {
                t = ((p[0] - o.cap_a[0]) * ab[0] + (p[1] - o.cap_a[1]) * ab[1] + (p[2] - o.cap_a[2]) * ab[2]) / l2;
                t = std::min(1.0, std::max(0.0, t));
            }
            const V3 q = {o.cap_a[0] + t * ab[0], o.cap_a[1] + t * ab[1], o.cap_a[2] + t * ab[2]};
            const V3 dv = {p[0] - q[0], p[1] - q[1], p[2] - q[2]};
            const double d = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
            if (!(d < o.cap_r)) continue;
            V3 nrm = d > 1e-12 ? V3{dv[0] / d, dv[1] / d, dv[2] / d} : V3{0, 0, 1};
            o.collided[i] = 1;
            o.c0[i] = o.fixed[i] ? 0.0 : (double)o.p.contact_stiffness;
            o.target[i] = {q[0] + o.cap_r * nrm[0], q[1] + o.cap_r * nrm[1], q[2] + o.cap_r * nrm[2]};
        }
        if (o.tri_contact) capsule_triangles(o);
    }
    // lumped contact weights on the coarse levels, coarsest factorisation
    const int L = o.p.levels;
    {
        std::vector<double> cf = o.c0;
        for (int l = 1; l < L; ++l) {
            OLevel& C = o.lev[l];
            C.c.assign(C.n, 0.0);
            for (size_t i = 0; i < cf.size(); ++i)
                for (int a = 0; a < 4; ++a)
                    if (C.pw[i][a] != 0) C.c[C.pid[i][a]] += C.pw[i][a] * cf[i];
            cf = C.c;
        }
        coarsest_factor(o);
    }
    // The global system A x = M/h^2 s + C p + sum_t w G^T R_t is solved for the
    // displacement from the prediction, d = x - s (same solution): A d = b_d with
    // b_d = C (p - s) + sum_t w G_t^T (R_t - F_t(s)), every term built from small
    // position differences.
    Vec d(V, V3{0, 0, 0});
    Vec bbase(V);
    for (int i = 0; i < V; ++i)
        for (int c = 0; c < 3; ++c) bbase[i][c] = o.c0[i] * (o.target[i][c] - o.s[i][c]);
    (void)ih2;
    std::vector<double> rot(9 * (size_t)o.T), Fs(9 * (size_t)o.T);
    auto defgrad = [&](int t, const Vec& p0, const Vec* p1, double* F) {
        const int* id = &o.tets[4 * t];
        const double* iv = &o.inv[9 * (size_t)t];
        double D[9];
        for (int rr = 0; rr < 3; ++rr)
            for (int c = 0; c < 3; ++c) {
                D[rr * 3 + c] = p0[id[c + 1]][rr] - p0[id[0]][rr];
                if (p1) D[rr * 3 + c] += (*p1)[id[c + 1]][rr] - (*p1)[id[0]][rr];
            }
        for (int rr = 0; rr < 3; ++rr)
            for (int c = 0; c < 3; ++c) F[rr * 3 + c] = D[rr * 3] * iv[c] + D[rr * 3 + 1] * iv[3 + c] + D[rr * 3 + 2] * iv[6 + c];
    };
#pragma omp parallel for schedule(static)
    for (int t = 0; t < o.T; ++t) defgrad(t, o.s, nullptr, &Fs[9 * (size_t)t]);
    Vec b(V), Ad, r(V), e;
    for (int it = 0; it < o.p.iterations; ++it) {
        // local step: R_t = closest rotation of F_t(s + d)
#pragma omp parallel for schedule(static)
        for (int t = 0; t < o.T; ++t) {
            double F[9];
            defgrad(t, o.s, &d, F);
            svd_rotation(F, &rot[9 * (size_t)t]);
        }
        b = bbase;
        for (int t = 0; t < o.T; ++t) {
            const int* id = &o.tets[4 * t];
            const double* A = &o.ac[12 * (size_t)t];
            const double* R = &rot[9 * (size_t)t];
            const double* F0 = &Fs[9 * (size_t)t];
            for (int j = 0; j < 4; ++j)
                for (int i = 0; i < 3; ++i)
                    b[id[j]][i] += o.w[t] * ((R[i * 3] - F0[i * 3]) * A[j] + (R[i * 3 + 1] - F0[i * 3 + 1]) * A[4 + j] +
                                             (R[i * 3 + 2] - F0[i * 3 + 2]) * A[8 + j]);
        }
        for (int pass = 0; pass < o.p.refinement_passes; ++pass) {
            spmv_level(o, 0, d, Ad);
#pragma omp parallel for schedule(static)
            for (int i = 0; i < V; ++i)
                for (int c = 0; c < 3; ++c) r[i][c] = b[i][c] - Ad[i][c];
            vcycle(o, 0, r, e);
#pragma omp parallel for schedule(static)
            for (int i = 0; i < V; ++i)
                for (int c = 0; c < 3; ++c) d[i][c] += e[i][c];
        }
        if (it == o.p.iterations - 1) {
            spmv_level(o, 0, d, Ad);
            double rr2 = 0;
            for (int i = 0; i < V; ++i)
                if (!o.fixed[i])
                    for (int c = 0; c < 3; ++c) rr2 += (b[i][c] - Ad[i][c]) * (b[i][c] - Ad[i][c]);
            o.last_residual = std::sqrt(rr2);
        }
    }
    // x = s + d and v = (x - last)/dt = v_predicted + d/dt
    for (int i = 0; i < V; ++i)
        for (int c = 0; c < 3; ++c) {
            o.x[i][c] = o.s[i][c] + d[i][c];
            o.v[i][c] += d[i][c] / dt;
        }
}

}  // namespace

struct oracle_solver {
    Oracle o;
};

extern "C" {

oracle_solver* oracle_create(const mgsb_mesh* mesh, const mgsb_params* params, char* err, int errlen) {
    auto fail = [&](const std::string& m) -> oracle_solver* {
        if (err && errlen > 0) std::snprintf(err, errlen, "%s", m.c_str());
        return nullptr;
    };
    if (!mesh || !params || mesh->num_verts <= 0 || mesh->num_tets <= 0) return fail("invalid mesh");
    oracle_solver* h = new oracle_solver();
    Oracle& o = h->o;
    o.p = *params;
    o.V = mesh->num_verts;
    o.T = mesh->num_tets;
    o.rest.assign(mesh->positions, mesh->positions + 3 * (size_t)o.V);
    o.tets.assign(mesh->tets, mesh->tets + 4 * (size_t)o.T);
    for (int v : o.tets)
        if (v < 0 || v >= o.V) {
            delete h;
            return fail("tet index out of range");
        }
    o.youngs.assign(o.T, params->youngs_modulus);
    o.poisson.assign(o.T, params->poisson_ratio);
    o.fixed.assign(o.V, 0);
    o.grid_hint = {mesh->grid_dims[0], mesh->grid_dims[1], mesh->grid_dims[2]};
    std::string e;
    if (!precompute(o, e)) {
        delete h;
        return fail(e);
    }
    if (o.grid_hint[0] <= 0 || o.grid_hint[1] <= 0 || o.grid_hint[2] <= 0) {
        // bounding box over mean edge length (same rule as the product's default)
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int i = 0; i < o.V; ++i)
            for (int c = 0; c < 3; ++c) {
                lo[c] = std::min(lo[c], o.rest[3 * i + c]);
                hi[c] = std::max(hi[c], o.rest[3 * i + c]);
            }
        double sum = 0;
        long cnt = 0;
        const int E[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
        for (int t = 0; t < o.T; ++t)
            for (auto& ed : E) {
                const int a = o.tets[4 * t + ed[0]], b = o.tets[4 * t + ed[1]];
                double d2 = 0;
                for (int c = 0; c < 3; ++c) d2 += (o.rest[3 * a + c] - o.rest[3 * b + c]) * (o.rest[3 * a + c] - o.rest[3 * b + c]);
                sum += std::sqrt(d2);
                ++cnt;
            }
        const double hm = sum / cnt;
        for (int c = 0; c < 3; ++c) o.grid_hint[c] = std::max(1, (int)std::lround((hi[c] - lo[c]) / hm));
    }
    o.x.resize(o.V);
    for (int i = 0; i < o.V; ++i) o.x[i] = {o.rest[3 * i], o.rest[3 * i + 1], o.rest[3 * i + 2]};
    o.v.assign(o.V, V3{0, 0, 0});
    o.s = o.x;
    o.last = o.x;
    o.prev = o.x;
    o.fext.assign(o.V, V3{0, 0, 0});
    o.collided.assign(o.V, 0);
    o.depth.assign(o.V, 0);
    o.cenergy.assign(o.V, 0);
    o.c0.assign(o.V, 0);
    o.target.assign(o.V, V3{0, 0, 0});
    if (o.p.solver == MGSB_SOLVER_MULTIGRID) {
        if (o.p.levels < 2) {
            delete h;
            return fail("multigrid needs >= 2 levels");
        }
        build_surface(o);
        assemble_L(o);
    }
    return h;
}

void oracle_destroy(oracle_solver* h) { delete h; }

int oracle_set_fixed(oracle_solver* h, const uint8_t* mask) {
    Oracle& o = h->o;
    for (int i = 0; i < o.V; ++i) o.fixed[i] = mask[i] ? 1 : 0;
    o.hierarchy_dirty = true;
    return 0;
}

int oracle_set_material(oracle_solver* h, const float* youngs, const float* poisson) {
    Oracle& o = h->o;
    for (int t = 0; t < o.T; ++t) {
        o.youngs[t] = youngs[t];
        o.poisson[t] = poisson[t];
    }
    if (o.p.solver == MGSB_SOLVER_MULTIGRID) assemble_L(o);
    o.hierarchy_dirty = true;
    return 0;
}

int oracle_set_params(oracle_solver* h, const mgsb_params* params) {
    Oracle& o = h->o;
    if (!params || params->solver != o.p.solver) return MGSB_NOT_SUPPORTED;
    const bool material = params->youngs_modulus != o.p.youngs_modulus || params->poisson_ratio != o.p.poisson_ratio;
    o.p = *params;
    if (material) {
        o.youngs.assign(o.T, params->youngs_modulus);
        o.poisson.assign(o.T, params->poisson_ratio);
    }
    std::string e;
    if (!precompute(o, e)) return MGSB_INVALID_ARG;
    if (o.p.solver == MGSB_SOLVER_MULTIGRID) assemble_L(o);
    o.hierarchy_dirty = true;
    return 0;
}

double oracle_segment_triangle(const double* p0p1, const double* abc, double* q, double* h) {
    const V3 P0 = {p0p1[0], p0p1[1], p0p1[2]}, P1 = {p0p1[3], p0p1[4], p0p1[5]};
    const V3 A = {abc[0], abc[1], abc[2]}, B = {abc[3], abc[4], abc[5]}, C = {abc[6], abc[7], abc[8]};
    V3 qq, hh;
    const double d = segment_triangle(P0, P1, A, B, C, qq, hh);
    for (int c = 0; c < 3; ++c) {
        q[c] = qq[c];
        h[c] = hh[c];
    }
    return d;
}

int oracle_set_surface_contact(oracle_solver* h, int mode) {
    h->o.tri_contact = mode == 1;
    return 0;
}

int oracle_set_tool_capsule(oracle_solver* h, const float a[3], const float b[3], float radius) {
    Oracle& o = h->o;
    o.have_capsule = radius > 0;
    o.cap_a = {a[0], a[1], a[2]};
    o.cap_b = {b[0], b[1], b[2]};
    o.cap_r = radius;
    return 0;
}

int oracle_set_tool_spheres(oracle_solver* h, int32_t count, const float* centers, const float* radii,
                            const uint8_t* active) {
    Oracle& o = h->o;
    o.spheres.clear();
    for (int i = 0; i < count; ++i)
        o.spheres.push_back({{centers[3 * i], centers[3 * i + 1], centers[3 * i + 2]}, radii[i], active ? active[i] != 0 : true});
    return 0;
}

int oracle_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int oracle_step(oracle_solver* h) {
    Oracle& o = h->o;
    if (o.p.solver == MGSB_SOLVER_REFERENCE_JACOBI)
        ref_frame(o);
    else
        mg_frame(o);
    for (int i = 0; i < o.V; ++i)
        for (int c = 0; c < 3; ++c)
            if (!std::isfinite(o.x[i][c])) return MGSB_DIVERGED;
    return 0;
}

int oracle_num_verts(const oracle_solver* h) { return h->o.V; }

void oracle_get_positions(const oracle_solver* h, double* out) {
    for (int i = 0; i < h->o.V; ++i)
        for (int c = 0; c < 3; ++c) out[3 * i + c] = h->o.x[i][c];
}

void oracle_get_velocities(const oracle_solver* h, double* out) {
    for (int i = 0; i < h->o.V; ++i)
        for (int c = 0; c < 3; ++c) out[3 * i + c] = h->o.v[i][c];
}

void oracle_get_contact_flags(const oracle_solver* h, int32_t* out) {
    for (int i = 0; i < h->o.V; ++i) out[i] = h->o.collided[i];
}

void oracle_get_collision_depth(const oracle_solver* h, double* out) {
    for (int i = 0; i < h->o.V; ++i) out[i] = h->o.depth[i];
}

void oracle_set_state(oracle_solver* h, const double* positions, const double* velocities) {
    Oracle& o = h->o;
    for (int i = 0; i < o.V; ++i)
        for (int c = 0; c < 3; ++c) {
            if (positions) o.x[i][c] = positions[3 * i + c];
            if (velocities) o.v[i][c] = velocities[3 * i + c];
        }
}

void oracle_get_precompute(const oracle_solver* h, double* inv, double* ac, double* volume, double* mass, double* diag) {
    const Oracle& o = h->o;
    if (inv) std::copy(o.inv.begin(), o.inv.end(), inv);
    if (ac) std::copy(o.ac.begin(), o.ac.end(), ac);
    if (volume) std::copy(o.vol.begin(), o.vol.end(), volume);
    if (mass) std::copy(o.mass.begin(), o.mass.end(), mass);
    if (diag) {
        if (o.p.solver == MGSB_SOLVER_REFERENCE_JACOBI)
            std::copy(o.diag.begin(), o.diag.end(), diag);
        else
            std::copy(o.Ldiag.begin(), o.Ldiag.end(), diag);
    }
}

void oracle_get_energy(const oracle_solver* h, double out[5]) {
    // runCalEnergy, PDSolver.cu:816-924 (FP64 throughout)
    const Oracle& o = h->o;
    const bool ref = o.p.solver == MGSB_SOLVER_REFERENCE_JACOBI;
    double Ek = 0, Ep = 0, Ec = 0, Nc = 0, dX = 0;
    for (int i = 0; i < o.V; ++i) {
        double a = 0, b = 0;
        for (int c = 0; c < 3; ++c) {
            a += (o.x[i][c] - o.prev[i][c]) * (o.x[i][c] - o.prev[i][c]);
            b += (o.x[i][c] - o.s[i][c]) * (o.x[i][c] - o.s[i][c]);
        }
        dX += a;
        Ek += o.mass[i] * b;
    }
    dX = std::sqrt(dX);
    Ek /= 2 * (double)o.p.dt * (double)o.p.dt;
    for (int t = 0; t < o.T; ++t) {
        const int* id = &o.tets[4 * t];
        double D[9], F[9], R[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) D[r * 3 + c] = o.x[id[c + 1]][r] - o.x[id[0]][r];
        const double* iv = &o.inv[9 * (size_t)t];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) F[r * 3 + c] = D[r * 3] * iv[c] + D[r * 3 + 1] * iv[3 + c] + D[r * 3 + 2] * iv[6 + c];
        if (ref)
            ref_rotation(F, R);
        else
            svd_rotation(F, R);
        double e = 0;
        for (int i = 0; i < 9; ++i) e += (F[i] - R[i]) * (F[i] - R[i]);
        Ep += ref ? e * o.vol[t] * o.p.volume_stiffness / 2 : e * o.w[t] / 2;
    }
    for (int i = 0; i < o.V; ++i) {
        if (ref)
            Ec += o.cenergy[i];
        else if (o.c0[i] > 0) {
            double d2 = 0;
            for (int c = 0; c < 3; ++c) d2 += (o.x[i][c] - o.target[i][c]) * (o.x[i][c] - o.target[i][c]);
            Ec += 0.5 * o.c0[i] * d2;
        }
        Nc += o.collided[i] > 0 ? 1 : 0;
    }
    out[0] = Ek;
    out[1] = Ep;
    out[2] = Ec;
    out[3] = Nc;
    out[4] = ref ? dX : o.last_residual;
}

double oracle_last_residual(const oracle_solver* h) { return h->o.last_residual; }

void oracle_surface_normals(const double* pos, int32_t V, const int32_t* tris, int32_t F, double* out) {
    // UpdateTriNormal (PDSolver.cu:394-424): unit normal (B-A) x (C-A) / |.| of
    // each triangle (normalize, utils.cu:293, has no epsilon test), summed into
    // its three vertices in triangle order; AvgOutsideTetVertNormal
    // (PDSolver.cu:438-450): divide by the length when it exceeds FLT_EPSILON.
    std::fill(out, out + 3 * (size_t)V, 0.0);
    for (int32_t f = 0; f < F; ++f) {
        const int32_t a = tris[3 * f], b = tris[3 * f + 1], c = tris[3 * f + 2];
        double ab[3], ac[3];
        for (int q = 0; q < 3; ++q) {
            ab[q] = pos[3 * b + q] - pos[3 * a + q];
            ac[q] = pos[3 * c + q] - pos[3 * a + q];
        }
        double n[3] = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]};
        const double len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        for (int q = 0; q < 3; ++q) n[q] /= len;
        for (int32_t v : {a, b, c})
            for (int q = 0; q < 3; ++q) out[3 * v + q] += n[q];
    }
    for (int32_t i = 0; i < V; ++i) {
        const double len = std::sqrt(out[3 * i] * out[3 * i] + out[3 * i + 1] * out[3 * i + 1] + out[3 * i + 2] * out[3 * i + 2]);
        if (len > 1.1920928955078125e-07)
            for (int q = 0; q < 3; ++q) out[3 * i + q] /= len;
    }
}

int oracle_level_size(const oracle_solver* h, int level, int32_t* n, int32_t* nnz) {
    Oracle& o = const_cast<Oracle&>(h->o);
    if (o.p.solver != MGSB_SOLVER_MULTIGRID || level < 0 || level >= o.p.levels) return MGSB_INVALID_ARG;
    if (o.hierarchy_dirty) build_levels(o);
    if (level == 0) {
        *n = o.V;
        size_t z = 0;
        for (auto& r : o.Loff) z += r.col.size();
        *nnz = (int32_t)z;
        return 0;
    }
    *n = o.lev[level].n;
    size_t z = 0;
    for (auto& r : o.lev[level].off) z += r.col.size();
    *nnz = (int32_t)z;
    return 0;
}

int oracle_level_prolongation(const oracle_solver* h, int level, int32_t* ids, double* w) {
    Oracle& o = const_cast<Oracle&>(h->o);
    if (o.p.solver != MGSB_SOLVER_MULTIGRID || level < 1 || level >= o.p.levels) return MGSB_INVALID_ARG;
    if (o.hierarchy_dirty) build_levels(o);
    const OLevel& C = o.lev[level];
    for (size_t i = 0; i < C.pid.size(); ++i)
        for (int a = 0; a < 4; ++a) {
            ids[4 * i + a] = C.pid[i][a];
            w[4 * i + a] = C.pw[i][a];
        }
    return 0;
}

int oracle_level_matrix(const oracle_solver* h, int level, double* diag, int32_t* ptr, int32_t* col, double* val) {
    Oracle& o = const_cast<Oracle&>(h->o);
    if (o.p.solver != MGSB_SOLVER_MULTIGRID || level < 0 || level >= o.p.levels) return MGSB_INVALID_ARG;
    if (o.hierarchy_dirty) build_levels(o);
    const std::vector<double>& dg = level == 0 ? o.Ldiag : o.lev[level].diag;
    const std::vector<Row>& rows = level == 0 ? o.Loff : o.lev[level].off;
    int z = 0;
    ptr[0] = 0;
    for (size_t i = 0; i < rows.size(); ++i) {
        diag[i] = dg[i];
        for (size_t q = 0; q < rows[i].col.size(); ++q) {
            col[z] = rows[i].col[q];
            val[z] = rows[i].val[q];
            ++z;
        }
        ptr[i + 1] = z;
    }
    return 0;
}

void oracle_ref_rotation(const double F[9], double R[9]) { ref_rotation(F, R); }
void oracle_svd_rotation(const double F[9], double R[9]) { svd_rotation(F, R); }
double oracle_inverse3(const double A[9], double R[9]) { return inverse3(A, R); }

}  // extern "C"


// ---------------------------------------------------------------------------
// Learned-smoother MLP (libmgsb's network; no reference counterpart)
// ---------------------------------------------------------------------------
namespace {
constexpr int kIn = 9, kHid = 64, kOut = 3;
constexpr int kW1 = 0, kB1 = kW1 + kHid * kIn, kW2 = kB1 + kHid, kB2 = kW2 + kHid * kHid, kW3 = kB2 + kHid,
              kB3 = kW3 + kOut * kHid, kNP = kB3 + kOut;

double bf16_round(double v) {
    float f = (float)v;
    uint32_t b;
    std::memcpy(&b, &f, 4);
    b += 0x7FFFu + ((b >> 16) & 1u);
    b &= 0xFFFF0000u;
    std::memcpy(&f, &b, 4);
    return (double)f;
}
// GELU, tanh form (Hendrycks & Gimpel 2016): x/2 (1 + tanh(sqrt(2/pi)(x + 0.044715 x^3)))
double gelu64(double x) {
    const double c = std::sqrt(2.0 / M_PI);
    return 0.5 * x * (1.0 + std::tanh(c * (x + 0.044715 * x * x * x)));
}
double gelu64_grad(double x) {
    const double c = std::sqrt(2.0 / M_PI);
    const double t = std::tanh(c * (x + 0.044715 * x * x * x));
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * c * (1.0 + 3.0 * 0.044715 * x * x);
}

struct MlpPass {
    double x[kIn], z1[kHid], h1[kHid], z2[kHid], h2[kHid], y[kOut];
};

void mlp_pass(const std::vector<double>& w, const double* xin, bool bf, MlpPass& P) {
    for (int k = 0; k < kIn; ++k) P.x[k] = bf ? bf16_round(xin[k]) : xin[k];
    for (int j = 0; j < kHid; ++j) {
        double a = w[kB1 + j];
        for (int k = 0; k < kIn; ++k) a += w[kW1 + j * kIn + k] * P.x[k];
        P.z1[j] = a;
        P.h1[j] = bf ? bf16_round(gelu64(a)) : gelu64(a);
    }
    for (int j = 0; j < kHid; ++j) {
        double a = w[kB2 + j];
        for (int k = 0; k < kHid; ++k) a += w[kW2 + j * kHid + k] * P.h1[k];
        P.z2[j] = a;
        P.h2[j] = bf ? bf16_round(gelu64(a)) : gelu64(a);
    }
    for (int o = 0; o < kOut; ++o) {
        double a = w[kB3 + o];
        for (int k = 0; k < kHid; ++k) a += w[kW3 + o * kHid + k] * P.h2[k];
        P.y[o] = a;
    }
}

std::vector<double> mlp_weights(const double* params, bool bf) {
    std::vector<double> w(params, params + kNP);
    if (bf) {
        for (int q = kW1; q < kB1; ++q) w[q] = bf16_round(w[q]);
        for (int q = kW2; q < kB2; ++q) w[q] = bf16_round(w[q]);
        for (int q = kW3; q < kB3; ++q) w[q] = bf16_round(w[q]);
    }
    return w;
}
}  // namespace

void oracle_mlp_forward(const double* params, const double* x, int32_t n, int32_t bf16, double* y) {
    const std::vector<double> w = mlp_weights(params, bf16 != 0);
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
        MlpPass P;
        mlp_pass(w, x + (size_t)i * kIn, bf16 != 0, P);
        for (int o = 0; o < kOut; ++o) y[(size_t)i * kOut + o] = P.y[o];
    }
}

double oracle_mlp_loss_grad(const double* params, const double* x, const double* t, int32_t n, int32_t bf16,
                            double* grad) {
    const std::vector<double> w = mlp_weights(params, bf16 != 0);
    std::vector<double> g(kNP, 0.0);
    double loss = 0.0;
    const double inv = 1.0 / ((double)n * kOut);
    for (int32_t i = 0; i < n; ++i) {
        MlpPass P;
        mlp_pass(w, x + (size_t)i * kIn, bf16 != 0, P);
        double dy[kOut];
        for (int o = 0; o < kOut; ++o) {
            const double d = P.y[o] - t[(size_t)i * kOut + o];
            loss += d * d;
            dy[o] = 2.0 * d * inv;
            g[kB3 + o] += dy[o];
            for (int k = 0; k < kHid; ++k) g[kW3 + o * kHid + k] += dy[o] * P.h2[k];
        }
        double dz2[kHid], dz1[kHid];
        for (int k = 0; k < kHid; ++k) {
            double a = 0.0;
            for (int o = 0; o < kOut; ++o) a += dy[o] * w[kW3 + o * kHid + k];
            dz2[k] = a * gelu64_grad(P.z2[k]);
            g[kB2 + k] += dz2[k];
            for (int j = 0; j < kHid; ++j) g[kW2 + k * kHid + j] += dz2[k] * P.h1[j];
        }
        for (int k = 0; k < kHid; ++k) {
            double a = 0.0;
            for (int j = 0; j < kHid; ++j) a += dz2[j] * w[kW2 + j * kHid + k];
            dz1[k] = a * gelu64_grad(P.z1[k]);
            g[kB1 + k] += dz1[k];
            for (int m = 0; m < kIn; ++m) g[kW1 + k * kIn + m] += dz1[k] * P.x[m];
        }
    }
    if (grad) std::copy(g.begin(), g.end(), grad);
    return loss * inv;
}


// ---------------------------------------------------------------------------
// Two-level schedule (PDSolver_MG, PDSolver_MG.cpp:5-253)
// ---------------------------------------------------------------------------
namespace {

// barycentricCoordinate(point, A, B, C, D) (utils.cu:335-364) in FP64.
void bary64(const double* p, const V3 v[4], double w[4], bool abs_volume = false) {
    auto sub = [](const V3& a, const V3& b) { return V3{a[0] - b[0], a[1] - b[1], a[2] - b[2]}; };
    auto dot = [](const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    auto cross = [](const V3& a, const V3& b) {
        return V3{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    };
    double Vol = dot(sub(v[1], v[0]), cross(sub(v[2], v[0]), sub(v[3], v[0]))) / 6.0;
    if (abs_volume) Vol = std::fabs(Vol);   // the face-area form of PDSolver_MG::Init uses |V|
    V3 ctr = {0, 0, 0};
    for (int k = 0; k < 4; ++k)
        for (int c = 0; c < 3; ++c) ctr[c] += 0.25 * v[k][c];
    const V3 P = {p[0], p[1], p[2]};
    for (int i = 0; i < 4; ++i) {
        const V3& q = v[i];
        const V3 &f0 = v[(i + 1) % 4], &f1 = v[(i + 2) % 4], &f2 = v[(i + 3) % 4];
        V3 n = cross(sub(f1, f0), sub(f2, f0));
        if (dot(n, sub(q, f0)) > 0)
            for (int c = 0; c < 3; ++c) n[c] = -n[c];
        const double l = std::sqrt(dot(n, n));
        for (int c = 0; c < 3; ++c) n[c] /= l;
        w[i] = 0.25 - dot(sub(P, ctr), n) * (0.5 * l) / (3 * Vol);
    }
}

}  // namespace

struct oracle_mg2 {
    oracle_solver* c = nullptr;
    oracle_solver* f = nullptr;
    std::vector<int> fid, cid;        // fine -> coarse tet ids, coarse -> fine tet ids
    std::vector<double> fw, cw;
};

extern "C" {

oracle_mg2* oracle_mg2_create(const mgsb_mesh* coarse, const mgsb_mesh* fine, const mgsb_params* params, char* err,
                              int errlen) {
    auto fail = [&](const std::string& m, oracle_mg2* h) -> oracle_mg2* {
        if (err && errlen > 0) std::snprintf(err, errlen, "%s", m.c_str());
        if (h) {
            delete h->c;
            delete h->f;
            delete h;
        }
        return nullptr;
    };
    oracle_mg2* h = new oracle_mg2();
    h->c = oracle_create(coarse, params, err, errlen);
    h->f = oracle_create(fine, params, err, errlen);
    if (!h->c || !h->f) return fail(err ? std::string(err) : "create failed", h);
    Oracle& C = h->c->o;
    Oracle& F = h->f->o;
    build_surface(C);
    C.tri_dcd = true;
    C.drop_small = F.drop_small = false;
    // PDSolver_MG::interpolate (PDSolver_MG.cpp:5-58): each fine vertex in the
    // first coarse tet (index order) whose weights lie in [-1e-5, 1 + 1e-5]
    h->fid.assign(4 * (size_t)F.V, -1);
    h->fw.assign(4 * (size_t)F.V, 0.0);
    for (int v = 0; v < F.V; ++v) {
        const double* P = &F.rest[3 * (size_t)v];
        bool found = false;
        for (int t = 0; t < C.T && !found; ++t) {
            const int* id = &C.tets[4 * t];
            V3 tv[4];
            for (int k = 0; k < 4; ++k) tv[k] = {C.rest[3 * id[k]], C.rest[3 * id[k] + 1], C.rest[3 * id[k] + 2]};
            double w[4];
            bary64(P, tv, w);
            bool in = true;
            for (int k = 0; k < 4; ++k)
                if (w[k] < -1e-5 || w[k] > 1 + 1e-5) in = false;
            if (!in) continue;
            for (int k = 0; k < 4; ++k) {
                h->fid[4 * (size_t)v + k] = id[k];
                h->fw[4 * (size_t)v + k] = w[k];
            }
            found = true;
        }
        if (!found) return fail("fine vertex outside the coarse mesh", h);
    }
    // PDSolver_MG::Init (PDSolver_MG.cpp:120-167): each coarse vertex in the first
    // fine tet whose four face planes (outward normals) it does not exceed by
    // more than 1e-6; weights from the face areas and normals.
    h->cid.assign(4 * (size_t)C.V, -1);
    h->cw.assign(4 * (size_t)C.V, 0.0);
    for (int v = 0; v < C.V; ++v) {
        const double* P = &C.rest[3 * (size_t)v];
        bool found = false;
        for (int t = 0; t < F.T && !found; ++t) {
            const int* id = &F.tets[4 * t];
            V3 tv[4];
            for (int k = 0; k < 4; ++k) tv[k] = {F.rest[3 * id[k]], F.rest[3 * id[k] + 1], F.rest[3 * id[k] + 2]};
            bool in = true;
            static const int face[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
            for (int k = 0; k < 4 && in; ++k) {
                const V3 &A = tv[face[k][0]], &B = tv[face[k][1]], &Cc = tv[face[k][2]], &D = tv[k];
                const V3 ab = {B[0] - A[0], B[1] - A[1], B[2] - A[2]}, ac = {Cc[0] - A[0], Cc[1] - A[1], Cc[2] - A[2]};
                V3 n = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]};
                if (n[0] * (D[0] - A[0]) + n[1] * (D[1] - A[1]) + n[2] * (D[2] - A[2]) > 0)
                    for (int c = 0; c < 3; ++c) n[c] = -n[c];
                const double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
                const V3& Af = tv[(k + 1) % 4];
                const double d = ((P[0] - Af[0]) * n[0] + (P[1] - Af[1]) * n[1] + (P[2] - Af[2]) * n[2]) / l;
                if (d > 1e-6) in = false;
            }
            if (!in) continue;
            double w[4];
            bary64(P, tv, w, true);   // face-area form (utils.cu:313-333) with the tet's |V|
            for (int k = 0; k < 4; ++k) {
                h->cid[4 * (size_t)v + k] = id[k];
                h->cw[4 * (size_t)v + k] = w[k];
            }
            found = true;
        }
        if (!found) return fail("coarse vertex outside the fine mesh", h);
    }
    return h;
}

void oracle_mg2_destroy(oracle_mg2* h) {
    if (!h) return;
    oracle_destroy(h->c);
    oracle_destroy(h->f);
    delete h;
}

oracle_solver* oracle_mg2_level(oracle_mg2* h, int level) { return level == 0 ? h->f : h->c; }

// PDSolver_MG::Step (PDSolver_MG.cpp:183-253)
void oracle_mg2_step(oracle_mg2* h) {
    Oracle& C = h->c->o;
    Oracle& F = h->f->o;
    ref_predict(C);
    ref_predict(F);
    auto iterate = [](Oracle& o) {
        std::vector<V3> force(o.V), cdiag(o.V), cforce(o.V);
        float omega = 1.0f;
        for (int it = 0; it < o.p.iterations; ++it) {
            omega = 4 / (4 - o.p.cheb_rho * o.p.cheb_rho * omega);
            ref_iteration(o, (double)omega, force, cdiag, cforce);
        }
    };
    auto transfer = [](Oracle& dst, const Oracle& src, const std::vector<int>& id, const std::vector<double>& w) {
        for (int v = 0; v < dst.V; ++v) {
            V3 q = {0, 0, 0};
            for (int k = 0; k < 4; ++k)
                for (int c = 0; c < 3; ++c) q[c] += w[4 * (size_t)v + k] * src.x[id[4 * (size_t)v + k]][c];
            dst.x[v] = q;
            dst.prev[v] = q;
        }
    };
    iterate(C);
    transfer(F, C, h->fid, h->fw);        // runInterpolate
    iterate(F);
    transfer(C, F, h->cid, h->cw);        // runAverage
    for (int v = 0; v < F.V; ++v) {       // runUpdateMapping
        V3 tv[4];
        for (int k = 0; k < 4; ++k) tv[k] = C.x[h->fid[4 * (size_t)v + k]];
        bary64(F.x[v].data(), tv, &h->fw[4 * (size_t)v]);
    }
    for (Oracle* o : {&C, &F})
        for (int i = 0; i < o->V; ++i)
            for (int c = 0; c < 3; ++c) o->v[i][c] = (o->x[i][c] - o->last[i][c]) / o->p.dt;
}

}  // extern "C"
