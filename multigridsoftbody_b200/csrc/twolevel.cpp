// Host binding of the two-level schedule's meshes (see twolevel.hpp).
#include "twolevel.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>

namespace mgsb {
namespace {

struct V3f {
    float x, y, z;
};
inline V3f ld(const float* p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
inline V3f sub(V3f a, V3f b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3f add(V3f a, V3f b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3f mul(V3f a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(V3f a, V3f b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3f cross(V3f a, V3f b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float len(V3f a) { return std::sqrt(dot(a, a)); }

// Uniform grid over the bounding boxes of a tet set: candidates of a point are
// the tets of its cell, in ascending index order.
struct TetGrid {
    float lo[3], cell;
    int dim[3];
    std::vector<int32_t> start, items;

    void build(const float* pos, const int32_t* tets, int T) {
        float hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = 1e30f;
            hi[a] = -1e30f;
        }
        std::vector<float> bb(6 * (size_t)T);
        double ext = 0.0;
        for (int t = 0; t < T; ++t) {
            float* b = &bb[6 * (size_t)t];
            for (int a = 0; a < 3; ++a) {
                b[a] = 1e30f;
                b[3 + a] = -1e30f;
            }
            for (int k = 0; k < 4; ++k) {
                const float* p = pos + 3 * tets[4 * t + k];
                for (int a = 0; a < 3; ++a) {
                    b[a] = std::min(b[a], p[a]);
                    b[3 + a] = std::max(b[3 + a], p[a]);
                }
            }
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::min(lo[a], b[a]);
                hi[a] = std::max(hi[a], b[3 + a]);
                ext += b[3 + a] - b[a];
            }
        }
        const float diag = std::sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                                     (hi[2] - lo[2]) * (hi[2] - lo[2]));
        const float margin = 1e-4f * diag + 1e-6f;   // covers the reference's 1e-5 / 1e-6 tolerances
        cell = std::max((float)(ext / (3.0 * std::max(T, 1))), 1e-6f);
        for (int a = 0; a < 3; ++a) {
            lo[a] -= margin;
            dim[a] = std::max(1, (int)std::ceil((hi[a] + margin - lo[a]) / cell));
        }
        const size_t ncell = (size_t)dim[0] * dim[1] * dim[2];
        std::vector<int32_t> cnt(ncell + 1, 0);
        auto cells = [&](int t, auto&& fn) {
            const float* b = &bb[6 * (size_t)t];
            int c0[3], c1[3];
            for (int a = 0; a < 3; ++a) {
                c0[a] = std::max(0, std::min(dim[a] - 1, (int)std::floor((b[a] - margin - lo[a]) / cell)));
                c1[a] = std::max(0, std::min(dim[a] - 1, (int)std::floor((b[3 + a] + margin - lo[a]) / cell)));
            }
            for (int k = c0[2]; k <= c1[2]; ++k)
                for (int j = c0[1]; j <= c1[1]; ++j)
                    for (int i = c0[0]; i <= c1[0]; ++i) fn(((size_t)k * dim[1] + j) * dim[0] + i);
        };
        for (int t = 0; t < T; ++t) cells(t, [&](size_t c) { ++cnt[c + 1]; });
        for (size_t c = 0; c < ncell; ++c) cnt[c + 1] += cnt[c];
        start = cnt;
        items.assign(cnt[ncell], 0);
        std::vector<int32_t> fill(cnt.begin(), cnt.end() - 1);
        for (int t = 0; t < T; ++t) cells(t, [&](size_t c) { items[fill[c]++] = t; });   // ascending t per cell
    }
    // candidates of point p: [b, e) in items
    void range(const float* p, int& b, int& e) const {
        int c[3];
        for (int a = 0; a < 3; ++a) c[a] = std::max(0, std::min(dim[a] - 1, (int)std::floor((p[a] - lo[a]) / cell)));
        const size_t id = ((size_t)c[2] * dim[1] + c[1]) * dim[0] + c[0];
        b = start[id];
        e = start[id + 1];
    }
};

}  // namespace

void tl_barycentric(const float p[3], const float a[3], const float b[3], const float c[3], const float d[3],
                    float w[4]) {
    const V3f P = {p[0], p[1], p[2]}, A = {a[0], a[1], a[2]}, B = {b[0], b[1], b[2]}, C = {c[0], c[1], c[2]},
              D = {d[0], d[1], d[2]};
    const float V = dot(sub(B, A), cross(sub(C, A), sub(D, A))) / 6.0f;
    const V3f centre = mul(add(add(A, B), add(C, D)), 0.25f);
    const V3f v[4] = {A, B, C, D};
    for (int i = 0; i < 4; ++i) {
        const V3f q = v[i], f0 = v[(i + 1) % 4], f1 = v[(i + 2) % 4], f2 = v[(i + 3) % 4];
        V3f nrm = cross(sub(f1, f0), sub(f2, f0));
        if (dot(nrm, sub(q, f0)) > 0.f) nrm = mul(nrm, -1.f);   // outward: away from the opposite vertex
        const float l = len(nrm);
        const float area = l * 0.5f;
        nrm = mul(nrm, 1.f / l);
        w[i] = 0.25f - dot(sub(P, centre), nrm) * area / (3.f * V);
    }
}

bool tl_bind_fine_to_coarse(const float* fine_pos, int nf, const float* coarse_pos, const int32_t* coarse_tets, int tc,
                            std::vector<int32_t>& ids, std::vector<float>& w, std::string& err) {
    TetGrid g;
    g.build(coarse_pos, coarse_tets, tc);
    ids.assign(4 * (size_t)nf, -1);
    w.assign(4 * (size_t)nf, 0.f);
    for (int v = 0; v < nf; ++v) {
        const float* P = fine_pos + 3 * v;
        int b, e;
        g.range(P, b, e);
        bool found = false;
        for (int q = b; q < e && !found; ++q) {
            const int t = g.items[q];
            const int32_t* id = coarse_tets + 4 * t;
            float wt[4];
            tl_barycentric(P, coarse_pos + 3 * id[0], coarse_pos + 3 * id[1], coarse_pos + 3 * id[2],
                           coarse_pos + 3 * id[3], wt);
            bool inside = true;
            for (int k = 0; k < 4; ++k)
                if (wt[k] < -1e-5f || wt[k] > 1.f + 1e-5f) inside = false;
            if (!inside) continue;
            for (int k = 0; k < 4; ++k) {
                ids[4 * (size_t)v + k] = id[k];
                w[4 * (size_t)v + k] = wt[k];
            }
            found = true;
        }
        if (!found) {
            char buf[160];
            std::snprintf(buf, sizeof buf, "fine vertex %d lies in no coarse tet", v);
            err = buf;
            return false;
        }
    }
    return true;
}

bool tl_bind_coarse_to_fine(const float* coarse_pos, int nc, const float* fine_pos, const int32_t* fine_tets, int tf,
                            std::vector<int32_t>& ids, std::vector<float>& w, std::string& err) {
    // per fine tet: centre, outward face normals (face k opposite vertex k) and
    // areas, |volume| (InitVolumeConstraint, PDSolver.cpp:86-130)
    std::vector<float> centre(3 * (size_t)tf), fn(12 * (size_t)tf), fa(4 * (size_t)tf), vol(tf);
    for (int t = 0; t < tf; ++t) {
        const int32_t* id = fine_tets + 4 * t;
        V3f v[4];
        for (int k = 0; k < 4; ++k) v[k] = ld(fine_pos, id[k]);
        V3f c = {0.f, 0.f, 0.f};
        for (int k = 0; k < 4; ++k) c = add(c, v[k]);
        centre[3 * (size_t)t] = c.x / 4;
        centre[3 * (size_t)t + 1] = c.y / 4;
        centre[3 * (size_t)t + 2] = c.z / 4;
        static const int face[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
        for (int k = 0; k < 4; ++k) {
            const V3f A = v[face[k][0]], B = v[face[k][1]], C = v[face[k][2]], Dk = v[k];
            V3f nrm = cross(sub(B, A), sub(C, A));
            if (dot(nrm, sub(Dk, A)) > 0.f) nrm = mul(nrm, -1.f);
            const float l = len(nrm);
            fa[4 * (size_t)t + k] = 0.5f * l;
            fn[12 * (size_t)t + 3 * k] = nrm.x / l;
            fn[12 * (size_t)t + 3 * k + 1] = nrm.y / l;
            fn[12 * (size_t)t + 3 * k + 2] = nrm.z / l;
        }
        vol[t] = std::fabs(dot(sub(v[1], v[0]), cross(sub(v[2], v[0]), sub(v[3], v[0])))) / 6.0f;
    }
    TetGrid g;
    g.build(fine_pos, fine_tets, tf);
    ids.assign(4 * (size_t)nc, -1);
    w.assign(4 * (size_t)nc, 0.f);
    for (int v = 0; v < nc; ++v) {
        const V3f P = ld(coarse_pos, v);
        int b, e;
        g.range(coarse_pos + 3 * v, b, e);
        bool found = false;
        for (int q = b; q < e && !found; ++q) {
            const int t = g.items[q];
            const int32_t* id = fine_tets + 4 * t;
            bool inside = true;
            for (int k = 0; k < 4 && inside; ++k) {
                const V3f A = ld(fine_pos, id[(k + 1) % 4]);
                const V3f nrm = {fn[12 * (size_t)t + 3 * k], fn[12 * (size_t)t + 3 * k + 1], fn[12 * (size_t)t + 3 * k + 2]};
                if (dot(sub(P, A), nrm) > 1e-6f) inside = false;
            }
            if (!inside) continue;
            const V3f c = {centre[3 * (size_t)t], centre[3 * (size_t)t + 1], centre[3 * (size_t)t + 2]};
            for (int k = 0; k < 4; ++k) {
                const V3f nrm = {fn[12 * (size_t)t + 3 * k], fn[12 * (size_t)t + 3 * k + 1], fn[12 * (size_t)t + 3 * k + 2]};
                ids[4 * (size_t)v + k] = id[k];
                w[4 * (size_t)v + k] = 0.25f - dot(sub(P, c), nrm) * fa[4 * (size_t)t + k] / (3.f * vol[t]);
            }
            found = true;
        }
        if (!found) {
            char buf[160];
            std::snprintf(buf, sizeof buf, "coarse vertex %d lies in no fine tet", v);
            err = buf;
            return false;
        }
    }
    return true;
}

}  // namespace mgsb
