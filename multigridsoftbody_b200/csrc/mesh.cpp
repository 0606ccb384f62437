// Host-side mesh generation and I/O (no GPU code).
#include "mesh.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <unordered_map>

namespace mgsb {

// Axis permutations with their parity; tet = path (0,0,0) -> +e_p0 -> +e_p1 -> (1,1,1).
static const int kPerm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
static const int kPermOdd[6] = {0, 1, 1, 0, 0, 1};

void kuhn_split(const int32_t corner[8], int32_t out[6][4]) {
    for (int t = 0; t < 6; ++t) {
        int c[3] = {0, 0, 0};
        int ids[4];
        ids[0] = corner[0];
        for (int s = 0; s < 3; ++s) {
            c[kPerm[t][s]] = 1;
            ids[s + 1] = corner[c[0] + 2 * c[1] + 4 * c[2]];
        }
        // det[e_p0, e_p0+e_p1, e_p0+e_p1+e_p2] = sign(perm); swap v1,v2 for odd perms.
        if (kPermOdd[t]) std::swap(ids[1], ids[2]);
        for (int s = 0; s < 4; ++s) out[t][s] = ids[s];
    }
}

HostMesh make_box(int nx, int ny, int nz, const double lo[3], const double hi[3]) {
    HostMesh m;
    const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
    m.pos.resize((size_t)3 * vx * vy * vz);
    auto vid = [&](int i, int j, int k) { return (int32_t)(i + vx * (k + vz * j)); };
    for (int j = 0; j < vy; ++j)
        for (int k = 0; k < vz; ++k)
            for (int i = 0; i < vx; ++i) {
                const int32_t v = vid(i, j, k);
                // Evaluate as lo + (hi-lo)*i/n so the end faces are exact.
                m.pos[3 * v + 0] = (i == nx) ? hi[0] : lo[0] + (hi[0] - lo[0]) * (double)i / nx;
                m.pos[3 * v + 1] = (j == ny) ? hi[1] : lo[1] + (hi[1] - lo[1]) * (double)j / ny;
                m.pos[3 * v + 2] = (k == nz) ? hi[2] : lo[2] + (hi[2] - lo[2]) * (double)k / nz;
            }
    m.tets.reserve((size_t)24 * nx * ny * nz);
    for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k)
            for (int i = 0; i < nx; ++i) {
                int32_t corner[8];
                for (int c = 0; c < 8; ++c) corner[c] = vid(i + (c & 1), j + ((c >> 1) & 1), k + ((c >> 2) & 1));
                int32_t tt[6][4];
                kuhn_split(corner, tt);
                for (int t = 0; t < 6; ++t)
                    for (int s = 0; s < 4; ++s) m.tets.push_back(tt[t][s]);
            }
    m.grid_dims[0] = nx;
    m.grid_dims[1] = ny;
    m.grid_dims[2] = nz;
    return m;
}

// splitmix64 finaliser as the lattice hash.
static inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline double lattice_value(int64_t i, int64_t j, int64_t k, uint64_t seed) {
    uint64_t h = mix64(seed);
    h = mix64(h ^ (uint64_t)i);
    h = mix64(h ^ (uint64_t)j);
    h = mix64(h ^ (uint64_t)k);
    return (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;  // [-1, 1)
}

static inline double smooth(double t) { return t * t * (3.0 - 2.0 * t); }

double value_noise(double x, double y, double z, double period, uint64_t seed) {
    const double u = x / period, v = y / period, w = z / period;
    const double fu = std::floor(u), fv = std::floor(v), fw = std::floor(w);
    const int64_t i = (int64_t)fu, j = (int64_t)fv, k = (int64_t)fw;
    const double a = smooth(u - fu), b = smooth(v - fv), c = smooth(w - fw);
    double acc = 0.0;
    for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
            for (int di = 0; di < 2; ++di) {
                const double wt = (di ? a : 1 - a) * (dj ? b : 1 - b) * (dk ? c : 1 - c);
                acc += wt * lattice_value(i + di, j + dj, k + dk, seed);
            }
    return acc;
}

HostMesh make_blob(int gx, int gy, int gz, double spacing, const double semi[3], double amp, double period,
                   uint64_t seed) {
    HostMesh m;
    const double ox = -0.5 * gx * spacing, oy = -0.5 * gy * spacing, oz = -0.5 * gz * spacing;
    const int vx = gx + 1, vy = gy + 1, vz = gz + 1;
    std::vector<int32_t> remap((size_t)vx * vy * vz, -1);
    auto gid = [&](int i, int j, int k) { return (size_t)i + (size_t)vx * ((size_t)k + (size_t)vz * j); };
    std::vector<std::array<int, 3>> kept;
    for (int j = 0; j < gy; ++j)
        for (int k = 0; k < gz; ++k)
            for (int i = 0; i < gx; ++i) {
                const double x = ox + (i + 0.5) * spacing, y = oy + (j + 0.5) * spacing, z = oz + (k + 0.5) * spacing;
                const double e = (x / semi[0]) * (x / semi[0]) + (y / semi[1]) * (y / semi[1]) +
                                 (z / semi[2]) * (z / semi[2]);
                if (e < 1.0 + amp * value_noise(x, y, z, period, seed)) kept.push_back({i, j, k});
            }
    // Mark used grid nodes, number them in grid order (y slowest, then z, then x).
    for (auto& c : kept)
        for (int q = 0; q < 8; ++q) remap[gid(c[0] + (q & 1), c[1] + ((q >> 1) & 1), c[2] + ((q >> 2) & 1))] = 0;
    int32_t nv = 0;
    for (int j = 0; j < vy; ++j)
        for (int k = 0; k < vz; ++k)
            for (int i = 0; i < vx; ++i) {
                const size_t g = gid(i, j, k);
                if (remap[g] < 0) continue;
                remap[g] = nv++;
                m.pos.push_back(ox + i * spacing);
                m.pos.push_back(oy + j * spacing);
                m.pos.push_back(oz + k * spacing);
            }
    for (auto& c : kept) {
        int32_t corner[8];
        for (int q = 0; q < 8; ++q) corner[q] = remap[gid(c[0] + (q & 1), c[1] + ((q >> 1) & 1), c[2] + ((q >> 2) & 1))];
        int32_t tt[6][4];
        kuhn_split(corner, tt);
        for (int t = 0; t < 6; ++t)
            for (int s = 0; s < 4; ++s) m.tets.push_back(tt[t][s]);
    }
    m.grid_dims[0] = gx;
    m.grid_dims[1] = gy;
    m.grid_dims[2] = gz;
    return m;
}

bool read_msh(const std::string& path, HostMesh& out, std::string& err) {
    std::ifstream f(path);
    if (!f) {
        err = "cannot open " + path;
        return false;
    }
    out = HostMesh();
    std::string tok;
    bool have_nodes = false;
    while (f >> tok) {
        if (tok == "$Nodes") {
            long n = 0;
            f >> n;
            if (!f || n < 0) {
                err = "bad $Nodes count";
                return false;
            }
            out.pos.resize((size_t)3 * n);
            for (long i = 0; i < n; ++i) {
                long idx;
                double x, y, z;
                f >> idx >> x >> y >> z;
                if (!f) {
                    err = "truncated $Nodes";
                    return false;
                }
                // Nodes are stored in file order, as the reference does (it ignores idx).
                out.pos[3 * i + 0] = x;
                out.pos[3 * i + 1] = y;
                out.pos[3 * i + 2] = z;
            }
            have_nodes = true;
        } else if (tok == "$Elements") {
            long n = 0;
            f >> n;
            for (long e = 0; e < n; ++e) {
                long idx, type, ntags;
                f >> idx >> type >> ntags;
                if (!f || ntags < 0) {
                    err = "bad element header";
                    return false;
                }
                for (long t = 0; t < ntags; ++t) {
                    long tag;
                    f >> tag;
                }
                int nnodes = 0;
                switch (type) {
                    case 15: nnodes = 1; break;  // point
                    case 1: nnodes = 2; break;   // line
                    case 2: nnodes = 3; break;   // triangle
                    case 3: nnodes = 4; break;   // quad
                    case 4: nnodes = 4; break;   // tet
                    case 5: nnodes = 8; break;   // hex
                    case 6: nnodes = 6; break;   // prism
                    case 7: nnodes = 5; break;   // pyramid
                    default: err = "unsupported gmsh element type " + std::to_string(type); return false;
                }
                long ids[8];
                for (int q = 0; q < nnodes; ++q) f >> ids[q];
                if (!f) {
                    err = "truncated $Elements";
                    return false;
                }
                if (type == 4)
                    for (int q = 0; q < 4; ++q) out.tets.push_back((int32_t)(ids[q] - 1));
            }
        }
    }
    if (!have_nodes) {
        err = "no $Nodes section";
        return false;
    }
    const long nv = (long)out.pos.size() / 3;
    for (int32_t v : out.tets)
        if (v < 0 || v >= nv) {
            err = "tet index out of range";
            return false;
        }
    return true;
}

void extract_surface(const int32_t* tets, int num_tets, std::vector<int32_t>& tris, std::vector<int32_t>& opposite) {
    struct Face {
        int32_t key[3];   // sorted ascending
        int32_t f[3];     // as emitted (outward for positively oriented tets)
        int32_t opp;
    };
    std::vector<Face> faces;
    faces.reserve((size_t)num_tets * 4);
    for (int t = 0; t < num_tets; ++t) {
        const int32_t* v = tets + 4 * t;
        const int32_t fv[4][4] = {{v[0], v[2], v[1], v[3]}, {v[0], v[1], v[3], v[2]}, {v[0], v[3], v[2], v[1]},
                                  {v[1], v[2], v[3], v[0]}};
        for (int q = 0; q < 4; ++q) {
            Face fc;
            for (int s = 0; s < 3; ++s) fc.f[s] = fc.key[s] = fv[q][s];
            fc.opp = fv[q][3];
            std::sort(fc.key, fc.key + 3);
            faces.push_back(fc);
        }
    }
    // Descending lexicographic order of the sorted key; stable so that for a
    // repeated key the first occurrence comes first.
    std::stable_sort(faces.begin(), faces.end(), [](const Face& a, const Face& b) {
        if (a.key[0] != b.key[0]) return a.key[0] > b.key[0];
        if (a.key[1] != b.key[1]) return a.key[1] > b.key[1];
        return a.key[2] > b.key[2];
    });
    tris.clear();
    opposite.clear();
    size_t i = 0;
    while (i < faces.size()) {
        size_t j = i + 1;
        while (j < faces.size() && faces[j].key[0] == faces[i].key[0] && faces[j].key[1] == faces[i].key[1] &&
               faces[j].key[2] == faces[i].key[2])
            ++j;
        if (j - i == 1) {
            for (int s = 0; s < 3; ++s) tris.push_back(faces[i].f[s]);
            opposite.push_back(faces[i].opp);
        }
        i = j;
    }
}

}  // namespace mgsb
