// C ABI of the host-side mesh utilities (see include/mgsb.h).
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/mgsb.h"
#include "mesh.hpp"

namespace {

mgsb_status export_mesh(const mgsb::HostMesh& m, mgsb_mesh_data** out) {
    mgsb_mesh_data* d = (mgsb_mesh_data*)std::calloc(1, sizeof(mgsb_mesh_data));
    if (!d) return MGSB_OUT_OF_MEMORY;
    d->num_verts = m.num_verts();
    d->num_tets = m.num_tets();
    d->positions = (float*)std::malloc(sizeof(float) * 3 * (size_t)(d->num_verts ? d->num_verts : 1));
    d->tets = (int32_t*)std::malloc(sizeof(int32_t) * 4 * (size_t)(d->num_tets ? d->num_tets : 1));
    if (!d->positions || !d->tets) {
        mgsb_mesh_free(d);
        return MGSB_OUT_OF_MEMORY;
    }
    for (size_t i = 0; i < m.pos.size(); ++i) d->positions[i] = (float)m.pos[i];
    if (!m.tets.empty()) std::memcpy(d->tets, m.tets.data(), m.tets.size() * sizeof(int32_t));
    for (int c = 0; c < 3; ++c) d->grid_dims[c] = m.grid_dims[c];
    *out = d;
    return MGSB_OK;
}

}  // namespace

extern "C" {

mgsb_status mgsb_mesh_box(int32_t nx, int32_t ny, int32_t nz, const float lo[3], const float hi[3], mgsb_mesh_data** out) {
    if (!out || !lo || !hi || nx <= 0 || ny <= 0 || nz <= 0) return MGSB_INVALID_ARG;
    if ((double)(nx + 1) * (ny + 1) * (nz + 1) > 2e9 || 6.0 * nx * ny * nz > 2e9) return MGSB_INVALID_ARG;
    for (int c = 0; c < 3; ++c)
        if (!(hi[c] > lo[c])) return MGSB_INVALID_ARG;
    const double l[3] = {lo[0], lo[1], lo[2]}, h[3] = {hi[0], hi[1], hi[2]};
    return export_mesh(mgsb::make_box(nx, ny, nz, l, h), out);
}

mgsb_status mgsb_mesh_blob(int32_t gx, int32_t gy, int32_t gz, float spacing, const float semi_axes[3], float noise_amp,
                           float noise_period, uint64_t seed, mgsb_mesh_data** out) {
    if (!out || !semi_axes || gx <= 0 || gy <= 0 || gz <= 0 || !(spacing > 0) || !(noise_period > 0)) return MGSB_INVALID_ARG;
    const double semi[3] = {semi_axes[0], semi_axes[1], semi_axes[2]};
    mgsb::HostMesh m = mgsb::make_blob(gx, gy, gz, spacing, semi, noise_amp, noise_period, seed);
    if (m.num_tets() == 0) return MGSB_INVALID_ARG;
    return export_mesh(m, out);
}

mgsb_status mgsb_mesh_read_msh(const char* path, mgsb_mesh_data** out) {
    if (!path || !out) return MGSB_INVALID_ARG;
    mgsb::HostMesh m;
    std::string err;
    if (!mgsb::read_msh(path, m, err)) return MGSB_IO_ERROR;
    return export_mesh(m, out);
}

mgsb_status mgsb_mesh_extract_surface(mgsb_mesh_data* m) {
    if (!m || !m->tets) return MGSB_INVALID_ARG;
    std::vector<int32_t> tris, opp;
    mgsb::extract_surface(m->tets, m->num_tets, tris, opp);
    std::free(m->tris);
    std::free(m->tri_opposite);
    m->num_tris = (int32_t)opp.size();
    m->tris = (int32_t*)std::malloc(sizeof(int32_t) * (tris.size() ? tris.size() : 1));
    m->tri_opposite = (int32_t*)std::malloc(sizeof(int32_t) * (opp.size() ? opp.size() : 1));
    if (!m->tris || !m->tri_opposite) return MGSB_OUT_OF_MEMORY;
    if (!tris.empty()) std::memcpy(m->tris, tris.data(), tris.size() * sizeof(int32_t));
    if (!opp.empty()) std::memcpy(m->tri_opposite, opp.data(), opp.size() * sizeof(int32_t));
    return MGSB_OK;
}

mgsb_status mgsb_mesh_free(mgsb_mesh_data* m) {
    if (!m) return MGSB_INVALID_ARG;
    std::free(m->positions);
    std::free(m->tets);
    std::free(m->tris);
    std::free(m->tri_opposite);
    std::free(m);
    return MGSB_OK;
}

double mgsb_value_noise(double x, double y, double z, double period, uint64_t seed) {
    return mgsb::value_noise(x, y, z, period, seed);
}

}  // extern "C"
