// Host-side mesh generation and I/O.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace mgsb {

struct HostMesh {
    std::vector<double> pos;      // 3V
    std::vector<int32_t> tets;    // 4T
    std::vector<int32_t> tris;    // 3F boundary faces
    std::vector<int32_t> tri_opposite;
    int32_t grid_dims[3] = {0, 0, 0};
    int num_verts() const { return (int)(pos.size() / 3); }
    int num_tets() const { return (int)(tets.size() / 4); }
};

// Box [lo,hi] -> nx*ny*nz hexes, each split into 6 Kuhn (Freudenthal) tets
// sharing the hex's (0,0,0)-(1,1,1) diagonal; tets positively oriented.
// Vertex id of grid node (i,j,k) = i + (nx+1)*(k + (nz+1)*j).
HostMesh make_box(int nx, int ny, int nz, const double lo[3], const double hi[3]);

// Voxel blob (see mgsb_mesh_blob in mgsb.h).
HostMesh make_blob(int gx, int gy, int gz, double spacing, const double semi[3], double amp, double period,
                   uint64_t seed);

double value_noise(double x, double y, double z, double period, uint64_t seed);

// gmsh 2.2 ASCII: $Nodes and $Elements (type 4 = tet; type 2 triangles skipped),
// indices 1-based in the file.  Returns false with err set on failure.
bool read_msh(const std::string& path, HostMesh& out, std::string& err);

// Boundary faces with the vertex opposite each face; a face is boundary when it
// occurs in exactly one tet.  Face order: by sorted vertex triple, descending
// lexicographic (the iteration order of the reference's std::set<FaceKey>).
void extract_surface(const int32_t* tets, int num_tets, std::vector<int32_t>& tris,
                     std::vector<int32_t>& opposite);

// The 6 Kuhn tets of a hex whose corner (a,b,c) has id corner[a + 2b + 4c].
void kuhn_split(const int32_t corner[8], int32_t out[6][4]);

}  // namespace mgsb
