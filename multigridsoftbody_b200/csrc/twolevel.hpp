// Binding between the two meshes of the reference's two-level schedule
// (PDSolver_MG::Init / interpolate, PDSolver_MG.cpp:5-181): every fine vertex
// to the coarse tet that contains it (barycentric weights, tolerance 1e-5), and
// every coarse vertex to the fine tet that contains it (face-plane test, then
// face-area barycentric weights).  FP32 like the reference; the first
// containing tet in index order wins, found through a uniform grid over the tet
// bounding boxes instead of the reference's O(V*T) scan (same result).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace mgsb {

// Barycentric weights of p in tet (a, b, c, d) — barycentricCoordinate
// (utils.cu:335-364): signed volume V = ab.(ac x ad)/6, per vertex i the
// outward normal n_i of the opposite face and its area F_i,
// w_i = 1/4 - (p - centre).n_i F_i / (3 V).
void tl_barycentric(const float p[3], const float a[3], const float b[3], const float c[3], const float d[3],
                    float w[4]);

// ids[4 * v], w[4 * v] for every fine vertex; false (with err) if a vertex lies
// in no coarse tet.
bool tl_bind_fine_to_coarse(const float* fine_pos, int nf, const float* coarse_pos, const int32_t* coarse_tets, int tc,
                            std::vector<int32_t>& ids, std::vector<float>& w, std::string& err);

// ids[4 * v], w[4 * v] for every coarse vertex (PDSolver_MG.cpp:120-167 with
// pointInTet, utils.cu:298-311, and the face-area barycentric form,
// utils.cu:313-333); false (with err) if a vertex lies in no fine tet.
bool tl_bind_coarse_to_fine(const float* coarse_pos, int nc, const float* fine_pos, const int32_t* fine_tets, int tf,
                            std::vector<int32_t>& ids, std::vector<float>& w, std::string& err);

}  // namespace mgsb
