// Host-side FP64 precompute: per-tet rest data, lumped mass, the scalar PD
// system matrix and the geometric-multigrid hierarchy.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace mgsb {

// Rest data of one tet.  Dm = [X1-X0, X2-X0, X3-X0] (columns), inv = Dm^-1
// (row-major).  F = Ds(x) * inv = sum_j x_j g_j^T with g_k = row k-1 of inv
// (k=1..3) and g_0 = -(g_1+g_2+g_3): the columns of the reference's 3x4 "Ac"
// matrix (PDSolver.cpp:53-64).
struct TetRest {
    double inv[9];
    double det;      // det Dm (signed)
    double volume;   // |det|/6
    double g[4][3];
};

// Inverse by adjugate / determinant, laid out like Matrix_Inverse_3
// (utils.cu:233-252).  Returns the determinant.
double inverse3(const double A[9], double R[9]);

bool tet_rest(const double* pos, const int32_t* tets, int num_tets, std::vector<TetRest>& out, std::string& err);

// Compressed sparse rows with the diagonal kept apart: row i has off-diagonal
// entries col[ptr[i]..ptr[i+1]) and diagonal diag[i].
struct SparseSym {
    int n = 0;
    std::vector<int32_t> ptr, col;
    std::vector<double> val, diag;
};

// L = diag(mass)/dt^2 + sum_t w_t G_t^T G_t  (scalar; the 3-D system is L (x) I3).
void assemble_pd_matrix(const std::vector<TetRest>& rest, const int32_t* tets, int num_verts, const double* w,
                        const double* mass, double dt, SparseSym& L);

// One coarse level of the hierarchy for one body.
struct CoarseLevel {
    int n = 0;                      // coarse vertices
    int dims[3] = {0, 0, 0};        // hex counts of this level's grid
    std::vector<double> pos;        // 3n, grid node positions
    // Prolongation from this level to the next finer one: 4 (id, weight) per
    // finer vertex; weight 0 for fixed/inactive finer vertices.
    std::vector<int32_t> p_ids;     // 4 * n_finer
    std::vector<double> p_w;        // 4 * n_finer
    SparseSym A;                    // Galerkin operator P^T A_finer P
    std::vector<uint8_t> active;    // n; 0 = no free finer support
};

// Grid hex counts of level 1.. derived by halving (ceil) dims0 per axis.
// Each coarse level is a Kuhn-split voxel grid over the body's bounding box
// keeping the hexes that contain a finer-level vertex; finer vertices are
// interpolated barycentrically inside the Kuhn tet that contains them.
void build_hierarchy(const double* pos, int num_verts, const SparseSym& A0, const uint8_t* fixed, int levels,
                     const int dims0[3], std::vector<CoarseLevel>& out);

// Default finest grid dims from the bounding box and the mean tet edge length.
void default_grid_dims(const double* pos, int num_verts, const int32_t* tets, int num_tets, int dims[3]);

// Row-major dense copy of a level matrix; inactive rows/cols become identity.
void dense_from_sparse(const SparseSym& A, const std::vector<uint8_t>& active, std::vector<double>& dense);
// Inverse of a row-major SPD matrix (Cholesky in FP64); false if not SPD.
bool spd_inverse(const std::vector<double>& A, int n, std::vector<double>& inv);

}  // namespace mgsb
