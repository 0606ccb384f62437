// Host-side plan of every device array a solver needs (no CUDA calls):
// precompute, RHS slot incidence, sliced-ELL matrices of all levels,
// prolongation / restriction operators, coarsest dense blocks.
#pragma once
#include <vector_types.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mgsb.h"
#include "setup.hpp"

namespace mgsb {

struct PlanBody {
    int V = 0, T = 0;
    int v_off = 0, t_off = 0;
    std::vector<double> rest;        // 3V
    std::vector<int32_t> tets;       // 4T (local ids)
    std::vector<float> youngs, poisson;
    std::vector<uint8_t> fixed;
    std::vector<int32_t> surface;    // surface vertex ids (local)
    int grid_dims[3] = {0, 0, 0};
    float gravity[3] = {0, 0, 0};
    float damping = 1.f;
    std::vector<TetRest> tr;
    std::vector<CoarseLevel> levels;  // multigrid levels 1..L-1
};

struct PlanLevel {
    int n = 0, nnz = 0;
    int S = 32;                      // slice height of the sliced ELL
    std::vector<int32_t> slice_ptr, ell_col;
    std::vector<float> ell_val, diag0;
    std::vector<double> ell_val64;   // level 0 only: FP64 copy for the mixed-precision residual
    // prolongation rows of the next finer level's vertices (coarse side = this level)
    std::vector<int4> pid;
    std::vector<float4> pw;
    // restriction CSR: children (finer vertices) of each vertex of this level
    std::vector<int32_t> rptr, rcol;
    std::vector<float> rw;
    // OP = Off(this level) * P(next coarser level) as sliced ELL with this
    // level's slice height; columns index the next coarser level (every level
    // but the coarsest).  With it the product A (d + P e) = A d + D (P e) + OP e
    // needs no neighbour of the prolonged vector: the prolongation and the first
    // post-smoothing sweep (or the learned cycle's post-smoothing residual) run
    // as one kernel from the residual of d.
    std::vector<int32_t> op_slice_ptr, op_col;
    std::vector<float> op_val;
    int op_nnz = 0;
    // level 1 only: RO = R * Off(level 0) as CSR over this level's rows
    // (columns: level-0 vertices, ascending).  With it the restriction of the
    // level-0 residual is R (b - D d) - RO d: the level-1 right-hand side comes
    // from b, D and d without the level-0 residual being formed first.
    std::vector<int32_t> ro_ptr, ro_col;
    std::vector<float> ro_val;
};

struct Plan {
    int N0 = 0, T = 0;
    std::vector<int32_t> body_of;
    std::vector<float> fixf, mass, diag;      // mg: mass = m/h^2, diag = L_ii; ref: density-1 mass, volume diagonal
    std::vector<int4> tets, slot_of;
    std::vector<float4> tA, tB;
    std::vector<float2> tC;
    std::vector<int32_t> slot_ptr;
    std::vector<PlanLevel> levels;            // [0] = finest (matrix only)
    std::vector<float> dense;                 // coarsest dense blocks (row-major per body)
    std::vector<double> dense64;              // the same in FP64
    std::vector<float> dense_inv;             // inverse of each block without contact (Woodbury base)
    std::vector<double> dense_inv64;
    std::vector<double> diag64;               // level-0 diagonal in FP64
    std::vector<uint8_t> is_surf;             // per vertex: on the boundary surface
    std::vector<int32_t> cl_off, cl_n, dense_off;
    std::vector<int2> range;                  // [body * L + level]: (first row, rows)
    int max_coarsest = 0;
    std::vector<int32_t> surf;                // global surface vertex ids
    // body-0 precompute for export
    std::vector<float> h_inv, h_ac, h_vol, h_mass, h_diag;
};

// Sliced ELL (slices of S rows, column-major inside a slice: entry k of row r
// at sptr[r / S] + k * S + r % S) from CSR rows.
// Padding entries get a zero coefficient and column pad_col[r] (default: the
// row itself, valid when rows and columns index the same level).
void build_ell(const std::vector<int32_t>& ptr, const std::vector<int32_t>& col, const std::vector<double>& val, int n,
               int S, std::vector<int32_t>& sptr, std::vector<int32_t>& ecol, std::vector<float>& eval,
               const std::vector<int32_t>* pad_col = nullptr);

constexpr int kSliceL0 = 8;       // 4 lanes per row at level 0
constexpr int kSliceCoarse = 4;   // 8 lanes per row on coarse levels

// Copies a mesh into a body (rest data, default material, no fixed vertex,
// surface vertices for the multigrid kind).  Returns a status.
mgsb_status make_body(const mgsb_mesh& m, const mgsb_params& p, bool multigrid, PlanBody& B, std::string& err);

// Builds the plan; also (re)builds each body's multigrid hierarchy.
bool build_plan(std::vector<PlanBody>& bodies, const mgsb_params& p, Plan& out, std::string& err);

}  // namespace mgsb
