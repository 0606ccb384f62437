/*
 * FP64 CPU oracle for the PD soft-body frame — TEST INFRASTRUCTURE ONLY.
 *
 * Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
 * the checker; never linked into or called by the product library.
 *
 * Two modes (params->solver):
 *   MGSB_SOLVER_REFERENCE_JACOBI — restatement in FP64 of the reference frame
 *     (buuugyellow/MultiGridSoftBody, MultiGridSoftBody/src):
 *       precompute            PDSolver.cpp:12-132 (density 1 lumped mass)
 *       inertial prediction   PDSolver.cu:72-116  (calculateST)
 *       sphere DCD            PDSolver.cu:277-331 (DCDByPoint_sphere)
 *       local step            PDSolverAc.cu:447-662 (getTetFRV2 + calTetIFV1)
 *       polar decomposition   utils.cu:123-226   (GetRotation_D)
 *       Jacobi + Chebyshev    PDSolver.cu:192-235, PDSolver.cpp:261-271
 *       velocity              PDSolver.cu:245-252
 *       energy diagnostics    PDSolver.cu:816-924 (runCalEnergy)
 *   MGSB_SOLVER_MULTIGRID — PD with a V-cycle global step exactly as
 *     configured (levels, sweeps, Galerkin operators on Kuhn voxel grids,
 *     lumped contact weights, dense Cholesky coarsest), corotational strain
 *     constraints with weight 2*mu*V, capsule contacts detected once per
 *     frame on the predicted positions.
 */
#ifndef MGSB_ORACLE_H_
#define MGSB_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#include "../include/mgsb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_solver oracle_solver;

oracle_solver* oracle_create(const mgsb_mesh* mesh, const mgsb_params* params, char* err, int errlen);
void oracle_destroy(oracle_solver* h);
int oracle_set_fixed(oracle_solver* h, const uint8_t* mask);
int oracle_set_material(oracle_solver* h, const float* youngs, const float* poisson);
/* Capsule narrow phase: 0 vertices, 1 vertices and surface triangles
 * (the rule of mgsb_set_surface_contact). */
int oracle_set_surface_contact(oracle_solver* h, int mode);
/* Distance between segment p0p1[6] and triangle abc[9], closest points q
 * (segment) and h (triangle). */
double oracle_segment_triangle(const double* p0p1, const double* abc, double* q, double* h);
/* Parameters changed between frames (same rules as mgsb_set_params). */
int oracle_set_params(oracle_solver* h, const mgsb_params* params);
int oracle_set_tool_capsule(oracle_solver* h, const float a[3], const float b[3], float radius);
int oracle_set_tool_spheres(oracle_solver* h, int32_t count, const float* centers, const float* radii,
                            const uint8_t* active);
int oracle_step(oracle_solver* h);
int oracle_num_verts(const oracle_solver* h);
void oracle_get_positions(const oracle_solver* h, double* out);
void oracle_get_velocities(const oracle_solver* h, double* out);
void oracle_get_contact_flags(const oracle_solver* h, int32_t* out);
void oracle_get_collision_depth(const oracle_solver* h, double* out);
void oracle_set_state(oracle_solver* h, const double* positions, const double* velocities);
/* inv [9T], ac [12T], volume [T], mass [V], diag [V]; NULL allowed. */
void oracle_get_precompute(const oracle_solver* h, double* inv, double* ac, double* volume, double* mass,
                           double* diag);
/* Ek, Ep, Ec, Nc, dX as in runCalEnergy. */
void oracle_get_energy(const oracle_solver* h, double out[5]);
/* Fine-level residual norm of the PD global system after the last iteration. */
double oracle_last_residual(const oracle_solver* h);
/* Host threads of the OpenMP loops (n <= 0: all); returns the count in force. */
int oracle_set_threads(int n);

/* Hierarchy inspection (level >= 1): sizes, and the Galerkin matrix in CSR
 * with the diagonal first in each row. */
int oracle_level_size(const oracle_solver* h, int level, int32_t* n, int32_t* nnz_offdiag);
int oracle_level_prolongation(const oracle_solver* h, int level, int32_t* ids, double* w);
int oracle_level_matrix(const oracle_solver* h, int level, double* diag, int32_t* ptr, int32_t* col, double* val);

/* Two-level schedule of the reference (PDSolver_MG): a coarse and a fine
 * reference-kind solver; level 0 = fine, 1 = coarse (use the oracle_solver
 * calls on oracle_mg2_level for fixed sets, spheres and readback). */
typedef struct oracle_mg2 oracle_mg2;
oracle_mg2* oracle_mg2_create(const mgsb_mesh* coarse, const mgsb_mesh* fine, const mgsb_params* params, char* err,
                              int errlen);
void oracle_mg2_destroy(oracle_mg2* h);
oracle_solver* oracle_mg2_level(oracle_mg2* h, int level);
void oracle_mg2_step(oracle_mg2* h);

/* Pure functions. */
/* Vertex normals of a triangle surface: UpdateTriNormal + AvgOutsideTetVertNormal
 * (PDSolver.cu:394-460).  pos [3V], tris [3F]; out [3V], zero where no triangle. */
void oracle_surface_normals(const double* pos, int32_t V, const int32_t* tris, int32_t F, double* out);
/* Learned-smoother MLP 9 -> 64 -> 64 -> 3 (GELU, tanh form), parameters in the libmgsb
 * layout W1[64][9] b1[64] W2[64][64] b2[64] W3[3][64] b3[3].  With bf16 != 0
 * the weights (not the biases), the inputs and the hidden activations are
 * rounded to BF16 (round to nearest even) as on the tensor cores, and the
 * gradient passes straight through the roundings. */
void oracle_mlp_forward(const double* params, const double* x, int32_t n, int32_t bf16, double* y);
/* Mean over samples and outputs of (y - t)^2 and its gradient. */
double oracle_mlp_loss_grad(const double* params, const double* x, const double* t, int32_t n, int32_t bf16,
                            double* grad);
void oracle_ref_rotation(const double F[9], double R[9]);
void oracle_svd_rotation(const double F[9], double R[9]);
double oracle_inverse3(const double A[9], double R[9]);

#ifdef __cplusplus
}
#endif

#endif
