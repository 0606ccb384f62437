/*
 * mgsb.h — C ABI of the B200-native projective-dynamics (PD) soft-body solver.
 *
 * One handle owns one or more independent bodies ("a batch"); a single-body
 * solver is a batch of one.  Every entry point takes plain pointers and sizes;
 * no CUDA or C++ types cross the boundary (the optional stream is a void*).
 *
 * Each entry point names the reference interface it replaces
 * (buuugyellow/MultiGridSoftBody, paths relative to MultiGridSoftBody/src).
 *
 * Two solver kinds are offered:
 *   MGSB_SOLVER_REFERENCE_JACOBI — the reference's frame: inertial prediction,
 *     per-iteration sphere DCD, corotational local step with the invariant-based
 *     polar decomposition, one under-relaxed diagonal-Jacobi update with
 *     Chebyshev acceleration (PDSolver.cpp:243-293).  Same constants, same
 *     clamps; float atomics replaced by an ordered gather.
 *   MGSB_SOLVER_MULTIGRID — PD with a geometric-multigrid V-cycle global step
 *     (Galerkin levels, sliced-ELL Jacobi smoother, dense Cholesky coarsest),
 *     E/nu material, capsule tool contacts as projection constraints, optional
 *     FP64 iterative refinement.
 *
 * Threading: one handle per host thread; no global state.
 * Errors: every call returns mgsb_status; mgsb_last_error_string() explains.
 */
#ifndef MGSB_H_
#define MGSB_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MGSB_ABI_VERSION 1

typedef enum mgsb_status {
    MGSB_OK = 0,
    MGSB_INVALID_ARG = 1,
    MGSB_DEGENERATE_TET = 2,   /* replaces exit(0) in Matrix_Inverse_3, utils.cu:244-247 */
    MGSB_CUDA_ERROR = 3,
    MGSB_DIVERGED = 4,         /* non-finite positions detected after a frame */
    MGSB_TIMEOUT = 5,
    MGSB_NOT_SUPPORTED = 6,
    MGSB_OUT_OF_MEMORY = 7,
    MGSB_IO_ERROR = 8
} mgsb_status;

typedef enum mgsb_solver_kind {
    MGSB_SOLVER_REFERENCE_JACOBI = 0,
    MGSB_SOLVER_MULTIGRID = 1
} mgsb_solver_kind;

typedef enum mgsb_precision {
    MGSB_PRECISION_FP32 = 0,   /* everything FP32 */
    MGSB_PRECISION_MIXED = 1   /* FP64 outer residual + positions, FP32 V-cycle correction */
} mgsb_precision;

/* Tetrahedral mesh (host memory, copied at create).
 * Replaces the vectors handed to PDSolver::Init, PDSolver.h:102. */
typedef struct mgsb_mesh {
    int32_t num_verts;
    int32_t num_tets;
    const float* positions;   /* [3*num_verts] xyz */
    const int32_t* tets;      /* [4*num_tets], 0-based */
    /* Optional structured-grid hint used to build the multigrid hierarchy.
     * grid_dims = hex counts of the finest voxel grid that generated the
     * mesh (0,0,0 = derive from the bounding box and mean edge length). */
    int32_t grid_dims[3];
} mgsb_mesh;

/* Solver parameters.  Replaces the constants set in PDSolver::Init
 * (PDSolver.cpp:166-176) and the public fields PDSolver.h:72-81. */
typedef struct mgsb_params {
    int32_t solver;             /* mgsb_solver_kind */
    int32_t iterations;         /* PD local/global iterations per frame (m_iterNum) */
    float dt;                   /* m_dt */
    float damping;              /* m_damping, velocity scale per frame */
    float gravity[3];           /* m_gravity{X,Y,Z} */
    /* reference-Jacobi kind */
    float volume_stiffness;     /* m_volumnStiffness (k) */
    float collision_stiffness;  /* m_collisionStiffness */
    float cheb_rho;             /* m_rho */
    float relaxation;           /* under-relaxation factor, 0.6 in calculatePOS */
    /* multigrid kind */
    float density;              /* kg/m^3 */
    float youngs_modulus;       /* default E for every tet (Pa) */
    float poisson_ratio;        /* default nu for every tet */
    float contact_stiffness;    /* weight of a contact projection constraint */
    int32_t levels;             /* multigrid levels incl. the finest */
    int32_t pre_sweeps;
    int32_t post_sweeps;
    float jacobi_omega;         /* weighted-Jacobi factor */
    int32_t precision;          /* mgsb_precision */
    int32_t refinement_passes;  /* V-cycles per PD iteration (mixed: FP64 refinement passes) */
    int32_t use_graph;          /* capture the frame in a CUDA graph */
    int32_t device;             /* CUDA device ordinal */
    void* stream;               /* cudaStream_t, NULL = solver-owned stream */
} mgsb_params;

/* Fill defaults for a solver kind.  Reference-Jacobi defaults are the
 * reference's own (20 iterations, dt 1/60, damping 0.95, k 8000, k_c 1000,
 * rho 0.9992, gravity -9.8 y, relaxation 0.6). */
mgsb_status mgsb_default_params(int32_t solver_kind, mgsb_params* out);

typedef struct mgsb_solver mgsb_solver;

/* Create one body.  Replaces PDSolver::Init (PDSolver.cpp:164-200) incl.
 * InitVolumeConstraint (PDSolver.cpp:12-132) and PDSolverData::Init
 * (PDSolver.cu:9-70). */
mgsb_status mgsb_create(const mgsb_mesh* mesh, const mgsb_params* params, mgsb_solver** out);

/* Create a batch of independent bodies that advance in one launch per phase.
 * params[i].solver must be MGSB_SOLVER_MULTIGRID and all bodies share
 * iterations/levels/sweeps/precision/dt of params[0]; material, gravity and
 * tool are per body.  No reference counterpart (the reference has one body). */
mgsb_status mgsb_batch_create(int32_t num_bodies, const mgsb_mesh* meshes, const mgsb_params* params,
                              mgsb_solver** out);

/* Frees all device memory.  The reference never frees (PDSolverData). */
mgsb_status mgsb_destroy(mgsb_solver* h);

mgsb_status mgsb_num_bodies(const mgsb_solver* h, int32_t* n);
mgsb_status mgsb_num_verts(const mgsb_solver* h, int32_t body, int32_t* n);
mgsb_status mgsb_num_tets(const mgsb_solver* h, int32_t body, int32_t* n);

/* Per-tet material (multigrid kind).  E, nu: [num_tets of body].
 * No reference counterpart (single scalar k, PDSolver.cpp:170). */
mgsb_status mgsb_set_material(mgsb_solver* h, int32_t body, const float* youngs, const float* poisson);

/* Change the solver's parameters between frames: the reference's public fields
 * m_iterNum, m_dt, m_damping, m_volumnStiffness, m_collisionStiffness, m_rho,
 * m_gravity{X,Y,Z} (PDSolver.h:72-81), which callers assign after Init, plus
 * the multigrid kind's density, contact weight, levels, sweep counts, Jacobi
 * factor, refinement passes and graph use.  Gravity and damping apply to every
 * body of a batch.  A changed youngs_modulus / poisson_ratio sets every tet of
 * every body to it (replacing mgsb_set_material); unchanged ones keep the
 * per-tet material.  The solver kind, precision, device and stream are fixed
 * at create (MGSB_NOT_SUPPORTED).  Invalid values: MGSB_INVALID_ARG, nothing
 * changed.  Waits for the solver's stream; the next step rebuilds the derived
 * data and the frame's CUDA graph.  Positions and velocities are kept. */
mgsb_status mgsb_set_params(mgsb_solver* h, const mgsb_params* params);
/* The parameters in force (the reference's public fields, read back). */
mgsb_status mgsb_get_params(const mgsb_solver* h, mgsb_params* out);

/* Fixed-vertex mask, 1 = fixed.  Replaces PDSolver::SetFixedVert
 * (PDSolver.cpp:134-162; flag 0.0f = fixed there). */
mgsb_status mgsb_set_fixed(mgsb_solver* h, int32_t body, const uint8_t* mask);

/* Capsule tool of a body (segment a-b, radius).  radius <= 0 disables it.
 * Replaces the sphere collider pose read in PDSolver::DCDByPoint
 * (PDSolver.cpp:228-233) / SphereCollider::MoveDelta (Collider.cpp:9-17);
 * CapsuleCollider is declared but unimplemented there (Collider.h:22-30). */
mgsb_status mgsb_set_tool_capsule(mgsb_solver* h, int32_t body, const float a[3], const float b[3], float radius);
/* All bodies at once: a[3n], b[3n], radius[n] (one host->device copy). */
mgsb_status mgsb_set_tool_capsules(mgsb_solver* h, const float* a, const float* b, const float* radius);

/* Sphere colliders for the reference-Jacobi kind (up to 8; active flag per
 * sphere).  Replaces g_simulator->m_sphereColliders (Simulator.cpp:57) as
 * read by DCDByPoint_sphere (PDSolver.cu:277-331). */
mgsb_status mgsb_set_tool_spheres(mgsb_solver* h, int32_t count, const float* centers, const float* radii,
                                  const uint8_t* active);

/* Advance one frame.  Replaces PDSolver::Step (PDSolver.cpp:243-293). */
mgsb_status mgsb_step(mgsb_solver* h);
/* Advance n frames back to back (tool pose fixed). */
mgsb_status mgsb_step_n(mgsb_solver* h, int32_t n);
/* Block until the solver's stream is idle. */
mgsb_status mgsb_synchronize(mgsb_solver* h);

/* Readback.  Replaces runCpyTetVertForRender (PDSolver.cu:261-268). */
mgsb_status mgsb_get_positions(mgsb_solver* h, int32_t body, float* out /* [3*V] */);
mgsb_status mgsb_get_velocities(mgsb_solver* h, int32_t body, float* out /* [3*V] */);
/* Positions of every body, concatenated in body order (one copy). */
mgsb_status mgsb_get_all_positions(mgsb_solver* h, float* out);
/* FP64 master positions (mixed precision only). */
mgsb_status mgsb_get_positions_f64(mgsb_solver* h, int32_t body, double* out);
/* Per-vertex contact flag (1 = in contact this frame) — m_tetVertIsCollide. */
mgsb_status mgsb_get_contact_flags(mgsb_solver* h, int32_t body, int32_t* out /* [V] */);
/* Contact flags of every body, concatenated in body order (one copy).  No
 * reference counterpart (the reference simulates one body). */
mgsb_status mgsb_get_all_contact_flags(mgsb_solver* h, int32_t* out /* [sum V] */);
/* The frame's result in one readback: positions (as mgsb_get_all_positions)
 * and contact flags (as mgsb_get_all_contact_flags) of every body, copied
 * with one stream synchronisation instead of two.  MGSB_DIVERGED as the
 * single readbacks.  No reference counterpart. */
mgsb_status mgsb_get_frame(mgsb_solver* h, float* positions /* [3 sum V] */, int32_t* contact_flags /* [sum V] */);
/* The same without a host copy: the positions are packed to xyz on the device
 * and copied with the contact flags into the solver's pinned readback buffer
 * (one synchronisation); *positions [3 sum V] and *contact_flags [sum V] point
 * into that buffer and stay valid until the next readback call on this solver
 * (any mgsb_get_* that returns host data) or mgsb_destroy.  No reference
 * counterpart. */
mgsb_status mgsb_get_frame_view(mgsb_solver* h, const float** positions, const int32_t** contact_flags);
/* Contact vertex indices, ascending.  *n receives the count; if cap < count
 * only cap entries are written and MGSB_INVALID_ARG is returned. */
mgsb_status mgsb_get_contacts(mgsb_solver* h, int32_t body, int32_t* idx, size_t cap, size_t* n);
/* Per-vertex collision depth (reference kind) — m_tetVertCollisionDepth. */
mgsb_status mgsb_get_collision_depth(mgsb_solver* h, int32_t body, float* out /* [V] */);
/* Device pointer to the body's positions (float4 xyzw per vertex, w unused),
 * valid until the next step/destroy — replaces the GL hand-off. */
mgsb_status mgsb_get_device_positions(mgsb_solver* h, int32_t body, const float** dptr);
/* Area-unweighted surface vertex normals — UpdateTriNormal +
 * AvgOutsideTetVertNormal (PDSolver.cu:394-460). */
mgsb_status mgsb_get_normals(mgsb_solver* h, int32_t body, float* out /* [3*V] */);
/* The same normals without allocating anything, for callers that cannot call
 * cudaMalloc while they run (a host that owns the GPU memory budget and forbids
 * driver allocations in its frame loop; a real-time thread that cannot take the
 * implicit synchronisation of cudaMalloc/cudaFree).  No counterpart in the
 * reference.  Scratch is a fixed 2 MiB device array inside the library, held by
 * every GPU that loads it until exit; a body may have at most 65,536 surface
 * triangles and 65,536 surface vertices, else MGSB_NOT_SUPPORTED.  A pending
 * set-up (after mgsb_set_fixed / mgsb_set_material) is not rebuilt here:
 * MGSB_INVALID_ARG until a mgsb_step or mgsb_get_normals call has done it.  The
 * first call on a device (and the first after its context was reset) looks up
 * the scratch address; make it outside any stream capture.  All calls on one
 * device share the scratch, so calls that overlap in time (other threads, other
 * handles) race. */
mgsb_status mgsb_get_normals_noalloc(mgsb_solver* h, int32_t body, float* out /* [3*V] */);

/* Checkpoint / resume: overwrite positions and velocities of a body. */
mgsb_status mgsb_set_state(mgsb_solver* h, int32_t body, const float* positions, const float* velocities);

/* Energy diagnostics of the current state — runCalEnergy (PDSolver.cu:816-924)
 * as a device reduction.  out[0]=Ek, out[1]=Ep, out[2]=Ec, out[3]=Nc,
 * out[4]=|x-prev| (reference kind) or last fine-level residual norm. */
mgsb_status mgsb_get_energy(mgsb_solver* h, int32_t body, double out[5]);

/* Timing of the last frame on the solver stream (CUDA events), ms. */
mgsb_status mgsb_last_frame_ms(mgsb_solver* h, float* ms);
/* Run one frame eagerly with CUDA events around every kernel launch and
 * report, per kernel name, the summed device time and the launch count
 * (names: cap entries of 48 chars).  The frame advances the simulation.
 * No reference counterpart (the reference times with std::chrono,
 * PDSolver.cpp:244-292). */
mgsb_status mgsb_profile_frame(mgsb_solver* h, int32_t cap, char* names, float* total_ms, int32_t* launches,
                               int32_t* count);
/* Device time of one kernel in the frame's own launch chain: one frame is
 * captured with every launch of the kernel `name` (a name mgsb_profile_frame
 * reports) repeated `reps` (1..1000) times back to back between two
 * event-record nodes, so the time per launch carries no event overhead;
 * us_per_launch = summed chain time / (reps x launches_per_frame).  The
 * solver state is saved before that frame and restored after it, so the
 * simulation does not advance.  The broad-phase kernels (k_bp_*) append to
 * shared lists and are refused (MGSB_NOT_SUPPORTED).  No reference
 * counterpart. */
mgsb_status mgsb_time_kernel(mgsb_solver* h, const char* name, int32_t reps, float* us_per_launch,
                             int32_t* launches_per_frame);
/* Number of kernel launches one frame issues. */
mgsb_status mgsb_launches_per_frame(const mgsb_solver* h, int32_t* n);

/* Export of the precomputed per-tet / per-vertex data of body 0 (test hook,
 * host copies): inv_dm [9T], ac [12T], volume [T], mass [V], diag [V].
 * Any pointer may be NULL.  Replaces reading PDSolver's m_tetInvD3x3,
 * m_tetInvD3x4, m_tetVolume, m_tetVertMass, m_tetVolumeDiag. */
mgsb_status mgsb_get_precompute(mgsb_solver* h, float* inv_dm, float* ac, float* volume, float* mass, float* diag);

/* Multigrid hierarchy inspection (body-concatenated arrays). */
mgsb_status mgsb_level_size(mgsb_solver* h, int32_t level, int32_t* num_verts, int32_t* nnz_offdiag);
/* info: [vertices, off-diagonal nnz, restriction entries, ELL slice height,
 * stored ELL entries, coarse-kernel cluster size, its block size, level-0
 * fusion flag].  No reference counterpart. */
mgsb_status mgsb_level_info(mgsb_solver* h, int32_t level, int32_t info[8]);
/* Rows of one body on one multigrid level (a batch's bodies have levels of
 * their own sizes).  No reference counterpart. */
mgsb_status mgsb_body_level_size(mgsb_solver* h, int32_t body, int32_t level, int32_t* n);

/* Project-written autotuner: times `frames` frames for each candidate shape
 * of the coarse V-cycle kernel (cluster size, block size, level-0 fusion,
 * coarse split — read back with mgsb_get_coarse_split) from the current
 * state, keeps the fastest and restores the state.
 * chosen (may be NULL): [cluster, block, fused].  No reference counterpart. */
mgsb_status mgsb_autotune(mgsb_solver* h, int32_t frames, int32_t chosen[3]);
/* Set the coarse-kernel shape explicitly: cluster size (0 = by size, else
 * 1..16), block size (0 = keep, 256/512/1024), level-0 fusion (-1 = by size,
 * 0, 1).  No reference counterpart. */
mgsb_status mgsb_set_kernel_shape(mgsb_solver* h, int32_t cluster, int32_t block, int32_t fuse_level0);
/* Coarse-level split of the V-cycle: levels 1..split-1 run as grid-wide
 * kernels over every SM, levels split..L-1 in the cluster kernel (split 1 =
 * all coarse levels in the cluster kernel; 0 = by size: levels whose largest
 * body has more than 1024 rows run grid-wide).  The autotuner also picks it.
 * Same arithmetic either way.  No reference counterpart. */
mgsb_status mgsb_set_coarse_split(mgsb_solver* h, int32_t split);
mgsb_status mgsb_get_coarse_split(mgsb_solver* h, int32_t* split);
/* Programmatic dependent launch between the frame's consecutive kernels
 * (default 1): the next kernel's blocks are scheduled while the previous one
 * finishes and wait for its completion on the device, which hides most of
 * the launch gap; 0 = plain stream order.  Same results either way.  No
 * reference counterpart. */
mgsb_status mgsb_set_launch_overlap(mgsb_solver* h, int32_t on);
/* Prolongation fused with the first post-smoothing sweep (default 1): with
 * OP = Off * P precomputed per level, A (d + P e) = (b - res) + D P e + OP e,
 * so the sweep after the prolongation needs no neighbour of the prolonged
 * vector and both run as one kernel (in the learned cycle: the prolongation
 * and the post-smoothing residual).  0 = separate launches.  The same
 * V-cycle; results agree to rounding.  No reference counterpart. */
mgsb_status mgsb_set_fused_prolongation(mgsb_solver* h, int32_t on);
/* Level-1 restriction straight from level 0 (default 0): with RO = R * Off(level 0)
 * precomputed, R (b - A d) = R (b - D d) - RO d, so when level 1 runs grid-wide
 * (coarse split >= 2) and the prolongation is fused, the level-0 residual is
 * not formed as a launch of its own (the fused prolongation forms the rows it
 * needs).  0 = the separate residual launch.  The same V-cycle; results agree
 * to rounding.  On config 1 the fused launch costs what the two it replaces
 * cost (4.9 vs 2.2 + 2.9 µs), hence off by default.  No reference counterpart. */
mgsb_status mgsb_set_fused_restriction(mgsb_solver* h, int32_t on);
/* Tool-contact broad phase of the multigrid kinds (default 0 = every
 * surface vertex against its body's capsule).  1: a uniform grid per body
 * over the rest bounding box of its surface, rebuilt every frame from the
 * predicted positions by a counting sort; each capsule tests only the
 * vertices in the cells its swept box covers.  The contact set, stiffness
 * and targets are the same either way; toggling clears the contact state
 * until the next frame.  Replaces the all-vertex loop of DCDByPoint
 * (PDSolver.cpp:228-233, PDSolver.cu:277-331). */
mgsb_status mgsb_set_broad_phase(mgsb_solver* h, int32_t on);

/* Dense coarse operator (one body): the V-cycle of the levels from the coarse
 * split down to the coarsest is a linear map M of the split level's
 * right-hand side.  With 1, M is formed once per frame after the coarse
 * diagonals and the coarsest inverse are refreshed (one CTA per column, each
 * the one-CTA V-cycle on a unit vector) and every V-cycle applies it as one
 * restriction + one dense product instead of the cluster kernel.  The same
 * V-cycle up to rounding.  At most 1,024 rows on the split level
 * (MGSB_NOT_SUPPORTED otherwise, and for batches).  The autotuner tries it at
 * every eligible split.  No reference counterpart. */
mgsb_status mgsb_set_coarse_dense(mgsb_solver* h, int32_t on);
mgsb_status mgsb_get_coarse_dense(mgsb_solver* h, int32_t* on);

/* Capsule narrow phase of the multigrid kinds.  MGSB_CONTACT_VERTICES (the
 * default): surface vertices inside the capsule are contacts, projected to its
 * surface.  MGSB_CONTACT_VERTICES_AND_TRIANGLES: in addition every surface
 * triangle closer to the capsule's segment than its radius is in contact (a
 * capsule entering a face between its vertices), and each vertex of such a
 * triangle that is not itself inside the capsule becomes a contact whose
 * target is its predicted position plus the mean push of its touching
 * triangles; a triangle's push moves it out along its closest-point line to
 * the segment by the penetration depth.  The capsule form of the reference's
 * sphere test DCDByTriangle_sphere_V2 (PDSolver.cu:612-680, response
 * :462-501), gathered per vertex instead of float atomics.  Evaluated once per
 * frame in FP64 on the predicted positions; not combined with the broad phase
 * (MGSB_NOT_SUPPORTED). */
enum { MGSB_CONTACT_VERTICES = 0, MGSB_CONTACT_VERTICES_AND_TRIANGLES = 1 };
mgsb_status mgsb_set_surface_contact(mgsb_solver* h, int32_t mode);

/* Host-only (no GPU): build the multigrid hierarchy of one mesh exactly as
 * mgsb_create would and return level `level`: vertex count, off-diagonal
 * count, prolongation rows of the next finer level (pid/pw: 4 per finer
 * vertex, level >= 1), the diagonal (L_ii at level 0, Galerkin diagonal
 * above; 0 = inactive) and the off-diagonal part in CSR.  Array pointers may
 * be NULL.  No reference counterpart (test and tooling hook). */
mgsb_status mgsb_inspect_level(const mgsb_mesh* mesh, const mgsb_params* params, const uint8_t* fixed, int32_t level,
                               int32_t* n, int32_t* nnz, int32_t* pid, float* pw, float* diag, int32_t* ptr,
                               int32_t* col, float* val);

const char* mgsb_last_error_string(const mgsb_solver* h);
const char* mgsb_status_string(mgsb_status s);

/* ---------------------------------------------------------------------------
 * Mesh utilities (host only; no GPU needed).
 * ------------------------------------------------------------------------- */
typedef struct mgsb_mesh_data {
    int32_t num_verts;
    int32_t num_tets;
    float* positions;       /* [3V] */
    int32_t* tets;          /* [4T] */
    int32_t num_tris;       /* boundary triangles (filled by mgsb_mesh_extract_surface) */
    int32_t* tris;          /* [3F] outward-oriented */
    int32_t* tri_opposite;  /* [F] vertex of the owning tet opposite the face */
    int32_t grid_dims[3];
} mgsb_mesh_data;

/* Box [lo,hi] split into nx*ny*nz hexes, 6 Kuhn tets per hex, vertex index
 * i + (nx+1)*(k + (nz+1)*j).  No reference counterpart (the reference loads
 * gmsh files). */
mgsb_status mgsb_mesh_box(int32_t nx, int32_t ny, int32_t nz, const float lo[3], const float hi[3],
                          mgsb_mesh_data** out);
/* Voxel blob: voxels of a grid whose centre satisfies
 * (x/ax)^2+(y/ay)^2+(z/az)^2 < 1 + amp*s(x,y,z), s = seeded value noise of the
 * given period; 6 Kuhn tets per kept voxel, unused vertices dropped. */
mgsb_status mgsb_mesh_blob(int32_t gx, int32_t gy, int32_t gz, float spacing, const float semi_axes[3],
                           float noise_amp, float noise_period, uint64_t seed, mgsb_mesh_data** out);
/* gmsh 2.2 ASCII reader — SoftObject::ReadFromFile (SoftObject.cpp:85-130). */
mgsb_status mgsb_mesh_read_msh(const char* path, mgsb_mesh_data** out);
/* Boundary faces + opposite vertex — SoftObject::TetFaceExtraction
 * (SoftObject.cpp:154-251); same face order as the reference's std::set. */
mgsb_status mgsb_mesh_extract_surface(mgsb_mesh_data* m);
mgsb_status mgsb_mesh_free(mgsb_mesh_data* m);

/* Seeded 3-D value noise used by the blob generator, exposed for tests. */
double mgsb_value_noise(double x, double y, double z, double period, uint64_t seed);

/* ------------------------------------------------------------------------
 * The reference's two-level nested-iteration schedule — PDSolver_MG
 * (PDSolver_MG.cpp:5-253, updatePointInTet / updateMapping PDSolver.cu:724-793,
 * DCDByTriangle_sphere_V2 PDSolver.cu:612-680).  Two reference-kind solvers
 * (mgsb_default_params(MGSB_SOLVER_REFERENCE_JACOBI) params, `iterations`
 * per level) on a coarse and a fine mesh of the same body.  Per frame: both
 * predict; the coarse level iterates with sphere-vs-surface-triangle
 * collision; fine positions are interpolated from the coarse tets that hold
 * them; the fine level iterates with per-vertex sphere collision; coarse
 * positions are averaged back from the fine tets; the fine-in-coarse weights
 * are recomputed; velocities follow.  The whole frame is one CUDA graph.
 * Level 0 = fine, 1 = coarse.
 * ------------------------------------------------------------------------ */
typedef struct mgsb_two_level mgsb_two_level;
/* PDSolver_MG::Init: binds every fine vertex to the coarse tet holding it and
 * every coarse vertex to the fine tet holding it (MGSB_INVALID_ARG if a vertex
 * lies outside the other mesh). */
mgsb_status mgsb_mg2_create(const mgsb_mesh* coarse, const mgsb_mesh* fine, const mgsb_params* params,
                            mgsb_two_level** out);
mgsb_status mgsb_mg2_destroy(mgsb_two_level* t);
const char* mgsb_mg2_last_error(const mgsb_two_level* t);
/* The level's solver handle for the getters (positions, contacts, energy, ...);
 * owned by t. */
mgsb_status mgsb_mg2_level(mgsb_two_level* t, int32_t level, mgsb_solver** out);
/* SetFixedVert of both PDSolvers (NULL leaves a level unchanged). */
mgsb_status mgsb_mg2_set_fixed(mgsb_two_level* t, const uint8_t* coarse_mask, const uint8_t* fine_mask);
/* g_simulator->m_sphereColliders for both levels. */
mgsb_status mgsb_mg2_set_tool_spheres(mgsb_two_level* t, int32_t count, const float* centers, const float* radii,
                                      const uint8_t* active);
/* PDSolver_MG::Step. */
mgsb_status mgsb_mg2_step(mgsb_two_level* t);
mgsb_status mgsb_mg2_get_positions(mgsb_two_level* t, int32_t level, float* out);

/* ------------------------------------------------------------------------
 * Learned smoother network (config 4).  No counterpart in the reference: its
 * multigrid smoother is plain Jacobi (PDSolver.cu:192-235).
 * A per-vertex MLP 9 -> 64 -> 64 -> 3 with GELU, BF16 weights/activations and
 * FP32 accumulation; inference runs as tcgen05 tensor-core GEMMs over 128-row
 * tiles, training as a hand-written forward/backward kernel plus Adam.
 * Parameters (FP32, mgsb_mlp_num_params() = 4995 floats), row-major:
 *   W1[64][9] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]
 * ------------------------------------------------------------------------ */
typedef struct mgsb_mlp mgsb_mlp;
int32_t mgsb_mlp_num_params(void);
/* Seeded uniform Glorot initialisation, zero biases. */
mgsb_status mgsb_mlp_create(int32_t device, uint64_t seed, mgsb_mlp** out);
mgsb_status mgsb_mlp_destroy(mgsb_mlp* h);
const char* mgsb_mlp_last_error(const mgsb_mlp* h);
mgsb_status mgsb_mlp_set_params(mgsb_mlp* h, const float* params, int32_t n);
mgsb_status mgsb_mlp_get_params(mgsb_mlp* h, float* params, int32_t n);
/* y[n][3] = MLP(x[n][9]) on the tensor cores (host buffers). */
mgsb_status mgsb_mlp_forward(mgsb_mlp* h, const float* x, int32_t n, float* y);
/* Mean squared error over all n samples and its gradient (host buffers). */
mgsb_status mgsb_mlp_loss_grad(mgsb_mlp* h, const float* x, const float* t, int32_t n, float* grad, float* loss);
/* Adam on minibatches of `batch` samples drawn uniformly (seeded) from the n
 * pairs; step size lr with cosine decay to 10 %.  losses (optional) receives
 * the minibatch loss of every step. */
mgsb_status mgsb_mlp_train(mgsb_mlp* h, const float* x, const float* t, int64_t n, int32_t steps, int32_t batch,
                           float lr, uint64_t seed, float* losses);

/* Attach (net != NULL) or detach the learned smoother of a multigrid solver.
 * Each V-cycle then smooths level 0 with one learned sweep before and one after
 * the coarse correction (in place of the Jacobi sweeps), and every V-cycle's
 * residual is checked: it fails unless |r_end| <= guard_ratio * |r_start|
 * (both finite).  When any V-cycle of a frame fails, the frame's global solve
 * is repeated from its start with the plain V-cycle, so that frame equals
 * the plain solver's frame (in a CUDA graph the repeat is the body of a
 * conditional node; eagerly the host reads the decision after the solve).
 * The network must live on the solver's device and outlive the attachment;
 * retraining it updates the solver in place.  No counterpart in the
 * reference. */
mgsb_status mgsb_set_learned_smoother(mgsb_solver* h, const mgsb_mlp* net, float guard_ratio);
/* Learned V-cycles checked, and checks failed, since the network was attached. */
mgsb_status mgsb_learned_stats(mgsb_solver* h, uint64_t out[2]);
/* The last frame's learned V-cycles (PD iteration-major, refinement pass
 * minor): before[c] = |r| where cycle c started, after[c] = |r| after it (the
 * quantities the guard compares: a cycle passes when after <= guard_ratio x
 * before).  *n receives the frame's cycle count; at most cap values are
 * written to each array.  Diagnostic: synchronises the solver's stream. */
mgsb_status mgsb_learned_cycle_norms(mgsb_solver* h, double* before, double* after, int32_t cap, int32_t* n);
/* Training pairs from the plain FP32 multigrid solver's current state: the
 * learned sweep is trained to reproduce `sweeps` weighted-Jacobi sweeps from
 * zero in one step.  Three residuals are used: r = b - A d of the last global
 * step, the residual left after plain pre-smoothing and the coarse correction
 * of r (what post-smoothing sees), and the residual a further PD iteration
 * would start from (local step at the current d; what pre-smoothing sees).  One
 * pair per free vertex whose residual scale s_i is at least 1e-2 of that
 * residual's RMS: features x[9] of the residual against the Jacobi result in
 * the network's output space, t = e_sweeps / (s_i / D_i).  *n receives the
 * count (up to 3 x vertices); with x = t = NULL only counts.  The call leaves
 * the solver's state as it was, but not its scratch: call it between frames. */
mgsb_status mgsb_smoother_pairs(mgsb_solver* h, int32_t sweeps, float* x, float* t, int64_t cap, int64_t* n);
/* Smoother comparison on the last global step: V-cycles on A e = r from e = 0;
 * mode 0 plain (configured sweeps), 1 plain with 1+1 sweeps, 2 learned (no
 * fallback).  out[0] = |r|, out[k] = residual norm after k cycles (cycles + 1
 * values).  Plain FP32 multigrid solver only. */
mgsb_status mgsb_vcycle_residuals(mgsb_solver* h, int32_t cycles, int32_t mode, double* out);

#ifdef __cplusplus
}
#endif

#endif /* MGSB_H_ */
