/*
 * lhi.h -- C-ABI of the B200 liquid step (drop-in for the reference's
 * LiquidModel<3> / CGSolver<3> pair).
 *
 * Every entry point returns an int status (LHI_OK == 0).  On failure the
 * message is available from lhi_last_error() (thread-local).  No torch types,
 * no C++ types: plain pointers and sizes only.
 *
 * Host buffers passed to the lhi_liquid_* calls are typed by the handle's
 * precision: float for LHI_PRECISION_FP32 and LHI_PRECISION_MIXED, double for
 * LHI_PRECISION_FP64 ("host scalar").  Integer fields are documented per field.
 *
 * Array layout of every grid field follows the reference's Array3
 * (Array.h:78-83): index (x * ny + y) * nz + z, z fastest.
 *   vx, wx, liquidWx, tempVx : (nx+1) x  ny    x  nz
 *   vy, wy, liquidWy, tempVy :  nx    x (ny+1) x  nz
 *   vz, wz, liquidWz, tempVz :  nx    x  ny    x (nz+1)
 *   pressure, liquidPhi      :  nx    x  ny    x  nz
 *   solidPhi, isValid        : (nx+1) x (ny+1) x (nz+1)
 * Particles cross the boundary as AoS triples (x, y, z) per particle, like
 * Particle<3>::position / velocity (ParticleSystem.h:5-22); the affine matrix
 * is 9 values per particle in Eigen's column-major order (col a = C[3a..3a+2]).
 *
 * Threading: one host thread drives a handle; calls on one handle are not
 * thread-safe; distinct handles are independent.  All device work of a handle
 * is ordered on its own CUDA stream; calls that return host data synchronise.
 */
#ifndef LHI_H_
#define LHI_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define LHI_API __declspec(dllexport)
#else
#define LHI_API __attribute__((visibility("default")))
#endif

/* ---------------------------------------------------------------- status */
#define LHI_OK 0
#define LHI_E_INVALID_ARG 1
#define LHI_E_CUDA 2
#define LHI_E_OOM 3
#define LHI_E_NOT_CONVERGED 4
#define LHI_E_TIMEOUT 5
#define LHI_E_NAN 6
#define LHI_E_UNSUPPORTED 7

/* ------------------------------------------------------------- precision */
#define LHI_PRECISION_FP32 0  /* everything float: reference-compatible      */
#define LHI_PRECISION_MIXED 1 /* float grid/particles/V-cycle, double CG x,
                                 dots, true residual and final check         */
#define LHI_PRECISION_FP64 2  /* everything double                            */

/* preconditioner: CGSolver<3>::PrecondType (PressureSolver.h:84-86) */
#define LHI_PRECOND_NONE 0
#define LHI_PRECOND_JACOBI 1
#define LHI_PRECOND_MULTIGRID 2
#define LHI_PRECOND_LEARNED 3 /* no counterpart in the reference: the network of
                                 lhi_solver_set_network inside flexible PCG, with
                                 the V-cycle as fallback (FP32 / MIXED handles) */

/* stopping rule */
#define LHI_TOL_ABSOLUTE 0 /* ||r|| < tol, as PressureSolver.cpp:871      */
#define LHI_TOL_RELATIVE 1 /* ||r|| < tol * ||r0||                         */

/* CG update of beta */
#define LHI_CG_REFERENCE 0 /* Fletcher-Reeves rz_new/rz_old (PressureSolver.cpp:906) */
#define LHI_CG_FLEXIBLE 1  /* Polak-Ribiere, safe for a varying preconditioner     */

/* cells on which PCG updates x and r and takes p.Ap and ||r|| */
#define LHI_REGION_INTERIOR 0 /* fluid cells of [1, N-2]^3, as PressureSolver.cpp:874-899 */
#define LHI_REGION_FLUID 1    /* every fluid cell: a consistent CG when fluid cells lie on
                                 the domain's outer layer (one-cell walls)               */

/* red-black smoother update */
#define LHI_SMOOTHER_REFERENCE 0 /* z = (1 - w) z + w (r - A z) / diag, as PressureSolver.cpp:832:
                                    A z includes the diagonal, so w = 0.5 gives z_GS / 2     */
#define LHI_SMOOTHER_DAMPED_GS 1 /* z = z + w (r - A z) / diag: damped Gauss-Seidel           */

/* Red-black sweep kernels of the FP32 V-cycle.  FUSED: one pass per sweep
   over shared-memory tiles staged by TMA, both colours, into a second
   solution buffer (levels whose z extent is a multiple of 4; other levels
   and FP64 use SPLIT).  SPLIT: one launch per colour, in place.  Both give
   the same values. */
#define LHI_SWEEP_FUSED 0
#define LHI_SWEEP_SPLIT 1
/* Coarse multigrid operators: the reference's re-discretisation from the
   level's approximated liquid SDF and face fractions (BuildLHS,
   PressureSolver.cpp:544-664), or the Galerkin operator of the finer level
   under the V-cycle's own transfers: A_c = P^T A P / 8 with P the constant
   injection (Prolong, :774-794), so the coarse correction of the averaging
   restriction (Restrict, :796-819) is the A-orthogonal projection.  The
   Galerkin levels stay consistent with the finest level where thin solids
   make the re-discretised ones disagree with it (the V-cycle then stops
   being a usable preconditioner); no counterpart in the reference. */
#define LHI_COARSE_REFERENCE 0
#define LHI_COARSE_GALERKIN 1
/* Initial guess of the PCG (lhi_solver_params.initial_guess).  ZERO is the
   reference's (x = 0, PressureSolver.cpp:841-856).  PREVIOUS starts from the
   last solve's solution on the cells that are fluid now (0 elsewhere); the
   relative stopping rule then measures ||r|| against ||b|| rather than
   ||r0||, so the solve still ends at ||r||/||b|| <= tolerance.  No
   counterpart in the reference. */
#define LHI_GUESS_ZERO 0
#define LHI_GUESS_PREVIOUS 1

typedef struct lhi_grid_desc {
    int32_t dim[3];        /* gridDimension (SceneParameter.h:137)          */
    int32_t reserved;
    double min_coord[3];   /* minCoord, converted to the handle's scalar    */
    double max_coord[3];   /* maxCoord                                      */
} lhi_grid_desc;

typedef struct lhi_solver_params {   /* SolverParameter<3> (SceneParameter.h:10-45) */
    int32_t max_iterations;
    int32_t preconditioner;          /* LHI_PRECOND_*                          */
    double tolerance;
    int32_t num_level;
    int32_t num_pre_smooth;
    int32_t num_post_smooth;
    int32_t num_final_smooth;
    double smoothing_factor;
    int32_t tolerance_mode;          /* LHI_TOL_*        (0 = reference)       */
    int32_t cg_variant;              /* LHI_CG_*         (0 = reference)       */
    int32_t true_residual_every;     /* recompute r = b - A x every k iterations
                                        (0 = never)                            */
    int32_t update_region;           /* LHI_REGION_* (0 = reference)           */
    int32_t smoother;                /* LHI_SMOOTHER_* (0 = reference)         */
    int32_t coarse_cells;            /* MG levels below the finest with at most
                                        this many cells are solved together by
                                        one CTA in shared memory (0 => 4096)   */
    int32_t eager;                   /* 1: the host drives the PCG loop (one
                                        synchronisation per iteration); 0: the
                                        loop runs on the device as a CUDA graph
                                        with a conditional while node          */
    int32_t sweep_kernel;            /* LHI_SWEEP_* (0 = fused where the level
                                        allows it)                             */
    int32_t coarse_operator;         /* LHI_COARSE_* (0 = reference)           */
    int32_t initial_guess;           /* LHI_GUESS_* (0 = reference)            */
} lhi_solver_params;

typedef struct lhi_liquid_params {   /* LiquidParameter<3> + SceneParameter<3> */
    double density;                  /* liquid density (rho)                   */
    double gravity;                  /* gravity along y                        */
    double particle_radius;          /* 0 => 2 * dx.x (ParticleSystem.cpp:8)   */
    int32_t extrapolate_iterations;  /* 0 => 5 (LiquidModel.cpp:948)           */
    int32_t correct_volume;          /* 1: Step ends with CorrectVolume, the call
                                        the reference's Step has commented out
                                        (LiquidModel.cpp:527); 0 (default): off */
    int32_t correct_cycle;           /* 0 => 8 (m_correctCycle, LiquidModel.cpp:486) */
    int32_t reserved[5];
} lhi_liquid_params;

/* Headless particle render (LiquidModel<3>::Render, LiquidModel.cpp:1138-1159,
   and Shader/Scene3D_vertex.glsl), lhi_liquid_render. */
typedef struct lhi_render_params {
    int32_t width, height;  /* viewport in pixels (main.cpp:11: 480 x 480)        */
    float point_size;       /* gl_PointSize in pixels (LiquidModel.cpp:1149: 5)   */
    uint8_t color[4];       /* RGBA of the points (Color::Blue: 0, 0, 255, 255)   */
    uint8_t background[4];  /* clear colour (main.cpp:12: Color::White)           */
} lhi_render_params;

typedef struct lhi_solve_stats {
    int32_t iterations;        /* PCG iterations taken                        */
    int32_t status;            /* LHI_OK or LHI_E_NOT_CONVERGED / LHI_E_NAN /
                                  LHI_E_TIMEOUT                               */
    double initial_residual;   /* ||r0|| over all cells (PressureSolver.cpp:868) */
    double final_residual;     /* recursive ||r|| over interior fluid cells   */
    double true_residual;      /* ||b - A x|| over interior fluid cells, or -1 */
    double solve_ms;           /* device time of the solve (CUDA events)      */
} lhi_solve_stats;

/* Boundary tree node: BaseBoundary<3> family (Boundary.h:6-96). */
#define LHI_BOUNDARY_RECT 0         /* RectBoundary                            */
#define LHI_BOUNDARY_SOLID 1        /* SolidBoundary stub: Compute() == 1      */
#define LHI_BOUNDARY_UNION 2        /* OperatorBoundary::Union  = min(l, r)    */
#define LHI_BOUNDARY_INTERSECTION 3 /* OperatorBoundary::Intersection = max    */
#define LHI_BOUNDARY_SUBTRACT 4     /* OperatorBoundary::Substract max(l, -r)  */
#define LHI_BOUNDARY_NONE 5         /* OperatorBoundary::None = left child     */
typedef struct lhi_boundary_node {
    int32_t kind;
    int32_t use_inside;
    int32_t left;              /* child node index, -1 if none */
    int32_t right;
    double center[3];
    double half_extent[3];
} lhi_boundary_node;

/* Fluid primitive for the seeded scene generator. */
#define LHI_FLUID_BOX 0     /* a = min corner, b = max corner (half-open [a, b)) */
#define LHI_FLUID_SPHERE 1  /* a = centre, b[0] = radius                        */
typedef struct lhi_fluid_prim {
    int32_t kind;
    int32_t reserved;
    double a[3];
    double b[3];
    double velocity[3];
} lhi_fluid_prim;

/* Grid / solver fields for lhi_liquid_get_field / lhi_liquid_set_field. */
#define LHI_FIELD_VX 0
#define LHI_FIELD_VY 1
#define LHI_FIELD_VZ 2
#define LHI_FIELD_WX 3
#define LHI_FIELD_WY 4
#define LHI_FIELD_WZ 5
#define LHI_FIELD_LIQUID_WX 6
#define LHI_FIELD_LIQUID_WY 7
#define LHI_FIELD_LIQUID_WZ 8
#define LHI_FIELD_TEMP_VX 9
#define LHI_FIELD_TEMP_VY 10
#define LHI_FIELD_TEMP_VZ 11
#define LHI_FIELD_PRESSURE 12
#define LHI_FIELD_LIQUID_PHI 13
#define LHI_FIELD_SOLID_PHI 14
#define LHI_FIELD_IS_VALID 15   /* uint8, (nx+1)(ny+1)(nz+1)                  */
#define LHI_FIELD_RHS 16        /* CGSolver m_rhs                             */
#define LHI_FIELD_X 17          /* CGSolver m_x                               */
#define LHI_FIELD_P 18          /* CGSolver m_p                               */
#define LHI_FIELD_R 19          /* CGSolver m_r[level]                        */
#define LHI_FIELD_Z 20          /* CGSolver m_z[level]                        */
#define LHI_FIELD_ADIAG 21      /* CGSolver m_Adiag[level]                    */
#define LHI_FIELD_ACOEF 22      /* CGSolver m_Acoef[level]: 6 per cell, order
                                   right, left, top, bottom, front, back
                                   (read-only; expanded from face storage)   */
#define LHI_FIELD_CELL_KEY 23   /* int32 per particle, device (sorted) order:
                                   linear cell index of Point2Index(pos)      */
#define LHI_FIELD_PARTICLE_ID 24 /* int32 per particle, device order: caller's
                                   particle index                             */
#define LHI_FIELD_CELL_START 25 /* int32, ncells + 1: first sorted particle of
                                   each cell                                  */
#define LHI_FIELD_AP 26         /* CG's A p of level 0 (lhi_solver_spmv)       */
#define LHI_FIELD_COUNT 27

typedef struct lhi_liquid lhi_liquid;  /* opaque handle: owns all device memory */

/* ------------------------------------------------------------ lifecycle */
/* LiquidModel<3>::LiquidModel (LiquidModel.cpp:479-504) + Grid<3>::Grid
   (Grid.cpp:86-98) + CGSolver<3>::CGSolver (PressureSolver.cpp:422-447). */
LHI_API int lhi_liquid_create(const lhi_grid_desc* grid, const lhi_solver_params* solver,
                              const lhi_liquid_params* liquid, int32_t precision,
                              lhi_liquid** out);
LHI_API int lhi_liquid_destroy(lhi_liquid* h);
LHI_API const char* lhi_last_error(void);
LHI_API int lhi_liquid_precision(const lhi_liquid* h, int32_t* precision);
LHI_API int lhi_liquid_sync(lhi_liquid* h);
/* Grid spacing dx (Grid.cpp:94-97) as the handle computed it. */
LHI_API int lhi_liquid_get_dx(const lhi_liquid* h, double dx[3]);

/* ---------------------------------------------------------- scene input */
/* LiquidModel<3>::ComputeSolidPhi (LiquidModel.cpp:563-611): evaluates the
   boundary tree at the (N+1)^3 nodes on the device, then the face fractions. */
LHI_API int lhi_liquid_set_boundary(lhi_liquid* h, const lhi_boundary_node* nodes,
                                    int32_t count, int32_t root);
/* Same, for a node SDF evaluated by the caller (BaseBoundary<3>::Compute on
   the host): uploads solidPhi then computes liquidWx/y/z on the device. */
LHI_API int lhi_liquid_set_solid_phi(lhi_liquid* h, const void* node_phi);
/* ParticleSystem<3>::Resize + Set* (ParticleSystem.cpp:11-21, .h:40-45).
   vel / affine may be NULL (zero).  Radius is the handle's particle radius. */
LHI_API int lhi_liquid_set_particles(lhi_liquid* h, int64_t n, const void* pos,
                                     const void* vel, const void* affine);
/* ParticleSystem<3>::Get* in the caller's particle order; NULL skips. */
LHI_API int lhi_liquid_get_particles(lhi_liquid* h, void* pos, void* vel, void* affine);
LHI_API int lhi_liquid_num_particles(const lhi_liquid* h, int64_t* n);

/* ------------------------------------------------------------ the step */
/* LiquidModel<3>::PreStep (LiquidModel.cpp:514-517): Clear + ComputeLiquidPhi */
LHI_API int lhi_liquid_pre_step(lhi_liquid* h, double dt);
/* LiquidModel<3>::Step (LiquidModel.cpp:520-528): P2G, gravity, projection,
   extrapolation, G2P, advection */
LHI_API int lhi_liquid_step(lhi_liquid* h, double dt);
/* LiquidModel<3>::PostStep (LiquidModel.cpp:531-537): divergence diagnostic */
LHI_API int lhi_liquid_post_step(lhi_liquid* h, double dt);

/* ------------------------------------------------------- stage entries */
LHI_API int lhi_liquid_clear(lhi_liquid* h);                      /* Grid.cpp:157-169     */
LHI_API int lhi_liquid_sort_particles(lhi_liquid* h);             /* cell-key radix sort  */
LHI_API int lhi_liquid_compute_liquid_phi(lhi_liquid* h);         /* LiquidModel.cpp:540  */
LHI_API int lhi_liquid_particle_to_grid(lhi_liquid* h);           /* LiquidModel.cpp:614  */
LHI_API int lhi_liquid_apply_gravity(lhi_liquid* h, double dt);   /* LiquidModel.cpp:899  */
LHI_API int lhi_liquid_projection(lhi_liquid* h, double dt);      /* LiquidModel.cpp:826-896 */
LHI_API int lhi_liquid_velocity_update(lhi_liquid* h, double dt); /* LiquidModel.cpp:834-889 */
LHI_API int lhi_liquid_extrapolate(lhi_liquid* h);                /* LiquidModel.cpp:938  */
LHI_API int lhi_liquid_grid_to_particle(lhi_liquid* h);           /* LiquidModel.cpp:724  */
LHI_API int lhi_liquid_advect_particles(lhi_liquid* h, double dt);/* LiquidModel.cpp:913  */
/* LiquidModel<3>::ComputeDivergence (LiquidModel.cpp:1066-1083): mean over
   fluid cells; max_abs is the max-norm of the same per-cell divergence over
   the fluid cells whose six faces the projection updates ([1, N-3]^3). */
LHI_API int lhi_liquid_compute_divergence(lhi_liquid* h, double* mean, double* max_abs);
/* LiquidModel<3>::GetCFL (LiquidModel.h:49-55) */
LHI_API int lhi_liquid_get_cfl(lhi_liquid* h, double* dt_out);
/* LiquidModel<3>::CorrectVolume (LiquidModel.cpp:1086-1132) with the
   neighbour search of HashNeighborSearch (NeighborSearch.h:22-108) done on
   the handle's cell-sorted particles.  The particles whose index (caller
   order) is step mod cycle move by the repulsion of their neighbours within
   one radius (every other particle keeps its position), then step advances.
   Off unless called, or unless lhi_liquid_params.correct_volume is set,
   which makes Step end with it (the reference's Step has the call commented
   out).  Where the reference differs: its neighbour table is the one built
   at the end of the previous call, not the current positions, and a hash
   collision can list a particle twice; here the neighbours are those of the
   current positions, each counted once per cell its 3x3x3 region shares
   with the particle's region, as the table lists it once per region cell.
   Coincident particles (distance <= 1e-4 radius) take a seeded counter-based
   uniform number (SplitMix64 of the two indices, the call count and the
   axis) where the reference draws from an unseeded std::mt19937. */
LHI_API int lhi_liquid_correct_volume(lhi_liquid* h, double dt);
/* LiquidModel<3>::Render without a graphics API: the vertex shader's
   normalised device coordinates, point = (pos - minCoord) / (maxCoord -
   minCoord) * 2 - 1 in float (Shader/Scene3D_vertex.glsl:9), per particle in
   the caller's order (ndc, n x 3, may be NULL), and the points drawn as GL
   draws them into an RGBA image (rgba, height x width x 4 bytes, row 0 at
   the bottom as in GL window coordinates, may be NULL): points outside
   [-1, 1]^3 are clipped, the viewport maps x to (x + 1) * width / 2, each
   point covers the pixels whose centres lie in the square of side
   point_size around it (left and bottom edges included), and every covered
   pixel takes the point colour (one uniform colour, no depth test, no
   blending: Scene3D_fragment.glsl), the rest the background. */
LHI_API int lhi_liquid_render(lhi_liquid* h, const lhi_render_params* params, float* ndc, uint8_t* rgba);

/* -------------------------------------------------------------- solver */
LHI_API int lhi_solver_init(lhi_liquid* h);                               /* PressureSolver.cpp:666 */
LHI_API int lhi_solver_build_rhs(lhi_liquid* h);                          /* PressureSolver.cpp:682 */
LHI_API int lhi_solver_build_lhs(lhi_liquid* h, double density, double dt); /* PressureSolver.cpp:544 */
LHI_API int lhi_solver_apply_preconditioner(lhi_liquid* h);               /* PressureSolver.cpp:719 */
/* CGSolver<3>::Solve (PressureSolver.cpp:839-934); stats may be NULL. */
LHI_API int lhi_solver_solve(lhi_liquid* h, double density, double dt, lhi_solve_stats* stats);
LHI_API int lhi_solver_get_stats(lhi_liquid* h, lhi_solve_stats* stats);
/* CGSolver<3>::GetAx (PressureSolver.cpp:700-717) applied to a whole level:
   out = A_level * x (host buffers, ncells(level) host scalars). */
LHI_API int lhi_solver_get_ax(lhi_liquid* h, int32_t level, const void* x, void* out);
/* One SpMV of the PCG body (the Ap = A p and p.Ap of PressureSolver.cpp:874-880)
   with the kernel the solve itself runs: the TMA-staged tile kernel on FP32
   grids the fused sweep takes, the row kernel elsewhere.  Reads the
   handle's p (LHI_FIELD_P), writes Ap (LHI_FIELD_AP) on every cell of the
   active tiles and returns p.Ap over the update region; *tma_kernel (may be
   NULL) is 1 when the TMA kernel ran.  Needs a BuildLHS first. */
LHI_API int lhi_solver_spmv(lhi_liquid* h, double* p_dot_ap, int32_t* tma_kernel);
/* Active tiles of one MG level after the last BuildLHS: tiles of 8 x 8 x 32
   cells (x, y, z) holding a cell with phi <= 0 or covering an active tile of
   the next finer level; the V-cycle and PCG kernels visit only these.
   Levels solved by the single-CTA coarse kernel report *coarse = 1. */
LHI_API int lhi_solver_active_tiles(lhi_liquid* h, int32_t level, int32_t* active, int32_t* total,
                                    int32_t* coarse);

/* -------------------------------------------------------------- fields */
LHI_API int lhi_liquid_field_size(const lhi_liquid* h, int32_t field, int32_t level,
                                  int64_t* count, int32_t* elem_bytes);
LHI_API int lhi_liquid_get_field(lhi_liquid* h, int32_t field, int32_t level, void* out);
LHI_API int lhi_liquid_set_field(lhi_liquid* h, int32_t field, int32_t level, const void* in);

/* Asynchronous steps (on = 1): lhi_liquid_step / lhi_liquid_projection /
   lhi_solver_solve enqueue the whole solve on the handle's stream and return
   at once with LHI_OK; the solve's status and statistics are read (with a
   synchronisation) by lhi_solver_get_stats.  Independent handles stepped in
   this mode run concurrently on the GPU (the batched form).  Solves that the
   host drives (learned preconditioner, residual recording, profiling, eager)
   still wait. */
LHI_API int lhi_liquid_set_async(lhi_liquid* h, int32_t on);
/* Empty string while solves run as CUDA graphs; otherwise why the solve
   graph could not be built, in which case every solve runs host-driven (or,
   for the learned preconditioner, why the graph of the iterations after its
   fallback could not be built, in which case those stay host-driven). */
LHI_API const char* lhi_solver_graph_error(lhi_liquid* h);

/* ------------------------------------------------------- measurement */
/* The handle's CUDA stream (cudaStream_t), e.g. to record events around
   calls; all of the handle's device work is ordered on it. */
LHI_API int lhi_liquid_stream(lhi_liquid* h, void** stream);
/* Number of kernels this library has launched in the process so far,
   counting the kernels a solve graph replay ran (its loop body once per
   PCG iteration; the V-cycle kernels of the final iteration, which return
   at once, included). */
LHI_API int lhi_kernel_launch_count(int64_t* count);
/* Limit, in milliseconds, of every bounded wait of the solver kernels on
   their TMA staging copies and of the network's brick convolution on its
   pipeline barriers, on the current device (default 200; 0 gives up at
   once).  A kernel that gives up records LHI_E_TIMEOUT (in the solve's
   status, or the network's, which the next network call or learned solve
   reports), waits (200 ms at most) for its own copies and MMAs in flight
   and returns, so the context stays usable.  For tests of that path. */
LHI_API int lhi_debug_set_stage_wait_limit(double ms);
/* Kernel categories timed by the optional profiler. */
#define LHI_KERNEL_SORT 0         /* cell keys, radix sort, permutation, cell ranges */
#define LHI_KERNEL_LIQUID_PHI 1   /* liquid SDF gather                               */
#define LHI_KERNEL_P2G 2          /* P2G accumulation + normalisation                */
#define LHI_KERNEL_G2P 3          /* G2P + advection                                 */
#define LHI_KERNEL_EXTRAPOLATE 4  /* velocity extrapolation sweeps                    */
#define LHI_KERNEL_GRID 5         /* clear, P2G normalisation + gravity, velocity update, RHS, divergence */
#define LHI_KERNEL_LHS 6          /* per-level matrix assembly                        */
#define LHI_KERNEL_SMOOTH_FINE 7  /* red-black smoothing on the finest level          */
#define LHI_KERNEL_SMOOTH_COARSE 8 /* smoothing on the coarser levels                 */
#define LHI_KERNEL_RESTRICT 9
#define LHI_KERNEL_PROLONG 10
#define LHI_KERNEL_SPMV 11        /* Ap and p.Ap                                      */
#define LHI_KERNEL_CG_VECTOR 12   /* x/r/p updates, dots, true residual, scalars      */
#define LHI_KERNEL_COUNT 13
/* enable = 1 starts (and resets) per-category timing with CUDA events on
   the handle's stream; enable = 0 stops it. */
LHI_API int lhi_liquid_profile(lhi_liquid* h, int32_t enable);
/* Launches and total device milliseconds of one category since the last
   reset (synchronises the handle's stream). */
LHI_API int lhi_liquid_profile_read(lhi_liquid* h, int32_t category, int64_t* launches, double* total_ms);

/* ------------------------------------------- learned preconditioner */
/* No counterpart in the reference: the network M(r, masks) -> search
   direction used by LHI_PRECOND_LEARNED inside flexible PCG.  Three-level 3D
   convolutional network, 3x3x3 kernels, 16/32/64 channels (about 140k
   parameters), BF16 activations and weights with FP32 accumulation on the
   tensor cores.  Parameters cross the ABI as FP32 in packed order: per layer
   l = 0..5, W[27][cout_l][cin_l] then b[cout_l], with (cin, cout) =
   (4,16) (16,32) (32,64) (64,32) (32,16) (16,1) and tap = (dx+1)*9 +
   (dy+1)*3 + (dz+1). */
typedef struct lhi_net lhi_net;
LHI_API int lhi_net_create(uint64_t seed, lhi_net** out);
LHI_API int lhi_net_destroy(lhi_net* net);
LHI_API int lhi_net_num_params(int64_t* count);
LHI_API int lhi_net_get_params(lhi_net* net, float* out);
/* Parameters to / from a file: 8-byte tag "LHINET01", int64 count, then the
   packed FP32 parameters (little-endian). */
LHI_API int lhi_net_save(lhi_net* net, const char* path);
LHI_API int lhi_net_load(lhi_net* net, const char* path);
LHI_API int lhi_net_set_params(lhi_net* net, const float* in);
/* Activation between layers: 0 = identity (default: a linear multilevel
   operator, a fixed preconditioner for each geometry), 1 = ReLU. */
LHI_API int lhi_net_set_relu(lhi_net* net, int32_t relu);
/* 1 (default): the forward passes of lhi_net_forward_host and of the solver
   evaluate each convolution only on the output tiles that the cells with
   type != 0 depend on (z is the same, bit for bit); 0: every tile. */
LHI_API int lhi_net_set_sparse(lhi_net* net, int32_t on);
/* z = M(r) on an n0 x n1 x n2 grid from host buffers: r (float per cell),
   type (uint8 per cell: 0 phi > 0, 1 phi == 0, 2 phi < 0), solid (uint8
   per cell, 1 = solid cell, may be NULL); scale > 0 fixes s, 0 uses the RMS
   of r over cells with type != 0. */
LHI_API int lhi_net_forward_host(lhi_net* net, const int32_t dims[3], const float* r, const uint8_t* type,
                                 const uint8_t* solid, double scale, float* z);
/* Attaches a network to a handle created with LHI_PRECOND_LEARNED (the
   handle does not own it; keep it alive while the handle solves).  The
   solve applies the network as the preconditioner until an iteration
   reduces ||r|| by less than 5% or the iteration count exceeds
   fallback_iterations (0 = the solver's max_iterations); from then on it
   applies the multigrid V-cycle of the handle's solver parameters.
   fallback_iterations = -1 turns the fallback off (network only).  The
   network's iterations are host-driven (one synchronisation each); after
   the fallback the rest of the solve is one replay of a CUDA graph of the
   V-cycle loop (from the second V-cycle iteration of the handle's first
   fallback on). */
LHI_API int lhi_solver_set_network(lhi_liquid* h, lhi_net* net, int32_t fallback_iterations);
/* Iterations of the last solve that used the network, and the iteration
   at which the fallback started (-1 if it did not). */
LHI_API int lhi_solver_learned_stats(lhi_liquid* h, int32_t* network_iterations, int32_t* fallback_iteration);
/* Keeps the PCG residual handed to the preconditioner at each iteration of
   the following solves (up to max_snapshots, FP32, device memory; 0 stops
   recording and frees them).  Recording solves run host-driven. */
LHI_API int lhi_solver_record_residuals(lhi_liquid* h, int32_t max_snapshots);
LHI_API int lhi_solver_num_snapshots(lhi_liquid* h, int32_t* count);
/* Recorded residual `index` (0 = oldest kept) as ncells floats (host). */
LHI_API int lhi_solver_get_snapshot(lhi_liquid* h, int32_t index, float* out);
/* Adam training of the network on the handle's recorded residuals with the
   handle's level-0 matrix A (from its last BuildLHS): each step draws
   `batch` snapshots r (seeded), accumulates the gradient of
   ||A M(r) - r||^2 / ||r||^2 / batch and takes one Adam step (beta1 0.9,
   beta2 0.999, eps 1e-8).  Returns the mean loss of the first and of the
   last step. */
LHI_API int lhi_net_train(lhi_net* net, lhi_liquid* h, int32_t steps, int32_t batch, double lr, uint64_t seed,
                          double* first_loss, double* last_loss);

/* Self-check of the tensor-core path: one CTA computes D = A B^T (A 128 x K,
   B N x K as BF16 bit patterns, row-major; D 128 x N float) with the same
   tcgen05 descriptors as the network; *stage reports the last step reached
   (1 TMEM allocated, 2 MMAs issued, 3 commit arrived, 4 result read). */
LHI_API int lhi_net_tensor_core_selftest(int32_t n, int32_t k, const uint16_t* a, const uint16_t* b, float* d,
                                         int32_t* stage);
/* Gradient of sum(dz * M(r)) with respect to the packed parameters. */
LHI_API int lhi_net_backward_host(lhi_net* net, const int32_t dims[3], const float* r, const uint8_t* type,
                                  const uint8_t* solid, double scale, const float* dz, float* grad);

/* ------------------------------------------- no-allocation divergence */
/* No counterpart in the reference: an added entry point for callers that
   cannot allocate device memory -- a host that owns all device memory in its
   own pool, or a frame loop that must not stall on cudaMalloc/cudaFree
   (which may synchronise the device).
   Computes what lhi_liquid_compute_divergence computes (mean over fluid
   cells, max-norm over fluid cells of [1, N-3]^3), but from DEVICE pointers
   the caller already holds, with no handle and no allocation of any kind.
   Fields are float for LHI_PRECISION_FP32 / MIXED and double for FP64, in
   the layouts listed at the top of this file; dx is the grid spacing of the
   x axis; stream is a cudaStream_t of the current device (NULL = the legacy
   default stream).
   Scratch is a fixed device array inside the library (about 192 KB, held by
   every GPU that loads the library until the process exits), so grids above
   LHI_NOALLOC_MAX_CELLS cells are rejected with LHI_E_INVALID_ARG.  The first
   call on each device looks up that array's device address; make that first
   call before any stream capture.  Every call shares the one array: calls
   that overlap on the GPU (other streams, other host threads) race and must
   be serialised by the caller.  The call synchronises the stream to return
   the two values. */
#define LHI_NOALLOC_MAX_CELLS 16777216 /* 256^3 */
LHI_API int lhi_divergence_noalloc(const int32_t dim[3], double dx, int32_t precision, const void* liquid_phi,
                                   const void* liquid_wx, const void* liquid_wy, const void* liquid_wz,
                                   const void* vx, const void* vy, const void* vz, void* stream, double* mean,
                                   double* max_abs);

/* ------------------------------------------------- seeded scene builder */
/* RectBoundary / OperatorBoundary::Compute (Boundary.h:38-90) on the host,
   in the given precision (0 float, 2 double), at n points (xyz triples). */
LHI_API int lhi_boundary_eval(const lhi_boundary_node* nodes, int32_t count, int32_t root,
                              int32_t precision, const void* points, int64_t n, void* out);
/* Seeds 8 jittered particles per fluid cell (2x2x2 sub-cells, jitter
   +-0.25 sub-cell, counter-based RNG keyed by seed): a cell is seeded when
   its centre is inside a fluid primitive and the boundary SDF there is >= 0.
   Call with pos == NULL to get the count; then with buffers of that size. */
LHI_API int lhi_scene_seed_particles(const lhi_grid_desc* grid, const lhi_boundary_node* nodes,
                                     int32_t count, int32_t root, const lhi_fluid_prim* prims,
                                     int32_t nprims, uint64_t seed, int32_t precision,
                                     int64_t* n_out, void* pos, void* vel);
/* ParticleSystem<3>::SpawnParticles (ParticleSystem.cpp:45-64): lattice of
   spacing 0.5 * default_radius over [min, max), capped at max_count. */
LHI_API int lhi_scene_spawn_lattice(const double min_coord[3], const double max_coord[3],
                                    double default_radius, int64_t max_count,
                                    int32_t precision, int64_t* n_out, void* pos);

#ifdef __cplusplus
}
#endif

#endif /* LHI_H_ */
