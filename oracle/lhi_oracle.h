/*
 * lhi_oracle.h -- CPU oracle for the liquid step.  TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of the reference's 3D liquid path
 * (LiquidModel.cpp:476-1134, PressureSolver.cpp:420-936, Grid.cpp:84-193,
 * Kernel.h:12-31, MathUtils.h:8-33, MathUtils.cpp:29-35,75-88,
 * Boundary.h:38-90, ParticleSystem.cpp:7-64), deterministic (bit-identical
 * for any thread count), in float (the reference's Scalar) or double.
 *
 * The library also carries the scene generator (lhi_scene_seed_particles and
 * friends, built from liquidhairinteration_b200/csrc/scene.cpp), so CPU-only
 * runs of the reference arm seed their particles without the CUDA library.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker.  The product never calls it.
 *
 * Pinning: the float build is checked bit-for-bit against the reference's own
 * sources compiled from the reference tree (oracle/refbuild, one OpenMP
 * thread, serial extrapolation flags) and against the reference's only
 * fixture (LiquidData.csv frame 0: the SpawnParticles lattice).
 */
#ifndef LHI_ORACLE_H_
#define LHI_ORACLE_H_

#include <stdint.h>
#include "lhi.h"

#ifdef __cplusplus
extern "C" {
#endif

#define LHO_API __attribute__((visibility("default")))

/* extrapolation flag semantics */
#define LHO_EXTRAP_JACOBI 0 /* flags read from the previous sweep (GPU semantics) */
#define LHO_EXTRAP_SERIAL 1 /* in-place flags in x-y-z loop order: the reference
                               run with one OpenMP thread (LiquidModel.cpp:964-975) */

typedef struct lho_model lho_model;

/* Threads of the oracle's parallel loops (0: every processor, the default).
   Results are bit-identical for any count: only loops whose iterations write
   disjoint data run in parallel, and every sum is taken serially. */
LHO_API void lho_set_threads(int32_t n);
LHO_API int32_t lho_get_threads(void);
/* OpenMP's default thread count for parallel regions the calling thread
   opens without a num_threads clause: the reference build's own loops. */
LHO_API void lho_set_omp_default_threads(int32_t n);
/* Message of the last failed scene-generator call in this library. */
LHO_API const char* lho_last_error(void);

/* dbl = 0: Scalar float; dbl = 1: Scalar double.  Host buffers use Scalar. */
LHO_API lho_model* lho_create(const lhi_grid_desc* grid, const lhi_solver_params* solver,
                              const lhi_liquid_params* liquid, int32_t dbl);
LHO_API void lho_destroy(lho_model* m);
LHO_API void lho_get_dx(const lho_model* m, double dx[3]);

LHO_API int lho_set_boundary(lho_model* m, const lhi_boundary_node* nodes, int32_t count,
                             int32_t root);
LHO_API int lho_set_solid_phi(lho_model* m, const void* node_phi);
LHO_API int lho_boundary_eval(const lhi_boundary_node* nodes, int32_t count, int32_t root,
                              int32_t dbl, const void* points, int64_t n, void* out);

LHO_API int lho_set_particles(lho_model* m, int64_t n, const void* pos, const void* vel,
                              const void* affine);
LHO_API int lho_get_particles(lho_model* m, void* pos, void* vel, void* affine);
LHO_API int64_t lho_num_particles(const lho_model* m);

LHO_API int lho_field_size(const lho_model* m, int32_t field, int32_t level, int64_t* count,
                           int32_t* elem_bytes);
LHO_API int lho_get_field(lho_model* m, int32_t field, int32_t level, void* out);
LHO_API int lho_set_field(lho_model* m, int32_t field, int32_t level, const void* in);

LHO_API int lho_clear(lho_model* m);
LHO_API int lho_compute_liquid_phi(lho_model* m);
LHO_API int lho_particle_to_grid(lho_model* m);
LHO_API int lho_apply_gravity(lho_model* m, double dt);
LHO_API int lho_velocity_update(lho_model* m, double dt);
LHO_API int lho_projection(lho_model* m, double dt, lhi_solve_stats* stats);
LHO_API int lho_extrapolate(lho_model* m, int32_t mode);
LHO_API int lho_grid_to_particle(lho_model* m);
LHO_API int lho_advect_particles(lho_model* m, double dt);
LHO_API int lho_pre_step(lho_model* m, double dt);
LHO_API int lho_step(lho_model* m, double dt, int32_t extrap_mode, lhi_solve_stats* stats);
LHO_API int lho_correct_volume(lho_model* m, double dt);
LHO_API int lho_compute_divergence(lho_model* m, double* mean, double* max_abs);
LHO_API int lho_get_cfl(lho_model* m, double* dt_out);

LHO_API int lho_solver_init(lho_model* m);
LHO_API int lho_solver_build_rhs(lho_model* m);
LHO_API int lho_solver_build_lhs(lho_model* m, double density, double dt);
LHO_API int lho_solver_apply_preconditioner(lho_model* m);
LHO_API int lho_solver_solve(lho_model* m, double density, double dt, lhi_solve_stats* stats);
LHO_API int lho_solver_get_ax(lho_model* m, int32_t level, const void* x, void* out);

/* Cell key of every particle (caller order) and the stable sort by key:
   sorted_ids[k] = caller index of the k-th particle, cell_start[ncells+1]. */
LHO_API int lho_cell_keys(lho_model* m, int32_t* keys);
LHO_API int lho_sort_by_cell(lho_model* m, int32_t* sorted_ids, int32_t* cell_start);

/* LiquidModel<3>::Render restated without a graphics API (see
   lhi_liquid_render in lhi.h): float positions (n x 3) -> the vertex
   shader's coordinates and the RGBA image (row 0 at the bottom). */
LHO_API int lho_render(const float* pos, int64_t n, const float mn[3], const float mx[3],
                       const lhi_render_params* params, float* ndc, uint8_t* rgba);

/* ParticleSystem<3>::SpawnParticles restated (ParticleSystem.cpp:45-64). */
LHO_API int64_t lho_spawn_lattice(const double min_coord[3], const double max_coord[3],
                                  double default_radius, int64_t max_count, int32_t dbl,
                                  void* pos);

#ifdef __cplusplus
}
#endif
#endif
