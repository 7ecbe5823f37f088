/*
 * mpm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement (f64, single thread, ordered-map sparse grid) of tessera-mpm's
 * deterministic reference pipeline: crates/tessera-mpm/src/world.rs,
 * material.rs and obstacle.rs.  The tests, `__graft_entry__.smoke()` and the
 * CPU-baseline leg of `bench.py` use it as the checker.  The product library
 * (libtmpm.so) never links or calls it.
 *
 * Parity of this restatement is pinned by the reference's own known-answer
 * tests, restated in tests/test_oracle.py (world.rs:659-968,
 * material.rs:547-665, sand_neo_hookean_tests.rs, obstacle.rs:793-1060).
 * The reference ships no golden vector files.
 */
#ifndef MPM_ORACLE_H
#define MPM_ORACLE_H

#include "../include/tmpm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrcWorld OrcWorld;

/* MpmWorld::new (world.rs:224-241). */
OrcWorld *orc_world_create(const TmpmParams *params, const TmpmParticleArrays *particles, int32_t *status);
void orc_world_destroy(OrcWorld *world);
OrcWorld *orc_world_clone(const OrcWorld *world);

/* MpmWorld::add_particles / remove_chunk / set_obstacles (world.rs:243-286). */
int32_t orc_world_add_particles(OrcWorld *world, const TmpmParticleArrays *particles, uint64_t *chunk);
int32_t orc_world_remove_chunk(OrcWorld *world, uint64_t chunk, size_t *removed);
int32_t orc_world_set_obstacles(OrcWorld *world, const TmpmObstacle *obstacles, size_t count);
void orc_world_set_use_cpic(OrcWorld *world, int32_t enabled);
int32_t orc_world_set_params(OrcWorld *world, const TmpmParams *params);

/* MpmWorld::stable_timestep (world.rs:288-303). */
double orc_world_stable_timestep(const OrcWorld *world);

/* MpmWorld::step / step_with_obstacle_reactions (world.rs:305-359). */
int32_t orc_world_step(OrcWorld *world, double dt);
int32_t orc_world_step_reactions(OrcWorld *world, double dt, double *reactions);

/* One MpmWorld::substep (world.rs:361-467) with a fixed dt, bypassing the CFL
 * split of `advance`.  reactions may be NULL. */
int32_t orc_world_substep_fixed(OrcWorld *world, double dt, double *reactions);

size_t orc_world_count(const OrcWorld *world);
uint64_t orc_world_substeps(const OrcWorld *world);
int32_t orc_world_read(const OrcWorld *world, TmpmParticleArrays *out);
int32_t orc_world_write(OrcWorld *world, const TmpmParticleArrays *in);
int32_t orc_world_set_force(OrcWorld *world, size_t index, const double force[3]);

/* P2G only (world.rs:369-399) with dt: number of grid nodes, then node data
 * (i, j, k, transfer key) and (mass, momentum xyz) in the BTreeMap key order. */
size_t orc_world_p2g(const OrcWorld *world, double dt, int64_t *keys_out, double *values_out, size_t capacity);

/* Material and obstacle primitives for known-answer tests. */
void orc_kirchhoff_stress(int32_t material, const double params[5], const double F_cm[9],
                          const double C_cm[9], const double plastic[3], double out_cm[9]);
void orc_project_deformation(int32_t material, const double params[5], const double F_cm[9],
                             const double plastic_in[3], double F_out_cm[9], double plastic_out[3]);
double orc_timestep_bound(int32_t material, const double params[5], double density,
                          const double velocity[3], double cell_width, double det);
int32_t orc_material_valid(int32_t material, const double params[5]);
int32_t orc_obstacle_valid(const TmpmObstacle *obstacle);
void orc_obstacle_surface(const TmpmObstacle *obstacle, const double point[3], double *distance, double normal[3]);
void orc_obstacle_contact_velocity(const TmpmObstacle *obstacle, const double point[3],
                                   const double velocity[3], const double normal[3], double out[3]);
int32_t orc_obstacle_may_contact(const TmpmObstacle *obstacle, const double point[3], double margin);

/* CPU baseline: `threads` independent copies of `world`, each advanced by
 * `substeps` fixed substeps of dt concurrently.  Returns wall seconds. */
double orc_bench_threads(const OrcWorld *world, int32_t threads, int32_t substeps, double dt);

#ifdef __cplusplus
}
#endif

#endif
