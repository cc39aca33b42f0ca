/*
 * CPU oracle for the LBM step -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference solver
 *   src/lattices.js  (direction tables, weights stored as float32)
 *   src/sim.js       (class Sim: init, gradient pass, the seven step phases, RG8 pack)
 *   src/solid.js     (class RigidSphere: contains / surfaceVelocity /
 *                     applyImpulseAtCell / absorbDeadCells / step)
 * with the reference's arithmetic semantics: every intermediate in double,
 * rounded to float only when stored into a Float32Array field, no FMA
 * contraction (build with -ffp-contract=off), scan order z, y, x, k.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * this library, and only as the checker or the timed CPU baseline.  The GPU
 * product path never calls it.
 *
 * Pinning: the reference ships no golden vectors (its test/ scripts only
 * check finiteness, phi range and max|u|), and no JavaScript engine exists on
 * this machine.  tests/golden/make_golden.py runs the reference's own
 * lattices.js / solid.js / sim.js, translated mechanically into Python by
 * tests/golden/jsmini.py, and commits the results as .npz fixtures in
 * tests/golden; tests/test_golden_cpu.py requires this oracle to reproduce
 * every field, set, sphere state and impulse of those fixtures bit for bit.
 *
 * Multi-sphere scenes (the batched workload) use a composite solid: a cell is
 * SOLID when any sphere contains it, and the first containing sphere (lowest
 * index) owns the cell's surface velocity and every impulse applied at it.
 * With one sphere this is exactly the reference's single-solid behaviour.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Element type of the Float32Array fields.  The default build stores float32
 * like the reference; building with -DOR_STORE_DOUBLE keeps every field in
 * double, giving an FP64 reference for the GPU's FP64 storage form. */
#ifdef OR_STORE_DOUBLE
typedef double or_real;
#else
typedef float or_real;
#endif

#define OR_Q27 27
#define OR_Q7 7
#define OR_TAG_FLUID 0
#define OR_TAG_SOLID 1
#define OR_TAG_WALL 2
#define OR_MAX_SPHERES 8

/* RigidSphere state (src/solid.js:8-47). All doubles, like the JS numbers. */
typedef struct {
  int nx, ny, nz;
  double cx, cy, cz, r;
  double vx, vy, vz, wx, wy, wz;
  double density;
  int dragging;
  double dragTargetX, dragTargetY, dragTargetZ;
  double Fx, Fy, Fz, Tx, Ty, Tz;
  double volume, mass, I;
} or_sphere;

/* Sim state (src/sim.js:30-96).  Arrays use the reference layout:
 * cell i = (z*ny + y)*nx + x, populations AoS f[i*27 + k], h[i*7 + k]. */
typedef struct {
  int nx, ny, nz, n;
  or_real *f, *f2, *h, *h2;
  or_real *rho, *ux, *uy, *uz, *phi, *phiPrev;
  uint8_t *tag, *tagPrev;
  or_real *usx, *usy, *usz;
  or_real *gx, *gy, *gz, *lap;
  or_real *bodyFx, *bodyFy, *bodyFz;
  int32_t neighOffset27[OR_Q27], fOffset27[OR_Q27];
  int32_t neighOffset7[OR_Q7], hOffset7[OR_Q7];
  double tau, tauPhi, sigma, gravity, rhoL, rhoG, W, mobility;
  int omp; /* >0: parallelise the order-free phases with OpenMP (timing only) */
} or_sim;

/* sizeof(or_real) of this build */
int or_store_bytes(void);

/* Lattice tables (src/lattices.js:31-104). */
void or_tables(int8_t ex27[27], int8_t ey27[27], int8_t ez27[27], float w27[27],
               int8_t opp27[27], int8_t ex7[7], int8_t ey7[7], int8_t ez7[7],
               float w7[7], int8_t opp7[7]);

or_sim *or_sim_create(int nx, int ny, int nz);
void or_sim_destroy(or_sim *s);
void or_sim_set_omp(or_sim *s, int nthreads);

void or_init_flat(or_sim *s, double waterlineY);
void or_seed_hydrostatic(or_sim *s);
void or_compute_phi_gradients(or_sim *s);
/* solids may be NULL / nsolids 0 (the reference's `solid === null`). */
void or_retag_cells(or_sim *s, const or_sphere *solids, int nsolids);
void or_handle_fresh_cells(or_sim *s);
void or_collide_phase(or_sim *s);
void or_stream_phase(or_sim *s);
void or_collide_hydro(or_sim *s);
void or_stream_hydro_and_macro(or_sim *s, or_sphere *solids, int nsolids);
void or_step(or_sim *s, or_sphere *solids, int nsolids);
void or_pack_volume(const or_sim *s, uint8_t *out);

/* RigidSphere (src/solid.js). */
void or_sphere_init(or_sphere *b, int nx, int ny, int nz, double cx, double cy,
                    double cz, double r, double density);
void or_sphere_recompute_mass(or_sphere *b);
int or_sphere_contains(const or_sphere *b, int x, int y, int z);
void or_sphere_surface_velocity(const or_sphere *b, int x, int y, int z, double out[3]);
void or_sphere_apply_impulse(or_sphere *b, int x, int y, int z, double px, double py,
                             double pz);
void or_absorb_dead_cells(or_sphere *solids, int nsolids, const or_sim *s);
void or_sphere_step(or_sphere *b, double dt, double gravity);

/* One worker tick (src/worker.js:96-100): sim.step, absorbDeadCells, solid.step. */
void or_worker_substep(or_sim *s, or_sphere *solids, int nsolids);

#ifdef __cplusplus
}
#endif
#endif
