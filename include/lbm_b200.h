/*
 * lbm_b200.h -- C ABI of the B200-native LBM step.
 *
 * Drop-in for the reference's `Sim` (src/sim.js:29-601) and the per-cell /
 * per-link work of `RigidSphere` (src/solid.js:50-101).  A Node N-API addon,
 * a ctypes module or a C program binds these symbols; every entry point takes
 * plain pointers and sizes and returns an int status (0 = ok, negative = error,
 * message via lbm_last_error).  A handle owns one CUDA stream and all device
 * state of one scene; it is not thread-safe (one owner thread, like the
 * reference's single Web Worker, src/worker.js:1-6).
 *
 * Layout seen through this ABI is the reference's: cell i = (z*ny + y)*nx + x,
 * populations array-of-structures f[i*27 + k], h[i*7 + k] (src/sim.js:35-38,
 * 98).  On the device the populations live structure-of-arrays.
 *
 * The sphere is passed as a descriptor (cx..wz); the device evaluates
 * RigidSphere.contains / surfaceVelocity in FP64 and returns the summed
 * momentum-exchange force and torque that RigidSphere.applyImpulseAtCell would
 * have accumulated (src/solid.js:70-80).  Several spheres form a composite
 * solid: the first sphere that contains a cell owns it.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define LBM_OK 0
#define LBM_ERR_ARG (-1)          /* bad argument (null, size, range)          */
#define LBM_ERR_OOM (-2)          /* device allocation refused                 */
#define LBM_ERR_CUDA (-3)         /* CUDA runtime error                        */
#define LBM_ERR_TIMEOUT (-4)      /* bounded device wait ran out               */
#define LBM_ERR_NAN (-5)          /* NaN/Inf watchdog tripped                  */
#define LBM_ERR_STATE (-6)        /* call not valid in the current state       */
#define LBM_ERR_UNSUPPORTED (-7)  /* option not built / not supported          */
#define LBM_ERR_CAPACITY (-8)     /* a fixed-size device list overflowed       */

/* ---- population storage forms -------------------------------------------- */
#define LBM_STORE_F32 0  /* plain FP32 drop-in                                    */
#define LBM_STORE_F16 1  /* FP16 offsets f-w_k, h-w_k*phi; FP32 arithmetic         */
#define LBM_STORE_BF16 2 /* BF16 offsets f-w_k, h-w_k*phi; FP32 arithmetic         */
#define LBM_STORE_F64 3  /* FP64 storage and arithmetic (GPU error reference)     */

/* ---- fields (lbm_upload_field / lbm_download_field) ----------------------- */
/* Element type is float32 for every field except TAG/TAG_PREV (uint8).       */
#define LBM_FIELD_F 0        /* n*27, AoS, current populations  (sim.f)       */
#define LBM_FIELD_F2 1       /* n*27, AoS, post-collision       (sim.f2)      */
#define LBM_FIELD_H 2        /* n*7                              (sim.h)      */
#define LBM_FIELD_H2 3       /* n*7                              (sim.h2)     */
#define LBM_FIELD_RHO 4      /* sum f, the pressure proxy        (sim.rho)    */
#define LBM_FIELD_UX 5
#define LBM_FIELD_UY 6
#define LBM_FIELD_UZ 7
#define LBM_FIELD_PHI 8
#define LBM_FIELD_PHI_PREV 9
#define LBM_FIELD_TAG 10     /* uint8: 0 FLUID, 1 SOLID, 2 WALL (src/lattices.js:102-104) */
#define LBM_FIELD_TAG_PREV 11
#define LBM_FIELD_USX 12     /* solid surface velocity at SOLID cells          */
#define LBM_FIELD_USY 13
#define LBM_FIELD_USZ 14
#define LBM_FIELD_GX 15      /* grad phi / lap phi scratch (sim.gx..sim.lap)   */
#define LBM_FIELD_GY 16
#define LBM_FIELD_GZ 17
#define LBM_FIELD_LAP 18
#define LBM_FIELD_BODY_FX 19 /* per-cell external force, consumed and zeroed by
                                the next hydro stream (src/sim.js:61-64, 581) */
#define LBM_FIELD_BODY_FY 20
#define LBM_FIELD_BODY_FZ 21
#define LBM_FIELD_COUNT 22

typedef struct lbm_sim lbm_sim;

/* Physics parameters (src/sim.js:88-95); plain doubles like the JS fields. */
typedef struct {
  double tau, tauPhi, sigma, gravity, rhoL, rhoG, W, mobility;
} lbm_params;

/* RigidSphere state (src/solid.js:9-44).  The per-cell kernels read only
 * cx..wz; the device-resident integrator (lbm_run_coupled) reads and writes
 * all of it, with RigidSphere.step's FP64 arithmetic (src/solid.js:104-210). */
typedef struct {
  double cx, cy, cz, r;
  double vx, vy, vz, wx, wy, wz;
  double density, mass, I;
  double dragTargetX, dragTargetY, dragTargetZ;
  double Fx, Fy, Fz, Tx, Ty, Tz;
  int32_t dragging;
  int32_t reserved;
} lbm_sphere;

/* Summed momentum exchange for one sphere. */
typedef struct {
  double Fx, Fy, Fz, Tx, Ty, Tz;
} lbm_impulse;

#define LBM_MAX_SPHERES 8

/* ---- lifetime ------------------------------------------------------------- */
/* new Sim(nx, ny, nz) (src/sim.js:30-96).  device: CUDA ordinal.  Every field
 * starts zeroed, params take the reference defaults. */
int lbm_create(int nx, int ny, int nz, int storage, int device, lbm_sim **out);
int lbm_destroy(lbm_sim *sim);
const char *lbm_last_error(const lbm_sim *sim);
int lbm_get_dims(const lbm_sim *sim, int *nx, int *ny, int *nz, int *storage);
/* Bytes of device memory this handle holds. */
int lbm_device_bytes(const lbm_sim *sim, size_t *bytes);
/* Bytes a handle of this size would hold (admission control). */
size_t lbm_footprint_bytes(int nx, int ny, int nz, int storage);

/* Plain property writes sim.tau = ... (src/sim.js:88-95, src/worker.js:139-145). */
int lbm_set_params(lbm_sim *sim, const lbm_params *p);
int lbm_get_params(const lbm_sim *sim, lbm_params *p);

/* ---- field transfer (reference layout, synchronous) ------------------------ */
int lbm_upload_field(lbm_sim *sim, int field, const void *host, size_t count);
int lbm_download_field(lbm_sim *sim, int field, void *host, size_t count);
/* Same, as double (exact for the FP64 storage form); not for the tag fields. */
int lbm_download_field_f64(lbm_sim *sim, int field, double *host, size_t count);

/* ---- init (src/sim.js:112-173) --------------------------------------------- */
int lbm_init_flat(lbm_sim *sim, double waterlineY);
int lbm_seed_hydrostatic(lbm_sim *sim);
/* initFlat with the caller's column profile instead of the waterline's tanh:
 * phi = phiPrev = phi_col[y] (ny doubles) on every cell of row y, h = w7 phi,
 * f = w27, rho 1, u 0, walls tagged, then seedHydrostatic -- what a host
 * that writes phi and h cell by cell after initFlat (the dam preset,
 * src/worker.js:57-73) gets for a profile that depends on y only, without
 * moving the fields through the host. */
int lbm_init_profile(lbm_sim *sim, const double *phi_col, int ny);

/* ---- the seven phases, callable one by one (src/sim.js:176-582) ------------- */
/* spheres may be NULL with nspheres 0 (the reference's solid === null). */
int lbm_retag_cells(lbm_sim *sim, const lbm_sphere *spheres, int nspheres);
int lbm_handle_fresh_cells(lbm_sim *sim);
/* retagCells(solid) for any duck-typed solid (src/sim.js:214-244, README.md:
 * 69-73), the generic fallback beside the sphere descriptors: the host has
 * called solid.contains(x, y, z) for every interior cell (solid_mask[i]
 * non-zero where it returned true; n bytes) and solid.surfaceVelocity for
 * those cells (surface_velocity[3*i .. 3*i+2], 3*n floats, or NULL for a
 * solid at rest).  Boundary cells become WALL whatever the mask says.  The
 * next fused lbm_step retags the whole grid. */
int lbm_retag_cells_mask(lbm_sim *sim, const uint8_t *solid_mask, const float *surface_velocity);
/* A rigid body given as a closed triangle mesh (README.md:65-73: the solid
 * interface is mesh-agnostic), voxelised on the device.  tri: 9 doubles per
 * triangle (three vertices, world coordinates in cells); a cell is inside
 * when the ray from its centre towards +x crosses the mesh an odd number of
 * times (edge functions with a top-left rule, every operation rounded
 * explicitly).  Inside cells get the rigid-body surface velocity
 * v + w x (centre - c) of src/solid.js:57-66 as float. */
typedef struct {
  double cx, cy, cz; /* the point the angular velocity turns about */
  double vx, vy, vz; /* linear velocity */
  double wx, wy, wz; /* angular velocity */
} lbm_rigid_motion;
/* the mask (n bytes) and, with us_out, the surface velocities (3n floats) */
int lbm_voxelize_mesh(lbm_sim *sim, const double *tri, int ntri, const lbm_rigid_motion *motion,
                      uint8_t *mask_out, float *us_out);
/* retagCells for the mesh body: lbm_retag_cells_mask with the mask and
 * velocities made on the device */
int lbm_retag_cells_mesh(lbm_sim *sim, const double *tri, int ntri, const lbm_rigid_motion *motion);
int lbm_compute_phi_gradients(lbm_sim *sim);
int lbm_collide_phase(lbm_sim *sim);
int lbm_stream_phase(lbm_sim *sim);
int lbm_collide_hydro(lbm_sim *sim);
/* out: one lbm_impulse per sphere (may be NULL). */
int lbm_stream_hydro_and_macro(lbm_sim *sim, const lbm_sphere *spheres, int nspheres,
                               lbm_impulse *out);

/* The momentum-exchange links of the last lbm_stream_hydro_and_macro, for a
 * duck-typed solid whose applyImpulseAtCell the host calls itself
 * (src/sim.js:517-536): in the reference's scan order (cells z, y, x, then
 * direction k), each FLUID cell i with a SOLID source i - e_k gives
 * (cells[j] = i, dirs[j] = k, mom[j] = f2_opp(i) + f_k(i)); the impulse at
 * the solid cell (x - ex, y - ey, z - ez) is -mom * e_k.  *count receives the
 * number of links; at most cap are written (cap = 0 only counts).  Valid
 * until the next call that changes f or f2. */
int lbm_solid_links(lbm_sim *sim, int32_t *cells, int8_t *dirs, double *mom, int cap, int *count);

/* ---- Sim.step (src/sim.js:202-210), fused ---------------------------------- */
/* retag + fresh cells on the spheres' bounding boxes, then one fused
 * gradient + collide + pull-stream + bounce-back + macro pass per step. */
int lbm_step(lbm_sim *sim, const lbm_sphere *spheres, int nspheres, lbm_impulse *out);
/* lbm_step in two halves, for z slabs of one scene (lbm_set_slab): begin =
 * retagCells + handleFreshCells (src/sim.js:203-204), end = the rest of the
 * step with the same spheres.  A slab's fresh cells are filled in the scene's
 * scan order when the slabs begin in z order with each slab's two top owned
 * planes copied into the next slab's copied planes after its begin, and the
 * two bottom owned planes copied down before the lower slab's end.
 * lbm_step = begin + end.  LBM_ERR_STATE for a begin after a begin or an end
 * without one. */
int lbm_step_begin(lbm_sim *sim, const lbm_sphere *spheres, int nspheres);
int lbm_step_end(lbm_sim *sim, const lbm_sphere *spheres, int nspheres, lbm_impulse *out);

/* RigidSphere.absorbDeadCells(sim) (src/solid.js:87-101): impulse rho(phi)*u
 * of every cell that turned FLUID -> SOLID at the last retag, summed in scan
 * order in FP64 per owning sphere.  lbm_step / lbm_step_end (fused path)
 * already compute this sum for the spheres they were given and fetch it with
 * their own impulses; called next with spheres of the same position, radius
 * and velocities, this returns that result without a launch or a wait.  Any
 * other call on the handle in between (or other spheres) makes it compute
 * anew; the bits are the same either way. */
int lbm_absorb_dead_cells(lbm_sim *sim, const lbm_sphere *spheres, int nspheres,
                          lbm_impulse *out);

/* Sim.packVolume(out) (src/sim.js:586-600): 2*n bytes, R = (clamp01(phi)*255)|0,
 * G = 255 on SOLID cells. */
int lbm_pack_volume(lbm_sim *sim, uint8_t *host_out);
/* Server start-up, no counterpart in the reference: load every fused kernel
 * of a storage form on the device (so no first launch waits for a module
 * load) and, with reserve_bytes > 0, grow the device's memory pool by that
 * much once (scene memory comes from the pool and stays there after a scene
 * is destroyed, so later scenes allocate without mapping new memory).
 * LBM_ERR_OOM when the reserve does not fit (the kernels are loaded
 * anyway).  lbm_trim_device_memory returns the pool's unused memory to the
 * device. */
int lbm_prepare_device(int device, int storage, uint64_t reserve_bytes);
int lbm_trim_device_memory(int device);
/* Page-locked host memory for the buffers a host reads every frame (packed
 * volumes, rendered images): device-to-host copies into it run at full link
 * speed, while a pageable destination is copied through driver staging
 * buffers at a fraction of that.  No counterpart in the reference (a Web
 * Worker posts an ArrayBuffer).  Free with lbm_host_free. */
int lbm_host_alloc(size_t bytes, void **out);
int lbm_host_free(void *p);
/* packVolume without waiting: the frame is packed on the handle's stream and
 * copied to host_out on a separate copy stream, so the copy overlaps the steps
 * queued after this call.  host_out (2*n bytes, best page-locked) holds the
 * frame once lbm_wait_frames (or lbm_synchronize) returns; the caller must not
 * read or reuse it before.  A later call waits on the device for the previous
 * copy before packing again.  No counterpart in the reference, whose worker
 * packs synchronously and posts the buffer (src/worker.js:102-111). */
int lbm_pack_volume_async(lbm_sim *sim, uint8_t *host_out);
/* lbm_step + lbm_pack_volume_async on a frame step, with the pack fused into
 * the step: the fused kernel writes the RG8 bytes of every cell it visits as
 * it writes the macros, a small launch adds the planes z = 0 and nz - 1, and
 * the volume is copied into host_frame on the copy stream.  The copy starts
 * when the next step's fused kernel is queued (it then runs beside that
 * kernel) or at the next lbm_wait_frames / lbm_wait_frame_slot, and is
 * complete after lbm_wait_frames.  The same bytes as lbm_step then
 * lbm_pack_volume. */
int lbm_step_frame(lbm_sim *sim, const lbm_sphere *spheres, int nspheres, lbm_impulse *out,
                   uint8_t *host_frame);
/* The asynchronous frames use two device buffers in turn.  Wait until the copy
 * out of the one the next lbm_step_frame / lbm_pack_volume_async will use has
 * reached its host buffer: a host that alternates two host buffers in the
 * same order thereby knows that the older one holds its frame (the worker's
 * pool of posted frame buffers, src/worker.js:17-21, 158-163). */
int lbm_wait_frame_slot(lbm_sim *sim);
int lbm_wait_frames(lbm_sim *sim);
/* Same, into device memory, asynchronous on the handle's stream. */
int lbm_pack_volume_device(lbm_sim *sim, void *device_out);

/* ---- device-resident coupled loop ------------------------------------------ */
/* nsteps x (sim.step, absorbDeadCells, RigidSphere.step(1, gravity)) entirely
 * on the device (src/worker.js:96-100); spheres in/out on the host.  When
 * frame_every > 0 and frames is non-NULL, the RG8 volume after every
 * frame_every-th step is copied to frames (2*n bytes per frame). */
int lbm_run_coupled(lbm_sim *sim, lbm_sphere *spheres, int nspheres, int nsteps,
                    int frame_every, uint8_t *frames);

/* RigidSphere.step(dt, gravity) (src/solid.js:104-210) on the host, in FP64
 * with the reference's operation order (the device-resident loop runs the
 * same code): for each sphere, gravity and the drag spring are added to the
 * accumulated Fx..Tz, then the capped, damped, snapped and wall-clamped
 * update of velocity, spin and centre; Fx..Tz are cleared.  nx, ny, nz give
 * the clamp walls.  Needs no device; for hosts (the Node addon) whose sphere
 * state lives in this struct. */
int lbm_sphere_step_host(lbm_sphere *spheres, int n, double dt, double gravity, int nx, int ny, int nz);

/* Wait for all work queued on the handle's stream.  Returns LBM_ERR_TIMEOUT
 * when a fused step since the last check was abandoned because one of its
 * bounded device waits ran out (its fields are not valid; the handle stays
 * usable, e.g. after lbm_init_flat).  lbm_step, lbm_run_coupled,
 * lbm_absorb_dead_cells and lbm_batch_run report the same when they return. */
int lbm_synchronize(lbm_sim *sim);
/* NaN/Inf watchdog, off by default (every = 0): the reference lets a
 * numerical blow-up show as NaN in the fields and raises nothing.  With
 * every > 0, once every steps have completed since the last scan, the call
 * that completed them (lbm_step, lbm_stream_hydro_and_macro, lbm_run_coupled
 * at its end, lbm_batch_run at its end, for each of its scenes) scans the
 * current phi, rho and u (one extra pass, 20 B per cell at FP32) and returns
 * LBM_ERR_NAN when one is NaN or infinite; lbm_last_error names the lowest
 * such cell.  The step itself has completed: its fields stay as computed.
 * Replaces nothing in the reference; the status code is listed with the
 * other error codes above. */
int lbm_set_nan_watchdog(lbm_sim *sim, int every);
/* CUDA stream of the handle (cudaStream_t), for callers that enqueue around it. */
void *lbm_stream(lbm_sim *sim);

/* ---- introspection used by tests and the bench ------------------------------ */
/* Sizes of the fresh (SOLID->FLUID) and dead (FLUID->SOLID) sets found at the
 * last retag, and the number of SOLID-source links seen by the last stream. */
int lbm_last_sets(lbm_sim *sim, int *n_fresh, int *n_dead);
/* Copy the last fresh / dead cell index lists (ascending scan order). */
int lbm_download_sets(lbm_sim *sim, int32_t *fresh, int cap_fresh, int32_t *dead,
                      int cap_dead);
/* Number of kernels this handle has launched since creation. */
int lbm_launch_count(const lbm_sim *sim, int64_t *count);
/* 1 when the library was built with bounds checks in the fused kernel
 * (make checked).  lbm_fault_record returns and clears the first recorded
 * violation: {location code, index, block (x | y<<20 | z<<40), thread
 * (x | y<<8)}, all zero when none. */
int lbm_checked_build(void);
int lbm_fault_record(lbm_sim *sim, int64_t out[4]);
/* Test hook for the bounded waits: while on, the fused kernel's staged forms
 * (rows 4 or 6 | LBM_FUSED_STAGED, 6 | LBM_FUSED_TMA) do not issue the first
 * plane copy of each tile, so that plane's wait runs out (about a second), the step is
 * abandoned and LBM_ERR_TIMEOUT is reported; the fault record then holds
 * location code 90.  No effect on the other forms. */
int lbm_test_withhold_stage_copy(lbm_sim *sim, int on);
/* Test hook for the fresh-cell fill: while on, the handle's fresh cells are
 * filled by one thread in scan order (the reference's loop) instead of in
 * parallel rounds; the results are the same bit for bit either way. */
int lbm_test_sequential_fill(lbm_sim *sim, int on);
/* Host->device and device->host bytes this handle has copied since creation. */
int lbm_transfer_bytes(const lbm_sim *sim, uint64_t *h2d, uint64_t *d2h);
/* Time the fused step kernel with CUDA events on the handle's stream.
 * enable = 1 starts recording (and clears the totals), 0 stops; the query
 * synchronises the stream and returns the summed kernel time and launch count. */
int lbm_fused_timing(lbm_sim *sim, int enable);
int lbm_fused_timing_query(lbm_sim *sim, double *total_ms, int64_t *launches);
/* Fused-kernel launch shape: rows per CTA and z planes per CTA.
 *   rows = 2, 4 or 8: the plain form (every storage form);
 *   rows = 4 or 6 | LBM_FUSED_COMPACT: the compact shared-memory ring (each
 *     direction keeps only the cells that can source it) with register loads
 *     of each plane (FP32/FP16/BF16 storage);
 *   rows = 4 or 6 | LBM_FUSED_ASYNC: the compact ring, each thread's loads of
 *     the next plane issued one plane ahead as per-thread asynchronous copies
 *     into shared memory (FP32/FP16/BF16);
 *   rows = 4 or 6 | LBM_FUSED_STAGED: the compact ring, the tile rows of the
 *     next plane staged by bulk asynchronous copies waited on with bounded
 *     mbarrier waits (FP32/FP16/BF16);
 *   rows = 6 | LBM_FUSED_TMA: the compact ring, the tile rows of the next
 *     plane staged by tensor-map (TMA) box copies, one per array, issued by a
 *     halo warp and waited on with bounded mbarrier waits (FP32/FP16/BF16);
 *     needs nx a multiple of 16, and a scene without it runs
 *     6 | LBM_FUSED_COMPACT instead (lbm_get_fused_config reports the shape
 *     that was set, lbm_get_launch_shape the one that runs);
 *   rows = 6 | LBM_FUSED_L2PF: the compact form with register loads, plus
 *     one lane per CTA that asks the tensor-copy unit, once per plane, to
 *     bring the tile's rows two planes ahead (three for FP16/BF16) into L2
 *     (tensor-map prefetches, nothing staged in shared memory, nothing
 *     waited on), so the cells' loads hit L2; needs nx a multiple of 16, otherwise it runs as
 *     6 | LBM_FUSED_COMPACT.  6 | LBM_FUSED_L2PF is the default for FP32
 *     (z-chunks of 22 planes), FP16 and BF16 (24); rows 4, z-chunks of 32
 *     for FP64.
 * Every shape gives the same results bit for bit. */
#define LBM_FUSED_STAGED 0x100
#define LBM_FUSED_COMPACT 0x400
#define LBM_FUSED_ASYNC 0x800
#define LBM_FUSED_TMA 0x1000
#define LBM_FUSED_L2PF 0x2000
int lbm_set_fused_config(lbm_sim *sim, int rows, int zchunk);
/* The tile shape the handle's fused launches use: the shape that was set,
 * or 6 | LBM_FUSED_COMPACT where 6 | LBM_FUSED_TMA or 6 | LBM_FUSED_L2PF was
 * set on a scene whose nx is not a multiple of 16. */
int lbm_get_launch_shape(const lbm_sim *sim, int *shape);
/* ---- one scene in z slabs (several handles, one or more GPUs) -------------- */
/* Declares the handle a z slab of a larger scene: its local plane k is the
 * scene's plane k + zoff; local planes own_lo .. own_hi (within 1 .. nz - 2)
 * are this slab's own, the planes below and above them copies of the
 * neighbouring slabs' (two planes each side, so the copied plane next to the
 * owned ones collides with a complete phi stencil; the outermost local plane
 * is the scene's wall or a copy whose results are discarded).  Spheres keep
 * the scene's coordinates: the library shifts them into the slab's frame
 * (exactly: zoff is an integer).  Impulses (lbm_step, lbm_absorb_dead_cells)
 * cover the owned planes only, so the slabs' impulses add up to the scene's.
 * Needs nx * ny divisible by 8.  The reference has no counterpart: it is one
 * scene in one typed-array set (src/sim.js:30-96); this splits scenes larger
 * than one GPU.  lbm_run_coupled and batches refuse slabs. */
int lbm_set_slab(lbm_sim *sim, int zoff, int own_lo, int own_hi);
/* After a step of both: copy nplanes planes (populations, phi, rho, u and tags
 * of the current state) from src's plane src_plane on to dst's plane
 * dst_plane -- the halo exchange between neighbouring slabs, device to device
 * (over NVLink between GPUs, with peer access enabled here).  Synchronous. */
int lbm_slab_copy_planes(lbm_sim *dst, int dst_plane, const lbm_sim *src, int src_plane, int nplanes);
/* The launch shape in use (the default or the last lbm_set_fused_config). */
int lbm_get_fused_config(const lbm_sim *sim, int *rows, int *zchunk);

/* ---- batches: many scenes stepped together ---------------------------------- */
/* The reference advances one scene per Web Worker (src/worker.js:94-115); a
 * batch advances many independent scenes of any sizes with one persistent
 * fused launch per step over the tiles of every scene (per-scene descriptors),
 * the per-scene plan / retag / fresh-cell / impulse / RigidSphere.step kernels
 * as parallel branches around it, and, with use_graph, the step sequence
 * captured once as a CUDA graph and replayed.  Each scene's results are the
 * same as lbm_run_coupled's on that scene alone.  All handles must be on one
 * device with one storage form; a handle belongs to at most one running batch.
 * rows / zchunk choose the fused tile shape (lbm_batch_time_fused times a
 * shape on the batch's current state, for an autotuner). */
typedef struct lbm_batch lbm_batch;
int lbm_batch_create(lbm_sim *const *sims, int n, lbm_batch **out);
int lbm_batch_destroy(lbm_batch *batch);
/* Replace the batch's scenes (same device and storage form), keeping its
 * stream, events, tables and page-locked frame buffer: a continuous-batching
 * server changes membership between ticks without building a new batch.  The
 * step graph is captured anew at the next lbm_batch_run. */
int lbm_batch_set_scenes(lbm_batch *batch, lbm_sim *const *sims, int n);
const char *lbm_batch_last_error(const lbm_batch *batch);
int lbm_batch_set_config(lbm_batch *batch, int rows, int zchunk);
/* nsteps coupled steps of every scene (lbm_run_coupled semantics): spheres[s]
 * holds nspheres[s] spheres of scene s (updated in place); with frame_every > 0
 * the RG8 volume of scene s after every frame_every-th step is appended to
 * frames[s] (2*n_s bytes per frame). */
int lbm_batch_run(lbm_batch *batch, lbm_sphere *const *spheres, const int *nspheres, int nsteps,
                  int frame_every, uint8_t *const *frames, int use_graph);
/* Average time of the batched fused kernel with the given tile shape, over
 * reps launches on the batch's current state (it rewrites the next half only;
 * run after lbm_batch_run). */
int lbm_batch_time_fused(lbm_batch *batch, int rows, int zchunk, int reps, double *ms);
/* Batched fused launches executed so far. */
int lbm_batch_launch_count(const lbm_batch *batch, int64_t *count);

/* ---- headless render of the RG8 volume -------------------------------------- */
/* Orbit camera of the reference's Renderer (src/render.js:405-412, 452-458):
 * azimuth and elevation in radians, distance in units of the largest grid
 * edge, light direction (normalised here).  lbm_camera_default fills the
 * reference's start view: azimuth pi/4, elevation -0.25, distance 2.4,
 * light (0.35, 0.75, 0.5). */
typedef struct {
  double azimuth, elev, dist;
  double light[3];
} lbm_camera;
void lbm_camera_default(lbm_camera *cam);
/* The reference's fragment shader (src/render.js:19-268: ray march of the
 * phi = 0.5 surface with refraction, reflection, Beer-Lambert tint, sphere
 * and sky shading, tonemap) over an RG8 volume in device memory (the
 * packVolume layout, 2*nx*ny*nz bytes), one thread per pixel, into
 * width*height RGBA8 pixels in device memory, top row first.  sphere may be
 * NULL.  Asynchronous on `stream` (a cudaStream_t). */
int lbm_render_volume(const uint8_t *d_vol, int nx, int ny, int nz, const lbm_sphere *sphere,
                      const lbm_camera *cam, int width, int height, uint8_t *d_out, void *stream);
/* Renderer.uploadVolume + draw (src/render.js:431-434, 484-513) for a handle:
 * packs its current state and renders it; the image (width*height*4 bytes,
 * top row first) goes to host memory. */
int lbm_render(lbm_sim *sim, const lbm_sphere *sphere, const lbm_camera *cam, int width, int height,
               uint8_t *host_out);

/* ---- allocation-free dead-cell sweep --------------------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory at the point of the call (an engine that owns all device memory
 * through its own pool, a host whose allocator belongs to another runtime, a
 * loop that must not pay cudaMalloc's synchronisation): the same sum as
 * lbm_absorb_dead_cells, on FP32 fields the caller owns, with no handle and no
 * allocation.  tag / tag_prev (uint8, n cells), phi, ux, uy, uz (float, n cells)
 * and out (6*nspheres doubles: Fx Fy Fz Tx Ty Tz per sphere, overwritten) are
 * device pointers in the reference's cell order; spheres is host memory.  The
 * work is queued on `stream` (a cudaStream_t, NULL for the default stream).
 * Its scratch is one fixed device array inside the library (about 8.4 MB per
 * GPU, held until exit): the spheres' search box may hold at most 2^20 cells,
 * larger boxes return LBM_ERR_CAPACITY.  The first call on each device sets
 * that array up and should come before any stream capture.  Calls share the
 * array, so calls that overlap on the GPU race.  A message for a non-zero
 * status goes to err (errlen bytes, may be NULL). */
int lbm_absorb_dead_cells_noalloc(int nx, int ny, int nz, double rho_liquid, double rho_gas,
                                  const uint8_t *tag, const uint8_t *tag_prev,
                                  const float *phi, const float *ux, const float *uy,
                                  const float *uz, const lbm_sphere *spheres, int nspheres,
                                  double *out, void *stream, char *err, size_t errlen);

#ifdef __cplusplus
}
#endif
#endif
