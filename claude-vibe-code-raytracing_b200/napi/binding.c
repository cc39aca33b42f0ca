/*
 * binding.c -- Node-API addon over the C ABI of include/lbm_b200.h.
 *
 * This is the "thin N-API C-ABI addon" through which the reference's own
 * JavaScript (src/worker.js and the test scripts test/NAME.mjs) drives the CUDA
 * step: napi/sim.js and napi/solid.js re-export classes with the reference's
 * names (src/sim.js:29, src/solid.js:8) built on the functions below.
 *
 * Conventions:
 *   - a scene handle is a JS external wrapping the lbm_sim pointer (destroyed
 *     by destroy() or, failing that, by the garbage collector's finalizer);
 *     a batch likewise;
 *   - fields travel as typed arrays in the reference's layout (Float32Array,
 *     Uint8Array for tags, Float64Array for the FP64 download);
 *   - spheres travel as a Float64Array of 23 numbers per sphere, the
 *     lbm_sphere struct's memory (22 doubles, then the int32 `dragging` in
 *     the low half of the 23rd) -- napi/solid.js keeps each RigidSphere's
 *     state in such an array; impulses come back in a Float64Array of 6 per
 *     sphere;
 *   - a non-zero status throws an Error whose code is "LBM_ERR_<n>" and whose
 *     message is lbm_last_error (the reference signals only by exceptions).
 * Entry points that take device pointers (lbm_pack_volume_device,
 * lbm_render_volume, lbm_absorb_dead_cells_noalloc, lbm_stream) have no
 * JavaScript caller and are not bound.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lbm_b200.h"
#include "napi_decls.h"

#define LBM_SPHERE_F64 23 /* sizeof(lbm_sphere) / sizeof(double) */
_Static_assert(sizeof(lbm_sphere) == LBM_SPHERE_F64 * sizeof(double), "lbm_sphere is 23 doubles");
_Static_assert(sizeof(lbm_impulse) == 6 * sizeof(double), "lbm_impulse is 6 doubles");
_Static_assert(sizeof(lbm_params) == 8 * sizeof(double), "lbm_params is 8 doubles");
_Static_assert(sizeof(lbm_camera) == 6 * sizeof(double), "lbm_camera is 6 doubles");
_Static_assert(sizeof(lbm_rigid_motion) == 9 * sizeof(double), "lbm_rigid_motion is 9 doubles");

#define MAX_ARGS 8

typedef struct {
  lbm_sim *sim;
} SimBox;
typedef struct {
  lbm_batch *batch;
} BatchBox;

/* ------------------------------------------------------------------ errors */
static napi_value undefined_value(napi_env env) {
  napi_value u = NULL;
  napi_get_undefined(env, &u);
  return u;
}

static napi_value throw_msg(napi_env env, int code, const char *msg) {
  char c[32];
  snprintf(c, sizeof c, "LBM_ERR_%d", code < 0 ? -code : code);
  napi_throw_error(env, c, msg && msg[0] ? msg : "lbm call failed");
  return NULL;
}

static napi_value check_sim(napi_env env, lbm_sim *h, int rc) {
  if (rc == LBM_OK) return undefined_value(env);
  return throw_msg(env, rc, h ? lbm_last_error(h) : "null handle");
}

/* ------------------------------------------------------------- arguments */
typedef struct {
  napi_env env;
  size_t argc;
  napi_value argv[MAX_ARGS];
  int failed;
} Args;

static int args_get(napi_env env, napi_callback_info info, Args *a, size_t need) {
  a->env = env;
  a->argc = MAX_ARGS;
  a->failed = 0;
  if (napi_get_cb_info(env, info, &a->argc, a->argv, NULL, NULL) != napi_ok) {
    napi_throw_error(env, "LBM_ERR_1", "could not read the call's arguments");
    return 0;
  }
  if (a->argc < need) {
    char m[64];
    snprintf(m, sizeof m, "expected %zu arguments, got %zu", need, a->argc);
    napi_throw_error(env, "LBM_ERR_1", m);
    return 0;
  }
  return 1;
}

static int arg_fail(Args *a, const char *msg) {
  if (!a->failed) napi_throw_error(a->env, "LBM_ERR_1", msg);
  a->failed = 1;
  return 0;
}

static double arg_f64(Args *a, size_t i) {
  double v = 0;
  if (i >= a->argc || napi_get_value_double(a->env, a->argv[i], &v) != napi_ok) arg_fail(a, "a number was expected");
  return v;
}

static int32_t arg_i32(Args *a, size_t i) {
  int32_t v = 0;
  if (i >= a->argc || napi_get_value_int32(a->env, a->argv[i], &v) != napi_ok) arg_fail(a, "an integer was expected");
  return v;
}

static int is_nullish(Args *a, size_t i) {
  napi_valuetype t;
  if (i >= a->argc) return 1;
  if (napi_typeof(a->env, a->argv[i], &t) != napi_ok) return 0;
  return t == napi_undefined || t == napi_null;
}

/* typed array of the given kind (or any kind when kind < 0): data, element count */
static void *arg_typed(Args *a, size_t i, int kind, size_t *count) {
  napi_typedarray_type t;
  size_t len = 0, off = 0;
  void *data = NULL;
  napi_value ab;
  if (i >= a->argc || napi_get_typedarray_info(a->env, a->argv[i], &t, &len, &data, &ab, &off) != napi_ok) {
    arg_fail(a, "a typed array was expected");
    return NULL;
  }
  if (kind >= 0 && (int)t != kind) {
    arg_fail(a, kind == napi_float64_array ? "a Float64Array was expected"
                : kind == napi_float32_array ? "a Float32Array was expected"
                : kind == napi_uint8_array   ? "a Uint8Array was expected"
                                             : "a typed array of another kind was expected");
    return NULL;
  }
  if (count) *count = len;
  return data;
}

/* spheres: null / undefined (none) or a Float64Array of 23 numbers per sphere */
static lbm_sphere *arg_spheres(Args *a, size_t i, int *n) {
  *n = 0;
  if (is_nullish(a, i)) return NULL;
  size_t len = 0;
  double *d = (double *)arg_typed(a, i, napi_float64_array, &len);
  if (!d) return NULL;
  if (len % LBM_SPHERE_F64 != 0 || len / LBM_SPHERE_F64 > LBM_MAX_SPHERES) {
    arg_fail(a, "spheres: a Float64Array of 23 numbers per sphere, at most 8 spheres");
    return NULL;
  }
  *n = (int)(len / LBM_SPHERE_F64);
  return (lbm_sphere *)d;
}

/* impulse output: a Float64Array of at least 6 numbers per sphere */
static lbm_impulse *arg_impulses(Args *a, size_t i, int n) {
  size_t len = 0;
  double *d = (double *)arg_typed(a, i, napi_float64_array, &len);
  if (!d) return NULL;
  if (len < (size_t)(6 * (n > 0 ? n : 1))) {
    arg_fail(a, "impulses: a Float64Array of 6 numbers per sphere");
    return NULL;
  }
  return (lbm_impulse *)d;
}

static lbm_sim *arg_sim(Args *a, size_t i) {
  void *p = NULL;
  if (i >= a->argc || napi_get_value_external(a->env, a->argv[i], &p) != napi_ok || !p) {
    arg_fail(a, "a scene handle was expected");
    return NULL;
  }
  SimBox *box = (SimBox *)p;
  if (!box->sim) arg_fail(a, "the scene handle was destroyed");
  return box->sim;
}

static lbm_batch *arg_batch(Args *a, size_t i) {
  void *p = NULL;
  if (i >= a->argc || napi_get_value_external(a->env, a->argv[i], &p) != napi_ok || !p) {
    arg_fail(a, "a batch handle was expected");
    return NULL;
  }
  BatchBox *box = (BatchBox *)p;
  if (!box->batch) arg_fail(a, "the batch handle was destroyed");
  return box->batch;
}

static napi_value num(napi_env env, double v) {
  napi_value r = NULL;
  napi_create_double(env, v, &r);
  return r;
}

/* ------------------------------------------------------------- lifetime */
static void sim_finalize(napi_env env, void *data, void *hint) {
  (void)env;
  (void)hint;
  SimBox *box = (SimBox *)data;
  if (box->sim) lbm_destroy(box->sim);
  free(box);
}

/* create(nx, ny, nz, storage, device) -> handle  (new Sim, src/sim.js:30-96) */
static napi_value js_create(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 3)) return NULL;
  int nx = arg_i32(&a, 0), ny = arg_i32(&a, 1), nz = arg_i32(&a, 2);
  int storage = a.argc > 3 && !is_nullish(&a, 3) ? arg_i32(&a, 3) : LBM_STORE_F32;
  int device = a.argc > 4 && !is_nullish(&a, 4) ? arg_i32(&a, 4) : 0;
  if (a.failed) return NULL;
  lbm_sim *h = NULL;
  int rc = lbm_create(nx, ny, nz, storage, device, &h);
  if (rc != LBM_OK) return throw_msg(env, rc, "lbm_create failed (grid size, storage form or device)");
  SimBox *box = (SimBox *)malloc(sizeof(SimBox));
  if (!box) {
    lbm_destroy(h);
    return throw_msg(env, LBM_ERR_OOM, "out of host memory");
  }
  box->sim = h;
  napi_value ext = NULL;
  if (napi_create_external(env, box, sim_finalize, NULL, &ext) != napi_ok) {
    lbm_destroy(h);
    free(box);
    return throw_msg(env, LBM_ERR_STATE, "could not create the handle object");
  }
  return ext;
}

static napi_value js_destroy(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 1)) return NULL;
  void *p = NULL;
  if (napi_get_value_external(env, a.argv[0], &p) != napi_ok || !p) return throw_msg(env, LBM_ERR_ARG, "not a handle");
  SimBox *box = (SimBox *)p;
  if (box->sim) lbm_destroy(box->sim);
  box->sim = NULL;
  return undefined_value(env);
}

static napi_value js_last_error(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 1)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  if (a.failed) return NULL;
  napi_value s = NULL;
  napi_create_string_utf8(env, lbm_last_error(h), (size_t)-1, &s);
  return s;
}

/* getDims(h, Int32Array(4)) -> nx, ny, nz, storage */
static napi_value js_get_dims(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t len = 0;
  int32_t *d = (int32_t *)arg_typed(&a, 1, napi_int32_array, &len);
  if (a.failed) return NULL;
  if (len < 4) return throw_msg(env, LBM_ERR_ARG, "getDims needs an Int32Array of 4");
  return check_sim(env, h, lbm_get_dims(h, &d[0], &d[1], &d[2], &d[3]));
}

static napi_value js_device_bytes(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 1)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  if (a.failed) return NULL;
  size_t b = 0;
  int rc = lbm_device_bytes(h, &b);
  if (rc != LBM_OK) return check_sim(env, h, rc);
  return num(env, (double)b);
}

static napi_value js_footprint_bytes(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 4)) return NULL;
  int nx = arg_i32(&a, 0), ny = arg_i32(&a, 1), nz = arg_i32(&a, 2), st = arg_i32(&a, 3);
  if (a.failed) return NULL;
  return num(env, (double)lbm_footprint_bytes(nx, ny, nz, st));
}

/* setParams(h, Float64Array(8)) / getParams(h, Float64Array(8)): tau, tauPhi,
 * sigma, gravity, rhoL, rhoG, W, mobility (src/sim.js:88-95) */
static napi_value js_set_params(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t len = 0;
  double *p = (double *)arg_typed(&a, 1, napi_float64_array, &len);
  if (a.failed) return NULL;
  if (len < 8) return throw_msg(env, LBM_ERR_ARG, "params: a Float64Array of 8");
  lbm_params q;
  memcpy(&q, p, sizeof q);
  return check_sim(env, h, lbm_set_params(h, &q));
}

static napi_value js_get_params(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t len = 0;
  double *p = (double *)arg_typed(&a, 1, napi_float64_array, &len);
  if (a.failed) return NULL;
  if (len < 8) return throw_msg(env, LBM_ERR_ARG, "params: a Float64Array of 8");
  lbm_params q;
  int rc = lbm_get_params(h, &q);
  if (rc == LBM_OK) memcpy(p, &q, sizeof q);
  return check_sim(env, h, rc);
}

/* ------------------------------------------------------------- fields */
/* uploadField(h, field, typedArray) / downloadField(h, field, typedArray):
 * the element count is the array's length (Float32Array; Uint8Array for the
 * tag fields) */
static napi_value js_upload_field(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 3)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  int field = arg_i32(&a, 1);
  size_t len = 0;
  void *d = arg_typed(&a, 2, field == LBM_FIELD_TAG || field == LBM_FIELD_TAG_PREV ? napi_uint8_array
                                                                                    : napi_float32_array, &len);
  if (a.failed) return NULL;
  return check_sim(env, h, lbm_upload_field(h, field, d, len));
}

static napi_value js_download_field(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 3)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  int field = arg_i32(&a, 1);
  size_t len = 0;
  void *d = arg_typed(&a, 2, field == LBM_FIELD_TAG || field == LBM_FIELD_TAG_PREV ? napi_uint8_array
                                                                                    : napi_float32_array, &len);
  if (a.failed) return NULL;
  return check_sim(env, h, lbm_download_field(h, field, d, len));
}

static napi_value js_download_field_f64(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 3)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  int field = arg_i32(&a, 1);
  size_t len = 0;
  double *d = (double *)arg_typed(&a, 2, napi_float64_array, &len);
  if (a.failed) return NULL;
  return check_sim(env, h, lbm_download_field_f64(h, field, d, len));
}

/* ------------------------------------------------------------- the step */
static napi_value js_init_flat(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  double y = arg_f64(&a, 1);
  if (a.failed) return NULL;
  return check_sim(env, h, lbm_init_flat(h, y));
}

/* the phases that take only the handle */
#define SIM_ONLY(jsname, call)                                   \
  static napi_value jsname(napi_env env, napi_callback_info info) { \
    Args a;                                                      \
    if (!args_get(env, info, &a, 1)) return NULL;                \
    lbm_sim *h = arg_sim(&a, 0);                                 \
    if (a.failed) return NULL;                                   \
    return check_sim(env, h, call(h));                           \
  }
SIM_ONLY(js_seed_hydrostatic, lbm_seed_hydrostatic)
SIM_ONLY(js_handle_fresh_cells, lbm_handle_fresh_cells)
SIM_ONLY(js_compute_phi_gradients, lbm_compute_phi_gradients)
SIM_ONLY(js_collide_phase, lbm_collide_phase)
SIM_ONLY(js_stream_phase, lbm_stream_phase)
SIM_ONLY(js_collide_hydro, lbm_collide_hydro)
SIM_ONLY(js_wait_frames, lbm_wait_frames)
SIM_ONLY(js_wait_frame_slot, lbm_wait_frame_slot)
SIM_ONLY(js_synchronize, lbm_synchronize)

static napi_value js_retag_cells(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 1)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  int n = 0;
  lbm_sphere *sp = arg_spheres(&a, 1, &n);
  if (a.failed) return NULL;
  return check_sim(env, h, lbm_retag_cells(h, sp, n));
}

/* the calls that take spheres and return their impulses */
#define SIM_SPHERES_OUT(jsname, call)                            \
  static napi_value jsname(napi_env env, napi_callback_info info) { \
    Args a;                                                      \
    if (!args_get(env, info, &a, 3)) return NULL;                \
    lbm_sim *h = arg_sim(&a, 0);                                 \
    int n = 0;                                                   \
    lbm_sphere *sp = arg_spheres(&a, 1, &n);                     \
    lbm_impulse *out = arg_impulses(&a, 2, n);                   \
    if (a.failed) return NULL;                                   \
    return check_sim(env, h, call(h, sp, n, out));               \
  }
SIM_SPHERES_OUT(js_stream_hydro_and_macro, lbm_stream_hydro_and_macro)
SIM_SPHERES_OUT(js_step, lbm_step)
SIM_SPHERES_OUT(js_absorb_dead_cells, lbm_absorb_dead_cells)

/* retagCellsMask(h, Uint8Array(n) mask, Float32Array(3n) | null velocities):
 * retagCells for a duck-typed solid evaluated on the host */
static napi_value js_retag_cells_mask(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t mlen = 0, ulen = 0;
  uint8_t *mask = (uint8_t *)arg_typed(&a, 1, napi_uint8_array, &mlen);
  float *us = NULL;
  if (a.argc > 2 && !is_nullish(&a, 2)) us = (float *)arg_typed(&a, 2, napi_float32_array, &ulen);
  if (a.failed) return NULL;
  int nx = 0, ny = 0, nz = 0, st = 0;
  lbm_get_dims(h, &nx, &ny, &nz, &st);
  const size_t n = (size_t)nx * ny * nz;
  if (mlen < n || (us && ulen < 3 * n)) return throw_msg(env, LBM_ERR_ARG, "retagCellsMask: n mask bytes, 3n velocities");
  return check_sim(env, h, lbm_retag_cells_mask(h, mask, us));
}

/* retagCellsMesh(h, Float64Array tri[9 * ntri], Float64Array motion[9]):
 * retagCells for a rigid triangle mesh, voxelised on the device */
static napi_value js_retag_cells_mesh(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 3)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t tlen = 0, mlen = 0;
  double *tri = (double *)arg_typed(&a, 1, napi_float64_array, &tlen);
  double *mo = (double *)arg_typed(&a, 2, napi_float64_array, &mlen);
  if (a.failed) return NULL;
  if (tlen % 9 != 0 || mlen < 9) return throw_msg(env, LBM_ERR_ARG, "retagCellsMesh: 9 numbers per triangle, 9 of motion");
  lbm_rigid_motion m;
  memcpy(&m, mo, sizeof m);
  return check_sim(env, h, lbm_retag_cells_mesh(h, tri, (int)(tlen / 9), &m));
}

/* voxelizeMesh(h, tri, motion, Uint8Array mask[n], Float32Array us[3n] | null) */
static napi_value js_voxelize_mesh(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 4)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t tlen = 0, mlen = 0, klen = 0, ulen = 0;
  double *tri = (double *)arg_typed(&a, 1, napi_float64_array, &tlen);
  double *mo = (double *)arg_typed(&a, 2, napi_float64_array, &mlen);
  uint8_t *mask = (uint8_t *)arg_typed(&a, 3, napi_uint8_array, &klen);
  float *us = NULL;
  if (a.argc > 4 && !is_nullish(&a, 4)) us = (float *)arg_typed(&a, 4, napi_float32_array, &ulen);
  if (a.failed) return NULL;
  int nx = 0, ny = 0, nz = 0, st = 0;
  lbm_get_dims(h, &nx, &ny, &nz, &st);
  const size_t n = (size_t)nx * ny * nz;
  if (tlen % 9 != 0 || mlen < 9 || klen < n || (us && ulen < 3 * n))
    return throw_msg(env, LBM_ERR_ARG, "voxelizeMesh: 9 numbers per triangle, 9 of motion, n mask bytes, 3n velocities");
  lbm_rigid_motion m;
  memcpy(&m, mo, sizeof m);
  return check_sim(env, h, lbm_voxelize_mesh(h, tri, (int)(tlen / 9), &m, mask, us));
}

/* solidLinks(h, Int32Array cells | null, Int8Array dirs | null, Float64Array mom | null)
 * -> number of links of the last streamHydroAndMacro (as many written as fit) */
static napi_value js_solid_links(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 1)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  int32_t *cells = NULL;
  int8_t *dirs = NULL;
  double *mom = NULL;
  size_t cl = 0, dl = 0, ml = 0;
  if (a.argc > 3 && !is_nullish(&a, 1)) {
    cells = (int32_t *)arg_typed(&a, 1, napi_int32_array, &cl);
    dirs = (int8_t *)arg_typed(&a, 2, napi_int8_array, &dl);
    mom = (double *)arg_typed(&a, 3, napi_float64_array, &ml);
  }
  if (a.failed) return NULL;
  size_t cap = cl < dl ? cl : dl;
  cap = cap < ml ? cap : ml;
  int count = 0;
  int rc = lbm_solid_links(h, cells, dirs, mom, cells ? (int)cap : 0, &count);
  if (rc != LBM_OK) return check_sim(env, h, rc);
  return num(env, (double)count);
}

/* packVolume(h, Uint8Array(2n)) (src/sim.js:586-600) */
static napi_value js_pack_volume(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t len = 0;
  uint8_t *d = (uint8_t *)arg_typed(&a, 1, napi_uint8_array, &len);
  if (a.failed) return NULL;
  int nx = 0, ny = 0, nz = 0, st = 0;
  lbm_get_dims(h, &nx, &ny, &nz, &st);
  if (len < 2 * (size_t)nx * ny * nz) return throw_msg(env, LBM_ERR_ARG, "packVolume needs 2 * nx * ny * nz bytes");
  return check_sim(env, h, lbm_pack_volume(h, d));
}

/* packVolumeAsync(h, Uint8Array(2n)): the array must stay referenced (and
 * unread) until waitFrames(h) */
static napi_value js_pack_volume_async(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t len = 0;
  uint8_t *d = (uint8_t *)arg_typed(&a, 1, napi_uint8_array, &len);
  if (a.failed) return NULL;
  int nx = 0, ny = 0, nz = 0, st = 0;
  lbm_get_dims(h, &nx, &ny, &nz, &st);
  if (len < 2 * (size_t)nx * ny * nz) return throw_msg(env, LBM_ERR_ARG, "packVolumeAsync needs 2 * nx * ny * nz bytes");
  return check_sim(env, h, lbm_pack_volume_async(h, d));
}

/* stepFrame(h, spheres, out, Uint8Array frame): step with packVolume fused
 * into it; the frame is copied into `frame` asynchronously (waitFrames) */
static napi_value js_step_frame(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 4)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  int n = 0;
  lbm_sphere *sp = arg_spheres(&a, 1, &n);
  lbm_impulse *out = arg_impulses(&a, 2, n);
  size_t len = 0;
  uint8_t *d = (uint8_t *)arg_typed(&a, 3, napi_uint8_array, &len);
  if (a.failed) return NULL;
  int nx = 0, ny = 0, nz = 0, st = 0;
  lbm_get_dims(h, &nx, &ny, &nz, &st);
  if (len < 2 * (size_t)nx * ny * nz) return throw_msg(env, LBM_ERR_ARG, "stepFrame needs 2 * nx * ny * nz bytes");
  return check_sim(env, h, lbm_step_frame(h, sp, n, out, d));
}

/* initProfile(h, Float64Array phiCol[ny]): initFlat with a column profile */
static napi_value js_init_profile(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t len = 0;
  double *col = (double *)arg_typed(&a, 1, napi_float64_array, &len);
  if (a.failed) return NULL;
  return check_sim(env, h, lbm_init_profile(h, col, (int)len));
}

/* runCoupled(h, spheres, nsteps, frameEvery, frames | null): the worker's tick
 * (src/worker.js:96-100) nsteps times on the device; spheres updated in place */
static napi_value js_run_coupled(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 3)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  int n = 0;
  lbm_sphere *sp = arg_spheres(&a, 1, &n);
  int nsteps = arg_i32(&a, 2);
  int every = a.argc > 3 && !is_nullish(&a, 3) ? arg_i32(&a, 3) : 0;
  uint8_t *frames = NULL;
  size_t flen = 0;
  if (every > 0 && !is_nullish(&a, 4)) frames = (uint8_t *)arg_typed(&a, 4, napi_uint8_array, &flen);
  if (a.failed) return NULL;
  if (frames) {
    int nx = 0, ny = 0, nz = 0, st = 0;
    lbm_get_dims(h, &nx, &ny, &nz, &st);
    if (flen < (size_t)(nsteps / every) * 2 * (size_t)nx * ny * nz)
      return throw_msg(env, LBM_ERR_ARG, "frames: 2 * nx * ny * nz bytes per frame");
  }
  return check_sim(env, h, lbm_run_coupled(h, sp, n, nsteps, frames ? every : 0, frames));
}

/* sphereStep(spheres, dt, gravity, nx, ny, nz): RigidSphere.step on the host */
static napi_value js_sphere_step(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 6)) return NULL;
  int n = 0;
  lbm_sphere *sp = arg_spheres(&a, 0, &n);
  double dt = arg_f64(&a, 1), g = arg_f64(&a, 2);
  int nx = arg_i32(&a, 3), ny = arg_i32(&a, 4), nz = arg_i32(&a, 5);
  if (a.failed) return NULL;
  int rc = lbm_sphere_step_host(sp, n, dt, g, nx, ny, nz);
  if (rc != LBM_OK) return throw_msg(env, rc, "sphereStep: bad arguments");
  return undefined_value(env);
}

static napi_value js_set_nan_watchdog(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  int every = arg_i32(&a, 1);
  if (a.failed) return NULL;
  return check_sim(env, h, lbm_set_nan_watchdog(h, every));
}

/* lastSets(h, counts Int32Array(2), fresh Int32Array | null, dead Int32Array | null):
 * the numbers of fresh and dead cells of the last retag into counts, and as
 * many of the scan-ordered cell indices as fit into fresh and dead */
static napi_value js_last_sets(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t clen = 0;
  int32_t *counts = (int32_t *)arg_typed(&a, 1, napi_int32_array, &clen);
  int32_t *fresh = NULL, *dead = NULL;
  size_t flen = 0, dlen = 0;
  if (a.argc > 2 && !is_nullish(&a, 2)) fresh = (int32_t *)arg_typed(&a, 2, napi_int32_array, &flen);
  if (a.argc > 3 && !is_nullish(&a, 3)) dead = (int32_t *)arg_typed(&a, 3, napi_int32_array, &dlen);
  if (a.failed) return NULL;
  if (clen < 2) return throw_msg(env, LBM_ERR_ARG, "lastSets needs an Int32Array(2) for the counts");
  int nf = 0, nd = 0;
  int rc = lbm_last_sets(h, &nf, &nd);
  if (rc != LBM_OK) return check_sim(env, h, rc);
  counts[0] = nf;
  counts[1] = nd;
  if (fresh || dead) rc = lbm_download_sets(h, fresh, (int)flen, dead, (int)dlen);
  return check_sim(env, h, rc);
}

/* launchCount(h), checkedBuild() */
static napi_value js_launch_count(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 1)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  if (a.failed) return NULL;
  int64_t c = 0;
  int rc = lbm_launch_count(h, &c);
  if (rc != LBM_OK) return check_sim(env, h, rc);
  return num(env, (double)c);
}

static napi_value js_checked_build(napi_env env, napi_callback_info info) {
  (void)info;
  return num(env, (double)lbm_checked_build());
}

/* faultRecord(h, Float64Array(4)) */
static napi_value js_fault_record(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t len = 0;
  double *d = (double *)arg_typed(&a, 1, napi_float64_array, &len);
  if (a.failed) return NULL;
  if (len < 4) return throw_msg(env, LBM_ERR_ARG, "faultRecord needs a Float64Array of 4");
  int64_t r[4] = {0, 0, 0, 0};
  int rc = lbm_fault_record(h, r);
  for (int i = 0; i < 4; i++) d[i] = (double)r[i];
  return check_sim(env, h, rc);
}

/* transferBytes(h, Float64Array(2)): host->device, device->host */
static napi_value js_transfer_bytes(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t len = 0;
  double *d = (double *)arg_typed(&a, 1, napi_float64_array, &len);
  if (a.failed) return NULL;
  if (len < 2) return throw_msg(env, LBM_ERR_ARG, "transferBytes needs a Float64Array of 2");
  uint64_t up = 0, down = 0;
  int rc = lbm_transfer_bytes(h, &up, &down);
  d[0] = (double)up;
  d[1] = (double)down;
  return check_sim(env, h, rc);
}

/* fusedTiming(h, on) ; fusedTimingQuery(h, Float64Array(2)): total ms, launches */
static napi_value js_fused_timing(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  int on = arg_i32(&a, 1);
  if (a.failed) return NULL;
  return check_sim(env, h, lbm_fused_timing(h, on));
}

static napi_value js_fused_timing_query(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t len = 0;
  double *d = (double *)arg_typed(&a, 1, napi_float64_array, &len);
  if (a.failed) return NULL;
  if (len < 2) return throw_msg(env, LBM_ERR_ARG, "fusedTimingQuery needs a Float64Array of 2");
  double ms = 0;
  int64_t n = 0;
  int rc = lbm_fused_timing_query(h, &ms, &n);
  d[0] = ms;
  d[1] = (double)n;
  return check_sim(env, h, rc);
}

static napi_value js_set_fused_config(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 3)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  int rows = arg_i32(&a, 1), zchunk = arg_i32(&a, 2);
  if (a.failed) return NULL;
  return check_sim(env, h, lbm_set_fused_config(h, rows, zchunk));
}

/* getFusedConfig(h, Int32Array(2)) -> rows, zchunk */
static napi_value js_get_fused_config(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  size_t len = 0;
  int32_t *d = (int32_t *)arg_typed(&a, 1, napi_int32_array, &len);
  if (a.failed) return NULL;
  if (len < 2) return throw_msg(env, LBM_ERR_ARG, "getFusedConfig needs an Int32Array of 2");
  return check_sim(env, h, lbm_get_fused_config(h, &d[0], &d[1]));
}

static napi_value js_test_withhold_stage_copy(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 2)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  int on = arg_i32(&a, 1);
  if (a.failed) return NULL;
  return check_sim(env, h, lbm_test_withhold_stage_copy(h, on));
}

/* ------------------------------------------------------------- rendering */
/* cameraDefault(Float64Array(6)); render(h, spheres | null, camera, width,
 * height, Uint8Array(width * height * 4)) */
static napi_value js_camera_default(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 1)) return NULL;
  size_t len = 0;
  double *d = (double *)arg_typed(&a, 0, napi_float64_array, &len);
  if (a.failed) return NULL;
  if (len < 6) return throw_msg(env, LBM_ERR_ARG, "camera: a Float64Array of 6");
  lbm_camera c;
  lbm_camera_default(&c);
  memcpy(d, &c, sizeof c);
  return undefined_value(env);
}

static napi_value js_render(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 6)) return NULL;
  lbm_sim *h = arg_sim(&a, 0);
  int n = 0;
  lbm_sphere *sp = arg_spheres(&a, 1, &n);
  size_t clen = 0, ilen = 0;
  double *cam = (double *)arg_typed(&a, 2, napi_float64_array, &clen);
  int w = arg_i32(&a, 3), hgt = arg_i32(&a, 4);
  uint8_t *img = (uint8_t *)arg_typed(&a, 5, napi_uint8_array, &ilen);
  if (a.failed) return NULL;
  if (clen < 6 || w <= 0 || hgt <= 0 || ilen < (size_t)w * hgt * 4)
    return throw_msg(env, LBM_ERR_ARG, "render: camera of 6, image of width * height * 4 bytes");
  lbm_camera c;
  memcpy(&c, cam, sizeof c);
  return check_sim(env, h, lbm_render(h, n ? sp : NULL, &c, w, hgt, img));
}

/* ------------------------------------------------------------- batches */
static void batch_finalize(napi_env env, void *data, void *hint) {
  (void)env;
  (void)hint;
  BatchBox *box = (BatchBox *)data;
  if (box->batch) lbm_batch_destroy(box->batch);
  free(box);
}

static napi_value check_batch(napi_env env, lbm_batch *b, int rc) {
  if (rc == LBM_OK) return undefined_value(env);
  return throw_msg(env, rc, b ? lbm_batch_last_error(b) : "null batch");
}

/* batchCreate(h0, h1, ...) -> batch: up to MAX_ARGS scene handles per call */
static napi_value js_batch_create(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 1)) return NULL;
  lbm_sim *sims[MAX_ARGS];
  for (size_t i = 0; i < a.argc; i++) sims[i] = arg_sim(&a, i);
  if (a.failed) return NULL;
  lbm_batch *b = NULL;
  int rc = lbm_batch_create(sims, (int)a.argc, &b);
  if (rc != LBM_OK) return throw_msg(env, rc, "lbm_batch_create failed (handles on different devices or storage forms?)");
  BatchBox *box = (BatchBox *)malloc(sizeof(BatchBox));
  if (!box) {
    lbm_batch_destroy(b);
    return throw_msg(env, LBM_ERR_OOM, "out of host memory");
  }
  box->batch = b;
  napi_value ext = NULL;
  if (napi_create_external(env, box, batch_finalize, NULL, &ext) != napi_ok) {
    lbm_batch_destroy(b);
    free(box);
    return throw_msg(env, LBM_ERR_STATE, "could not create the batch object");
  }
  return ext;
}

static napi_value js_batch_destroy(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 1)) return NULL;
  void *p = NULL;
  if (napi_get_value_external(env, a.argv[0], &p) != napi_ok || !p) return throw_msg(env, LBM_ERR_ARG, "not a batch");
  BatchBox *box = (BatchBox *)p;
  if (box->batch) lbm_batch_destroy(box->batch);
  box->batch = NULL;
  return undefined_value(env);
}

static napi_value js_batch_set_config(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 3)) return NULL;
  lbm_batch *b = arg_batch(&a, 0);
  int rows = arg_i32(&a, 1), zchunk = arg_i32(&a, 2);
  if (a.failed) return NULL;
  return check_batch(env, b, lbm_batch_set_config(b, rows, zchunk));
}

/* batchRun(batch, spheresAll, counts, nsteps, useGraph): spheresAll is one
 * Float64Array holding every scene's spheres back to back, counts an
 * Int32Array with the number of spheres of each scene (frames are taken by
 * the caller between runs with packVolume) */
static napi_value js_batch_run(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 5)) return NULL;
  lbm_batch *b = arg_batch(&a, 0);
  size_t slen = 0, clen = 0;
  double *all = is_nullish(&a, 1) ? NULL : (double *)arg_typed(&a, 1, napi_float64_array, &slen);
  int32_t *counts = (int32_t *)arg_typed(&a, 2, napi_int32_array, &clen);
  int nsteps = arg_i32(&a, 3), graph = arg_i32(&a, 4);
  if (a.failed) return NULL;
  lbm_sphere **sp = (lbm_sphere **)calloc(clen ? clen : 1, sizeof(lbm_sphere *));
  if (!sp) return throw_msg(env, LBM_ERR_OOM, "out of host memory");
  size_t at = 0;
  for (size_t s = 0; s < clen; s++) {
    if (counts[s] < 0 || counts[s] > LBM_MAX_SPHERES || at + (size_t)counts[s] * LBM_SPHERE_F64 > slen) {
      free(sp);
      return throw_msg(env, LBM_ERR_ARG, "batchRun: counts do not match the sphere array");
    }
    sp[s] = counts[s] ? (lbm_sphere *)(all + at) : NULL;
    at += (size_t)counts[s] * LBM_SPHERE_F64;
  }
  int rc = lbm_batch_run(b, sp, (const int *)counts, nsteps, 0, NULL, graph);
  free(sp);
  return check_batch(env, b, rc);
}

static napi_value js_batch_time_fused(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 4)) return NULL;
  lbm_batch *b = arg_batch(&a, 0);
  int rows = arg_i32(&a, 1), zchunk = arg_i32(&a, 2), reps = arg_i32(&a, 3);
  if (a.failed) return NULL;
  double ms = 0;
  int rc = lbm_batch_time_fused(b, rows, zchunk, reps, &ms);
  if (rc != LBM_OK) return check_batch(env, b, rc);
  return num(env, ms);
}

static napi_value js_batch_launch_count(napi_env env, napi_callback_info info) {
  Args a;
  if (!args_get(env, info, &a, 1)) return NULL;
  lbm_batch *b = arg_batch(&a, 0);
  if (a.failed) return NULL;
  int64_t c = 0;
  int rc = lbm_batch_launch_count(b, &c);
  if (rc != LBM_OK) return check_batch(env, b, rc);
  return num(env, (double)c);
}

/* ------------------------------------------------------------- module */
#define FN(name, fn) {name, NULL, fn, NULL, NULL, NULL, napi_default, NULL}

static const napi_property_descriptor kExports[] = {
    FN("create", js_create),
    FN("destroy", js_destroy),
    FN("lastError", js_last_error),
    FN("getDims", js_get_dims),
    FN("deviceBytes", js_device_bytes),
    FN("footprintBytes", js_footprint_bytes),
    FN("setParams", js_set_params),
    FN("getParams", js_get_params),
    FN("uploadField", js_upload_field),
    FN("downloadField", js_download_field),
    FN("downloadFieldF64", js_download_field_f64),
    FN("initFlat", js_init_flat),
    FN("seedHydrostatic", js_seed_hydrostatic),
    FN("retagCells", js_retag_cells),
    FN("retagCellsMask", js_retag_cells_mask),
    FN("retagCellsMesh", js_retag_cells_mesh),
    FN("voxelizeMesh", js_voxelize_mesh),
    FN("solidLinks", js_solid_links),
    FN("handleFreshCells", js_handle_fresh_cells),
    FN("computePhiGradients", js_compute_phi_gradients),
    FN("collidePhase", js_collide_phase),
    FN("streamPhase", js_stream_phase),
    FN("collideHydro", js_collide_hydro),
    FN("streamHydroAndMacro", js_stream_hydro_and_macro),
    FN("step", js_step),
    FN("absorbDeadCells", js_absorb_dead_cells),
    FN("packVolume", js_pack_volume),
    FN("packVolumeAsync", js_pack_volume_async),
    FN("stepFrame", js_step_frame),
    FN("initProfile", js_init_profile),
    FN("waitFrames", js_wait_frames),
    FN("waitFrameSlot", js_wait_frame_slot),
    FN("runCoupled", js_run_coupled),
    FN("sphereStep", js_sphere_step),
    FN("synchronize", js_synchronize),
    FN("setNanWatchdog", js_set_nan_watchdog),
    FN("lastSets", js_last_sets),
    FN("launchCount", js_launch_count),
    FN("checkedBuild", js_checked_build),
    FN("faultRecord", js_fault_record),
    FN("transferBytes", js_transfer_bytes),
    FN("fusedTiming", js_fused_timing),
    FN("fusedTimingQuery", js_fused_timing_query),
    FN("setFusedConfig", js_set_fused_config),
    FN("getFusedConfig", js_get_fused_config),
    FN("testWithholdStageCopy", js_test_withhold_stage_copy),
    FN("cameraDefault", js_camera_default),
    FN("render", js_render),
    FN("batchCreate", js_batch_create),
    FN("batchDestroy", js_batch_destroy),
    FN("batchSetConfig", js_batch_set_config),
    FN("batchRun", js_batch_run),
    FN("batchTimeFused", js_batch_time_fused),
    FN("batchLaunchCount", js_batch_launch_count),
};

/* Node looks up this symbol when it loads the addon (Node-API module
 * registration by symbol, version 1). */
__attribute__((visibility("default"))) napi_value napi_register_module_v1(napi_env env, napi_value exports) {
  if (napi_define_properties(env, exports, sizeof kExports / sizeof kExports[0], kExports) != napi_ok) {
    napi_throw_error(env, "LBM_ERR_7", "could not define the addon's functions");
    return NULL;
  }
  return exports;
}
