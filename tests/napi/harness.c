/*
 * Drives the Node-API addon through the Node-API stand-in (napi_stub.c) the
 * way Node would: dlopen the .node file, call napi_register_module_v1, then
 * call the exported functions with stub values.  Test infrastructure only.
 *
 *   harness ADDON exports      print the exported names
 *   harness ADDON cpu          argument checks and the host sphere integrator
 *   harness ADDON gpu          the smoke scene, 10 worker ticks, on cuda:0
 */
#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lbm_b200.h"
#include "napi_stub.h"

typedef napi_value (*RegisterFn)(napi_env, napi_value);

static napi_value N(double v) { return stub_number(v); }

static void expect_throw(napi_env env, const char *what, const char *code_prefix) {
  if (!env->thrown) {
    printf("FAIL %s: nothing thrown\n", what);
    exit(1);
  }
  if (code_prefix && strncmp(env->code, code_prefix, strlen(code_prefix)) != 0) {
    printf("FAIL %s: code %s (%s)\n", what, env->code, env->msg);
    exit(1);
  }
  printf("threw %s: %s: %s\n", what, env->code, env->msg);
}

static void expect_ok(napi_env env, const char *what) {
  if (env->thrown) {
    printf("FAIL %s: %s %s\n", what, env->code, env->msg);
    exit(1);
  }
}

/* a RigidSphere's state as the addon's Float64Array (lbm_sphere memory) */
static void sphere_init(lbm_sphere *s, double cx, double cy, double cz, double r, double density) {
  memset(s, 0, sizeof *s);
  s->cx = cx, s->cy = cy, s->cz = cz, s->r = r, s->density = density;
  double V = (4.0 / 3.0) * M_PI * r * r * r;  /* src/solid.js:39-47 */
  s->mass = density * V;
  s->I = 0.4 * s->mass * r * r;
}

static void print_sphere(const char *tag, const lbm_sphere *s) {
  printf("%s %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", tag, s->cx, s->cy, s->cz, s->vx, s->vy,
         s->vz, s->wx, s->wy, s->wz);
}

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  void *lib = dlopen(argv[1], RTLD_NOW | RTLD_LOCAL);
  if (!lib) {
    printf("dlopen: %s\n", dlerror());
    return 2;
  }
  RegisterFn reg = (RegisterFn)dlsym(lib, "napi_register_module_v1");
  if (!reg) return 2;
  struct napi_env__ envs;
  memset(&envs, 0, sizeof envs);
  napi_env env = &envs;
  reg(env, stub_null());
  const char *mode = argv[2];

  if (!strcmp(mode, "exports")) {
    for (int i = 0; i < env->nfns; i++) printf("%s\n", env->names[i]);
    return 0;
  }

  if (!strcmp(mode, "cpu")) {
    /* the host integrator: one falling, one dragged sphere */
    lbm_sphere sp[2];
    sphere_init(&sp[0], 20.0, 14.0, 20.0, 4.0, 2.0);
    sp[0].Fy = -0.3;
    sp[0].Tx = 0.02;
    sphere_init(&sp[1], 10.0, 8.0, 30.0, 3.0, 1.4);
    sp[1].dragging = 1;
    sp[1].dragTargetX = 30, sp[1].dragTargetY = 20, sp[1].dragTargetZ = 10;
    napi_value a[6] = {stub_typed(napi_float64_array, sp, 2 * 23), N(1.0), N(-0.001), N(40), N(28), N(40)};
    for (int t = 0; t < 3; t++) {
      stub_call(env, "sphereStep", 6, a);
      expect_ok(env, "sphereStep");
    }
    print_sphere("sphere0", &sp[0]);
    print_sphere("sphere1", &sp[1]);

    /* argument checks */
    float wrong[23];
    napi_value b[6] = {stub_typed(napi_float32_array, wrong, 23), N(1.0), N(-0.001), N(40), N(28), N(40)};
    stub_call(env, "sphereStep", 6, b);
    expect_throw(env, "float32 spheres", "LBM_ERR_1");
    double odd[22];
    napi_value c[6] = {stub_typed(napi_float64_array, odd, 22), N(1.0), N(-0.001), N(40), N(28), N(40)};
    stub_call(env, "sphereStep", 6, c);
    expect_throw(env, "22 numbers", "LBM_ERR_1");
    double imp[6];
    napi_value d[3] = {N(1.0), stub_null(), stub_typed(napi_float64_array, imp, 6)};
    stub_call(env, "step", 3, d);
    expect_throw(env, "number as handle", "LBM_ERR_1");
    napi_value e[1] = {N(3.0)};
    stub_call(env, "initFlat", 1, e);
    expect_throw(env, "too few arguments", "LBM_ERR_1");
    napi_value f[3] = {N(2), N(2), N(2)};
    stub_call(env, "create", 3, f);
    expect_throw(env, "2x2x2 grid", "LBM_ERR_");
    return 0;
  }

  if (!strcmp(mode, "gpu")) {
    /* test/smoke.mjs scene: 12^3, liquid at y > 6, sphere r = 2 at (6, 3, 6) */
    napi_value ca[3] = {N(12), N(12), N(12)};
    napi_value h = stub_call(env, "create", 3, ca);
    expect_ok(env, "create");
    /* test/smoke.mjs:7-15 order: initFlat runs with the constructor's
     * parameters, the scene's parameters are set after it */
    napi_value ia[2] = {h, N(6)};
    stub_call(env, "initFlat", 2, ia);
    expect_ok(env, "initFlat");
    double params[8] = {0.7, 0.7, 0.012, 0.0012, 1.0, 0.1, 4.0, 0.02};
    napi_value pa[2] = {h, stub_typed(napi_float64_array, params, 8)};
    stub_call(env, "setParams", 2, pa);
    expect_ok(env, "setParams");
    lbm_sphere sp;
    sphere_init(&sp, 6, 3, 6, 2.0, 1.5);
    double imp[6];
    napi_value spv = stub_typed(napi_float64_array, &sp, 23), impv = stub_typed(napi_float64_array, imp, 6);
    for (int t = 0; t < 10; t++) {
      /* src/worker.js:96-100: sim.step(solid); solid.absorbDeadCells(sim); solid.step(1, g);
       * the impulses of the first two are what applyImpulseAtCell accumulates */
      napi_value sa[3] = {h, spv, impv};
      stub_call(env, "step", 3, sa);
      expect_ok(env, "step");
      sp.Fx += imp[0], sp.Fy += imp[1], sp.Fz += imp[2], sp.Tx += imp[3], sp.Ty += imp[4], sp.Tz += imp[5];
      stub_call(env, "absorbDeadCells", 3, sa);
      expect_ok(env, "absorbDeadCells");
      sp.Fx += imp[0], sp.Fy += imp[1], sp.Fz += imp[2], sp.Tx += imp[3], sp.Ty += imp[4], sp.Tz += imp[5];
      napi_value ss[6] = {spv, N(1.0), N(params[3]), N(12), N(12), N(12)};
      stub_call(env, "sphereStep", 6, ss);
      expect_ok(env, "sphereStep");
    }
    static float phi[12 * 12 * 12];
    napi_value da[3] = {h, N(LBM_FIELD_PHI), stub_typed(napi_float32_array, phi, 12 * 12 * 12)};
    stub_call(env, "downloadField", 3, da);
    expect_ok(env, "downloadField");
    double sum = 0;
    for (int i = 0; i < 12 * 12 * 12; i++) sum += phi[i];
    printf("phisum %.17g\n", sum);
    printf("phi777 %.9g\n", phi[(7 * 12 + 7) * 12 + 7]);
    print_sphere("sphere", &sp);
    napi_value xa[1] = {h};
    stub_call(env, "destroy", 1, xa);
    expect_ok(env, "destroy");
    stub_call(env, "seedHydrostatic", 1, xa);
    expect_throw(env, "destroyed handle", "LBM_ERR_1");
    stub_finalize_all(env);
    return 0;
  }
  return 2;
}
