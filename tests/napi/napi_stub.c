/*
 * A stand-in for Node's side of Node-API, enough to load and drive the addon
 * (claude-vibe-code-raytracing_b200/napi/binding.c) from C without Node: values
 * are small tagged structs, typed arrays wrap caller memory, a thrown error is
 * recorded in the environment.  Test infrastructure only.
 */
#include "napi_stub.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static struct napi_value__ g_undefined = {V_UNDEFINED};

napi_value stub_number(double v) {
  napi_value x = (napi_value)calloc(1, sizeof *x);
  x->kind = V_NUMBER;
  x->num = v;
  return x;
}
napi_value stub_null(void) {
  napi_value x = (napi_value)calloc(1, sizeof *x);
  x->kind = V_NULL;
  return x;
}
napi_value stub_typed(napi_typedarray_type t, void *data, size_t len) {
  napi_value x = (napi_value)calloc(1, sizeof *x);
  x->kind = V_TYPED;
  x->ttype = t;
  x->data = data;
  x->len = len;
  return x;
}

napi_status napi_get_cb_info(napi_env env, napi_callback_info cbinfo, size_t *argc, napi_value *argv,
                             napi_value *this_arg, void **data) {
  (void)env;
  size_t cap = *argc;
  for (size_t i = 0; i < cap; i++) argv[i] = i < cbinfo->argc ? cbinfo->argv[i] : &g_undefined;
  *argc = cbinfo->argc;
  if (this_arg) *this_arg = &g_undefined;
  if (data) *data = NULL;
  return napi_ok;
}
napi_status napi_typeof(napi_env env, napi_value v, napi_valuetype *r) {
  (void)env;
  switch (v->kind) {
    case V_UNDEFINED: *r = napi_undefined; break;
    case V_NULL: *r = napi_null; break;
    case V_NUMBER: *r = napi_number; break;
    case V_STRING: *r = napi_string; break;
    case V_EXTERNAL: *r = napi_external; break;
    default: *r = napi_object; break;
  }
  return napi_ok;
}
napi_status napi_get_value_double(napi_env env, napi_value v, double *r) {
  (void)env;
  if (v->kind != V_NUMBER) return napi_number_expected;
  *r = v->num;
  return napi_ok;
}
napi_status napi_get_value_int32(napi_env env, napi_value v, int32_t *r) {
  (void)env;
  if (v->kind != V_NUMBER) return napi_number_expected;
  *r = (int32_t)v->num;
  return napi_ok;
}
napi_status napi_create_int32(napi_env env, int32_t v, napi_value *r) {
  (void)env;
  *r = stub_number(v);
  return napi_ok;
}
napi_status napi_create_double(napi_env env, double v, napi_value *r) {
  (void)env;
  *r = stub_number(v);
  return napi_ok;
}
napi_status napi_create_string_utf8(napi_env env, const char *s, size_t n, napi_value *r) {
  (void)env;
  napi_value x = (napi_value)calloc(1, sizeof *x);
  x->kind = V_STRING;
  if (n == (size_t)-1) n = strlen(s);
  x->str = (char *)calloc(n + 1, 1);
  memcpy(x->str, s, n);
  *r = x;
  return napi_ok;
}
napi_status napi_create_external(napi_env env, void *data, napi_finalize fin, void *hint, napi_value *r) {
  napi_value x = (napi_value)calloc(1, sizeof *x);
  x->kind = V_EXTERNAL;
  x->data = data;
  x->fin = fin;
  x->hint = hint;
  env->externals[env->nexternals++ % STUB_MAX_EXTERNALS] = x;
  *r = x;
  return napi_ok;
}
napi_status napi_get_value_external(napi_env env, napi_value v, void **r) {
  (void)env;
  if (v->kind != V_EXTERNAL) return napi_invalid_arg;
  *r = v->data;
  return napi_ok;
}
napi_status napi_get_typedarray_info(napi_env env, napi_value v, napi_typedarray_type *t, size_t *len, void **data,
                                     napi_value *ab, size_t *off) {
  (void)env;
  if (v->kind != V_TYPED) return napi_invalid_arg;
  if (t) *t = v->ttype;
  if (len) *len = v->len;
  if (data) *data = v->data;
  if (ab) *ab = &g_undefined;
  if (off) *off = 0;
  return napi_ok;
}
napi_status napi_get_undefined(napi_env env, napi_value *r) {
  (void)env;
  *r = &g_undefined;
  return napi_ok;
}
napi_status napi_throw_error(napi_env env, const char *code, const char *msg) {
  if (env->thrown) return napi_pending_exception;
  env->thrown = 1;
  snprintf(env->code, sizeof env->code, "%s", code ? code : "");
  snprintf(env->msg, sizeof env->msg, "%s", msg ? msg : "");
  return napi_ok;
}
napi_status napi_define_properties(napi_env env, napi_value obj, size_t n, const napi_property_descriptor *p) {
  (void)obj;
  for (size_t i = 0; i < n && env->nfns < STUB_MAX_FNS; i++) {
    env->names[env->nfns] = p[i].utf8name;
    env->fns[env->nfns] = p[i].method;
    env->nfns++;
  }
  return napi_ok;
}

napi_callback stub_fn(napi_env env, const char *name) {
  for (int i = 0; i < env->nfns; i++)
    if (strcmp(env->names[i], name) == 0) return env->fns[i];
  return NULL;
}

napi_value stub_call(napi_env env, const char *name, size_t argc, napi_value *argv) {
  napi_callback f = stub_fn(env, name);
  if (!f) {
    fprintf(stderr, "no export %s\n", name);
    exit(2);
  }
  struct napi_callback_info__ ci = {argc, argv};
  env->thrown = 0;
  env->code[0] = env->msg[0] = 0;
  return f(env, &ci);
}

void stub_finalize_all(napi_env env) {
  int n = env->nexternals < STUB_MAX_EXTERNALS ? env->nexternals : STUB_MAX_EXTERNALS;
  for (int i = 0; i < n; i++) {
    napi_value x = env->externals[i];
    if (x && x->fin) x->fin(env, x->data, x->hint);
    env->externals[i] = NULL;
  }
}
