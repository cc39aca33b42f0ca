/* Test stand-in for Node's side of Node-API (see napi_stub.c). */
#ifndef NAPI_STUB_H
#define NAPI_STUB_H
#include "napi_decls.h"

enum { V_UNDEFINED, V_NULL, V_NUMBER, V_STRING, V_EXTERNAL, V_TYPED };
#define STUB_MAX_FNS 128
#define STUB_MAX_EXTERNALS 64

struct napi_value__ {
  int kind;
  double num;
  char *str;
  void *data;
  size_t len;
  napi_typedarray_type ttype;
  napi_finalize fin;
  void *hint;
};
struct napi_env__ {
  int thrown;
  char code[64], msg[512];
  int nfns;
  const char *names[STUB_MAX_FNS];
  napi_callback fns[STUB_MAX_FNS];
  int nexternals;
  napi_value externals[STUB_MAX_EXTERNALS];
};
struct napi_callback_info__ {
  size_t argc;
  napi_value *argv;
};

napi_value stub_number(double v);
napi_value stub_null(void);
napi_value stub_typed(napi_typedarray_type t, void *data, size_t len);
napi_callback stub_fn(napi_env env, const char *name);
napi_value stub_call(napi_env env, const char *name, size_t argc, napi_value *argv);
void stub_finalize_all(napi_env env);
#endif
