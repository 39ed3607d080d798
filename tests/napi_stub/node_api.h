/* Declarations of the Node-API (N-API) functions, types and macros that
 * courant_b200/napi/courant_napi.cc uses, as documented at
 * https://nodejs.org/api/n-api.html. Node's own headers are not installed
 * here; this file lets a CPU test compile the module's source (syntax and
 * types only, nothing is linked or run). Test infrastructure. */
#pragma once
#include <stddef.h>
#include <stdint.h>

typedef struct napi_env__ *napi_env;
typedef struct napi_value__ *napi_value;
typedef struct napi_ref__ *napi_ref;
typedef struct napi_callback_info__ *napi_callback_info;
typedef enum { napi_ok, napi_invalid_arg, napi_object_expected, napi_string_expected, napi_generic_failure } napi_status;
typedef enum { napi_undefined, napi_null, napi_boolean, napi_number, napi_string, napi_symbol, napi_object,
               napi_function, napi_external, napi_bigint } napi_valuetype;
typedef napi_value (*napi_callback)(napi_env env, napi_callback_info info);
typedef void (*napi_finalize)(napi_env env, void *finalize_data, void *finalize_hint);
#define NAPI_AUTO_LENGTH SIZE_MAX

#ifdef __cplusplus
extern "C" {
#endif
napi_status napi_create_object(napi_env env, napi_value *result);
napi_status napi_create_function(napi_env env, const char *utf8name, size_t length, napi_callback cb, void *data,
                                 napi_value *result);
napi_status napi_get_cb_info(napi_env env, napi_callback_info cbinfo, size_t *argc, napi_value *argv,
                             napi_value *this_arg, void **data);
napi_status napi_get_value_double(napi_env env, napi_value value, double *result);
napi_status napi_get_value_string_utf8(napi_env env, napi_value value, char *buf, size_t bufsize, size_t *result);
napi_status napi_create_double(napi_env env, double value, napi_value *result);
napi_status napi_get_undefined(napi_env env, napi_value *result);
napi_status napi_typeof(napi_env env, napi_value value, napi_valuetype *result);
napi_status napi_set_named_property(napi_env env, napi_value object, const char *utf8name, napi_value value);
napi_status napi_create_arraybuffer(napi_env env, size_t byte_length, void **data, napi_value *result);
napi_status napi_create_reference(napi_env env, napi_value value, uint32_t initial_refcount, napi_ref *result);
napi_status napi_delete_reference(napi_env env, napi_ref ref);
napi_status napi_add_finalizer(napi_env env, napi_value js_object, void *finalize_data, napi_finalize finalize_cb,
                               void *finalize_hint, napi_ref *result);
napi_status napi_throw_error(napi_env env, const char *code, const char *msg);
#ifdef __cplusplus
}
#endif

#define NAPI_MODULE(modname, regfunc) \
    extern "C" napi_value napi_register_module_v1(napi_env env, napi_value exports) { return regfunc(env, exports); }
