// A plain C ABI over the Node shim's call translation, so that it can be
// driven and tested without node (tests/test_napi_shim.py uses it through
// ctypes exactly as courant.ts uses the module: numbers in, numbers out,
// buffers in the arena). The N-API module (courant_napi.cc) calls the same
// Shim class.
#include <cstring>
#include <exception>
#include <string>

#include "shim.hpp"

namespace {
thread_local std::string g_err;

template <class F>
auto guarded(F f, decltype(f()) fail) -> decltype(f()) {
    try {
        return f();
    } catch (const std::exception &e) {
        g_err = e.what();
        return fail;
    }
}
}  // namespace

extern "C" {

__attribute__((visibility("default"))) void *cnapi_open(const char *library, double arena_mb) {
    return guarded([&]() -> void * { return new cnapi::Shim(library, (size_t)(arena_mb * 1048576.0)); }, nullptr);
}

__attribute__((visibility("default"))) void cnapi_close(void *shim) { delete static_cast<cnapi::Shim *>(shim); }

__attribute__((visibility("default"))) const char *cnapi_error(void) { return g_err.c_str(); }

// base address and size of the arena (JavaScript's memory.buffer)
__attribute__((visibility("default"))) void *cnapi_memory(void *shim, double *bytes) {
    cnapi::Arena &a = static_cast<cnapi::Shim *>(shim)->memory();
    if (bytes) *bytes = (double)a.size();
    return a.base();
}

__attribute__((visibility("default"))) double cnapi_malloc(void *shim, double n) {
    return static_cast<cnapi::Shim *>(shim)->malloc(n);
}

__attribute__((visibility("default"))) int cnapi_free(void *shim, double off) {
    return guarded([&]() { static_cast<cnapi::Shim *>(shim)->free(off); return 0; }, -1);
}

__attribute__((visibility("default"))) int cnapi_find(const char *name) { return cnapi::Shim::find(name); }

__attribute__((visibility("default"))) int cnapi_arity(int index) { return cnapi::Shim::arity(index); }

// call export `index` with `nargs` numbers; *status: 0 value, 1 undefined (void), -1 error (cnapi_error)
__attribute__((visibility("default"))) double cnapi_call(void *shim, int index, const double *args, int nargs,
                                                         int *status) {
    if (nargs != cnapi::Shim::arity(index)) {
        g_err = "wrong number of arguments";
        *status = -1;
        return 0;
    }
    return guarded([&]() {
        bool undef = false;
        const double r = static_cast<cnapi::Shim *>(shim)->call(index, args, &undef);
        *status = undef ? 1 : 0;
        return r;
    }, (*status = -1, 0.0));
}

}  // extern "C"
