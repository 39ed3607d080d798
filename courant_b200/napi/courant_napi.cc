// Node-API module presenting libcourant_b200 as the `Exports` object of the
// reference's TypeScript wrapper (skyhoffert/CourantEM
// web/src/solver/courant.ts:19-85), so that the board runner
// (web/tools/run-board.ts:53) only changes its loader:
//
//   const napi = require('./courant_napi.node');
//   const cem = new Courant({ exports: napi.load() } as unknown as WebAssembly.Instance);
//
// napi.load(library?, arenaMB?) dlopens a courant.h library (default: the
// libcourant_b200.so beside this module) and returns an object with
//   memory  { buffer: ArrayBuffer }  the arena (see arena.hpp): an ArrayBuffer
//                                    Node allocates once and never detaches
//   malloc(n), free(p)               offsets into memory.buffer
//   cem_*(...)                       one function per Exports entry (shim_exports.cpp)
// Pointers are offsets into memory.buffer, exactly as in the wasm build.
// Errors of the translation (unknown handle, pointer outside the buffer) throw
// a JS Error; the solver's own errors keep the courant.h convention
// (-1 and cem_last_error()).
#include <node_api.h>

#include <dlfcn.h>

#include <exception>
#include <string>
#include <vector>

#include "shim.hpp"

namespace {

struct Bound {
    cnapi::Shim *shim;
    int index;   // export index, -1 malloc, -2 free
};

bool check(napi_env env, napi_status st, const char *what) {
    if (st == napi_ok) return true;
    napi_throw_error(env, nullptr, what);
    return false;
}

napi_value number(napi_env env, double v) {
    napi_value out;
    napi_create_double(env, v, &out);
    return out;
}

napi_value undefined(napi_env env) {
    napi_value out;
    napi_get_undefined(env, &out);
    return out;
}

// every exported function: read the arguments as numbers, call, return a number
napi_value dispatch(napi_env env, napi_callback_info info) {
    size_t argc = 24;
    napi_value argv[24];
    void *data = nullptr;
    if (!check(env, napi_get_cb_info(env, info, &argc, argv, nullptr, &data), "courant: bad call")) return nullptr;
    const Bound *b = static_cast<const Bound *>(data);
    double args[24] = {};
    for (size_t q = 0; q < argc && q < 24; q++)
        if (!check(env, napi_get_value_double(env, argv[q], &args[q]), "courant: arguments must be numbers"))
            return nullptr;
    try {
        if (b->index == -1) return number(env, b->shim->malloc(args[0]));
        if (b->index == -2) {
            b->shim->free(args[0]);
            return undefined(env);
        }
        if ((int)argc < cnapi::Shim::arity(b->index)) {
            napi_throw_error(env, nullptr, "courant: too few arguments");
            return nullptr;
        }
        bool undef = false;
        const double r = b->shim->call(b->index, args, &undef);
        return undef ? undefined(env) : number(env, r);
    } catch (const std::exception &e) {
        napi_throw_error(env, nullptr, e.what());
        return nullptr;
    }
}

// the shim and the ArrayBuffer its arena lives in: the buffer is held by a
// reference until the exports object (and with it the shim) is collected
struct Holder {
    cnapi::Shim *shim = nullptr;
    napi_ref buffer = nullptr;
};

void free_holder(napi_env env, void *data, void *) {
    Holder *h = static_cast<Holder *>(data);
    delete h->shim;
    if (h->buffer) napi_delete_reference(env, h->buffer);
    delete h;
}
void free_bound(napi_env, void *data, void *) { delete static_cast<Bound *>(data); }

bool add_function(napi_env env, napi_value obj, const char *name, cnapi::Shim *shim, int index) {
    Bound *b = new Bound{shim, index};
    napi_value fn;
    if (!check(env, napi_create_function(env, name, NAPI_AUTO_LENGTH, dispatch, b, &fn), "courant: function")) {
        delete b;
        return false;
    }
    return check(env, napi_add_finalizer(env, fn, b, free_bound, nullptr, nullptr), "courant: finalizer") &&
           check(env, napi_set_named_property(env, obj, name, fn), "courant: property");
}

// the directory of this module, for the default library path
std::string module_dir() {
    Dl_info di;
    if (!dladdr(reinterpret_cast<void *>(&module_dir), &di) || !di.dli_fname) return ".";
    std::string p = di.dli_fname;
    const size_t s = p.rfind('/');
    return s == std::string::npos ? "." : p.substr(0, s);
}

napi_value load(napi_env env, napi_callback_info info) {
    size_t argc = 2;
    napi_value argv[2];
    if (!check(env, napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr), "courant: bad call")) return nullptr;
    std::string lib = module_dir() + "/libcourant_b200.so";
    double arena_mb = 1024;
    if (argc > 0) {
        napi_valuetype t;
        napi_typeof(env, argv[0], &t);
        if (t == napi_string) {
            char buf[4096];
            size_t n = 0;
            if (!check(env, napi_get_value_string_utf8(env, argv[0], buf, sizeof buf, &n), "courant: library path"))
                return nullptr;
            lib.assign(buf, n);
        }
    }
    if (argc > 1 && !check(env, napi_get_value_double(env, argv[1], &arena_mb), "courant: arena size")) return nullptr;
    // the arena is the backing store of an ArrayBuffer Node allocates (the
    // operating system commits its pages as they are touched)
    const size_t bytes = (size_t)(arena_mb * 1048576.0);
    void *base = nullptr;
    napi_value ex, memory, buffer;
    if (!check(env, napi_create_arraybuffer(env, bytes, &base, &buffer), "courant: cannot allocate the memory buffer"))
        return nullptr;
    Holder *h = new Holder;
    try {
        h->shim = new cnapi::Shim(lib, bytes, base);
    } catch (const std::exception &e) {
        delete h;
        napi_throw_error(env, nullptr, e.what());
        return nullptr;
    }
    cnapi::Shim *shim = h->shim;
    if (!check(env, napi_create_object(env, &ex), "courant: object") ||
        !check(env, napi_create_reference(env, buffer, 1, &h->buffer), "courant: reference") ||
        !check(env, napi_add_finalizer(env, ex, h, free_holder, nullptr, nullptr), "courant: finalizer")) {
        if (h->buffer) napi_delete_reference(env, h->buffer);
        delete h->shim;
        delete h;
        return nullptr;
    }
    if (!check(env, napi_create_object(env, &memory), "courant: object") ||
        !check(env, napi_set_named_property(env, memory, "buffer", buffer), "courant: property") ||
        !check(env, napi_set_named_property(env, ex, "memory", memory), "courant: property"))
        return nullptr;
    if (!add_function(env, ex, "malloc", shim, -1) || !add_function(env, ex, "free", shim, -2)) return nullptr;
    const std::vector<std::string> &names = cnapi::Shim::names();
    for (size_t q = 0; q < names.size(); q++)
        if (!add_function(env, ex, names[q].c_str(), shim, (int)q)) return nullptr;
    return ex;
}

napi_value init(napi_env env, napi_value exports) {
    napi_value fn;
    if (!check(env, napi_create_function(env, "load", NAPI_AUTO_LENGTH, load, nullptr, &fn), "courant: load") ||
        !check(env, napi_set_named_property(env, exports, "load", fn), "courant: property"))
        return nullptr;
    return exports;
}

}  // namespace

NAPI_MODULE(NODE_GYP_MODULE_NAME, init)
