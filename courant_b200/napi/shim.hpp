// The call translation behind the Node N-API module (courant_napi.cc): the
// `Exports` object of the reference's TypeScript wrapper
// (skyhoffert/CourantEM web/src/solver/courant.ts:19-85), served by any
// library with the courant.h ABI (libcourant_b200.so by default) loaded with
// dlopen. Kept free of Node headers, so it builds and is tested without node.
//
// Conventions, as courant.ts expects them of its wasm module:
//  * every argument and result is a JS number (double);
//  * pointer arguments are offsets into the arena's ArrayBuffer (`memory`),
//    from `malloc`; they are translated to host addresses by adding the base;
//  * a simulation handle is a small integer (a table of cem_sim pointers);
//  * a pointer the library returns into its own memory (spectra, plan arrays,
//    field and state arrays, the error string) comes back as the offset of an
//    arena mirror holding a copy. Field and state arrays are live in the
//    reference (callers write initial conditions and read every step), so their
//    mirrors are synchronised around every later call on that simulation:
//    copied into the library before the call, and back after it.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../../include/courant.h"
#include "arena.hpp"

namespace cnapi {

// courant.h entry points resolved from the loaded library
struct Lib {
    void *handle = nullptr;
#define CNAPI_FN(name) decltype(&::name) name = nullptr;
#include "shim_functions.inc"
#undef CNAPI_FN
};

class Shim {
 public:
    // arena of `arena_bytes`, its own or `borrowed` (which must outlive the shim)
    Shim(const std::string &library, size_t arena_bytes, void *borrowed = nullptr);
    ~Shim();

    Arena &memory() { return arena_; }

    // malloc/free of the Exports interface
    double malloc(double n);
    void free(double off);

    // names of the callable exports (besides malloc and free), in table order
    static const std::vector<std::string> &names();
    // index of an export, -1 if unknown
    static int find(const std::string &name);
    // number of arguments the export takes
    static int arity(int index);
    // call an export; `undefined_result` is set for void functions
    double call(int index, const double *args, bool *undefined_result);

    // handle table
    double new_handle(cem_sim *s);
    cem_sim *sim(double handle) const;
    void drop_handle(double handle);

    // arena helpers used by the exports
    void *ptr(double off) const;
    double mirror(double handle, int kind, int a, int b, const double *src, size_t n, bool live);
    double string_mirror(const char *text);
    void sync_in(double handle);
    void sync_out(double handle);

    const Lib &lib() const { return lib_; }

 private:
    struct Mirror {
        uint64_t off = 0;
        size_t n = 0;
        double *lib = nullptr;   // the library's array (live mirrors only)
        bool live = false;
    };
    Lib lib_;
    Arena arena_;
    std::unordered_map<uint32_t, cem_sim *> sims_;
    uint32_t next_ = 1;
    std::map<std::tuple<uint32_t, int, int, int>, Mirror> mirrors_;
    uint64_t err_off_ = 0;
    size_t err_cap_ = 0;
};

}  // namespace cnapi
