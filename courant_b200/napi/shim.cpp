// Call translation of the Node shim (see shim.hpp).
#include "shim.hpp"

#include <dlfcn.h>

#include <cstring>
#include <stdexcept>

namespace cnapi {

Shim::Shim(const std::string &library, size_t arena_bytes, void *borrowed) : arena_(arena_bytes, borrowed) {
    lib_.handle = dlopen(library.c_str(), RTLD_NOW | RTLD_LOCAL);
    if (!lib_.handle) throw std::runtime_error(std::string("cannot load ") + library + ": " + dlerror());
#define CNAPI_FN(name)                                                                       \
    lib_.name = reinterpret_cast<decltype(lib_.name)>(dlsym(lib_.handle, #name));            \
    if (!lib_.name) throw std::runtime_error(std::string(library) + " does not export " #name);
#include "shim_functions.inc"
#undef CNAPI_FN
}

Shim::~Shim() {
    for (auto &kv : sims_) lib_.cem_destroy(kv.second);
    if (lib_.handle) dlclose(lib_.handle);
}

double Shim::malloc(double n) {
    if (!(n >= 0)) return 0;
    return (double)arena_.alloc((size_t)n);
}

void Shim::free(double off) { arena_.release((uint64_t)off); }

void *Shim::ptr(double off) const { return arena_.ptr((uint64_t)off); }

double Shim::new_handle(cem_sim *s) {
    if (!s) return 0;
    const uint32_t h = next_++;
    sims_[h] = s;
    return h;
}

cem_sim *Shim::sim(double handle) const {
    auto it = sims_.find((uint32_t)handle);
    if (it == sims_.end()) throw std::invalid_argument("unknown simulation handle");
    return it->second;
}

void Shim::drop_handle(double handle) {
    const uint32_t h = (uint32_t)handle;
    for (auto it = mirrors_.begin(); it != mirrors_.end();) {
        if (std::get<0>(it->first) == h) {
            arena_.release(it->second.off);
            it = mirrors_.erase(it);
        } else {
            ++it;
        }
    }
    sims_.erase(h);
}

// Arena copy of n doubles of library memory, one slot per (handle, kind, a, b),
// reused by later calls; live mirrors remember the library array.
double Shim::mirror(double handle, int kind, int a, int b, const double *src, size_t n, bool live) {
    if (!src) return 0;
    Mirror &m = mirrors_[std::make_tuple((uint32_t)handle, kind, a, b)];
    if (m.off && m.n != n) {
        arena_.release(m.off);
        m.off = 0;
    }
    if (!m.off) {
        m.off = arena_.alloc(n * sizeof(double));
        m.n = n;
        if (!m.off) throw std::runtime_error("arena full: raise COURANT_ARENA_MB");
    }
    m.live = live;
    m.lib = live ? const_cast<double *>(src) : nullptr;
    std::memcpy(arena_.ptr(m.off), src, n * sizeof(double));
    return (double)m.off;
}

double Shim::string_mirror(const char *text) {
    const size_t n = std::strlen(text ? text : "") + 1;
    if (n > err_cap_) {
        arena_.release(err_off_);
        err_cap_ = n < 256 ? 256 : n;
        err_off_ = arena_.alloc(err_cap_);
    }
    std::memcpy(arena_.ptr(err_off_), text ? text : "", n);
    return (double)err_off_;
}

// live arrays: what JavaScript wrote goes into the library before a call on the simulation ...
void Shim::sync_in(double handle) {
    const uint32_t h = (uint32_t)handle;
    for (auto &kv : mirrors_)
        if (std::get<0>(kv.first) == h && kv.second.live)
            std::memcpy(kv.second.lib, arena_.ptr(kv.second.off), kv.second.n * sizeof(double));
}

// ... and what the call changed comes back after it
void Shim::sync_out(double handle) {
    const uint32_t h = (uint32_t)handle;
    for (auto &kv : mirrors_)
        if (std::get<0>(kv.first) == h && kv.second.live)
            std::memcpy(arena_.ptr(kv.second.off), kv.second.lib, kv.second.n * sizeof(double));
}

}  // namespace cnapi
