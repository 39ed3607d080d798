// Arena of host memory addressed by offsets (see arena.hpp).
#include "arena.hpp"

#include <sys/mman.h>

namespace cnapi {

namespace {
constexpr uint64_t kAlign = 16;
constexpr uint64_t kReserved = 64;   // offsets below this are never handed out (0 is NULL)
}  // namespace

Arena::Arena(size_t bytes, void *borrowed) {
    if (bytes <= kReserved) throw std::invalid_argument("arena: too small");
    if (borrowed) {
        owned_ = false;
        size_ = bytes;
        base_ = static_cast<uint8_t *>(borrowed);
    } else {
        size_ = (bytes + 4095) / 4096 * 4096;
        void *p = mmap(nullptr, size_, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
        if (p == MAP_FAILED) throw std::runtime_error("arena: cannot reserve host memory");
        base_ = static_cast<uint8_t *>(p);
    }
    free_[kReserved] = size_ - kReserved;
}

Arena::~Arena() {
    if (base_ && owned_) munmap(base_, size_);
}

uint64_t Arena::alloc(size_t n) {
    const uint64_t need = ((uint64_t)(n ? n : 1) + kAlign - 1) / kAlign * kAlign;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
        if (it->second < need) continue;
        const uint64_t off = it->first, left = it->second - need;
        free_.erase(it);
        if (left) free_[off + need] = left;
        used_[off] = need;
        used_bytes_ += need;
        return off;
    }
    return 0;
}

void Arena::release(uint64_t off) {
    if (!off) return;
    auto u = used_.find(off);
    if (u == used_.end()) throw std::invalid_argument("arena: free of a pointer that malloc did not return");
    uint64_t size = u->second;
    used_bytes_ -= size;
    used_.erase(u);
    // coalesce with the free neighbours
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + size == next->first) {
        size += next->second;
        next = free_.erase(next);
    }
    if (next != free_.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == off) {
            prev->second += size;
            return;
        }
    }
    free_[off] = size;
}

void *Arena::ptr(uint64_t off) const {
    if (!off) return nullptr;
    if (off >= size_) throw std::out_of_range("arena: pointer outside the memory buffer");
    return base_ + off;
}

}  // namespace cnapi
