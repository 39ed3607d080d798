// Arena of host memory that JavaScript sees as one ArrayBuffer.
//
// The reference's TypeScript wrapper (skyhoffert/CourantEM
// web/src/solver/courant.ts:19-85, :166-176) talks to the solver core as a
// WebAssembly module: every pointer is a number, an offset into
// `memory.buffer`, and buffers come from the module's malloc/free. A native
// library has real pointers instead. The arena gives the Node shim the same
// picture: one fixed, never-moving block of host memory (committed by the OS
// as it is touched) that JavaScript sees as one ArrayBuffer, with a
// first-fit allocator whose offsets play the role of wasm pointers. Offset 0
// stays unused, so it can mean NULL. The memory is reserved here, or
// borrowed: the Node module hands in the backing store of an ArrayBuffer
// that Node allocated.
#pragma once

#include <cstddef>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <unordered_map>

namespace cnapi {

class Arena {
 public:
    // `bytes` of fresh memory, or of `borrowed` memory that stays the caller's
    // (and must outlive the arena)
    explicit Arena(size_t bytes, void *borrowed = nullptr);
    ~Arena();
    Arena(const Arena &) = delete;
    Arena &operator=(const Arena &) = delete;

    uint8_t *base() const { return base_; }
    size_t size() const { return size_; }

    // offset of a fresh block of n bytes (16-byte aligned), or 0 when full
    uint64_t alloc(size_t n);
    // return a block from alloc (0 is ignored, like free(NULL))
    void release(uint64_t off);
    // native address of an offset (nullptr for 0); throws for offsets outside the arena
    void *ptr(uint64_t off) const;
    // bytes in use (blocks handed out)
    size_t in_use() const { return used_bytes_; }

 private:
    uint8_t *base_ = nullptr;
    size_t size_ = 0;
    bool owned_ = true;
    std::map<uint64_t, uint64_t> free_;            // offset -> size, coalesced
    std::unordered_map<uint64_t, uint64_t> used_;  // offset -> size
    size_t used_bytes_ = 0;
};

}  // namespace cnapi
