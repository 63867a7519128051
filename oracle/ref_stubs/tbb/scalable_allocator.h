// Stand-in for TBB's scalable allocator, which the reference's
// common/DRAM.cpp uses for its host sequence arena: aligned malloc/free.
// Test infrastructure (the shim test links the reference's DRAM.cpp).
#pragma once
#include <cstdlib>

inline void* scalable_aligned_malloc(size_t size, size_t alignment) {
    void* p = nullptr;
    return posix_memalign(&p, alignment < sizeof(void*) ? sizeof(void*) : alignment, size) == 0 ? p : nullptr;
}
inline void scalable_aligned_free(void* p) { free(p); }
