/* Windows aligned allocator used by the reference's Memory.h:10-32. */
#pragma once
#include <stdlib.h>
static inline void* _aligned_malloc(size_t size, size_t align)
{
    void* p = nullptr;
    if (posix_memalign(&p, align < sizeof(void*) ? sizeof(void*) : align, size ? size : 1) != 0) return nullptr;
    return p;
}
static inline void _aligned_free(void* p) { free(p); }
