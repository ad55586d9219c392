/*
 * Stand-in for the two VOLK entry points the reference decoder calls
 * (reference lib/ldpc_decoder.cc:6-7,34,36,63,130,242). VOLK itself is not
 * vendored by the reference, not pinned (reference CMakeLists.txt:14) and not
 * installed here, so this header restates the documented semantics:
 *   volk_32f_binary_slicer_8i(out, in, n): out[i] = (in[i] >= 0) ? 1 : 0
 *   volk_malloc / volk_free / volk_get_alignment: aligned heap memory.
 * Test infrastructure only: used to compile the reference sources into
 * oracle/_ref, never linked into the product library.
 */
#ifndef WLDPC_ORACLE_VOLK_SHIM_H
#define WLDPC_ORACLE_VOLK_SHIM_H
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>

static inline size_t volk_get_alignment(void) { return 64; }

static inline void* volk_malloc(size_t size, size_t alignment)
{
    void* p = NULL;
    if (size == 0) size = alignment;
    if (posix_memalign(&p, alignment, size) != 0) return NULL;
    return p;
}

static inline void volk_free(void* p) { free(p); }

static inline void volk_32f_binary_slicer_8i(int8_t* c, const float* a, unsigned int n)
{
    for (unsigned int i = 0; i < n; i++) c[i] = (a[i] >= 0.0f) ? 1 : 0;
}
#endif
