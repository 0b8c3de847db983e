/*
 * Test infrastructure only (oracle): force-included (-include) when the
 * reference's operator builder (operators.cpp, operators_c.cpp) is compiled
 * from its own sources into oracle/_ref/.
 *
 * The reference's types.h pulls in asd.h (MPI, Lua, logging).  The operator
 * builder only needs the scalar typedefs and the aligned allocator, so this
 * header claims the TYPES_H include guard first and supplies exactly those:
 *   - dfloat_t = double      (types.h:33 with USE_DFLOAT_DOUBLE set to 1, the
 *                             FP64 "dfloat build" the hot path is quoted on)
 *   - uintloc_t = uint32_t   (types.h:12)
 *   - asd_malloc / asd_malloc_aligned / asd_free / asd_free_aligned
 *                            (asd.c:236-280; plain malloc semantics)
 */
#ifndef WADG_REF_SHIM_H
#define WADG_REF_SHIM_H

#define TYPES_H 1
#define USE_DFLOAT_DOUBLE 1

#ifdef __cplusplus
#include <cstdint>
#include <cstdlib>
#else
#include <stdint.h>
#include <stdlib.h>
#endif

typedef uint32_t uintloc_t;
typedef uint64_t uintglo_t;
typedef double dfloat_t;

static inline void *asd_malloc(size_t n) { return malloc(n ? n : 1); }
static inline void asd_free(void *p) { free(p); }
static inline void *asd_malloc_aligned(size_t n)
{
  void *p = NULL;
  if (posix_memalign(&p, 64, n ? n : 64) != 0)
    abort();
  return p;
}
static inline void asd_free_aligned(void *p) { free(p); }

#endif
