/*
 * Stand-in for CRoaring's header, used ONLY to compile the reference's src/utils.cpp for the
 * oracle.  The roaring helpers there (utils.cpp:15-157) are never called on the partitioning
 * path; every function here aborts so that an unexpected call is loud.
 */
#ifndef ORACLE_SHIM_ROARING_H
#define ORACLE_SHIM_ROARING_H

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

typedef struct roaring_bitmap_s {
    int unused;
} roaring_bitmap_t;

static inline void oracle_roaring_unreachable(const char *fn) {
    fprintf(stderr, "[oracle-roaring] %s called: not on the partitioning path\n", fn);
    abort();
}
static inline roaring_bitmap_t *roaring_bitmap_create(void) { oracle_roaring_unreachable(__func__); return 0; }
static inline void roaring_bitmap_add(roaring_bitmap_t *, uint32_t) { oracle_roaring_unreachable(__func__); }
static inline void roaring_bitmap_clear(roaring_bitmap_t *) { oracle_roaring_unreachable(__func__); }
static inline void roaring_bitmap_free(const roaring_bitmap_t *) { oracle_roaring_unreachable(__func__); }
static inline bool roaring_bitmap_is_empty(const roaring_bitmap_t *) { oracle_roaring_unreachable(__func__); return true; }
static inline roaring_bitmap_t *roaring_bitmap_or(const roaring_bitmap_t *, const roaring_bitmap_t *) {
    oracle_roaring_unreachable(__func__);
    return 0;
}
static inline void roaring_bitmap_or_inplace(roaring_bitmap_t *, const roaring_bitmap_t *) {
    oracle_roaring_unreachable(__func__);
}
static inline size_t roaring_bitmap_portable_size_in_bytes(const roaring_bitmap_t *) {
    oracle_roaring_unreachable(__func__);
    return 0;
}
static inline size_t roaring_bitmap_portable_serialize(const roaring_bitmap_t *, char *) {
    oracle_roaring_unreachable(__func__);
    return 0;
}
static inline roaring_bitmap_t *roaring_bitmap_portable_deserialize(const char *) {
    oracle_roaring_unreachable(__func__);
    return 0;
}

#endif
