/*
 * Test-infrastructure shim: a minimal stand-in for libnuma's <numa.h>.
 *
 * libnuma is not installed on this image, and the reference's CPU SpGEMM only
 * uses it to place buffers on NUMA nodes (src/inc/utils.c:200-232,
 * src/inc/utils.c:356-381).  Placement has no effect on results, so every
 * call here is a no-op that reports a single node.  Project-written; used only
 * to build the reference as an oracle under oracle/_ref.
 */
#ifndef CAS_SHIM_NUMA_H
#define CAS_SHIM_NUMA_H
#include <stdlib.h>
#include <string.h>

struct bitmask {
	unsigned long size;
	unsigned long *maskp;
};

static inline int numa_available(void) { return 0; }
static inline int numa_num_configured_nodes(void) { return 1; }

static inline struct bitmask *numa_bitmask_alloc(unsigned int n) {
	struct bitmask *b = (struct bitmask *) calloc(1, sizeof(struct bitmask));
	unsigned long words = (n + 8 * sizeof(unsigned long) - 1) / (8 * sizeof(unsigned long));
	if (words == 0) words = 1;
	b->size = words * 8 * sizeof(unsigned long);
	b->maskp = (unsigned long *) calloc(words, sizeof(unsigned long));
	return b;
}
static inline void numa_bitmask_free(struct bitmask *b) {
	if (b) { free(b->maskp); free(b); }
}
static inline struct bitmask *numa_bitmask_clearall(struct bitmask *b) {
	memset(b->maskp, 0, b->size / 8);
	return b;
}
static inline struct bitmask *numa_bitmask_setbit(struct bitmask *b, unsigned int i) {
	if (i < b->size) b->maskp[i / (8 * sizeof(unsigned long))] |= 1UL << (i % (8 * sizeof(unsigned long)));
	return b;
}
static inline int numa_bitmask_isbitset(const struct bitmask *b, unsigned int i) {
	if (i >= b->size) return 0;
	return (b->maskp[i / (8 * sizeof(unsigned long))] >> (i % (8 * sizeof(unsigned long)))) & 1UL;
}
#endif
