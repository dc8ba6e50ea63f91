/*
 * Test-infrastructure shim for <numaif.h>: mbind() accepts and ignores the
 * policy (page placement does not change any result of the reference's
 * SpGEMM, src/inc/utils.c:210).  Project-written.
 */
#ifndef CAS_SHIM_NUMAIF_H
#define CAS_SHIM_NUMAIF_H
#define MPOL_DEFAULT 0
#define MPOL_PREFERRED 1
#define MPOL_BIND 2
#define MPOL_INTERLEAVE 3
static inline long mbind(void *addr, unsigned long len, int mode,
	const unsigned long *nodemask, unsigned long maxnode, unsigned flags) {
	(void) addr; (void) len; (void) mode; (void) nodemask; (void) maxnode; (void) flags;
	return 0;
}
#endif
