/*
 * Test-infrastructure shim for <libpmem.h>.  Persistent memory is only used
 * under -DUSE_NVM (src/inc/utils.c:157-198), which the oracle build never
 * defines; these stubs exist so the translation units compile.
 * Project-written.
 */
#ifndef CAS_SHIM_LIBPMEM_H
#define CAS_SHIM_LIBPMEM_H
#include <stddef.h>
#include <sys/types.h>
#define PMEM_FILE_CREATE (1 << 0)
#define PMEM_FILE_EXCL (1 << 1)
static inline void *pmem_map_file(const char *path, size_t len, int flags, mode_t mode,
	size_t *mapped_lenp, int *is_pmemp) {
	(void) path; (void) len; (void) flags; (void) mode;
	if (mapped_lenp) *mapped_lenp = 0;
	if (is_pmemp) *is_pmemp = 0;
	return NULL;
}
static inline int pmem_unmap(void *addr, size_t len) { (void) addr; (void) len; return 0; }
#endif
