/*
 * Test-infrastructure shim for <libconfig.h>.  The reference reads a core-ID
 * map from a libconfig file to pin its threads (src/inc/utils.c:100-131,
 * src/inc/utils.c:134-155).  This shim ignores the file and returns core
 * IDs i % nproc (at most SOCKET_CORE_NUM of them, the size of the arrays
 * the reference fills), so thread i is pinned to core i.  Project-written.
 */
#ifndef CAS_SHIM_LIBCONFIG_H
#define CAS_SHIM_LIBCONFIG_H
#include <unistd.h>

typedef struct { int unused; } config_t;
typedef struct { int length; } config_setting_t;

static config_setting_t cas_shim_core_setting;

static inline void config_init(config_t *c) { (void) c; }
static inline void config_destroy(config_t *c) { (void) c; }
static inline int config_read_file(config_t *c, const char *path) { (void) c; (void) path; return 1; }
static inline const char *config_error_file(const config_t *c) { (void) c; return ""; }
static inline int config_error_line(const config_t *c) { (void) c; return 0; }
static inline const char *config_error_text(const config_t *c) { (void) c; return ""; }
static inline config_setting_t *config_lookup(const config_t *c, const char *path) {
	(void) c; (void) path;
	long n = sysconf(_SC_NPROCESSORS_ONLN);
	if (n < 1) n = 1;
#ifdef SOCKET_CORE_NUM
	/* the reference copies this many IDs into int[SOCKET_CORE_NUM] arrays */
	if (n > SOCKET_CORE_NUM) n = SOCKET_CORE_NUM;
#endif
	cas_shim_core_setting.length = (int) n;
	return &cas_shim_core_setting;
}
static inline int config_setting_length(const config_setting_t *s) { return s ? s->length : 0; }
static inline int config_setting_get_int_elem(const config_setting_t *s, int idx) {
	return s && s->length > 0 ? idx % s->length : 0;
}
#endif
