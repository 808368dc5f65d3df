/* Stand-in for <numa.h> so the reference's reference_omp backend builds and
 * runs without libnuma: interleaved allocation becomes an ordinary aligned
 * allocation (one NUMA node on the hosts used here).  Test infrastructure
 * for oracle/_ref only. */
#ifndef ALP_ORACLE_NUMA_SHIM_H
#define ALP_ORACLE_NUMA_SHIM_H
#include <stdlib.h>
static inline void *numa_alloc_interleaved(size_t size) {
	void *p = NULL;
	if (posix_memalign(&p, 4096, size ? size : 1) != 0) return NULL;
	return p;
}
static inline void numa_free(void *p, size_t size) { (void) size; free(p); }
static inline void numa_set_localalloc(void) {}
#endif
