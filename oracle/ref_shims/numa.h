/* Stand-in for <numa.h> (libnuma is absent in this image). The reference uses it only to
 * count NUMA nodes for its per-node compact data copies (cpu/common.cpp:139-174); one node. */
#ifndef Q1_REF_SHIM_NUMA_H_
#define Q1_REF_SHIM_NUMA_H_
static inline int numa_available(void) { return 0; }
static inline int numa_num_configured_nodes(void) { return 1; }
#endif
