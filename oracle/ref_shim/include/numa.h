/* numa.h — the libnuma queries the reference makes, for the oracle shim
 * (test infrastructure only): one node holding every online CPU. */
#ifndef PLATO_ORACLE_SHIM_NUMA_H
#define PLATO_ORACLE_SHIM_NUMA_H
#include <unistd.h>
struct bitmask { unsigned long size; unsigned long* maskp; };
inline int numa_available(void) { return 0; }
inline int numa_num_configured_cpus(void) { return static_cast<int>(sysconf(_SC_NPROCESSORS_ONLN)); }
inline int numa_num_configured_nodes(void) { return 1; }
inline int numa_max_node(void) { return 0; }
inline struct bitmask* numa_parse_nodestring(const char*) { return nullptr; }
inline void numa_set_interleave_mask(struct bitmask*) {}
inline void numa_bitmask_free(struct bitmask*) {}
#endif
