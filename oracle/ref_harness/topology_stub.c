/*
 * Test-infrastructure stub (oracle only): a fixed host topology for the reference's DIV-RF
 * checker (libref_div_rf.so).
 *
 * The reference's DIVArray constructor reads the host CPU topology (lib/topology/
 * hardware_topology.c: sysfs caches, cores, memory nodes; lib/topology/task_topology.c:
 * the CPU each thread is pinned to) only to fill per-thread statistics and NUMA hints
 * (src/spmv_kernels/DIV/div.cpp:226-279, :528); the packet bytes, the packet groups and y do
 * not depend on them.  On hosts whose sysfs layout or thread placement that reader does not
 * accept it stops the process, so the checker is linked with this stub instead: one memory
 * node, one L3 cache node of 32 MiB shared by every thread, task number = OpenMP thread
 * number (what the reference's own code gives with one thread pinned to each CPU of one
 * socket).  Prototypes are the reference's (lib/topology/hardware_topology.h:125-155,
 * task_topology.h:91-124).
 */
#include <omp.h>

#include "topology/hardware_topology.h"
#include "topology/task_topology.h"

struct topohw_topology * topohw_get_topology()
{
	return 0;
}

struct topotk_topology * topotk_get_topology()
{
	return 0;
}

long topohw_get_cache_size(long cpu_id, long level, enum cache_types type)
{
	(void) cpu_id;
	(void) type;
	return level == 3 ? 32L << 20 : level == 2 ? 2L << 20 : 48L << 10;
}

long topotk_get_task_num()
{
	return omp_get_thread_num();
}

long topotk_get_num_tasks()
{
	return omp_get_max_threads();
}

long topotk_get_task_cache_node_num(long level)
{
	(void) level;
	return 0;
}

long topotk_get_num_task_cache_nodes(long level)
{
	(void) level;
	return 1;
}

long topotk_get_task_mem_node_num()
{
	return 0;
}

long topotk_get_num_task_mem_nodes()
{
	return 1;
}
