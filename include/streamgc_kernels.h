/*
 * streamgc_kernels.h -- kernel-level drop-in (libsgc_dropin.a, relocatable
 * device code). The reference's seven __global__ entry points with their exact
 * names and signatures (algorithms/streamgc/src/streamgc.cu:80-87), each taking
 * a DEVICE copy of GPUPartition as the reference kernels do. Link a program
 * built against the reference kernels with -rdc=true and libsgc_dropin.a in
 * place of the reference's kernel sources. CUDA C++ only (these are kernels).
 */
#ifndef STREAMGC_KERNELS_H
#define STREAMGC_KERNELS_H

#include "streamgc_types.h"

#ifdef __CUDACC__
/* local_update.cu:61-147 -- warp per update, grid-stride over updates. */
__global__ void local_update_kernel(EdgeUpdate* updates, uint32_t num_updates, GPUPartition* partition,
                                    uint32_t histogram_threshold);
/* epoch_maintenance.cu:5-16 -- thread per owned vertex. */
__global__ void epoch_snapshot_kernel(GPUPartition* partition, uint32_t num_vertices_global);
/* epoch_maintenance.cu:20-61 -- thread per owned vertex (row). */
__global__ void compact_csr_kernel(GPUPartition* partition);
/* epoch_maintenance.cu:66-87 -- thread per overflow entry. */
__global__ void drain_overflow_local_kernel(GPUPartition* partition, uint32_t overflow_count, uint32_t* num_failed);
/* epoch_maintenance.cu:90-110 -- thread per ghost overflow entry. */
__global__ void drain_overflow_ghost_kernel(GPUPartition* partition, uint32_t overflow_count, uint32_t* num_failed);
/* epoch_maintenance.cu:113-128 -- thread per owned vertex. */
__global__ void rebuild_bitmaps_kernel(GPUPartition* partition);
/* conflict_repair.cu:10-114 -- thread per owned vertex. */
__global__ void conflict_repair_kernel(GPUPartition* partition, uint32_t histogram_threshold, uint32_t* num_conflicts);
#endif

#endif /* STREAMGC_KERNELS_H */
