/* Host -> device copy of a large pageable buffer through pinned staging buffers (hostcopy.c). */
#ifndef SPMV_HOSTCOPY_H
#define SPMV_HOSTCOPY_H

#include <stddef.h>

#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Copies bytes from pageable host src to device dst on stream s.  Large copies return once
 * the whole copy has reached the device (the staging buffers are then free); copies below
 * 8 MB are enqueued as a plain cudaMemcpyAsync. */
__attribute__((visibility("hidden")))
cudaError_t spmv_h2d_pageable(void * dst, const void * src, size_t bytes, cudaStream_t s);

#ifdef __cplusplus
}
#endif

#endif
