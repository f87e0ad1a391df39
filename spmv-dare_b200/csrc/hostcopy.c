/*
 * Host -> device copies of large pageable buffers (the CSR arrays a conversion receives).
 *
 * A plain cudaMemcpyAsync from pageable memory is staged by the driver through its own
 * small pinned buffers, one host thread at a time (about 11 GB/s on the B200 hosts).  Here
 * the copy runs through two pinned staging buffers of STAGE_BYTES: the host threads of an
 * OpenMP team fill one (a parallel memcpy) while the DMA engine drains the other, so the
 * host-side copy and the PCIe transfer overlap.  The staging buffers are allocated once per
 * process (cudaHostAlloc, portable) and shared under a mutex; copies below SMALL_BYTES, or
 * any copy when pinned memory cannot be had, take the plain path.
 */
#include <pthread.h>
#include <stdint.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "hostcopy.h"

#define STAGE_BYTES ((size_t) 32 << 20)
#define SMALL_BYTES ((size_t) 8 << 20)
#define PIECE_BYTES ((size_t) 1 << 20)

static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;
static void * g_stage[2];
static int g_state;            /* 0: not tried, 1: staging buffers ready, -1: unavailable */

static int stage_ready(void)
{
	if (g_state == 0) {
		g_state = -1;
		if (cudaHostAlloc(&g_stage[0], STAGE_BYTES, cudaHostAllocPortable) == cudaSuccess) {
			if (cudaHostAlloc(&g_stage[1], STAGE_BYTES, cudaHostAllocPortable) == cudaSuccess)
				g_state = 1;
			else
				cudaFreeHost(g_stage[0]);
		}
		if (g_state < 0)
			cudaGetLastError();   /* a failed pinned allocation is not the caller's error */
	}
	return g_state > 0;
}

/* memcpy of len bytes by the OpenMP team, in PIECE_BYTES pieces */
static void parallel_copy(void * dst, const void * src, size_t len)
{
	const long pieces = (long) ((len + PIECE_BYTES - 1) / PIECE_BYTES);
	#pragma omp parallel for schedule(static) num_threads(pieces < 16 ? (int) pieces : 16)
	for (long p = 0; p < pieces; p++) {
		const size_t o = (size_t) p * PIECE_BYTES;
		const size_t n = len - o < PIECE_BYTES ? len - o : PIECE_BYTES;
		memcpy((char *) dst + o, (const char *) src + o, n);
	}
}

cudaError_t spmv_h2d_pageable(void * dst, const void * src, size_t bytes, cudaStream_t s)
{
	if (bytes < SMALL_BYTES)
		return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
	pthread_mutex_lock(&g_lock);
	if (!stage_ready()) {
		pthread_mutex_unlock(&g_lock);
		return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
	}
	cudaEvent_t done[2] = {0, 0};
	cudaError_t e = cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming);
	if (e == cudaSuccess)
		e = cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming);
	size_t off = 0;
	for (int k = 0; e == cudaSuccess && off < bytes; k ^= 1) {
		const size_t len = bytes - off < STAGE_BYTES ? bytes - off : STAGE_BYTES;
		if (off >= 2 * STAGE_BYTES)
			e = cudaEventSynchronize(done[k]);      /* the DMA out of this buffer has finished */
		if (e != cudaSuccess)
			break;
		parallel_copy(g_stage[k], (const char *) src + off, len);
		e = cudaMemcpyAsync((char *) dst + off, g_stage[k], len, cudaMemcpyHostToDevice, s);
		if (e == cudaSuccess)
			e = cudaEventRecord(done[k], s);
		off += len;
	}
	/* the staging buffers are reused by the next copy: wait until this one has drained */
	for (int k = 0; k < 2; k++)
		if (done[k]) {
			if (e == cudaSuccess)
				e = cudaEventSynchronize(done[k]);
			cudaEventDestroy(done[k]);
		}
	pthread_mutex_unlock(&g_lock);
	return e;
}
