// Shared device/host helpers of libspmv_b200: error plumbing, PTX wrappers for the
// Blackwell bulk-copy engine (cp.async.bulk + mbarrier), small integer utilities.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "spmv_b200.h"

namespace spmv {

// ------------------------------------------------------------------ host error plumbing
void set_error(int code, const char * fmt, ...);
void clear_error();
int  last_status();

#define SPMV_CUDA_TRY(expr)                                                                      \
	do {                                                                                     \
		cudaError_t _e = (expr);                                                         \
		if (_e != cudaSuccess) {                                                         \
			spmv::set_error(_e == cudaErrorMemoryAllocation ? SPMV_ERR_NOMEM : SPMV_ERR_CUDA, \
				"%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__, __LINE__); \
			return spmv::last_status();                                              \
		}                                                                                \
	} while (0)

#define SPMV_TRY(expr)                                                                           \
	do {                                                                                     \
		int _s = (expr);                                                                 \
		if (_s != SPMV_OK)                                                               \
			return _s;                                                               \
	} while (0)

// Device-side error word (one per handle): first error wins.
#define DEV_ERR_TIMEOUT 1
#define DEV_ERR_BOUNDS  2
#define DEV_ERR_FORMAT  3

__device__ __forceinline__ void dev_flag_error(int * err, int code)
{
	if (err)
		atomicCAS(err, 0, code);
}

// ------------------------------------------------------------------ bulk copy / mbarrier
__device__ __forceinline__ uint32_t smem_u32(const void * p)
{
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t * bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t * bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
	             : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t * bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t * bar, uint32_t parity)
{
	uint32_t ok;
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
	    "selp.u32 %0, 1, 0, p;\n\t}"
	    : "=r"(ok)
	    : "r"(smem_u32(bar)), "r"(parity)
	    : "memory");
	return ok != 0;
}

// try_wait that suspends the warp in hardware (up to `hint_ns` nanoseconds, or until the
// phase completes) instead of returning at once: a waiting warp takes no issue slots from
// the warps that work.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t * bar, uint32_t parity, uint32_t hint_ns)
{
	uint32_t ok;
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
	    "selp.u32 %0, 1, 0, p;\n\t}"
	    : "=r"(ok)
	    : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
	    : "memory");
	return ok != 0;
}

// Bounded wait on an mbarrier phase: gives up after ~`budget` clock cycles and returns
// false (the caller records DEV_ERR_TIMEOUT and leaves), so no wait can spin forever.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t * bar, uint32_t parity, long long budget)
{
	if (mbar_try_wait(bar, parity))
		return true;
	long long t0 = clock64();
	while (!mbar_try_wait_sleep(bar, parity, 20000u)) {
		if (clock64() - t0 > budget)
			return false;
	}
	return true;
}

// Before a CTA (or warp) that gave up on a wait leaves: waits, bounded, for the `pending`
// bulk copies it issued that nobody has waited for, ring slots s, s+1, ... (mod S) from
// phase `parity` on, so that no copy is still writing into the shared memory of a CTA
// that has exited.  A slot whose copy already landed returns at once.
__device__ __forceinline__ void drain_ring(uint64_t * bars, int S, int s, uint32_t parity, int pending,
		long long budget)
{
	for (int q = 0; q < pending; q++) {
		(void) mbar_wait_bounded(&bars[s], parity, budget);
		if (++s == S) {
			s = 0;
			parity ^= 1u;
		}
	}
}

// Named barrier over n threads (a multiple of 32) of the CTA.
__device__ __forceinline__ void named_bar_sync(int id, int n)
{
	asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// Named barrier over n threads that also returns whether any of them passed `pred` true
// (so a decision to leave is taken by all of them together).
__device__ __forceinline__ bool named_bar_or(int id, int n, bool pred)
{
	uint32_t out;
	asm volatile(
	    "{\n\t.reg .pred p, q;\n\t"
	    "setp.ne.u32 p, %1, 0;\n\t"
	    "bar.red.or.pred q, %2, %3, p;\n\t"
	    "selp.u32 %0, 1, 0, q;\n\t}"
	    : "=r"(out)
	    : "r"((uint32_t) pred), "r"(id), "r"(n)
	    : "memory");
	return out != 0;
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Global -> shared bulk copy (TMA, non-tensor form) completing on `bar`.
// Requirements: both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void * dst_smem, const void * src_gmem, uint32_t bytes, uint64_t * bar)
{
	asm volatile(
	    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
	        smem_u32(dst_smem)),
	    "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
	    : "memory");
}

// Read-only path load of x (L1/texture path, stays in L2 across CTAs).
template <typename T>
__device__ __forceinline__ T ldg(const T * p)
{
	return __ldg(p);
}

// ------------------------------------------------------------------ misc
__host__ __device__ __forceinline__ int64_t ceil_div(int64_t a, int64_t b)
{
	return (a + b - 1) / b;
}

// x loads a gather thread of the warp-specialised kernels keeps in flight per round.
#ifndef SPMV_WS_GATHER_SLOTS
#define SPMV_WS_GATHER_SLOTS 4
#endif
static constexpr int WS_GATHER_SLOTS = SPMV_WS_GATHER_SLOTS;

static constexpr long long kWaitBudgetCycles = 4000000000LL;  // ~2 s at 1.9 GHz

// Bound of a device wait in clock cycles for a limit given in microseconds (0: the default
// ~2 s).  2,000 cycles a microsecond is at or above the B200's top SM clock (1,965 MHz), so
// a wait lasts at least the stated time.
__host__ __device__ __forceinline__ long long wait_budget_cycles(int limit_us)
{
	return limit_us > 0 ? (long long) limit_us * 2000LL : kWaitBudgetCycles;
}


}  // namespace spmv
