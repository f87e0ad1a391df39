// Device primitives used by the GPU conversions: exclusive scans, a stable LSD radix
// sort of (uint64 key, uint32 value) pairs, and the reference's nnz-balanced partitioner.
#pragma once

#include "common.cuh"

namespace spmv {

// Exclusive scan of n int32 (or int64) items into out[0..n]; out[n] receives the total.
int scan_exclusive(const int32_t * in, int64_t * out, int64_t n, cudaStream_t s);
int scan_exclusive(const int64_t * in, int64_t * out, int64_t n, cudaStream_t s);

// Inclusive max-scan of n int32 items (out may alias in).
int scan_inclusive_max(const int32_t * in, int32_t * out, int64_t n, cudaStream_t s);

// Maximum of n int32 row lengths rp[i+1]-rp[i] (0 for n == 0), written to *d_out.
int max_row_length(const int32_t * d_rp, int64_t n, int32_t * d_out, cudaStream_t s);

// Stable ascending sort of keys[0..n) (bits [0, key_bits) significant) carrying vals.
// Sorted in place (temporaries are stream-ordered allocations).
int radix_sort_pairs(uint64_t * keys, uint32_t * vals, int64_t n, int key_bits, cudaStream_t s);

// loop_partitioner_balance_prefix_sums (lib/parallel_util.h:156-181) for all T workers at
// once: ranges[2t], ranges[2t+1] = [start, end) of worker t over the ascending sums[0..N).
int partition_prefix_sums(const int32_t * d_sums, int64_t N, int64_t total, int T, int64_t * d_ranges,
		cudaStream_t s);

// Nearest-index binary search over an ascending array, inclusive bounds
// (lib/macros/macrolib.h:537-588, default compare/distance :506-514).
__device__ __forceinline__ int64_t nearest_index(const int32_t * A, int64_t lo, int64_t hi, int64_t target)
{
	int64_t s = lo, e = hi, mid;
	if (target < (int64_t) A[s])
		return s;
	if (target > (int64_t) A[e])
		return e;
	for (;;) {
		mid = (s + e) / 2;
		if (mid == s || mid == e)
			break;
		if (target > (int64_t) A[mid])
			s = mid;
		else
			e = mid;
	}
	if (target == (int64_t) A[s])
		return s;
	if (target == (int64_t) A[e])
		return e;
	int64_t ds = target - (int64_t) A[s], de = target - (int64_t) A[e];
	ds = ds < 0 ? -ds : ds;
	de = de < 0 ? -de : de;
	return (ds < de) ? s : e;
}

// First index i in [lo, hi] with A[i] >= v (A ascending); hi if none.
__device__ __forceinline__ int64_t lower_bound_i32(const int32_t * A, int64_t lo, int64_t hi, int64_t v)
{
	while (lo < hi) {
		int64_t mid = (lo + hi) >> 1;
		if ((int64_t) A[mid] < v)
			lo = mid + 1;
		else
			hi = mid;
	}
	return lo;
}

// Stream-ordered scratch allocation helper (freed by its destructor on the same stream).
struct DevBuf {
	void * p = nullptr;
	cudaStream_t s = nullptr;
	DevBuf() = default;
	DevBuf(const DevBuf &) = delete;
	DevBuf & operator=(const DevBuf &) = delete;
	int alloc(size_t bytes, cudaStream_t stream)
	{
		s = stream;
		cudaError_t e = cudaMallocAsync(&p, bytes ? bytes : 16, stream);
		if (e != cudaSuccess) {
			p = nullptr;
			set_error(SPMV_ERR_NOMEM, "scratch allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
			return SPMV_ERR_NOMEM;
		}
		return SPMV_OK;
	}
	template <typename T>
	T * as() const
	{
		return static_cast<T *>(p);
	}
	~DevBuf()
	{
		if (p)
			cudaFreeAsync(p, s);
	}
};

}  // namespace spmv
