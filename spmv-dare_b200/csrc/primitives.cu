// Device primitives: exclusive scan, stable LSD radix sort, nnz-balanced partitioner.
#include "primitives.cuh"

namespace spmv {

namespace {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// Inclusive block scan of one int64 per thread; returns the inclusive prefix and sets
// *total to the block sum.
__device__ __forceinline__ int64_t block_inclusive_scan(int64_t v, int64_t * total)
{
	__shared__ int64_t warp_tot[SCAN_THREADS / 32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		int64_t t = __shfl_up_sync(0xffffffffu, v, o);
		if (lane >= o)
			v += t;
	}
	if (lane == 31)
		warp_tot[w] = v;
	__syncthreads();
	if (w == 0) {
		int64_t t = (lane < (int) (blockDim.x >> 5)) ? warp_tot[lane] : 0;
		#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			int64_t u = __shfl_up_sync(0xffffffffu, t, o);
			if (lane >= o)
				t += u;
		}
		warp_tot[lane] = t;   // inclusive warp prefix
	}
	__syncthreads();
	int64_t add = (w > 0) ? warp_tot[w - 1] : 0;
	*total = warp_tot[(blockDim.x >> 5) - 1];
	__syncthreads();
	return v + add;
}

template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) scan_reduce_kernel(const T * in, int64_t n, int64_t * partial)
{
	int64_t base = (int64_t) blockIdx.x * SCAN_TILE;
	int64_t sum = 0;
	#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; k++) {
		int64_t i = base + (int64_t) threadIdx.x * SCAN_ITEMS + k;
		if (i < n)
			sum += (int64_t) in[i];
	}
	int64_t tot;
	block_inclusive_scan(sum, &tot);
	if (threadIdx.x == 0)
		partial[blockIdx.x] = tot;
}

// Exclusive scan of a tile with a per-tile offset; the last tile writes out[n] = total.
template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) scan_apply_kernel(const T * in, int64_t n, const int64_t * offsets,
		int64_t * out)
{
	int64_t base = (int64_t) blockIdx.x * SCAN_TILE;
	int64_t loc[SCAN_ITEMS];
	int64_t sum = 0;
	#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; k++) {
		int64_t i = base + (int64_t) threadIdx.x * SCAN_ITEMS + k;
		loc[k] = (i < n) ? (int64_t) in[i] : 0;
		sum += loc[k];
	}
	int64_t tot;
	int64_t incl = block_inclusive_scan(sum, &tot);
	int64_t run = incl - sum + (offsets ? offsets[blockIdx.x] : 0);
	#pragma unroll
	for (int k = 0; k < SCAN_ITEMS; k++) {
		int64_t i = base + (int64_t) threadIdx.x * SCAN_ITEMS + k;
		if (i < n)
			out[i] = run;
		run += loc[k];
		if (i == n - 1)
			out[n] = run;
	}
}

__global__ void set_zero_total(int64_t * out)
{
	out[0] = 0;
}

template <typename T>
int scan_impl(const T * in, int64_t * out, int64_t n, cudaStream_t s)
{
	if (n == 0) {
		set_zero_total<<<1, 1, 0, s>>>(out);
		SPMV_CUDA_TRY(cudaGetLastError());
		return SPMV_OK;
	}
	int64_t tiles = ceil_div(n, SCAN_TILE);
	if (tiles == 1) {
		scan_apply_kernel<T><<<1, SCAN_THREADS, 0, s>>>(in, n, nullptr, out);
		SPMV_CUDA_TRY(cudaGetLastError());
		return SPMV_OK;
	}
	DevBuf partial, poff;
	SPMV_TRY(partial.alloc(tiles * sizeof(int64_t), s));
	SPMV_TRY(poff.alloc((tiles + 1) * sizeof(int64_t), s));
	scan_reduce_kernel<T><<<(unsigned) tiles, SCAN_THREADS, 0, s>>>(in, n, partial.as<int64_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(scan_impl<int64_t>(partial.as<int64_t>(), poff.as<int64_t>(), tiles, s));
	scan_apply_kernel<T><<<(unsigned) tiles, SCAN_THREADS, 0, s>>>(in, n, poff.as<int64_t>(), out);
	SPMV_CUDA_TRY(cudaGetLastError());
	return SPMV_OK;
}

// ------------------------------------------------------------------ radix sort
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_CHUNKS = 16;                      // 32-item chunks per warp
constexpr int RS_WARP_ITEMS = 32 * RS_CHUNKS;      // 512
constexpr int RS_TILE = RS_WARPS * RS_WARP_ITEMS;  // 4096

__global__ void __launch_bounds__(RS_THREADS) radix_hist_kernel(const uint64_t * keys, int64_t n, int shift,
		int32_t * counts, int64_t ntiles)
{
	__shared__ int32_t h[256];
	h[threadIdx.x] = 0;
	__syncthreads();
	int64_t base = (int64_t) blockIdx.x * RS_TILE;
	for (int i = threadIdx.x; i < RS_TILE; i += RS_THREADS) {
		int64_t idx = base + i;
		if (idx < n)
			atomicAdd(&h[(keys[idx] >> shift) & 255], 1);
	}
	__syncthreads();
	counts[(int64_t) threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: items of a tile are ranked in index order (warp-major, chunk, lane).
__global__ void __launch_bounds__(RS_THREADS) radix_scatter_kernel(const uint64_t * kin, const uint32_t * vin,
		uint64_t * kout, uint32_t * vout, int64_t n, int shift, const int64_t * offs, int64_t ntiles)
{
	__shared__ int32_t wh[RS_WARPS][256];
	__shared__ int64_t tbase[256];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_THREADS)
		(&wh[0][0])[i] = 0;
	__syncthreads();
	const int64_t base = (int64_t) blockIdx.x * RS_TILE + (int64_t) w * RS_WARP_ITEMS;
	const unsigned lt_mask = (1u << lane) - 1u;
	for (int c = 0; c < RS_CHUNKS; c++) {
		int64_t idx = base + c * 32 + lane;
		bool valid = idx < n;
		int d = valid ? (int) ((kin[idx] >> shift) & 255) : 256 + lane;
		unsigned peers = __match_any_sync(0xffffffffu, d);
		int leader = __ffs(peers) - 1;
		if (valid && lane == leader)
			wh[w][d] += __popc(peers);
	}
	__syncthreads();
	{
		int d = threadIdx.x;   // RS_THREADS == 256 digits
		int32_t run = 0;
		for (int ww = 0; ww < RS_WARPS; ww++) {
			int32_t t = wh[ww][d];
			wh[ww][d] = run;
			run += t;
		}
		tbase[d] = offs[(int64_t) d * ntiles + blockIdx.x];
	}
	__syncthreads();
	for (int c = 0; c < RS_CHUNKS; c++) {
		int64_t idx = base + c * 32 + lane;
		bool valid = idx < n;
		uint64_t k = valid ? kin[idx] : 0;
		int d = valid ? (int) ((k >> shift) & 255) : 256 + lane;
		unsigned peers = __match_any_sync(0xffffffffu, d);
		int leader = __ffs(peers) - 1;
		if (valid) {
			int64_t pos = tbase[d] + wh[w][d] + __popc(peers & lt_mask);
			kout[pos] = k;
			vout[pos] = vin[idx];
		}
		__syncwarp();
		if (valid && lane == leader)
			wh[w][d] += __popc(peers);
		__syncwarp();
	}
}

__global__ void partition_kernel(const int32_t * sums, int64_t N, int64_t total, int T, int64_t * ranges)
{
	int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= T)
		return;
	int64_t target = (int64_t) sums[0] + (total * t) / T;
	int64_t target_next = (int64_t) sums[0] + (total * (t + 1)) / T;
	ranges[2 * t] = (t == 0) ? 0 : nearest_index(sums, 0, N - 1, target);
	ranges[2 * t + 1] = (t == T - 1) ? N : nearest_index(sums, 0, N - 1, target_next);
}

// ------------------------------------------------------------------ max scan
constexpr int MS_THREADS = 1024;

__device__ __forceinline__ int32_t block_inclusive_max(int32_t v, int32_t * total)
{
	__shared__ int32_t wt[MS_THREADS / 32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		int32_t t = __shfl_up_sync(0xffffffffu, v, o);
		if (lane >= o)
			v = max(v, t);
	}
	if (lane == 31)
		wt[w] = v;
	__syncthreads();
	if (w == 0) {
		int32_t t = (lane < (int) (blockDim.x >> 5)) ? wt[lane] : INT32_MIN;
		#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			int32_t u = __shfl_up_sync(0xffffffffu, t, o);
			if (lane >= o)
				t = max(t, u);
		}
		wt[lane] = t;
	}
	__syncthreads();
	int32_t r = (w > 0) ? max(v, wt[w - 1]) : v;
	*total = wt[(blockDim.x >> 5) - 1];
	__syncthreads();
	return r;
}

__global__ void __launch_bounds__(MS_THREADS) max_reduce_kernel(const int32_t * in, int64_t n, int32_t * partial)
{
	int64_t i = (int64_t) blockIdx.x * MS_THREADS + threadIdx.x;
	int32_t v = (i < n) ? in[i] : INT32_MIN;
	int32_t tot;
	block_inclusive_max(v, &tot);
	if (threadIdx.x == 0)
		partial[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(MS_THREADS) max_apply_kernel(const int32_t * in, int64_t n, const int32_t * carry,
		int32_t * out)
{
	int64_t i = (int64_t) blockIdx.x * MS_THREADS + threadIdx.x;
	int32_t v = (i < n) ? in[i] : INT32_MIN;
	int32_t tot;
	int32_t r = block_inclusive_max(v, &tot);
	if (carry && blockIdx.x > 0)
		r = max(r, carry[blockIdx.x - 1]);
	if (i < n)
		out[i] = r;
}

__global__ void row_len_max_kernel(const int32_t * rp, int64_t n, int32_t * out)
{
	int32_t best = 0;
	for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
		best = max(best, rp[i + 1] - rp[i]);
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
	if ((threadIdx.x & 31) == 0)
		atomicMax(out, best);
}

}  // namespace

int scan_inclusive_max(const int32_t * in, int32_t * out, int64_t n, cudaStream_t s)
{
	if (n == 0)
		return SPMV_OK;
	int64_t tiles = ceil_div(n, MS_THREADS);
	if (tiles == 1) {
		max_apply_kernel<<<1, MS_THREADS, 0, s>>>(in, n, nullptr, out);
		SPMV_CUDA_TRY(cudaGetLastError());
		return SPMV_OK;
	}
	DevBuf partial;
	SPMV_TRY(partial.alloc(tiles * sizeof(int32_t), s));
	max_reduce_kernel<<<(unsigned) tiles, MS_THREADS, 0, s>>>(in, n, partial.as<int32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(scan_inclusive_max(partial.as<int32_t>(), partial.as<int32_t>(), tiles, s));
	max_apply_kernel<<<(unsigned) tiles, MS_THREADS, 0, s>>>(in, n, partial.as<int32_t>(), out);
	SPMV_CUDA_TRY(cudaGetLastError());
	return SPMV_OK;
}

int max_row_length(const int32_t * d_rp, int64_t n, int32_t * d_out, cudaStream_t s)
{
	SPMV_CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(int32_t), s));
	if (n == 0)
		return SPMV_OK;
	int64_t grid = ceil_div(n, 256);
	if (grid > 4096)
		grid = 4096;
	row_len_max_kernel<<<(unsigned) grid, 256, 0, s>>>(d_rp, n, d_out);
	SPMV_CUDA_TRY(cudaGetLastError());
	return SPMV_OK;
}

int scan_exclusive(const int32_t * in, int64_t * out, int64_t n, cudaStream_t s)
{
	return scan_impl<int32_t>(in, out, n, s);
}

int scan_exclusive(const int64_t * in, int64_t * out, int64_t n, cudaStream_t s)
{
	return scan_impl<int64_t>(in, out, n, s);
}

int radix_sort_pairs(uint64_t * keys, uint32_t * vals, int64_t n, int key_bits, cudaStream_t s)
{
	if (n <= 1 || key_bits <= 0)
		return SPMV_OK;
	int64_t ntiles = ceil_div(n, RS_TILE);
	DevBuf k2, v2, counts, offs;
	SPMV_TRY(k2.alloc(n * sizeof(uint64_t), s));
	SPMV_TRY(v2.alloc(n * sizeof(uint32_t), s));
	SPMV_TRY(counts.alloc(256 * ntiles * sizeof(int32_t), s));
	SPMV_TRY(offs.alloc((256 * ntiles + 1) * sizeof(int64_t), s));
	uint64_t * ka = keys, * kb = k2.as<uint64_t>();
	uint32_t * va = vals, * vb = v2.as<uint32_t>();
	int passes = (key_bits + 7) / 8;
	for (int p = 0; p < passes; p++) {
		int shift = 8 * p;
		radix_hist_kernel<<<(unsigned) ntiles, RS_THREADS, 0, s>>>(ka, n, shift, counts.as<int32_t>(), ntiles);
		SPMV_CUDA_TRY(cudaGetLastError());
		SPMV_TRY(scan_exclusive(counts.as<int32_t>(), offs.as<int64_t>(), 256 * ntiles, s));
		radix_scatter_kernel<<<(unsigned) ntiles, RS_THREADS, 0, s>>>(ka, va, kb, vb, n, shift, offs.as<int64_t>(),
				ntiles);
		SPMV_CUDA_TRY(cudaGetLastError());
		uint64_t * kt = ka; ka = kb; kb = kt;
		uint32_t * vt = va; va = vb; vb = vt;
	}
	if (ka != keys) {
		SPMV_CUDA_TRY(cudaMemcpyAsync(keys, ka, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
		SPMV_CUDA_TRY(cudaMemcpyAsync(vals, va, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
	}
	return SPMV_OK;
}

int partition_prefix_sums(const int32_t * d_sums, int64_t N, int64_t total, int T, int64_t * d_ranges, cudaStream_t s)
{
	if (N < 1 || T < 1) {
		set_error(SPMV_ERR_ARG, "partition of an empty range");
		return SPMV_ERR_ARG;
	}
	partition_kernel<<<(T + 127) / 128, 128, 0, s>>>(d_sums, N, total, T, d_ranges);
	SPMV_CUDA_TRY(cudaGetLastError());
	return SPMV_OK;
}

}  // namespace spmv
