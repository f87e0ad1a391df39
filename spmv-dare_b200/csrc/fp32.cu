// FP32 storage variant of CSR SpMV: values rounded once from FP64 to FP32, int32 column
// indices kept exact, x and y in FP32.  Each row is accumulated with the compensated dot
// product Dot2 of Ogita, Rump and Oishi ("Accurate sum and dot product", SIAM J. Sci.
// Comput. 26(6), 2005): every FP32 product's rounding error is recovered exactly with an
// FMA (TwoProduct) and every addition's with Knuth's TwoSum, and the errors are summed in
// a second FP32 accumulator.  The result is as accurate as if computed in twice the
// working precision and then rounded, so the row error is dominated by the one-time
// rounding of the stored values and of x.
//
// Staging follows the FP64 kernel (spmv_kernels.cu): persistent CTAs, bulk copies of each
// block's contiguous (values, columns) range into shared memory, a CTA-wide x gather, then
// one thread per row; a row longer than a block is reduced by the whole CTA with a
// compensated tree.
#include "internal.h"
#include "primitives.cuh"

namespace spmv {

int build_exec(Handle & h, const int32_t * d_P, int64_t U, int V);

namespace {

constexpr int F32_THREADS = 256;

struct F32Args {
	const StagedBlock * blocks;
	int64_t nblocks;
	const int32_t * rp;
	const int32_t * cols;
	const float * vals;
	const float * x;
	float * y;
	int cap_al;
	int stages;
	int stage_bytes;
	int * err;
};

// Knuth's TwoSum: s + e == a + b exactly.
__device__ __forceinline__ void two_sum(float a, float b, float & s, float & e)
{
	s = __fadd_rn(a, b);
	const float z = __fsub_rn(s, a);
	e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, z)), __fsub_rn(b, z));
}

// One Dot2 step: (s, c) += a * x.
__device__ __forceinline__ void dot2_step(float a, float x, float & s, float & c)
{
	const float p = __fmul_rn(a, x);
	const float pe = __fmaf_rn(a, x, -p);          // TwoProduct error, exact
	float t, e;
	two_sum(s, p, t, e);
	s = t;
	c = __fadd_rn(c, __fadd_rn(e, pe));
}

// (s1, c1) + (s2, c2) as a compensated pair.
__device__ __forceinline__ void merge(float & s1, float & c1, float s2, float c2)
{
	float t, e;
	two_sum(s1, s2, t, e);
	s1 = t;
	c1 = __fadd_rn(__fadd_rn(c1, c2), e);
}

__device__ __forceinline__ void issue_f32(const F32Args & a, int64_t b, int s, uint8_t * smem, uint64_t * bars)
{
	const StagedBlock d = a.blocks[b];
	if (d.units < 0 || d.elems == 0) {
		mbar_arrive(&bars[s]);
		return;
	}
	const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
	const int64_t e1 = ((int64_t) d.elem0 + d.elems + 3) & ~(int64_t) 3;
	const uint32_t cnt = (uint32_t) (e1 - e0);
	float * sv = reinterpret_cast<float *>(smem + (size_t) s * a.stage_bytes);
	int32_t * sc = reinterpret_cast<int32_t *>(smem + (size_t) s * a.stage_bytes + (size_t) a.cap_al * 4);
	fence_proxy_async_smem();
	mbar_arrive_expect_tx(&bars[s], cnt * 8u);
	bulk_g2s(sv, a.vals + e0, cnt * 4u, &bars[s]);
	bulk_g2s(sc, a.cols + e0, cnt * 4u, &bars[s]);
}

__global__ void __launch_bounds__(F32_THREADS) f32_kernel(F32Args a)
{
	extern __shared__ __align__(128) uint8_t smem[];
	__shared__ float red_s[F32_THREADS / 32], red_c[F32_THREADS / 32];
	float * xb = reinterpret_cast<float *>(smem + (size_t) a.stages * a.stage_bytes);
	uint64_t * bars = reinterpret_cast<uint64_t *>(smem + (size_t) a.stages * a.stage_bytes + (size_t) a.cap_al * 4);
	if (threadIdx.x == 0) {
		for (int s = 0; s < a.stages; s++)
			mbar_init(&bars[s], 1);
		mbar_fence_init();
	}
	__syncthreads();
	if (threadIdx.x == 0)
		for (int s = 0; s < a.stages; s++) {
			const int64_t b = (int64_t) blockIdx.x + (int64_t) s * gridDim.x;
			if (b < a.nblocks)
				issue_f32(a, b, s, smem, bars);
		}
	int s = 0;
	uint32_t parity = 0;
	for (int64_t b = blockIdx.x; b < a.nblocks; b += gridDim.x) {
		const StagedBlock d = a.blocks[b];
		const bool ok = mbar_wait_bounded(&bars[s], parity, kWaitBudgetCycles);
		if (__syncthreads_or(!ok)) {
			if (threadIdx.x == 0)
				dev_flag_error(a.err, DEV_ERR_TIMEOUT);
			return;
		}
		if (d.units >= 0) {
			const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
			const int off = (int) (d.elem0 - e0);
			const float * sv = reinterpret_cast<const float *>(smem + (size_t) s * a.stage_bytes);
			const int32_t * sc = reinterpret_cast<const int32_t *>(smem + (size_t) s * a.stage_bytes + (size_t) a.cap_al * 4);
			int js0 = 0, je0 = 0;
			if ((int) threadIdx.x < d.units) {
				const int64_t r = (int64_t) d.unit0 + threadIdx.x;
				js0 = (int) ((int64_t) __ldg(a.rp + r) - e0);
				je0 = (int) ((int64_t) __ldg(a.rp + r + 1) - e0);
			}
			#pragma unroll 4
			for (int e = threadIdx.x; e < d.elems; e += blockDim.x)
				xb[off + e] = __ldg(a.x + sc[off + e]);
			__syncthreads();
			for (int u = threadIdx.x; u < d.units; u += blockDim.x) {
				const int64_t r = (int64_t) d.unit0 + u;
				const int js = (u == (int) threadIdx.x) ? js0 : (int) ((int64_t) a.rp[r] - e0);
				const int je = (u == (int) threadIdx.x) ? je0 : (int) ((int64_t) a.rp[r + 1] - e0);
				float sum = 0.0f, c = 0.0f;
				#pragma unroll 4
				for (int j = js; j < je; j++)
					dot2_step(sv[j], xb[j], sum, c);
				a.y[r] = __fadd_rn(sum, c);
			}
		} else {
			// one long row: every thread a strided compensated partial, then a compensated tree
			const int64_t r = d.unit0;
			float sum = 0.0f, c = 0.0f;
			for (int64_t j = (int64_t) a.rp[r] + threadIdx.x; j < a.rp[r + 1]; j += blockDim.x)
				dot2_step(a.vals[j], __ldg(a.x + a.cols[j]), sum, c);
			#pragma unroll
			for (int o = 16; o > 0; o >>= 1) {
				const float s2 = __shfl_down_sync(0xffffffffu, sum, o);
				const float c2 = __shfl_down_sync(0xffffffffu, c, o);
				merge(sum, c, s2, c2);
			}
			if ((threadIdx.x & 31) == 0) {
				red_s[threadIdx.x >> 5] = sum;
				red_c[threadIdx.x >> 5] = c;
			}
			__syncthreads();
			if (threadIdx.x == 0) {
				float ts = red_s[0], tc = red_c[0];
				for (int w = 1; w < (int) (blockDim.x >> 5); w++)
					merge(ts, tc, red_s[w], red_c[w]);
				a.y[r] = __fadd_rn(ts, tc);
			}
		}
		__syncthreads();
		if (threadIdx.x == 0) {
			const int64_t nb = b + (int64_t) a.stages * gridDim.x;
			if (nb < a.nblocks)
				issue_f32(a, nb, s, smem, bars);
		}
		if (++s == a.stages) {
			s = 0;
			parity ^= 1u;
		}
	}
}

// ------------------------------------------------------------------ warp-specialised FP32 kernel
// The FP64 warp-specialised kernel's structure (spmv_kernels.cu: gather warps fetch x for
// block k+1 while row warps sum block k; long rows as chunk runs in per-CTA group order)
// with FP32 entries: the stage holds values (4 B) | columns (4 B) | gathered x (4 B).
// Every row, long ones included, is one sequential Dot2 chain.
struct F32WsArgs {
	const StagedBlock * blocks;
	const int64_t * ranges;
	const int32_t * rp;
	const int32_t * cols;
	const float * vals;
	const float * x;
	float * y;
	int cap_al;
	int stages;
	int stage_bytes;
	int row_threads;
	int * err;
};

__device__ __forceinline__ void f32ws_issue(const F32WsArgs & a, const StagedBlock & d, int s, uint8_t * smem, uint64_t * bars)
{
	if (d.elems == 0) {
		mbar_arrive(&bars[s]);
		return;
	}
	const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
	const int64_t e1 = ((int64_t) d.elem0 + d.elems + 3) & ~(int64_t) 3;
	const uint32_t cnt = (uint32_t) (e1 - e0);
	float * sv = reinterpret_cast<float *>(smem + (size_t) s * a.stage_bytes);
	int32_t * sc = reinterpret_cast<int32_t *>(smem + (size_t) s * a.stage_bytes + (size_t) a.cap_al * 4);
	fence_proxy_async_smem();
	mbar_arrive_expect_tx(&bars[s], cnt * 8u);
	bulk_g2s(sv, a.vals + e0, cnt * 4u, &bars[s]);
	bulk_g2s(sc, a.cols + e0, cnt * 4u, &bars[s]);
}

__global__ void __launch_bounds__(512) ws_f32_kernel(F32WsArgs a)
{
	extern __shared__ __align__(128) uint8_t smem[];
	__shared__ StagedBlock sdesc[8];
	const int S = a.stages;
	uint64_t * full = reinterpret_cast<uint64_t *>(smem + (size_t) S * a.stage_bytes);
	uint64_t * prod = full + S;
	const int nr = a.row_threads;
	const int ng = (int) blockDim.x - nr;
	if (threadIdx.x == 0) {
		for (int s = 0; s < S; s++) {
			mbar_init(&full[s], 1);
			mbar_init(&prod[s], (uint32_t) ng);
		}
		mbar_fence_init();
	}
	__syncthreads();
	int s = 0;
	uint32_t parity = 0;
	const int64_t b_begin = a.ranges[blockIdx.x], b_end = a.ranges[blockIdx.x + 1];
	if ((int) threadIdx.x < ng) {
		// ---- gather warps: x of every staged entry, WS_GATHER_SLOTS loads in flight per thread
		const int gt = threadIdx.x;
		for (int64_t b = b_begin; b < b_end; b++) {
			if (!mbar_wait_bounded(&full[s], parity, kWaitBudgetCycles)) {
				dev_flag_error(a.err, DEV_ERR_TIMEOUT);
				return;
			}
			const StagedBlock d = sdesc[s];
			if (d.elems > 0) {
				uint8_t * st = smem + (size_t) s * a.stage_bytes;
				const int32_t * sc = reinterpret_cast<const int32_t *>(st + (size_t) a.cap_al * 4);
				float * xg = reinterpret_cast<float *>(st + (size_t) a.cap_al * 8);
				const int off = d.elem0 & 3;
				for (int e0 = gt; e0 < d.elems; e0 += WS_GATHER_SLOTS * ng) {
					float xv[WS_GATHER_SLOTS];
					#pragma unroll
					for (int k = 0; k < WS_GATHER_SLOTS; k++) {
						const int e = e0 + k * ng;
						if (e < d.elems)
							xv[k] = __ldg(a.x + sc[off + e]);
					}
					#pragma unroll
					for (int k = 0; k < WS_GATHER_SLOTS; k++) {
						const int e = e0 + k * ng;
						if (e < d.elems)
							xg[off + e] = xv[k];
					}
				}
			}
			mbar_arrive(&prod[s]);
			if (++s == S) {
				s = 0;
				parity ^= 1u;
			}
		}
		return;
	}
	// ---- row warps
	const int rt = (int) threadIdx.x - ng;
	if (rt == 0)
		for (int q = 0; q < S; q++) {
			const int64_t b = b_begin + q;
			if (b < b_end) {
				const StagedBlock d = a.blocks[b];
				sdesc[q] = d;
				f32ws_issue(a, d, q, smem, full);
			}
		}
	named_bar_sync(1, nr);
	float ls = 0.0f, lc = 0.0f;      // running Dot2 pair of a long row across its chunks
	for (int64_t b = b_begin; b < b_end; b++) {
		const int64_t nb = b + S;
		StagedBlock dnext{};
		if (rt == 0 && nb < b_end)
			dnext = a.blocks[nb];
		const StagedBlock d = sdesc[s];
		const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
		int js = 0, je = 0;
		if (d.units >= 0 && rt < d.units) {
			const int64_t r = (int64_t) d.unit0 + rt;
			js = (int) ((int64_t) __ldg(a.rp + r) - e0);
			je = (int) ((int64_t) __ldg(a.rp + r + 1) - e0);
		}
		const bool ok = mbar_wait_bounded(&prod[s], parity, kWaitBudgetCycles);
		if (named_bar_or(1, nr, !ok)) {      // all row threads leave together
			if (rt == 0)
				dev_flag_error(a.err, DEV_ERR_TIMEOUT);
			return;
		}
		const uint8_t * st = smem + (size_t) s * a.stage_bytes;
		const float * sv = reinterpret_cast<const float *>(st);
		const float * xg = reinterpret_cast<const float *>(st + (size_t) a.cap_al * 8);
		if (d.units >= 0) {
			if (rt < d.units) {
				float sum = 0.0f, c = 0.0f;
				#pragma unroll 4
				for (int j = js; j < je; j++)
					dot2_step(sv[j], xg[j], sum, c);
				a.y[(int64_t) d.unit0 + rt] = __fadd_rn(sum, c);
			}
		} else if (rt == 0) {
			const int flags = -d.units - 1;
			const int off = d.elem0 & 3;
			if (flags & 1) {
				ls = 0.0f;
				lc = 0.0f;
			}
			#pragma unroll 4
			for (int e = 0; e < d.elems; e++)
				dot2_step(sv[off + e], xg[off + e], ls, lc);
			if (flags & 2)
				a.y[d.unit0] = __fadd_rn(ls, lc);
		}
		named_bar_sync(1, nr);
		if (rt == 0 && nb < b_end) {
			sdesc[s] = dnext;
			f32ws_issue(a, dnext, s, smem, full);
		}
		if (++s == S) {
			s = 0;
			parity ^= 1u;
		}
	}
}

__global__ void f64_to_f32_kernel(const double * in, float * out, int64_t n)
{
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		out[i] = __double2float_rn(in[i]);
}

__global__ void conv_kernel_d2f(const double * in, float * out, int64_t n)
{
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		out[i] = __double2float_rn(in[i]);
}

__global__ void conv_kernel_f2d(const float * in, double * out, int64_t n)
{
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		out[i] = (double) in[i];
}

}  // namespace

const void * ws_f32_kernel_fn()
{
	return (const void *) ws_f32_kernel;
}

// Rounds the stored FP64 values to FP32 and builds the staged block table: by default
// (kernel -1 or 4) the warp-specialised kernel's chunk-run table in per-CTA group order;
// kernel 0 keeps the CTA staged kernel (blocks of up to 2048 entries, 8 bytes staged each).
int convert_f32(Handle & h)
{
	cudaStream_t s = h.stream;
	SPMV_TRY(h.alloc(&h.d_vf, h.nnz + 8));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_vf, 0, (h.nnz + 8) * sizeof(float), s));
	if (h.nnz > 0) {
		f64_to_f32_kernel<<<(unsigned) ceil_div(h.nnz, 256), 256, 0, s>>>(h.d_v, h.d_vf, h.nnz);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	if (h.desc.kernel < 0 || h.desc.kernel == 4) {
		spmv_format_desc saved = h.desc;
		h.desc.kernel = 4;
		const int st = build_exec(h, h.d_rp, h.m, 1);     // geometry of ws_f32_kernel (values F32)
		h.desc = saved;
		if (st != SPMV_OK)
			return st;
		h.kernels_per_run = h.num_blocks > 0 ? 1 : 0;
		return SPMV_OK;
	}
	spmv_format_desc saved = h.desc;
	if (h.desc.block_nnz == 0)
		h.desc.block_nnz = 2048;
	h.desc.kernel = 0;
	int st = build_exec(h, h.d_rp, h.m, 1);
	h.desc = saved;
	if (st != SPMV_OK)
		return st;
	// shared memory of the FP32 kernel: 8 bytes per staged entry + a 4-byte x buffer
	const int cap_al = h.block_cap + 8;
	const int stage_bytes = (int) (ceil_div((int64_t) cap_al * 8, 128) * 128);
	const int max_stages = (int) ((220 * 1024 - 64 - cap_al * 4) / stage_bytes);
	if (h.stages > max_stages)
		h.stages = max_stages > 0 ? max_stages : 1;
	h.smem_bytes = (size_t) h.stages * stage_bytes + (size_t) cap_al * 4 + 64;
	SPMV_CUDA_TRY(cudaFuncSetAttribute(f32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) h.smem_bytes));
	int per_sm = 0;
	SPMV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f32_kernel, F32_THREADS, h.smem_bytes));
	if (h.desc.ctas_per_sm > 0)
		per_sm = h.desc.ctas_per_sm;
	int64_t g = (int64_t) h.num_sms * (per_sm > 0 ? per_sm : 1);
	if (g > h.num_blocks)
		g = h.num_blocks;
	h.grid = (int) (g > 0 ? g : 1);
	h.kernels_per_run = h.num_blocks > 0 ? 1 : 0;
	return SPMV_OK;
}

int launch_spmv_f32(Handle & h, const float * d_x, float * d_y, cudaStream_t s)
{
	if (h.num_blocks == 0)
		return SPMV_OK;
	if (h.exec_kernel == 4) {
		F32WsArgs w{};
		w.blocks = h.d_blocks;
		w.ranges = h.d_cta_ranges;
		w.rp = h.d_rp;
		w.cols = h.d_ci;
		w.vals = h.d_vf;
		w.x = d_x;
		w.y = d_y;
		w.cap_al = h.block_cap + 8;
		w.stages = h.stages;
		w.stage_bytes = (int) (ceil_div((int64_t) w.cap_al * 12, 128) * 128);
		w.row_threads = h.row_threads;
		w.err = h.d_err;
		ws_f32_kernel<<<h.grid, h.threads, h.smem_bytes, s>>>(w);
		SPMV_CUDA_TRY(cudaGetLastError());
		return SPMV_OK;
	}
	F32Args a{};
	a.blocks = h.d_blocks;
	a.nblocks = h.num_blocks;
	a.rp = h.d_rp;
	a.cols = h.d_ci;
	a.vals = h.d_vf;
	a.x = d_x;
	a.y = d_y;
	a.cap_al = h.block_cap + 8;
	a.stages = h.stages;
	a.stage_bytes = (int) (ceil_div((int64_t) a.cap_al * 8, 128) * 128);
	a.err = h.d_err;
	f32_kernel<<<h.grid, F32_THREADS, h.smem_bytes, s>>>(a);
	SPMV_CUDA_TRY(cudaGetLastError());
	return SPMV_OK;
}

// ------------------------------------------------------------------ allocation-free entry
// Scratch of spmv_run_device_mixed_noalloc: the FP32 copy of x followed by the FP32 y,
// in one file-scope device array that every GPU loading this library holds until exit.
static __device__ __align__(256) float g_mixed_scratch[SPMV_NOALLOC_MAX_ELEMS];

// Device address of g_mixed_scratch per device, resolved once per device (with that
// device current) by the first call on it.
static float * g_mixed_scratch_addr[64];

static int mixed_scratch(float ** out)
{
	int dev = 0;
	SPMV_CUDA_TRY(cudaGetDevice(&dev));
	if (dev < 0 || dev >= 64) {
		set_error(SPMV_ERR_ARG, "no-alloc entry: device ordinal %d out of range", dev);
		return SPMV_ERR_ARG;
	}
	if (!g_mixed_scratch_addr[dev]) {
		void * ptr = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&ptr, g_mixed_scratch);
		if (e != cudaSuccess) {
			set_error(SPMV_ERR_CUDA, "no-alloc entry: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
			return SPMV_ERR_CUDA;
		}
		g_mixed_scratch_addr[dev] = static_cast<float *>(ptr);
	}
	*out = g_mixed_scratch_addr[dev];
	return SPMV_OK;
}

int run_mixed_noalloc(Handle & h, const double * d_x, double * d_y, cudaStream_t s)
{
	if (h.desc.values != SPMV_VALUES_F32) {
		set_error(SPMV_ERR_ARG, "no-alloc entry: the handle must store FP32 values (value type SPMV_VALUES_F32)");
		return SPMV_ERR_ARG;
	}
	if (h.n + h.m > (int64_t) SPMV_NOALLOC_MAX_ELEMS) {
		set_error(SPMV_ERR_ARG, "no-alloc entry: n + m = %lld exceeds its static scratch of %d FP32 elements",
				(long long) (h.n + h.m), (int) SPMV_NOALLOC_MAX_ELEMS);
		return SPMV_ERR_ARG;
	}
	float * scratch = nullptr;
	SPMV_TRY(mixed_scratch(&scratch));
	float * xf = scratch;            // x rounded to FP32: written in full before it is read
	float * yf = scratch + h.n;      // FP32 y: every row is written by the SpMV kernel
	SPMV_TRY(convert_vector_d2f(d_x, xf, h.n, s));
	SPMV_TRY(launch_spmv_f32(h, xf, yf, s));
	SPMV_TRY(convert_vector_f2d(yf, d_y, h.m, s));
	return SPMV_OK;
}

int convert_vector_d2f(const double * in, float * out, int64_t n, cudaStream_t s)
{
	if (n > 0) {
		conv_kernel_d2f<<<(unsigned) ceil_div(n, 256), 256, 0, s>>>(in, out, n);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	return SPMV_OK;
}

int convert_vector_f2d(const float * in, double * out, int64_t n, cudaStream_t s)
{
	if (n > 0) {
		conv_kernel_f2d<<<(unsigned) ceil_div(n, 256), 256, 0, s>>>(in, out, n);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	return SPMV_OK;
}

}  // namespace spmv
