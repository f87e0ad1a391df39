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
#include <atomic>

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
			if (threadIdx.x == 0) {
				dev_flag_error(a.err, DEV_ERR_TIMEOUT);
				int pending = 0;          // copies issued for blocks b, b + grid, ... not yet waited for
				while (pending < a.stages && b + (int64_t) pending * gridDim.x < a.nblocks)
					pending++;
				drain_ring(bars, a.stages, s, parity, pending, kWaitBudgetCycles);
			}
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
// with FP32 entries: the stage holds values (4 B) | columns (4 B), and each gather thread
// overwrites the column it has read with the gathered x (4 B as well), so a stage takes 8
// bytes an entry (against 12 with a separate x buffer: 1.5 times the entries in flight for
// the same shared memory).  Every row, long ones included, is one sequential Dot2 chain.
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
	long long wait_budget;   // bound of the kernel's waits, clock cycles
	int hold;                // SPMV_DEBUG_WITHHOLD_HANDOFF: gather warps never hand a stage over
	const int4 * pinfo;      // packed columns: per block {16-byte offset, base, bits, stream bytes}
	const uint32_t * pcols;  // packed columns: the streams (pack.cu)
	const uint16_t * rassign;  // row_assign 1: local row of each row thread, longest rows first
};

// Column of entry e of a packed block stream (pack.cu): two whole words and a funnel shift.
__device__ __forceinline__ int32_t packed_col(const uint32_t * words, int e, int bits, int32_t base)
{
	const uint32_t bit = (uint32_t) e * (uint32_t) bits;
	const uint32_t w = bit >> 5;
	const uint32_t v = __funnelshift_r(words[w], words[w + 1], bit & 31);
	return base + (int32_t) (bits >= 32 ? v : (v & ((1u << bits) - 1u)));
}

// Packed variant: the stage holds values | x, and the block's packed column stream is copied
// to the top of the x region, so that x of stage position p only overwrites stream words
// of entries below p + 1 (x at byte 4p, the stream at 4 cap - bytes + e * bits / 8).
__device__ __forceinline__ void f32ws_issue_packed(const F32WsArgs & a, const StagedBlock & d, const int4 & pi, int s,
		uint8_t * smem, uint64_t * bars)
{
	if (d.elems == 0) {
		mbar_arrive(&bars[s]);
		return;
	}
	const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
	const int64_t e1 = ((int64_t) d.elem0 + d.elems + 3) & ~(int64_t) 3;
	const uint32_t cnt = (uint32_t) (e1 - e0);
	uint8_t * st = smem + (size_t) s * a.stage_bytes;
	uint8_t * words = st + (size_t) a.cap_al * 8 - (size_t) pi.w;
	fence_proxy_async_smem();
	mbar_arrive_expect_tx(&bars[s], cnt * 4u + (uint32_t) pi.w);
	bulk_g2s(st, a.vals + e0, cnt * 4u, &bars[s]);
	bulk_g2s(words, a.pcols + (int64_t) pi.x * 4, (uint32_t) pi.w, &bars[s]);
}

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

template <bool PACKED>
__global__ void __launch_bounds__(512) ws_f32_kernel(F32WsArgs a)
{
	extern __shared__ __align__(128) uint8_t smem[];
	__shared__ StagedBlock sdesc[8];
	__shared__ int4 spack[8];
	const int S = a.stages;
	uint64_t * full = reinterpret_cast<uint64_t *>(smem + (size_t) S * a.stage_bytes);
	uint64_t * prod = full + S;
	const int nr = a.row_threads;
	const int ng = (int) blockDim.x - nr;
	if (threadIdx.x == 0) {
		for (int s = 0; s < S; s++) {
			mbar_init(&full[s], 1);
			mbar_init(&prod[s], (uint32_t) (ng / 32));      // one arrival per gather warp
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
			const bool ok = mbar_wait_bounded(&full[s], parity, a.wait_budget);
			if (named_bar_or(2, ng, !ok)) {                // the gather warps leave together
				if (gt == 0)
					dev_flag_error(a.err, DEV_ERR_TIMEOUT);
				return;
			}
			const StagedBlock d = sdesc[s];
			if (PACKED && d.elems > 0) {
				// rounds of WS_GATHER_SLOTS * ng consecutive entries, the same count for every
				// gather thread: a round's x is stored only once every gather thread has
				// decoded the round's columns (named barrier 2), since x may overwrite them
				uint8_t * st = smem + (size_t) s * a.stage_bytes;
				float * xg = reinterpret_cast<float *>(st + (size_t) a.cap_al * 4);
				const int4 pi = spack[s];
				const uint32_t * words = reinterpret_cast<const uint32_t *>(st + (size_t) a.cap_al * 8 - (size_t) pi.w);
				const int off = d.elem0 & 3;
				const int per_round = WS_GATHER_SLOTS * ng;
				for (int rb = 0; rb < d.elems; rb += per_round) {
					float xv[WS_GATHER_SLOTS];
					#pragma unroll
					for (int k = 0; k < WS_GATHER_SLOTS; k++) {
						const int e = rb + gt + k * ng;
						if (e < d.elems)
							xv[k] = __ldg(a.x + packed_col(words, e, pi.z, pi.y));
					}
					named_bar_sync(2, ng);
					#pragma unroll
					for (int k = 0; k < WS_GATHER_SLOTS; k++) {
						const int e = rb + gt + k * ng;
						if (e < d.elems)
							xg[off + e] = xv[k];
					}
				}
			} else if (d.elems > 0) {
				uint8_t * st = smem + (size_t) s * a.stage_bytes;
				int32_t * sc = reinterpret_cast<int32_t *>(st + (size_t) a.cap_al * 4);
				float * xg = reinterpret_cast<float *>(sc);     // x of entry e replaces its column
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
			__syncwarp();                                  // the warp's stores before its arrival
			if ((gt & 31) == 0 && !a.hold)
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
				if (PACKED) {
					const int4 pi = a.pinfo[b];
					spack[q] = pi;
					f32ws_issue_packed(a, d, pi, q, smem, full);
				} else {
					f32ws_issue(a, d, q, smem, full);
				}
			}
		}
	named_bar_sync(1, nr);
	float ls = 0.0f, lc = 0.0f;      // running Dot2 pair of a long row across its chunks
	for (int64_t b = b_begin; b < b_end; b++) {
		const int64_t nb = b + S;
		StagedBlock dnext{};
		int4 pnext{};
		if (rt == 0 && nb < b_end) {
			dnext = a.blocks[nb];
			if (PACKED)
				pnext = a.pinfo[nb];
		}
		const StagedBlock d = sdesc[s];
		const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
		int js = 0, je = 0;
		int64_t r = -1;                  // this thread's row: by position, or longest first (rassign)
		if (d.units >= 0 && rt < d.units) {
			r = (int64_t) d.unit0 + (a.rassign ? (int64_t) a.rassign[(int64_t) d.unit0 + rt] : rt);
			js = (int) ((int64_t) __ldg(a.rp + r) - e0);
			je = (int) ((int64_t) __ldg(a.rp + r + 1) - e0);
		}
		const bool ok = mbar_wait_bounded(&prod[s], parity, a.wait_budget);
		if (named_bar_or(1, nr, !ok)) {      // all row threads leave together
			if (rt == 0) {
				dev_flag_error(a.err, DEV_ERR_TIMEOUT);
				// rt 0 issued the copies of blocks b .. b + S - 1: wait until they have landed
				drain_ring(full, S, s, parity, (int) (b_end - b < S ? b_end - b : S), kWaitBudgetCycles);
			}
			return;
		}
		const uint8_t * st = smem + (size_t) s * a.stage_bytes;
		const float * sv = reinterpret_cast<const float *>(st);
		const float * xg = reinterpret_cast<const float *>(st + (size_t) a.cap_al * 4);
		if (d.units >= 0) {
			if (rt < d.units) {
				float sum = 0.0f, c = 0.0f;
				#pragma unroll 4
				for (int j = js; j < je; j++)
					dot2_step(sv[j], xg[j], sum, c);
				a.y[r] = __fadd_rn(sum, c);
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
			if (PACKED) {
				spack[s] = pnext;
				f32ws_issue_packed(a, dnext, pnext, s, smem, full);
			} else {
				f32ws_issue(a, dnext, s, smem, full);
			}
		}
		if (++s == S) {
			s = 0;
			parity ^= 1u;
		}
	}
}

// ------------------------------------------------------------------ segmented FP32 kernel
// Kernel 7 (an option; kernel 4 stays the FP32 default, 0.207 ms vs 0.36 ms on the 4M-row
// matrix).  The FP32 variant fixes no summation order (only compensated FP32 rows), so it
// does not need one thread per row, and one very long row is spread over the whole GPU.  The CSR arrays are cut into 256-entry
// chunks; every warp streams a contiguous range of chunks through its own ring of bulk-copy
// stages (values and columns, 2 KB per chunk), and each lane takes 8 consecutive entries of a
// chunk (16-byte shared-memory reads), whose x it has already requested while the previous
// chunk was summed.  A lane runs Dot2 over its entries, closing rows at their boundaries; a
// row that spans lanes is joined by a compensated segmented scan over the warp, a row that
// spans chunks leaves per-chunk partials (head: the chunk's first row when it began earlier;
// tail: the chunk's last row when it goes on), merged in chunk order by a fix-up kernel.
// Empty rows are zeroed from a precomputed list.
constexpr int SEG_K = 8;
constexpr int SEG_CHUNK = 32 * SEG_K;
constexpr int SEG_THREADS = 128;             // 4 independent warps per CTA
constexpr int SEG_STAGE_BYTES = SEG_CHUNK * 8;

struct SegArgs {
	const int32_t * rp;
	const int32_t * ci;
	const float * v;
	const float * x;
	float * y;
	const int32_t * chunk_row;
	int64_t nchunks;
	int64_t nwarps;
	int64_t m;
	int64_t nnz;
	float2 * head;
	float2 * tail;
	int stages;
	int warp_bytes;
	int * err;
};

// Rows of one chunk from the lane's 8 entries (values vv, gathered x xv).
__device__ __forceinline__ void seg_chunk(const SegArgs & a, int64_t chunk, const float (&vv)[SEG_K], const float (&xv)[SEG_K])
{
	const unsigned FULL = 0xffffffffu;
	const int lane = threadIdx.x & 31;
	const int64_t e0 = chunk * SEG_CHUNK;
	const int64_t el = e0 + (int64_t) SEG_K * lane;
	// row of the lane's first entry: the largest r with rp[r] <= el, searched in windows of 32
	// row boundaries from the chunk's first row (a 5-step binary search over shuffles)
	int64_t row = -1;
	for (int64_t base = a.chunk_row[chunk];; base += 32) {
		const int64_t bi = base + 1 + lane;
		const int64_t b = bi <= a.m ? (int64_t) a.rp[bi] : INT64_MAX;
		int pos = 0;
		#pragma unroll
		for (int step = 16; step > 0; step >>= 1) {
			const int64_t bm = __shfl_sync(FULL, b, pos + step - 1);
			if (bm <= el)
				pos += step;
		}
		const int64_t b31 = __shfl_sync(FULL, b, 31);
		if (pos == 31 && b31 <= el)
			pos = 32;
		if (row < 0 && pos < 32)
			row = base + pos;
		if (!__any_sync(FULL, row < 0))
			break;
	}
	// the next 9 row ends: a boundary equal to el + k + 1 closes the current row after entry k
	int64_t nbv[SEG_K + 1];
	#pragma unroll
	for (int j = 0; j <= SEG_K; j++)
		nbv[j] = row + 1 + j <= a.m ? (int64_t) a.rp[row + 1 + j] : INT64_MAX;
	int64_t r = row;
	const int64_t hrow = row;
	float hs = 0.0f, hc = 0.0f;
	bool head_closed = false;
	float s = 0.0f, c = 0.0f;
	if (nbv[SEG_K] > el + SEG_K) {
		#pragma unroll
		for (int k = 0; k < SEG_K; k++) {
			if (el + k < a.nnz)
				dot2_step(vv[k], xv[k], s, c);
			int cnt = 0;
			#pragma unroll
			for (int j = 0; j <= SEG_K; j++)
				cnt += (nbv[j] == el + k + 1) ? 1 : 0;
			if (cnt > 0) {
				if (!head_closed) {
					hs = s;
					hc = c;
					head_closed = true;
				} else if (r < a.m) {
					a.y[r] = __fadd_rn(s, c);        // a row begun and ended inside the lane
				}
				s = 0.0f;
				c = 0.0f;
				r += cnt;                            // rows in between are empty (zeroed from the list)
			}
		}
	} else {
		// more row ends inside the lane than tracked (empty rows): walk the boundaries
		int64_t nb = r < a.m ? (int64_t) a.rp[r + 1] : INT64_MAX;
		for (int k = 0; k < SEG_K; k++) {
			const int64_t e = el + k;
			if (e < a.nnz)
				dot2_step(vv[k], xv[k], s, c);
			if (nb == e + 1) {
				if (!head_closed) {
					hs = s;
					hc = c;
					head_closed = true;
				} else if (r < a.m) {
					a.y[r] = __fadd_rn(s, c);
				}
				s = 0.0f;
				c = 0.0f;
				while (nb == e + 1) {
					r++;
					nb = r < a.m ? (int64_t) a.rp[r + 1] : INT64_MAX;
				}
			}
		}
	}
	const int64_t trow = r;
	const bool single = !head_closed;
	const int64_t tstart = trow < a.m ? (int64_t) a.rp[trow] : INT64_MAX;
	// segmented inclusive scan of the open tails: a lane inside one row that began before it
	// continues its left neighbour's partial
	int f = (single && tstart < el) ? 0 : 1;
	float vs = s, vc = c;
	#pragma unroll
	for (int d = 1; d < 32; d <<= 1) {
		const float s2 = __shfl_up_sync(FULL, vs, d);
		const float c2 = __shfl_up_sync(FULL, vc, d);
		const int f2 = __shfl_up_sync(FULL, f, d);
		if (lane >= d && !f) {
			float t = s2, tc = c2;
			merge(t, tc, vs, vc);
			vs = t;
			vc = tc;
			f = f2;
		}
	}
	const float cs = __shfl_up_sync(FULL, vs, 1);
	const float ccar = __shfl_up_sync(FULL, vc, 1);
	if (head_closed && hrow < a.m) {
		const int64_t hstart = a.rp[hrow];
		if (hstart < el && lane > 0) {           // the head continues the left lane's row
			float t = cs, tc = ccar;
			merge(t, tc, hs, hc);
			hs = t;
			hc = tc;
		}
		if (hstart < e0)
			a.head[chunk] = make_float2(hs, hc);   // the chunk's first row began in an earlier chunk
		else
			a.y[hrow] = __fadd_rn(hs, hc);
	}
	// the open tail of lane 31 goes on past the chunk
	if (lane == 31 && trow < a.m) {
		if (tstart < e0)
			a.head[chunk] = make_float2(vs, vc);     // the whole chunk lies inside one row
		else
			a.tail[chunk] = make_float2(vs, vc);
	}
}

__device__ __forceinline__ void seg_issue(const SegArgs & a, int64_t chunk, uint8_t * stage, uint64_t * bar)
{
	fence_proxy_async_smem();
	mbar_arrive_expect_tx(bar, SEG_STAGE_BYTES);
	bulk_g2s(stage, a.v + chunk * SEG_CHUNK, SEG_CHUNK * 4u, bar);
	bulk_g2s(stage + SEG_CHUNK * 4, a.ci + chunk * SEG_CHUNK, SEG_CHUNK * 4u, bar);
}

__global__ void __launch_bounds__(SEG_THREADS) f32seg_kernel(SegArgs a)
{
	extern __shared__ __align__(128) uint8_t smem[];
	const unsigned FULL = 0xffffffffu;
	const int lane = threadIdx.x & 31;
	const int wib = threadIdx.x >> 5;
	const int64_t w = (int64_t) blockIdx.x * (SEG_THREADS / 32) + wib;
	if (w >= a.nwarps)
		return;
	const int64_t cb = w * a.nchunks / a.nwarps, ce = (w + 1) * a.nchunks / a.nwarps;
	if (cb >= ce)
		return;
	const int S = a.stages;
	uint8_t * wsm = smem + (size_t) wib * a.warp_bytes;
	uint64_t * bars = reinterpret_cast<uint64_t *>(wsm + (size_t) S * SEG_STAGE_BYTES);
	if (lane == 0) {
		for (int q = 0; q < S; q++)
			mbar_init(&bars[q], 1);
		mbar_fence_init();
	}
	__syncwarp();
	if (lane == 0)
		for (int q = 0; q < S && cb + q < ce; q++)
			seg_issue(a, cb + q, wsm + (size_t) q * SEG_STAGE_BYTES, &bars[q]);
	// x of the first chunk
	float xc[SEG_K], xn[SEG_K];
	{
		const bool ok = mbar_wait_bounded(&bars[0], 0u, kWaitBudgetCycles);
		if (!__all_sync(FULL, ok)) {
			if (lane == 0) {
				dev_flag_error(a.err, DEV_ERR_TIMEOUT);
				drain_ring(bars, S, 0, 0u, (int) (ce - cb < S ? ce - cb : S), kWaitBudgetCycles);
			}
			return;
		}
		const int4 * sc = reinterpret_cast<const int4 *>(wsm + SEG_CHUNK * 4) + 2 * lane;
		const int4 ca = sc[0], cbv = sc[1];
		const int32_t cc[SEG_K] = {ca.x, ca.y, ca.z, ca.w, cbv.x, cbv.y, cbv.z, cbv.w};
		#pragma unroll
		for (int k = 0; k < SEG_K; k++)
			xc[k] = __ldg(a.x + cc[k]);
	}
	int s = 0;                       // stage of the current chunk
	int ns = S > 1 ? 1 : 0;          // stage and phase of the next chunk
	uint32_t nparity = S > 1 ? 0u : 1u;
	for (int64_t ch = cb; ch < ce; ch++) {
		uint8_t * stage = wsm + (size_t) s * SEG_STAGE_BYTES;
		if (ch + 1 < ce) {
			// request x of the next chunk before summing this one
			const bool ok = mbar_wait_bounded(&bars[ns], nparity, kWaitBudgetCycles);
			if (!__all_sync(FULL, ok)) {
				if (lane == 0) {
					dev_flag_error(a.err, DEV_ERR_TIMEOUT);
					// copies in flight: chunks ch + 1 .. ch + S - 1 (the next one with S == 1)
					const int64_t span = S > 1 ? S - 1 : 1;
					drain_ring(bars, S, ns, nparity, (int) (ce - ch - 1 < span ? ce - ch - 1 : span), kWaitBudgetCycles);
				}
				return;
			}
			const int4 * sc = reinterpret_cast<const int4 *>(wsm + (size_t) ns * SEG_STAGE_BYTES + SEG_CHUNK * 4) + 2 * lane;
			const int4 ca = sc[0], cbv = sc[1];
			const int32_t cc[SEG_K] = {ca.x, ca.y, ca.z, ca.w, cbv.x, cbv.y, cbv.z, cbv.w};
			#pragma unroll
			for (int k = 0; k < SEG_K; k++)
				xn[k] = __ldg(a.x + cc[k]);
		}
		const float4 * sv = reinterpret_cast<const float4 *>(stage) + 2 * lane;
		const float4 va = sv[0], vb = sv[1];
		const float vv[SEG_K] = {va.x, va.y, va.z, va.w, vb.x, vb.y, vb.z, vb.w};
		__syncwarp();
		if (lane == 0 && ch + S < ce)
			seg_issue(a, ch + S, stage, &bars[s]);   // the stage's values and columns are read
		seg_chunk(a, ch, vv, xc);
		#pragma unroll
		for (int k = 0; k < SEG_K; k++)
			xc[k] = xn[k];
		s = ns;
		if (++ns == S) {
			ns = 0;
			nparity ^= 1u;
		}
	}
}

// Rows across chunk boundaries: their pieces in chunk order (tail of the first chunk, then
// the head partial of every later chunk the row reaches).
__global__ void f32seg_fixup_kernel(const int32_t * rp, const int32_t * rows, int64_t count, const float2 * head,
		const float2 * tail, float * y)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= count)
		return;
	const int64_t r = rows[i];
	const int64_t ca = (int64_t) rp[r] / SEG_CHUNK, cb = ((int64_t) rp[r + 1] - 1) / SEG_CHUNK;
	float s = tail[ca].x, c = tail[ca].y;
	for (int64_t k = ca + 1; k <= cb; k++)
		merge(s, c, head[k].x, head[k].y);
	y[r] = __fadd_rn(s, c);
}

__global__ void zero_rows_f32_kernel(const int32_t * rows, int64_t count, float * y)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < count)
		y[rows[i]] = 0.0f;
}

// First row of every chunk: the largest r with rp[r] <= chunk * SEG_CHUNK.
__global__ void seg_chunk_row_kernel(const int32_t * rp, int64_t m, int64_t nchunks, int32_t * out)
{
	const int64_t cidx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (cidx >= nchunks)
		return;
	const int64_t e0 = cidx * SEG_CHUNK;
	int64_t lo = 0, hi = m;           // rp[0] = 0 <= e0
	while (lo < hi) {
		const int64_t mid = (lo + hi + 1) >> 1;
		if ((int64_t) rp[mid] <= e0)
			lo = mid;
		else
			hi = mid - 1;
	}
	out[cidx] = (int32_t) lo;
}

// flags[r] for the row lists: 1 = the row crosses a chunk boundary (kind 0) / is empty (kind 1)
__global__ void seg_row_flags_kernel(const int32_t * rp, int64_t m, int kind, int64_t * flags)
{
	const int64_t r = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (r >= m)
		return;
	const int64_t a = rp[r], b = rp[r + 1];
	flags[r] = kind == 0 ? (b > a && a / SEG_CHUNK != (b - 1) / SEG_CHUNK) : (b == a);
}

__global__ void seg_row_scatter_kernel(const int64_t * flags, const int64_t * pos, int64_t m, int32_t * out)
{
	const int64_t r = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (r < m && flags[r])
		out[pos[r]] = (int32_t) r;
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

// ------------------------------------------------------------------ FP32 over 32-row slices
// The FP32 variant on SELL-C-sigma slices of 32 rows (format sell_c_s, C = 32): FP32 values
// column-major per slice as the FP64 layout, and the column indices packed per tile of 8
// slice columns x 32 rows: the tile's smallest column (base) and a fixed bit width, each
// entry's offset from the base in tiled row-major order (entry (r, k) of a full tile at
// position r * 8 + k - k8, as the tiled copy of kernels 8-10).  Padding entries pack 0.
// Warps claim work items as in kernel 10; per full tile lane L decodes its 8 tiled
// positions q * 32 + L (row 4q + L/8, column L % 8), loads x, and an 8 x 8 transpose
// between lanes leaves it its row's 8 x values; its row's Dot2 chain then runs over the
// row's own entries in column order (padding skipped), so y is the CSR row's sequential
// Dot2 bit for bit.  The next tile's packed words and values are loaded one tile ahead,
// the lines two tiles ahead prefetched into L1.
constexpr int F32S_THREADS = 256;

struct F32SArgs {
	const int2 * items;
	int64_t nitems;
	const int32_t * sptr;     // slice pointers (entries)
	const int32_t * tptr;     // first tile of each slice
	const int4 * thdr;        // per tile: {first word (low 32 bits), high bits, base, bit width}
	const uint32_t * words;   // packed offsets
	int64_t nwords;
	const float * vals;       // FP32 values, column-major per slice
	const int32_t * rlen;     // row length of every sliced row (0 past the last row)
	const int32_t * ymap;     // row_order
	const float * x;
	float * y;
	int64_t m;
	unsigned int * queue;
	unsigned int total_warps;
	int64_t heavy_min;
};

__device__ __forceinline__ void transpose8f(float (&X)[8], int lane)
{
	#pragma unroll
	for (int b = 1; b < 8; b <<= 1) {
		const bool up = (lane & b) != 0;
		#pragma unroll
		for (int q = 0; q < 8; q++) {
			if (q & b)
				continue;
			const float send = up ? X[q] : X[q | b];
			const float recv = __shfl_xor_sync(0xffffffffu, send, b);
			if (up)
				X[q] = recv;
			else
				X[q | b] = recv;
		}
	}
}

__device__ __forceinline__ uint32_t f32s_field(const uint32_t * w, int64_t off, uint32_t bit, int bits)
{
	const int64_t i = off + (bit >> 5);
	const uint32_t v = __funnelshift_r(__ldg(w + i), __ldg(w + i + 1), bit & 31);   // neighbouring lanes share words
	return bits >= 32 ? v : (v & ((1u << bits) - 1u));
}

// columns and values of full tile t0 (tile header hd) for lane L
__device__ __forceinline__ void f32s_tile_load(const F32SArgs & a, const int4 & hd, int64_t t0, int lane, int R,
		int32_t (&c)[8], float (&v)[8])
{
	const int64_t off = (int64_t) (uint32_t) hd.x | ((int64_t) hd.y << 32);
	#pragma unroll
	for (int q = 0; q < 8; q++)
		c[q] = hd.z + (int32_t) f32s_field(a.words, off, (uint32_t) (q * 32 + lane) * (uint32_t) hd.w, hd.w);
	#pragma unroll
	for (int j = 0; j < 8; j++)
		v[j] = __ldcs(a.vals + t0 + j * 32 + R);
}

__device__ __forceinline__ void f32s_slice(const F32SArgs & a, int64_t sl, int64_t e_end, int lane, int R, int dist)
{
	const int64_t b = a.sptr[sl];
	const int W = (int) (((int64_t) a.sptr[sl + 1] - b) >> 5);
	const int nt = W >> 3, rem = W & 7;
	const int64_t tp = a.tptr[sl];
	const int len = a.rlen[sl * 32 + R];
	float s = 0.0f, cc = 0.0f;
	int32_t c[8], cn[8];
	float v[8], vn[8];
	int4 hn = nt > 1 ? a.thdr[tp + 1] : make_int4(0, 0, 0, 0);
	if (nt > 0)
		f32s_tile_load(a, a.thdr[tp], b, lane, R, c, v);
	for (int t = 0; t < nt; t++) {
		const int64_t t0 = b + (int64_t) t * 256;
		// the values, header and (about) the packed words of the tile dist entries on into L1
		// (never past the item's entries or the packed words)
		if (t0 + dist + 256 <= e_end) {
			const int ahead = dist >> 8;
			if (lane < 8) {
				asm volatile("prefetch.global.L1 [%0];" ::"l"(a.vals + t0 + dist + lane * 32));
			} else if (lane == 8) {
				asm volatile("prefetch.global.L1 [%0];" ::"l"(a.thdr + tp + t + ahead));
			} else if (lane < 14 && hn.w > 0) {
				const int64_t w = ((int64_t) (uint32_t) hn.x | ((int64_t) hn.y << 32)) + (int64_t) (ahead - 1) * (8 * hn.w + 1) +
						(int64_t) (lane - 9) * 32;
				if (w < a.nwords)
					asm volatile("prefetch.global.L1 [%0];" ::"l"(a.words + w));
			}
		}
		int4 hnn = make_int4(0, 0, 0, 0);
		if (t + 1 < nt) {
			f32s_tile_load(a, hn, t0 + 256, lane, R, cn, vn);
			if (t + 2 < nt)
				hnn = a.thdr[tp + t + 2];
		}
		float X[8];
		#pragma unroll
		for (int q = 0; q < 8; q++)
			X[q] = __ldg(a.x + c[q]);
		transpose8f(X, lane);
		#pragma unroll
		for (int j = 0; j < 8; j++)
			if (t * 8 + j < len)
				dot2_step(v[j], X[j], s, cc);
		#pragma unroll
		for (int j = 0; j < 8; j++) {
			c[j] = cn[j];
			v[j] = vn[j];
		}
		hn = hnn;
	}
	if (rem > 0) {                               // the narrower last tile: rows at R * rem
		const int64_t t0 = b + (int64_t) nt * 256;
		const int4 hd = a.thdr[tp + nt];
		const int64_t off = (int64_t) (uint32_t) hd.x | ((int64_t) hd.y << 32);
		#pragma unroll
		for (int j = 0; j < 8; j++) {
			if (j < rem && nt * 8 + j < len) {
				const int32_t col = hd.z + (int32_t) f32s_field(a.words, off, (uint32_t) (R * rem + j) * (uint32_t) hd.w, hd.w);
				dot2_step(__ldcs(a.vals + t0 + j * 32 + R), __ldg(a.x + col), s, cc);
			}
		}
	}
	const int64_t row = sl * 32 + R;
	if (row < a.m)
		a.y[a.ymap[row]] = __fadd_rn(s, cc);
}

__global__ void __launch_bounds__(F32S_THREADS, 2) f32s_kernel(F32SArgs a)
{
	const int lane = threadIdx.x & 31;
	const int R = 4 * (lane & 7) + (lane >> 3);
	for (;;) {
		unsigned int it = 0;
		if (lane == 0)
			it = atomicAdd(&a.queue[0], 1u);
		it = __shfl_sync(0xffffffffu, it, 0);
		if ((int64_t) it >= a.nitems)
			break;
		const int2 r = a.items[it];
		const int64_t e_end = a.sptr[r.y];
		// a heavy slice (an item of its own) prefetches four times as far ahead
		const int dist = (r.y - r.x == 1 && e_end - a.sptr[r.x] >= a.heavy_min) ? 2048 : 512;
		for (int64_t sl = r.x; sl < r.y; sl++)
			f32s_slice(a, sl, e_end, lane, R, dist);
	}
	if (lane == 0 && atomicAdd(&a.queue[1], 1u) == a.total_warps - 1) {
		atomicExch(&a.queue[0], 0u);
		atomicExch(&a.queue[1], 0u);
	}
}

// ---- conversion kernels of the FP32 slices

// row length of every sliced row (rows past m: 0)
__global__ void f32s_rowlen_kernel(const int32_t * rp, const int32_t * order, int64_t m, int64_t nrows, int32_t * rlen)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nrows)
		return;
	rlen[i] = i < m ? rp[order[i] + 1] - rp[order[i]] : 0;
}

__global__ void f32s_tilecount_kernel(const int32_t * sptr, int64_t ns, int64_t * cnt)
{
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= ns)
		return;
	const int W = (int) (((int64_t) sptr[s + 1] - sptr[s]) >> 5);
	cnt[s] = (W + 7) >> 3;
}

// one warp per slice, lane = slice row: each tile's base, bit width and packed words
__global__ void f32s_tilebits_kernel(const int32_t * sptr, const int64_t * tptr, const int32_t * scols,
		const int32_t * rlen, int64_t ns, int4 * thdr, int64_t * nwords)
{
	const int64_t sl = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (sl >= ns)
		return;
	const int64_t b = sptr[sl];
	const int W = (int) (((int64_t) sptr[sl + 1] - b) >> 5);
	const int len = rlen[sl * 32 + lane];
	for (int k8 = 0, t = 0; k8 < W; k8 += 8, t++) {
		const int tw = W - k8 < 8 ? W - k8 : 8;
		int lo = INT32_MAX, hi = INT32_MIN;
		for (int j = 0; j < tw; j++)
			if (k8 + j < len) {
				const int32_t col = scols[b + (int64_t) (k8 + j) * 32 + lane];
				lo = min(lo, col);
				hi = max(hi, col);
			}
		#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
			hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
		}
		if (lane == 0) {
			int bits = 0;
			if (hi > lo) {
				const uint32_t span = (uint32_t) (hi - lo);
				bits = 32 - __clz(span);
			}
			thdr[tptr[sl] + t] = make_int4(0, 0, hi >= lo ? lo : 0, bits);
			nwords[tptr[sl] + t] = (int64_t) tw * bits + 1;   // 32 tw fields of `bits` bits, one spare word
		}
	}
}

__global__ void f32s_tileoff_kernel(const int64_t * off, int64_t ntiles, int4 * thdr)
{
	const int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= ntiles)
		return;
	thdr[t].x = (int) (uint32_t) (off[t] & 0xffffffffLL);
	thdr[t].y = (int) (off[t] >> 32);
}

// one warp per slice, lane = slice row: the offsets from the base packed (atomicOr, the
// words zeroed first)
__global__ void f32s_pack_kernel(const int32_t * sptr, const int64_t * tptr, const int32_t * scols, const int32_t * rlen,
		const int4 * thdr, int64_t ns, uint32_t * words)
{
	const int64_t sl = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (sl >= ns)
		return;
	const int64_t b = sptr[sl];
	const int W = (int) (((int64_t) sptr[sl + 1] - b) >> 5);
	const int len = rlen[sl * 32 + lane];
	for (int k8 = 0, t = 0; k8 < W; k8 += 8, t++) {
		const int tw = W - k8 < 8 ? W - k8 : 8;
		const int4 hd = thdr[tptr[sl] + t];
		const int bits = hd.w;
		if (bits == 0)
			continue;
		const int64_t off = (int64_t) (uint32_t) hd.x | ((int64_t) hd.y << 32);
		for (int j = 0; j < tw; j++) {
			const uint32_t val = k8 + j < len ? (uint32_t) (scols[b + (int64_t) (k8 + j) * 32 + lane] - hd.z) : 0u;
			const uint64_t bit = (uint64_t) (lane * tw + j) * (uint64_t) bits;
			const int64_t wi = off + (int64_t) (bit >> 5);
			const int sh = (int) (bit & 31);
			atomicOr(&words[wi], val << sh);
			if (sh + bits > 32)
				atomicOr(&words[wi + 1], (uint32_t) ((uint64_t) val >> (32 - sh)));
		}
	}
}

__global__ void f32s_i64_to_i32_kernel(const int64_t * in, int32_t * out, int64_t n)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		out[i] = (int32_t) in[i];
}

// row_assign 1: per staged block of whole rows, its rows ranked longest first (ties in row
// order); rassign[unit0 + rank] = local row, so the 32 threads of a row warp take rows of
// similar length and the warp's Dot2 loops run nearly as long as its threads' rows.  One CTA
// a block, the block's row lengths in shared memory.
__global__ void row_rank_kernel(const StagedBlock * blocks, const int32_t * rp, uint16_t * rassign)
{
	__shared__ int32_t len[1024];
	const StagedBlock d = blocks[blockIdx.x];
	if (d.units <= 0 || d.units > 1024)
		return;
	for (int i = threadIdx.x; i < d.units; i += blockDim.x)
		len[i] = rp[(int64_t) d.unit0 + i + 1] - rp[(int64_t) d.unit0 + i];
	__syncthreads();
	for (int i = threadIdx.x; i < d.units; i += blockDim.x) {
		const int li = len[i];
		int rank = 0;
		for (int j = 0; j < d.units; j++)
			rank += (len[j] > li) || (len[j] == li && j < i);
		rassign[(int64_t) d.unit0 + rank] = (uint16_t) i;
	}
}

__global__ void f64_to_f32_copy_kernel(const double * in, float * out, int64_t n)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		out[i] = __double2float_rn(in[i]);
}

}  // namespace

const void * ws_f32_kernel_fn(bool packed)
{
	return packed ? (const void *) ws_f32_kernel<true> : (const void *) ws_f32_kernel<false>;
}

int f32ws_stage_bytes(int cap_al)
{
	return (int) (ceil_div((int64_t) cap_al * 8, 128) * 128);
}

// Rounds the stored FP64 values to FP32 and builds the kernel's tables: by default (kernel
// -1 or 4) the warp-specialised kernel's chunk-run table in per-CTA group order; kernel 7
// the segmented kernel's chunk rows and cross-chunk / empty row lists; kernel 0 the CTA
// staged kernel (blocks of up to 2048 entries, 8 bytes staged each).
int convert_f32(Handle & h)
{
	cudaStream_t s = h.stream;
	SPMV_TRY(h.alloc(&h.d_vf, h.nnz + SPMV_ENTRY_PAD));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_vf, 0, (h.nnz + SPMV_ENTRY_PAD) * sizeof(float), s));
	if (h.nnz > 0) {
		f64_to_f32_kernel<<<(unsigned) ceil_div(h.nnz, 256), 256, 0, s>>>(h.d_v, h.d_vf, h.nnz);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	if (h.desc.kernel == 7) {
		h.exec_kernel = 7;
		h.num_seg_chunks = ceil_div(h.nnz, SEG_CHUNK);
		const int64_t nch = h.num_seg_chunks, m = h.m;
		SPMV_TRY(h.alloc(&h.d_chunk_row, nch > 0 ? nch : 1));
		SPMV_TRY(h.alloc(&h.d_chunk_head, nch > 0 ? nch : 1));
		SPMV_TRY(h.alloc(&h.d_chunk_tail, nch > 0 ? nch : 1));
		if (nch > 0) {
			seg_chunk_row_kernel<<<(unsigned) ceil_div(nch, 256), 256, 0, s>>>(h.d_rp, m, nch, h.d_chunk_row);
			SPMV_CUDA_TRY(cudaGetLastError());
		}
		DevBuf flags, pos;
		SPMV_TRY(flags.alloc((m + 1) * sizeof(int64_t), s));
		SPMV_TRY(pos.alloc((m + 1) * sizeof(int64_t), s));
		for (int kind = 0; kind < 2; kind++) {
			int64_t cnt = 0;
			if (m > 0) {
				seg_row_flags_kernel<<<(unsigned) ceil_div(m, 256), 256, 0, s>>>(h.d_rp, m, kind, flags.as<int64_t>());
				SPMV_CUDA_TRY(cudaGetLastError());
				SPMV_TRY(scan_exclusive(flags.as<int64_t>(), pos.as<int64_t>(), m, s));
				SPMV_CUDA_TRY(cudaMemcpyAsync(&cnt, pos.as<int64_t>() + m, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
				SPMV_CUDA_TRY(cudaStreamSynchronize(s));
			}
			int32_t ** dst = kind == 0 ? &h.d_cross_rows : &h.d_empty_rows;
			SPMV_TRY(h.alloc(dst, cnt > 0 ? cnt : 1));
			if (cnt > 0) {
				seg_row_scatter_kernel<<<(unsigned) ceil_div(m, 256), 256, 0, s>>>(flags.as<int64_t>(), pos.as<int64_t>(),
						m, *dst);
				SPMV_CUDA_TRY(cudaGetLastError());
			}
			(kind == 0 ? h.num_cross_rows : h.num_empty_rows) = cnt;
		}
		h.kernels_per_run = (nch > 0 ? 1 : 0) + (h.num_cross_rows > 0 ? 1 : 0) + (h.num_empty_rows > 0 ? 1 : 0);
		// geometry: a ring of `stages` 2 KB chunk stages per warp, 4 warps per CTA
		h.stages = h.desc.stages > 0 ? h.desc.stages : 6;
		if (h.stages < 2)
			h.stages = 2;                             // the next chunk's columns are read while this one is summed
		const int warp_bytes = (int) (ceil_div((int64_t) h.stages * SEG_STAGE_BYTES + 8 * h.stages, 128) * 128);
		h.smem_bytes = (size_t) warp_bytes * (SEG_THREADS / 32);
		if (h.smem_bytes > 220 * 1024) {
			set_error(SPMV_ERR_ARG, "segmented FP32 kernel: %d stages exceed shared memory", h.stages);
			return SPMV_ERR_ARG;
		}
		SPMV_CUDA_TRY(cudaFuncSetAttribute(f32seg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) h.smem_bytes));
		int per_sm = h.desc.ctas_per_sm;
		if (per_sm <= 0) {
			SPMV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f32seg_kernel, SEG_THREADS, h.smem_bytes));
			if (per_sm < 1)
				per_sm = 1;
		}
		int64_t g = (int64_t) h.num_sms * per_sm;
		const int64_t need = ceil_div(nch, SEG_THREADS / 32);
		h.grid = (int) (g < need ? g : (need > 0 ? need : 1));
		return SPMV_OK;
	}
	if (h.desc.kernel < 0 || h.desc.kernel == 4) {
		spmv_format_desc saved = h.desc;
		h.desc.kernel = 4;
		// FP32 stages are 8 bytes an entry: 1536-entry blocks and 5 gather warps (0.164 ms on the
		// 4M-row matrix; 768-entry blocks 0.186 ms)
		if (h.desc.block_nnz == 0)
			h.desc.block_nnz = 1536;
		if (h.desc.threads == 0)
			h.desc.threads = 224;
		const int st = build_exec(h, h.d_rp, h.m, 1);     // geometry of ws_f32_kernel (values F32)
		h.desc = saved;
		if (st != SPMV_OK)
			return st;
		if (h.desc.pack_cols == 1)
			SPMV_TRY(build_packed_cols(h));
		if (h.desc.row_assign == 1 && h.num_blocks > 0) {
			if (h.row_threads > 1024) {
				set_error(SPMV_ERR_ARG, "row_assign 1 takes at most 1024 row threads (got %d)", h.row_threads);
				return SPMV_ERR_ARG;
			}
			SPMV_TRY(h.alloc(&h.d_rassign, h.m > 0 ? h.m : 1));
			row_rank_kernel<<<(unsigned) h.num_blocks, 128, 0, s>>>(h.d_blocks, h.d_rp, h.d_rassign);
			SPMV_CUDA_TRY(cudaGetLastError());
		}
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

// FP32 variant on SELL-C-sigma slices of 32 rows: after convert_sellcs has built the FP64
// slices (row_order, slice pointers, column-major columns and values), the FP32 values,
// the row lengths, the packed tiles and kernel 10's work items.
int build_sliced_f32(Handle & h)
{
	cudaStream_t s = h.stream;
	const int64_t ns = h.nslices, total = h.sellcs_size, nrows = ns * 32;
	h.exec_kernel = 10;
	SPMV_TRY(h.alloc(&h.d_svals_f, total + 8));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_svals_f, 0, (total + 8) * sizeof(float), s));
	if (total > 0) {
		f64_to_f32_copy_kernel<<<(unsigned) ceil_div(total, 256), 256, 0, s>>>(h.d_svals, h.d_svals_f, total);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	SPMV_TRY(h.alloc(&h.d_srlen, nrows > 0 ? nrows : 1));
	SPMV_TRY(h.alloc(&h.d_stptr, ns + 1));
	if (ns > 0) {
		f32s_rowlen_kernel<<<(unsigned) ceil_div(nrows, 256), 256, 0, s>>>(h.d_rp, h.d_order, h.m, nrows, h.d_srlen);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	DevBuf cnt, tptr64;
	SPMV_TRY(cnt.alloc((ns + 1) * sizeof(int64_t), s));
	SPMV_TRY(tptr64.alloc((ns + 1) * sizeof(int64_t), s));
	if (ns > 0) {
		f32s_tilecount_kernel<<<(unsigned) ceil_div(ns, 256), 256, 0, s>>>(h.d_sptr32, ns, cnt.as<int64_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	SPMV_TRY(scan_exclusive(cnt.as<int64_t>(), tptr64.as<int64_t>(), ns, s));
	int64_t ntiles = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&ntiles, tptr64.as<int64_t>() + ns, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	if (ntiles > INT32_MAX) {
		set_error(SPMV_ERR_OVERFLOW, "FP32 slices: %lld tiles, beyond the 32-bit range", (long long) ntiles);
		return SPMV_ERR_OVERFLOW;
	}
	f32s_i64_to_i32_kernel<<<(unsigned) ceil_div(ns + 1, 256), 256, 0, s>>>(tptr64.as<int64_t>(), h.d_stptr, ns + 1);
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(h.alloc(&h.d_sthdr, ntiles + 2));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_sthdr, 0, (ntiles + 2) * sizeof(int4), s));
	DevBuf nw, woff;
	SPMV_TRY(nw.alloc((ntiles + 1) * sizeof(int64_t), s));
	SPMV_TRY(woff.alloc((ntiles + 1) * sizeof(int64_t), s));
	if (ns > 0) {
		f32s_tilebits_kernel<<<(unsigned) ceil_div(nrows, 256), 256, 0, s>>>(h.d_sptr32, tptr64.as<int64_t>(), h.d_scols,
				h.d_srlen, ns, h.d_sthdr, nw.as<int64_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	SPMV_TRY(scan_exclusive(nw.as<int64_t>(), woff.as<int64_t>(), ntiles, s));
	int64_t nwords = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&nwords, woff.as<int64_t>() + ntiles, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	if (ntiles > 0) {
		f32s_tileoff_kernel<<<(unsigned) ceil_div(ntiles, 256), 256, 0, s>>>(woff.as<int64_t>(), ntiles, h.d_sthdr);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	h.swords = nwords;
	SPMV_TRY(h.alloc(&h.d_swords, nwords + 2));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_swords, 0, (nwords + 2) * sizeof(uint32_t), s));
	if (ns > 0) {
		f32s_pack_kernel<<<(unsigned) ceil_div(nrows, 256), 256, 0, s>>>(h.d_sptr32, tptr64.as<int64_t>(), h.d_scols,
				h.d_srlen, h.d_sthdr, ns, h.d_swords);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	SPMV_TRY(build_tile_reg(h, h.d_sptr32, ns, 32));
	int per_sm = h.desc.ctas_per_sm;
	if (per_sm <= 0) {
		SPMV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f32s_kernel, F32S_THREADS, 0));
		if (per_sm < 1)
			per_sm = 1;
	}
	h.grid = h.num_sms * per_sm;
	h.threads = F32S_THREADS;
	h.kernels_per_run = h.num_items > 0 ? 1 : 0;
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	return SPMV_OK;
}

static int launch_sliced_f32(Handle & h, const float * d_x, float * d_y, cudaStream_t s)
{
	if (h.num_items == 0)
		return SPMV_OK;
	F32SArgs a{};
	a.items = h.d_items;
	a.nitems = h.num_items;
	a.sptr = h.d_sptr32;
	a.tptr = h.d_stptr;
	a.thdr = h.d_sthdr;
	a.words = h.d_swords;
	a.nwords = h.swords;
	a.vals = h.d_svals_f;
	a.rlen = h.d_srlen;
	a.ymap = h.d_order;
	a.x = d_x;
	a.y = d_y;
	a.m = h.m;
	a.queue = h.d_queue;
	a.total_warps = (unsigned int) h.grid * (F32S_THREADS / 32);
	a.heavy_min = h.tile_heavy_min;
	f32s_kernel<<<h.grid, F32S_THREADS, 0, s>>>(a);
	SPMV_CUDA_TRY(cudaGetLastError());
	return SPMV_OK;
}

int launch_spmv_f32(Handle & h, const float * d_x, float * d_y, cudaStream_t s)
{
	if (h.desc.format == SPMV_FMT_SELL_C_S)
		return launch_sliced_f32(h, d_x, d_y, s);
	if (h.exec_kernel == 7) {
		if (h.num_empty_rows > 0) {
			zero_rows_f32_kernel<<<(unsigned) ceil_div(h.num_empty_rows, 256), 256, 0, s>>>(h.d_empty_rows,
					h.num_empty_rows, d_y);
			SPMV_CUDA_TRY(cudaGetLastError());
		}
		if (h.num_seg_chunks > 0) {
			SegArgs g{};
			g.rp = h.d_rp;
			g.ci = h.d_ci;
			g.v = h.d_vf;
			g.x = d_x;
			g.y = d_y;
			g.chunk_row = h.d_chunk_row;
			g.nchunks = h.num_seg_chunks;
			g.nwarps = (int64_t) h.grid * (SEG_THREADS / 32);
			g.m = h.m;
			g.nnz = h.nnz;
			g.head = h.d_chunk_head;
			g.tail = h.d_chunk_tail;
			g.stages = h.stages;
			g.warp_bytes = (int) (h.smem_bytes / (SEG_THREADS / 32));
			g.err = h.d_err;
			f32seg_kernel<<<h.grid, SEG_THREADS, h.smem_bytes, s>>>(g);
			SPMV_CUDA_TRY(cudaGetLastError());
		}
		if (h.num_cross_rows > 0) {
			f32seg_fixup_kernel<<<(unsigned) ceil_div(h.num_cross_rows, 256), 256, 0, s>>>(h.d_rp, h.d_cross_rows,
					h.num_cross_rows, h.d_chunk_head, h.d_chunk_tail, d_y);
			SPMV_CUDA_TRY(cudaGetLastError());
		}
		return SPMV_OK;
	}
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
		w.stage_bytes = f32ws_stage_bytes(w.cap_al);
		w.row_threads = h.row_threads;
		w.err = h.d_err;
		w.wait_budget = wait_budget_cycles(h.desc.wait_limit_us);
		w.hold = (h.desc.debug_flags & SPMV_DEBUG_WITHHOLD_HANDOFF) != 0;
		w.pinfo = h.d_pinfo;
		w.pcols = h.d_pcols;
		w.rassign = h.d_rassign;
		if (h.d_pcols)
			ws_f32_kernel<true><<<h.grid, h.threads, h.smem_bytes, s>>>(w);
		else
			ws_f32_kernel<false><<<h.grid, h.threads, h.smem_bytes, s>>>(w);
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
// device current) by the first call on it.  Host threads that race on the first call
// resolve the same address and store it atomically.  The cache does not survive
// cudaDeviceReset(): the module is then loaded again and the array may move.
static std::atomic<float *> g_mixed_scratch_addr[64];

static int mixed_scratch(int dev, float ** out)
{
	if (dev < 0 || dev >= 64) {
		set_error(SPMV_ERR_ARG, "no-alloc entry: device ordinal %d out of range", dev);
		return SPMV_ERR_ARG;
	}
	float * p = g_mixed_scratch_addr[dev].load(std::memory_order_acquire);
	if (!p) {
		void * ptr = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&ptr, g_mixed_scratch);
		if (e != cudaSuccess) {
			set_error(SPMV_ERR_CUDA, "no-alloc entry: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
			return SPMV_ERR_CUDA;
		}
		p = static_cast<float *>(ptr);
		g_mixed_scratch_addr[dev].store(p, std::memory_order_release);
	}
	*out = p;
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
	int dev = -1;
	SPMV_CUDA_TRY(cudaGetDevice(&dev));
	if (dev != h.device) {
		// the array is per device: another GPU's copy would be read through peer access or fault
		set_error(SPMV_ERR_ARG, "no-alloc entry: the handle lives on device %d but device %d is current", h.device, dev);
		return SPMV_ERR_ARG;
	}
	float * scratch = nullptr;
	SPMV_TRY(mixed_scratch(dev, &scratch));
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
