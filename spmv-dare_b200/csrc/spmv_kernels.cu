// SpMV kernels for B200 (sm_100a).
//
// staged_kernel  -- CSR (csr_naive, csr_vec) and narrow SELL slices (sell, sell_sorted with
//                   V < 32).  Persistent CTAs walk a table of row blocks; each block's
//                   stored entries are one contiguous range, brought into shared memory by
//                   the bulk-copy engine (cp.async.bulk, mbarrier completion) while the CTA
//                   computes the previous block.  Every output row is then summed by ONE
//                   thread in the reference format's own operation order, so y is
//                   bit-identical to the reference:
//                     csr_naive  : sum = sum + a*x, product and sum rounded separately
//                                  (subkernel_csr_scalar, src/spmv_kernels/csr.cpp:167-182,
//                                  as the reference's x86 build evaluates it);
//                     csr_vec    : L lanes of fused a*x+s, (s0+s2)+(s1+s3), split tail
//                                  (subkernel_row_csr_vec, csr_vec.cpp:183-211);
//                     sell(_sorted): one fused a*x+s per slice column, padding included
//                                  (compute_sell, sell.cpp:240-280, sell_sorted.cpp:346-427).
// sliced_kernel  -- slices of >= 32 rows (SELL-C-sigma; SELL with V >= 32): one thread per
//                   row, a warp reads 32 consecutive column-major entries per step
//                   (coalesced), fused multiply-add over the slice width as vfmacc does
//                   (sellcs_mv_d, sell-C-s/sellcs_mv_kernels_epi.c:209-317).
#include <algorithm>

#include "internal.h"
#include "primitives.cuh"

namespace spmv {

namespace {

constexpr int STAGED_MAX_THREADS = 512;

struct StagedArgs {
	const StagedBlock * blocks;
	int64_t nblocks;
	const int32_t * ptr;     // CSR: row_ptr; SLICED: row_cluster_ptr
	const int32_t * cols;
	const double * vals;
	const int32_t * ymap;    // sell_sorted: rev_permutation
	const double * x;
	double * y;
	int64_t m;
	int V;                   // slice height (SLICED)
	int cap_al;              // staged entries per stage buffer (capacity + alignment slack)
	int stages;
	int stage_bytes;
	int exact;
	int row_threads;         // warp-specialised kernel: threads of the row warps
	int cols_off;            // warp-specialised kernel: byte offset of the staged columns in a stage
	const int64_t * ranges;  // warp-specialised kernel: each CTA's contiguous block range
	int * err;
	long long wait_budget;   // bound of the warp-specialised kernel's waits, clock cycles
	int hold;                // SPMV_DEBUG_WITHHOLD_HANDOFF: gather warps never hand a stage over
	const int4 * pinfo;      // packed columns (csr_naive): per block {16-byte offset, base, bits, bytes}
	const uint32_t * pcols;  // packed columns: the block streams (pack.cu)
};

// Column of entry e of a packed block stream (pack.cu): two whole words and a funnel shift.
__device__ __forceinline__ int32_t packed_col64(const uint32_t * words, int e, int bits, int32_t base)
{
	const uint32_t bit = (uint32_t) e * (uint32_t) bits;
	const uint32_t w = bit >> 5;
	const uint32_t v = __funnelshift_r(words[w], words[w + 1], bit & 31);
	return base + (int32_t) (bits >= 32 ? v : (v & ((1u << bits) - 1u)));
}

// Sequential sum of s[0..n) in index order.
__device__ __forceinline__ double seq_add(const double * s, int n, double sum)
{
	#pragma unroll 4
	for (int j = 0; j < n; j++)
		sum = __dadd_rn(sum, s[j]);
	return sum;
}

// Sequential fused chain sum = fma(v[j * vs], x[j * xs], sum), j = 0..n-1.
__device__ __forceinline__ double seq_fma(const double * v, int vs, const double * x, int xs, int n, double sum)
{
	#pragma unroll 4
	for (int j = 0; j < n; j++)
		sum = __fma_rn(v[j * vs], x[j * xs], sum);
	return sum;
}

template <int L>
__device__ __forceinline__ double lanes_reduce(const double * s)
{
	if (L == 1)
		return s[0];
	if (L == 2)
		return s[0] + s[1];
	if (L == 4)
		return (s[0] + s[2]) + (s[1] + s[3]);
	double tot = 0;
	#pragma unroll
	for (int h = 0; h < L; h += 4)
		tot = tot + ((s[h] + s[h + 2]) + (s[h + 1] + s[h + 3]));
	return tot;
}

// Sum of one CSR row whose entries are vals[js..je), cols[js..je) (shared or global).
template <Arith A, int L>
__device__ __forceinline__ double csr_row(const double * __restrict__ vals, const int32_t * __restrict__ cols, int64_t js,
		int64_t je, const double * __restrict__ x)
{
	if (A == Arith::LANES_FMA) {
		double s[L];
		#pragma unroll
		for (int l = 0; l < L; l++)
			s[l] = 0.0;
		int64_t jv = js + ((je - js) & ~(int64_t) (L - 1));
		for (int64_t j = js; j < jv; j += L) {
			#pragma unroll
			for (int l = 0; l < L; l++)
				s[l] = __fma_rn(vals[j + l], ldg(x + cols[j + l]), s[l]);
		}
		double sum = lanes_reduce<L>(s);
		for (int64_t j = jv; j < je; j++)
			sum = __dadd_rn(sum, __dmul_rn(vals[j], ldg(x + cols[j])));
		return sum;
	} else if (A == Arith::SEQ_FMA) {
		double sum = 0.0;
		#pragma unroll 4
		for (int64_t j = js; j < je; j++)
			sum = __fma_rn(vals[j], ldg(x + cols[j]), sum);
		return sum;
	} else {
		double sum = 0.0;
		#pragma unroll 4
		for (int64_t j = js; j < je; j++)
			sum = __dadd_rn(sum, __dmul_rn(vals[j], ldg(x + cols[j])));
		return sum;
	}
}

__device__ __forceinline__ void staged_issue_d(const StagedArgs & a, const StagedBlock & d, int s, uint8_t * smem,
		uint64_t * bars)
{
	if (d.units < 0 || d.elems == 0) {
		mbar_arrive(&bars[s]);
		return;
	}
	int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
	int64_t e1 = ((int64_t) d.elem0 + d.elems + 3) & ~(int64_t) 3;
	uint32_t cnt = (uint32_t) (e1 - e0);
	double * sv = reinterpret_cast<double *>(smem + (size_t) s * a.stage_bytes);
	int32_t * sc = reinterpret_cast<int32_t *>(smem + (size_t) s * a.stage_bytes + (size_t) a.cap_al * 8);
	fence_proxy_async_smem();
	mbar_arrive_expect_tx(&bars[s], cnt * 12u);
	bulk_g2s(sv, a.vals + e0, cnt * 8u, &bars[s]);
	bulk_g2s(sc, a.cols + e0, cnt * 4u, &bars[s]);
}

__device__ __forceinline__ void staged_issue(const StagedArgs & a, int64_t b, int s, uint8_t * smem, uint64_t * bars)
{
	const StagedBlock d = a.blocks[b];
	staged_issue_d(a, d, s, smem, bars);
}

// Deterministic CTA sum (fixed tree order).
__device__ __forceinline__ double cta_sum(double v, double * red)
{
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		v += __shfl_down_sync(0xffffffffu, v, o);
	if (lane == 0)
		red[w] = v;
	__syncthreads();
	double t = 0;
	if (threadIdx.x == 0) {
		for (int i = 0; i < (int) (blockDim.x >> 5); i++)
			t += red[i];
	}
	__syncthreads();
	return t;
}

// Long unit (a row / slice larger than one staged block) streamed through the gather
// buffer in chunks; every row is still summed by one thread in the reference order.
template <Kind K, Arith A, int L, bool YMAP>
__device__ __forceinline__ void staged_long_unit(const StagedArgs & a, const StagedBlock & d, double * xb)
{
	const int half = a.cap_al / 2;            // entries per chunk: values in xb[0,half), x in xb[half, 2 half)
	double * cv = xb;
	double * cx = xb + half;
	if (K == Kind::CSR && !a.exact) {
		// tolerance mode: every thread a strided partial, then a fixed-order CTA sum
		const int64_t r = d.unit0;
		double part = 0.0;
		for (int64_t j = a.ptr[r] + threadIdx.x; j < a.ptr[r + 1]; j += blockDim.x)
			part = __fma_rn(a.vals[j], ldg(a.x + a.cols[j]), part);
		double t = cta_sum(part, cv);
		if (threadIdx.x == 0)
			a.y[r] = t;
		return;
	}
	if (K == Kind::CSR) {
		const int64_t r = d.unit0;
		const int64_t js = a.ptr[r], je = a.ptr[r + 1];
		const int64_t jv = js + ((je - js) & ~(int64_t) (L - 1));
		double sum = 0.0;
		double lane[L];
		#pragma unroll
		for (int l = 0; l < L; l++)
			lane[l] = 0.0;
		for (int64_t c0 = js; c0 < je; c0 += half) {
			const int cnt = (int) ((je - c0) < half ? (je - c0) : half);
			for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
				const double v = a.vals[c0 + e];
				const double xv = ldg(a.x + a.cols[c0 + e]);
				cv[e] = v;
				cx[e] = xv;
			}
			__syncthreads();
			if (threadIdx.x == 0) {
				for (int e = 0; e < cnt; e++) {
					const int64_t j = c0 + e;
					if (A == Arith::LANES_FMA) {
						if (j < jv) {
							const int l = (int) ((j - js) & (L - 1));
							#pragma unroll
							for (int q = 0; q < L; q++)
								if (q == l)
									lane[q] = __fma_rn(cv[e], cx[e], lane[q]);
						} else {
							if (j == jv)
								sum = lanes_reduce<L>(lane);
							sum = __dadd_rn(sum, __dmul_rn(cv[e], cx[e]));
						}
					} else if (A == Arith::SEQ_FMA) {
						sum = __fma_rn(cv[e], cx[e], sum);
					} else {
						sum = __dadd_rn(sum, __dmul_rn(cv[e], cx[e]));
					}
				}
			}
			__syncthreads();
		}
		if (threadIdx.x == 0) {
			if (A == Arith::LANES_FMA && jv == je)
				sum = lanes_reduce<L>(lane);
			a.y[r] = sum;
		}
	} else {
		const int V = a.V;
		const int64_t sl = d.unit0;
		const int64_t p0 = a.ptr[sl];
		const int w = (a.ptr[sl + 1] - a.ptr[sl]) / V;
		const int kc = half / V > 0 ? half / V : 1;     // slice columns per chunk
		double acc = 0.0;
		for (int k0 = 0; k0 < w; k0 += kc) {
			const int kn = (w - k0) < kc ? (w - k0) : kc;
			const int cnt = kn * V;
			const int64_t base = p0 + (int64_t) k0 * V;
			for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
				cv[e] = a.vals[base + e];
				cx[e] = ldg(a.x + a.cols[base + e]);
			}
			__syncthreads();
			if (threadIdx.x < V)
				for (int k = 0; k < kn; k++)
					acc = __fma_rn(cv[k * V + threadIdx.x], cx[k * V + threadIdx.x], acc);
			__syncthreads();
		}
		if (threadIdx.x < V) {
			const int64_t row = sl * V + threadIdx.x;
			if (row < a.m)
				a.y[(YMAP && a.ymap) ? a.ymap[row] : row] = acc;
		}
	}
}

// Rows of one staged block whose gather is complete: one thread per row (CSR) or per
// slice row (SLICED), in the reference order, operands in shared memory (`sv` values or
// products, `xb` gathered x).  js0 / je0: bounds of this thread's first row relative to
// the stage start, loaded ahead by the caller.
template <Kind K, Arith A, int L, bool YMAP>
__device__ __forceinline__ void block_rows(const StagedArgs & a, const StagedBlock & d, const double * sv,
		const double * xb, int js0, int je0)
{
	const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
	if (K == Kind::CSR) {
		for (int u = threadIdx.x; u < d.units; u += blockDim.x) {
			const int64_t r = (int64_t) d.unit0 + u;
			const int js = (u == (int) threadIdx.x) ? js0 : (int) ((int64_t) a.ptr[r] - e0);
			const int je = (u == (int) threadIdx.x) ? je0 : (int) ((int64_t) a.ptr[r + 1] - e0);
			double sum = 0.0;
			if (A == Arith::SEQ_SPLIT) {
				sum = seq_add(sv + js, je - js, sum);
			} else if (A == Arith::SEQ_FMA) {
				sum = seq_fma(sv + js, 1, xb + js, 1, je - js, sum);
			} else {
				double ln[L];
				#pragma unroll
				for (int l = 0; l < L; l++)
					ln[l] = 0.0;
				const int jv = js + ((je - js) & ~(L - 1));
				for (int j = js; j < jv; j += L) {
					#pragma unroll
					for (int l = 0; l < L; l++)
						ln[l] = __fma_rn(sv[j + l], xb[j + l], ln[l]);
				}
				sum = lanes_reduce<L>(ln);
				for (int j = jv; j < je; j++)
					sum = __dadd_rn(sum, __dmul_rn(sv[j], xb[j]));
			}
			a.y[r] = sum;
		}
	} else {
		const int V = a.V;
		const int nrow = d.units * V;
		for (int u = threadIdx.x; u < nrow; u += blockDim.x) {
			const int64_t sl = (int64_t) d.unit0 + u / V;
			const int lane = u % V;
			const int64_t row = sl * V + lane;
			if (row >= a.m)
				continue;
			const int ks = (int) ((int64_t) a.ptr[sl] - e0) + lane;
			const int w = (a.ptr[sl + 1] - a.ptr[sl]) / V;
			double acc = 0.0;
			acc = seq_fma(sv + ks, V, xb + ks, V, w, acc);
			a.y[(YMAP && a.ymap) ? a.ymap[row] : row] = acc;
		}
	}
}

// Rows of one staged block, each row thread loading its own x entries (8 independent loads
// in flight) straight from the staged columns: no CTA-wide gather phase and no barrier
// between gather and rows.  Same per-row operation order as block_rows.
template <Kind K, Arith A, int L, bool YMAP>
__device__ __forceinline__ void own_rows(const StagedArgs & a, const StagedBlock & d, const double * sv, const int32_t * sc,
		int js0, int je0)
{
	const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
	const double * __restrict__ x = a.x;
	if (K == Kind::CSR) {
		for (int u = threadIdx.x; u < d.units; u += blockDim.x) {
			const int64_t r = (int64_t) d.unit0 + u;
			const int js = (u == (int) threadIdx.x) ? js0 : (int) ((int64_t) a.ptr[r] - e0);
			const int je = (u == (int) threadIdx.x) ? je0 : (int) ((int64_t) a.ptr[r + 1] - e0);
			double sum = 0.0;
			if (A == Arith::SEQ_SPLIT) {
				#pragma unroll 8
				for (int j = js; j < je; j++)
					sum = __dadd_rn(sum, __dmul_rn(sv[j], ldg(x + sc[j])));
			} else if (A == Arith::SEQ_FMA) {
				#pragma unroll 8
				for (int j = js; j < je; j++)
					sum = __fma_rn(sv[j], ldg(x + sc[j]), sum);
			} else {
				double ln[L];
				#pragma unroll
				for (int l = 0; l < L; l++)
					ln[l] = 0.0;
				const int jv = js + ((je - js) & ~(L - 1));
				#pragma unroll 2
				for (int j = js; j < jv; j += L) {
					#pragma unroll
					for (int l = 0; l < L; l++)
						ln[l] = __fma_rn(sv[j + l], ldg(x + sc[j + l]), ln[l]);
				}
				sum = lanes_reduce<L>(ln);
				for (int j = jv; j < je; j++)
					sum = __dadd_rn(sum, __dmul_rn(sv[j], ldg(x + sc[j])));
			}
			a.y[r] = sum;
		}
	} else {
		const int V = a.V;
		const int nrow = d.units * V;
		for (int u = threadIdx.x; u < nrow; u += blockDim.x) {
			const int64_t sl = (int64_t) d.unit0 + u / V;
			const int lane = u % V;
			const int64_t row = sl * V + lane;
			if (row >= a.m)
				continue;
			const int ks = (int) ((int64_t) a.ptr[sl] - e0) + lane;
			const int w = (a.ptr[sl + 1] - a.ptr[sl]) / V;
			double acc = 0.0;
			#pragma unroll 8
			for (int k = 0; k < w; k++)
				acc = __fma_rn(sv[ks + k * V], ldg(x + sc[ks + k * V]), acc);
			a.y[(YMAP && a.ymap) ? a.ymap[row] : row] = acc;
		}
	}
}

// One staged block (or one long unit) of a staged kernel: gather, then rows in the
// reference order.  `smem_stage` is the block's stage buffer, `xb` the gather buffer.
template <Kind K, Arith A, int L, bool YMAP, bool OWNX = false>
__device__ __forceinline__ void staged_block(const StagedArgs & a, const StagedBlock & d, uint8_t * smem_stage, double * xb)
{
	if (OWNX && d.units >= 0) {
		const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
		int js0 = 0, je0 = 0;
		if (K == Kind::CSR && (int) threadIdx.x < d.units) {
			const int64_t r = (int64_t) d.unit0 + threadIdx.x;
			js0 = (int) ((int64_t) __ldg(a.ptr + r) - e0);
			je0 = (int) ((int64_t) __ldg(a.ptr + r + 1) - e0);
		}
		own_rows<K, A, L, YMAP>(a, d, reinterpret_cast<const double *>(smem_stage),
				reinterpret_cast<const int32_t *>(smem_stage + (size_t) a.cap_al * 8), js0, je0);
	} else if (d.units >= 0) {
		const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
		const int off = (int) (d.elem0 - e0);
		const int cnt = d.elems;
		double * sv = reinterpret_cast<double *>(smem_stage);
		const int32_t * sc = reinterpret_cast<const int32_t *>(smem_stage + (size_t) a.cap_al * 8);
		// row bounds of this thread's first row, loaded before the gather so their
		// latency overlaps it
		int js0 = 0, je0 = 0;
		if (K == Kind::CSR && (int) threadIdx.x < d.units) {
			const int64_t r = (int64_t) d.unit0 + threadIdx.x;
			js0 = (int) ((int64_t) __ldg(a.ptr + r) - e0);
			je0 = (int) ((int64_t) __ldg(a.ptr + r + 1) - e0);
		}
		// 1) gather x for every staged entry, all threads, many loads in flight
		#pragma unroll 4
		for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
			const double xv = ldg(a.x + sc[off + e]);
			if (A == Arith::SEQ_SPLIT)
				sv[off + e] = __dmul_rn(sv[off + e], xv);   // the reference's rounded product
			else
				xb[off + e] = xv;
		}
		__syncthreads();
		// 2) one thread per row, reference order, operands in shared memory
		block_rows<K, A, L, YMAP>(a, d, sv, xb, js0, je0);
	} else {
		staged_long_unit<K, A, L, YMAP>(a, d, xb);
	}
}

template <Kind K, Arith A, int L, bool YMAP, bool OWNX = false>
__global__ void __launch_bounds__(STAGED_MAX_THREADS) staged_kernel(StagedArgs a)
{
	extern __shared__ __align__(128) uint8_t smem[];
	double * xb = reinterpret_cast<double *>(smem + (size_t) a.stages * a.stage_bytes);
	uint64_t * bars = reinterpret_cast<uint64_t *>(smem + (size_t) a.stages * a.stage_bytes + (size_t) a.cap_al * 8);

	if (threadIdx.x == 0) {
		for (int s = 0; s < a.stages; s++)
			mbar_init(&bars[s], 1);
		mbar_fence_init();
	}
	__syncthreads();
	// descriptors of the blocks in the ring, written by the issuing thread: the compute
	// threads read them from shared memory instead of waiting on a global load per block
	__shared__ StagedBlock sdesc[8];
	if (threadIdx.x == 0) {
		for (int s = 0; s < a.stages; s++) {
			int64_t b = (int64_t) blockIdx.x + (int64_t) s * gridDim.x;
			if (b < a.nblocks) {
				const StagedBlock d = a.blocks[b];
				sdesc[s] = d;
				staged_issue_d(a, d, s, smem, bars);
			}
		}
	}

	// ring slot and mbarrier phase of the current block, advanced incrementally (a runtime
	// division per block costs more issue slots than the rest of the block's bookkeeping)
	int s = 0;
	uint32_t parity = 0;
	for (int64_t b = blockIdx.x; b < a.nblocks; b += gridDim.x) {
		// the descriptor this iteration will issue, loaded now so its latency overlaps the block
		const int64_t nb = b + (int64_t) a.stages * gridDim.x;
		StagedBlock dnext{};
		if (threadIdx.x == 0 && nb < a.nblocks)
			dnext = a.blocks[nb];
		bool ok = mbar_wait_bounded(&bars[s], parity, kWaitBudgetCycles);
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
		const StagedBlock d = sdesc[s];
		staged_block<K, A, L, YMAP, OWNX>(a, d, smem + (size_t) s * a.stage_bytes, xb);
		__syncthreads();
		if (threadIdx.x == 0 && nb < a.nblocks) {
			sdesc[s] = dnext;
			staged_issue_d(a, dnext, s, smem, bars);
		}
		if (++s == a.stages) {
			s = 0;
			parity ^= 1u;
		}
	}
}

// ------------------------------------------------------------------ pipelined staged kernel
// Same blocks, stage ring and per-row operation order as staged_kernel, but the x gather
// of block i+1 is issued (into registers) before the rows of block i are summed, and
// stored to shared memory after them, so the gather's L2 latency overlaps the dependent
// add chains instead of following them.  Stage layout: values (8 B) | columns (4 B) |
// gathered x (8 B; not for SEQ_SPLIT, whose products replace the values in place).
// Requires block capacity <= PIPE_G * threads (one register slot per staged entry).
constexpr int PIPE_G = 8;

template <Kind K>
__device__ __forceinline__ void first_row_bounds(const StagedArgs & a, const StagedBlock & d, int & js0, int & je0)
{
	js0 = 0;
	je0 = 0;
	if (K == Kind::CSR && d.units >= 0 && (int) threadIdx.x < d.units) {
		const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
		const int64_t r = (int64_t) d.unit0 + threadIdx.x;
		js0 = (int) ((int64_t) __ldg(a.ptr + r) - e0);
		je0 = (int) ((int64_t) __ldg(a.ptr + r + 1) - e0);
	}
}

__device__ __forceinline__ void gather_load(const StagedArgs & a, const StagedBlock & d, const uint8_t * stage,
		double (&xr)[PIPE_G])
{
	const int32_t * sc = reinterpret_cast<const int32_t *>(stage + (size_t) a.cap_al * 8);
	const int off = d.elem0 & 3;
	#pragma unroll
	for (int k = 0; k < PIPE_G; k++) {
		const int e = (int) threadIdx.x + k * (int) blockDim.x;
		if (e < d.elems)
			xr[k] = ldg(a.x + sc[off + e]);
	}
}

template <Arith A>
__device__ __forceinline__ void gather_store(const StagedArgs & a, const StagedBlock & d, uint8_t * stage,
		const double (&xr)[PIPE_G])
{
	double * sv = reinterpret_cast<double *>(stage);
	double * xg = reinterpret_cast<double *>(stage + (size_t) a.cap_al * 12);
	const int off = d.elem0 & 3;
	#pragma unroll
	for (int k = 0; k < PIPE_G; k++) {
		const int e = (int) threadIdx.x + k * (int) blockDim.x;
		if (e < d.elems) {
			if (A == Arith::SEQ_SPLIT)
				sv[off + e] = __dmul_rn(sv[off + e], xr[k]);   // the reference's rounded product
			else
				xg[off + e] = xr[k];
		}
	}
}

template <Kind K, Arith A, int L, bool YMAP>
__global__ void __launch_bounds__(STAGED_MAX_THREADS) pipe_kernel(StagedArgs a)
{
	extern __shared__ __align__(128) uint8_t smem[];
	uint64_t * bars = reinterpret_cast<uint64_t *>(smem + (size_t) a.stages * a.stage_bytes);
	const int S = a.stages;
	if (threadIdx.x == 0) {
		for (int s = 0; s < S; s++)
			mbar_init(&bars[s], 1);
		mbar_fence_init();
	}
	__syncthreads();
	if (threadIdx.x == 0)
		for (int s = 0; s < S; s++) {
			const int64_t b = (int64_t) blockIdx.x + (int64_t) s * gridDim.x;
			if (b < a.nblocks)
				staged_issue(a, b, s, smem, bars);
		}
	int64_t b = blockIdx.x;
	if (b >= a.nblocks)
		return;
	StagedBlock d = a.blocks[b];
	double xr[PIPE_G];
	{
		const bool ok = mbar_wait_bounded(&bars[0], 0u, kWaitBudgetCycles);
		if (__syncthreads_or(!ok)) {
			if (threadIdx.x == 0) {
				dev_flag_error(a.err, DEV_ERR_TIMEOUT);
				int pending = 0;          // the first S blocks' copies
				while (pending < S && b + (int64_t) pending * gridDim.x < a.nblocks)
					pending++;
				drain_ring(bars, S, 0, 0u, pending, kWaitBudgetCycles);
			}
			return;
		}
		if (d.units >= 0) {
			gather_load(a, d, smem, xr);
			gather_store<A>(a, d, smem, xr);
		}
		__syncthreads();
	}
	int s = 0;                          // ring slot of the current block
	int ns = S > 1 ? 1 : 0;             // ring slot and mbarrier phase of the next block
	uint32_t nparity = S > 1 ? 0u : 1u;
	for (;;) {
		uint8_t * stage = smem + (size_t) s * a.stage_bytes;
		const int64_t nb = b + gridDim.x;
		const bool has_next = nb < a.nblocks;
		int js0, je0;
		first_row_bounds<K>(a, d, js0, je0);
		StagedBlock dn{};
		uint8_t * nstage = smem + (size_t) ns * a.stage_bytes;
		if (has_next) {
			dn = a.blocks[nb];
			const bool ok = mbar_wait_bounded(&bars[ns], nparity, kWaitBudgetCycles);
			if (__syncthreads_or(!ok)) {
				if (threadIdx.x == 0) {
					dev_flag_error(a.err, DEV_ERR_TIMEOUT);
					// copies in flight: blocks nb, nb + grid, ... up to the last one issued,
					// b + (S - 1) * grid (S - 1 of them; the one next block with S == 1)
					const int span = S > 1 ? S - 1 : 1;
					int pending = 0;
					while (pending < span && nb + (int64_t) pending * gridDim.x < a.nblocks)
						pending++;
					drain_ring(bars, S, ns, nparity, pending, kWaitBudgetCycles);
				}
				return;
			}
			if (dn.units >= 0)
				gather_load(a, dn, nstage, xr);
		}
		if (d.units >= 0)
			block_rows<K, A, L, YMAP>(a, d, reinterpret_cast<double *>(stage),
					reinterpret_cast<const double *>(stage + (size_t) a.cap_al * 12), js0, je0);
		else
			staged_long_unit<K, A, L, YMAP>(a, d, reinterpret_cast<double *>(stage));  // no staged data: chunk buffer
		if (has_next && dn.units >= 0)
			gather_store<A>(a, dn, nstage, xr);
		__syncthreads();
		if (threadIdx.x == 0) {
			const int64_t fb = b + (int64_t) S * gridDim.x;
			if (fb < a.nblocks)
				staged_issue(a, fb, s, smem, bars);
		}
		if (!has_next)
			break;
		b = nb;
		d = dn;
		s = ns;
		if (++ns == S) {
			ns = 0;
			nparity ^= 1u;
		}
	}
}

// Row bounds of row thread `t`'s row in block d, relative to the stage start (CSR).
// What row thread t needs of block d before the block's gather is done, loaded while it
// waits: CSR, its row's bounds (relative to the stage start); slices, its slice's start and
// width; the y index of its row (ymap applied; -1: no row).  Chunk blocks of a slice: the
// y index of the last chunk's row.
template <Kind K, bool YMAP>
__device__ __forceinline__ void row_pre_t(const StagedArgs & a, const StagedBlock & d, int t, int & js0, int & je0,
		int64_t & yi)
{
	js0 = 0;
	je0 = 0;
	yi = -1;
	const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
	if (K == Kind::CSR) {
		if (d.units >= 0 && t < d.units) {
			const int64_t r = (int64_t) d.unit0 + t;
			js0 = (int) ((int64_t) __ldg(a.ptr + r) - e0);
			je0 = (int) ((int64_t) __ldg(a.ptr + r + 1) - e0);
			yi = r;
		}
		return;
	}
	const int V = a.V;
	int64_t row = -1;
	if (d.units >= 0) {
		if (t < d.units * V) {
			const int64_t sl = (int64_t) d.unit0 + t / V;
			const int64_t p0 = __ldg(a.ptr + sl);
			js0 = (int) (p0 - e0);
			je0 = (int) (((int64_t) __ldg(a.ptr + sl + 1) - p0) / V);
			row = sl * V + t % V;
		}
	} else if (((-d.units - 1) & 2) && t < V) {
		row = (int64_t) d.unit0 * V + t;
	}
	if (row >= 0 && row < a.m)
		yi = (YMAP && a.ymap) ? (int64_t) __ldg(a.ymap + row) : row;
}

// One slice row over w slice columns staged from entry sb (a slice start, or a chunk start
// on a tile boundary): values column-major (vp[k * V]), x in the tiled order of the column
// indices (tile of 8 columns at sb + t8 * V, row `lane` at lane * tw inside it), stored at
// e + e / 8 so that the 32 rows of a full tile (stride 9 doubles) read without bank
// conflicts.  One fused multiply-add per column, in column order.
__device__ __forceinline__ double tiled_row(const double * vp, const double * xb, int sb, int w, int V, int lane,
		double acc)
{
	for (int t8 = 0; t8 < w; t8 += 8) {
		const int tw = w - t8 < 8 ? w - t8 : 8;
		const int eb = sb + t8 * V + lane * tw;
		#pragma unroll
		for (int j = 0; j < 8; j++) {
			if (j < tw) {
				const int e = eb + j;
				acc = __fma_rn(vp[(t8 + j) * V], xb[e + (e >> 3)], acc);
			}
		}
	}
	return acc;
}

// block_rows for row thread t of nt (the block holds at most nt rows).  TX: the x of tiled
// stage entry e sits at e + e / 8 (ws_kernel); row `lane` of a slice reads tile by tile.
template <Kind K, Arith A, int L, bool YMAP, bool TX = false>
__device__ __forceinline__ void rows_t(const StagedArgs & a, const StagedBlock & d, const double * sv, const double * xb,
		int js0, int je0, int64_t yi, int t, int nt)
{
	const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
	if (K == Kind::CSR) {
		if (t < d.units) {
			const int64_t r = (int64_t) d.unit0 + t;
			const int js = js0, je = je0;
			double sum = 0.0;
			if (A == Arith::SEQ_SPLIT) {
				sum = seq_add(sv + js, je - js, sum);
			} else if (A == Arith::SEQ_FMA) {
				sum = seq_fma(sv + js, 1, xb + js, 1, je - js, sum);
			} else {
				double ln[L];
				#pragma unroll
				for (int l = 0; l < L; l++)
					ln[l] = 0.0;
				const int jv = js + ((je - js) & ~(L - 1));
				for (int j = js; j < jv; j += L) {
					#pragma unroll
					for (int l = 0; l < L; l++)
						ln[l] = __fma_rn(sv[j + l], xb[j + l], ln[l]);
				}
				sum = lanes_reduce<L>(ln);
				for (int j = jv; j < je; j++)
					sum = __dadd_rn(sum, __dmul_rn(sv[j], xb[j]));
			}
			a.y[r] = sum;
		}
	} else {
		// a block holds at most nt / V slices (row_pre_t loaded this thread's slice and y index)
		const int V = a.V;
		if (yi >= 0) {
			const int lane = t % V;
			const int sb = js0, w = je0, ks = sb + lane;
			double acc = 0.0;
			if (TX)
				acc = tiled_row(sv + ks, xb, sb, w, V, lane, acc);
			else
				acc = seq_fma(sv + ks, V, xb + ks, V, w, acc);
			a.y[yi] = acc;
		}
	}
}

// ------------------------------------------------------------------ warp-specialised staged kernel
// The CTA's first warps gather (x loads, products or x into the stage), its last
// `row_threads / 32` warps sum rows, so block k's rows run while block k+1 is gathered and
// block k+2 is in flight.  Hand-offs: full[s] (bulk copy landed, with the block's
// descriptor in sdesc[s]), prod[s] (every gather thread has written its entries; count =
// gather threads).  The row warps give a stage back with a named barrier among themselves
// and their first thread issues the stage's next copy.  Same per-row operation order as
// staged_kernel; a block holds at most `row_threads` rows, and a unit longer than a block
// is a run of chunk blocks.  Each CTA walks a contiguous range of the block table.
// Bulk copy of a block's entries for the warp-specialised kernel (chunk blocks of long
// units included; only an empty block completes the stage without a copy).
// Packed variant (csr_naive): the block's packed column stream lands where the columns would.
__device__ __forceinline__ void ws_issue_packed(const StagedArgs & a, const StagedBlock & d, const int4 & pi, int s,
		uint8_t * smem, uint64_t * bars)
{
	if (d.elems == 0) {
		mbar_arrive(&bars[s]);
		return;
	}
	const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
	const int64_t e1 = ((int64_t) d.elem0 + d.elems + 3) & ~(int64_t) 3;
	const uint32_t cnt = (uint32_t) (e1 - e0);
	double * sv = reinterpret_cast<double *>(smem + (size_t) s * a.stage_bytes);
	uint8_t * sc = smem + (size_t) s * a.stage_bytes + (size_t) a.cols_off;
	fence_proxy_async_smem();
	mbar_arrive_expect_tx(&bars[s], cnt * 8u + (uint32_t) pi.w);
	bulk_g2s(sv, a.vals + e0, cnt * 8u, &bars[s]);
	bulk_g2s(sc, a.pcols + (int64_t) pi.x * 4, (uint32_t) pi.w, &bars[s]);
}

__device__ __forceinline__ void ws_issue(const StagedArgs & a, const StagedBlock & d, int s, uint8_t * smem, uint64_t * bars)
{
	if (d.elems == 0) {
		mbar_arrive(&bars[s]);
		return;
	}
	const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
	const int64_t e1 = ((int64_t) d.elem0 + d.elems + 3) & ~(int64_t) 3;
	const uint32_t cnt = (uint32_t) (e1 - e0);
	double * sv = reinterpret_cast<double *>(smem + (size_t) s * a.stage_bytes);
	int32_t * sc = reinterpret_cast<int32_t *>(smem + (size_t) s * a.stage_bytes + (size_t) a.cols_off);
	fence_proxy_async_smem();
	mbar_arrive_expect_tx(&bars[s], cnt * 12u);
	bulk_g2s(sv, a.vals + e0, cnt * 8u, &bars[s]);
	bulk_g2s(sc, a.cols + e0, cnt * 4u, &bars[s]);
}

// One chunk block of a unit longer than a staged block (units = -1 - flags; bit 0: first
// chunk, bit 1: last).  The unit's running state (sum, lanes) lives in the row thread's
// registers between consecutive chunks, which the same CTA processes in order, so every
// row is still summed by one thread in the reference order.
template <Kind K, Arith A, int L, bool YMAP, bool TX = false>
__device__ __forceinline__ void ws_chunk(const StagedArgs & a, const StagedBlock & d, const double * sv, const double * xg,
		int64_t yi, int rt, double & acc, double (&ln)[L])
{
	const int flags = -d.units - 1;
	const int off = d.elem0 & 3;
	if (K == Kind::CSR) {
		if (rt != 0)
			return;
		const int64_t r = d.unit0;
		if (flags & 1) {
			acc = 0.0;
			#pragma unroll
			for (int l = 0; l < L; l++)
				ln[l] = 0.0;
		}
		if (A == Arith::SEQ_SPLIT) {
			acc = seq_add(sv + off, d.elems, acc);
		} else if (A == Arith::SEQ_FMA) {
			acc = seq_fma(sv + off, 1, xg + off, 1, d.elems, acc);
		} else {
			const int64_t js = a.ptr[r], je = a.ptr[r + 1];
			const int64_t jv = js + ((je - js) & ~(int64_t) (L - 1));
			for (int e = 0; e < d.elems; e++) {
				const int64_t j = (int64_t) d.elem0 + e;
				if (j < jv) {
					const int l = (int) ((j - js) & (L - 1));
					#pragma unroll
					for (int q = 0; q < L; q++)
						if (q == l)
							ln[q] = __fma_rn(sv[off + e], xg[off + e], ln[q]);
				} else {
					if (j == jv)
						acc = lanes_reduce<L>(ln);
					acc = __dadd_rn(acc, __dmul_rn(sv[off + e], xg[off + e]));
				}
			}
			if ((flags & 2) && jv == je)
				acc = lanes_reduce<L>(ln);
		}
		if (flags & 2)
			a.y[r] = acc;
	} else {
		const int V = a.V;
		if (rt >= V)
			return;
		if (flags & 1)
			acc = 0.0;
		const int kn = d.elems / V;
		if (TX)
			acc = tiled_row(sv + rt, xg, 0, kn, V, rt, acc);   // chunks start on a tile boundary, off = 0
		else
			acc = seq_fma(sv + off + rt, V, xg + off + rt, V, kn, acc);
		if ((flags & 2) && yi >= 0)
			a.y[yi] = acc;
	}
}

// TX (kernel 8, slices only): the column indices are stored row-major in tiles of 8 slice
// columns (tile_cols_kernel), so 32 consecutive gather threads read 4 rows x 8 neighbouring
// columns instead of 32 rows x 1 column.  The gather keeps that order (x of stage entry e
// at e + e / 8) and the row threads walk the tiles (tiled_row).  Blocks start at slice
// boundaries and chunks at tile boundaries, so off == 0.
template <Kind K, Arith A, int L, bool YMAP, bool TX = false, bool PK = false>
__global__ void __launch_bounds__(STAGED_MAX_THREADS) ws_kernel(StagedArgs a)
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
		// ---- gather warps
		const int gt = threadIdx.x;
		for (int64_t b = b_begin; b < b_end; b++) {
			const bool ok = mbar_wait_bounded(&full[s], parity, a.wait_budget);
			if (named_bar_or(2, ng, !ok)) {                // the gather warps leave together
				if (gt == 0)
					dev_flag_error(a.err, DEV_ERR_TIMEOUT);
				return;
			}
			const StagedBlock d = sdesc[s];
			if (d.elems > 0) {
				uint8_t * st = smem + (size_t) s * a.stage_bytes;
				double * sv = reinterpret_cast<double *>(st);
				const int32_t * sc = reinterpret_cast<const int32_t *>(st + (size_t) a.cols_off);
				double * xg = reinterpret_cast<double *>(st + (size_t) a.cap_al * 8);
				const int off = d.elem0 & 3;
				const int4 pi = PK ? spack[s] : int4{};
				const uint32_t * words = reinterpret_cast<const uint32_t *>(st + (size_t) a.cols_off);
				// Rounds of WS_GATHER_SLOTS * ng consecutive entries, the same count for every gather
				// thread; WS_GATHER_SLOTS independent loads in flight per thread.  The FMA formats'
				// columns sit at the top of the x buffer: x of position p covers column positions
				// below p + 1 only, so once every gather thread has read the round's columns (named
				// barrier 2) the round's x overwrites columns already read.
				const int per_round = WS_GATHER_SLOTS * ng;
				for (int rb = 0; rb < d.elems; rb += per_round) {
					const int e0 = rb + gt;
					double xv[WS_GATHER_SLOTS];
					#pragma unroll
					for (int k = 0; k < WS_GATHER_SLOTS; k++) {
						const int e = e0 + k * ng;
						if (e < d.elems)
							xv[k] = ldg(a.x + (PK ? packed_col64(words, e, pi.z, pi.y) : sc[off + e]));
					}
					if (A != Arith::SEQ_SPLIT)
						named_bar_sync(2, ng);
					#pragma unroll
					for (int k = 0; k < WS_GATHER_SLOTS; k++) {
						const int e = e0 + k * ng;
						if (e < d.elems) {
							if (A == Arith::SEQ_SPLIT)
								sv[off + e] = __dmul_rn(sv[off + e], xv[k]);   // the reference's rounded product
							else if (TX)
								xg[e + (e >> 3)] = xv[k];
							else
								xg[off + e] = xv[k];
						}
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
				if (PK) {
					const int4 pi = a.pinfo[b];
					spack[q] = pi;
					ws_issue_packed(a, d, pi, q, smem, full);
				} else {
					ws_issue(a, d, q, smem, full);
				}
			}
		}
	named_bar_sync(1, nr);
	double acc = 0.0;          // running state of a long unit across its chunk blocks
	double ln[L];
	#pragma unroll
	for (int l = 0; l < L; l++)
		ln[l] = 0.0;
	for (int64_t b = b_begin; b < b_end; b++) {
		const int64_t nb = b + S;
		StagedBlock dnext{};
		int4 pnext{};
		if (rt == 0 && nb < b_end) {
			dnext = a.blocks[nb];
			if (PK)
				pnext = a.pinfo[nb];
		}
		const StagedBlock d = sdesc[s];
		int js0 = 0, je0 = 0;
		int64_t yi = -1;
		row_pre_t<K, YMAP>(a, d, rt, js0, je0, yi);
		const bool ok = mbar_wait_bounded(&prod[s], parity, a.wait_budget);
		if (named_bar_or(1, nr, !ok)) {      // all row threads leave together
			if (rt == 0) {
				dev_flag_error(a.err, DEV_ERR_TIMEOUT);
				// rt 0 issued the copies of blocks b .. b + S - 1: wait until they have landed
				drain_ring(full, S, s, parity, (int) (b_end - b < S ? b_end - b : S), kWaitBudgetCycles);
			}
			return;
		}
		uint8_t * st = smem + (size_t) s * a.stage_bytes;
		if (d.units >= 0)
			rows_t<K, A, L, YMAP, TX>(a, d, reinterpret_cast<const double *>(st),
					reinterpret_cast<const double *>(st + (size_t) a.cap_al * 8), js0, je0, yi, rt, nr);
		else
			ws_chunk<K, A, L, YMAP, TX>(a, d, reinterpret_cast<const double *>(st),
					reinterpret_cast<const double *>(st + (size_t) a.cap_al * 8), yi, rt, acc, ln);
		named_bar_sync(1, nr);
		if (rt == 0 && nb < b_end) {
			sdesc[s] = dnext;
			if (PK) {
				spack[s] = pnext;
				ws_issue_packed(a, dnext, pnext, s, smem, full);
			} else {
				ws_issue(a, dnext, s, smem, full);
			}
		}
		if (++s == S) {
			s = 0;
			parity ^= 1u;
		}
	}
}

// ------------------------------------------------------------------ batched SpMV
// Many matrices in one persistent launch.  The staged blocks of every matrix form one
// work queue (long units first); CTAs claim blocks with an atomic counter (dynamic, so
// uneven matrices balance), prefetch `stages` claims ahead through the bulk-copy ring, and
// run the block with its matrix's format: kind 0 = csr_naive order, kind 1 = slices with
// one FMA per column (sell, sell_sorted, sell_c_s).
__device__ __forceinline__ void batch_issue(const BatchArgs & b, int64_t c, int s, uint8_t * smem, uint64_t * bars,
		int64_t * claim)
{
	claim[s] = c < b.nblocks ? c : -1;
	if (c >= b.nblocks) {
		mbar_arrive(&bars[s]);
		return;
	}
	const StagedBlock d = b.blocks[c];
	if (d.units < 0 || d.elems == 0) {
		mbar_arrive(&bars[s]);
		return;
	}
	const BatchMat mt = b.mats[b.bmat[c]];
	const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
	const int64_t e1 = ((int64_t) d.elem0 + d.elems + 3) & ~(int64_t) 3;
	const uint32_t cnt = (uint32_t) (e1 - e0);
	double * sv = reinterpret_cast<double *>(smem + (size_t) s * b.stage_bytes);
	int32_t * sc = reinterpret_cast<int32_t *>(smem + (size_t) s * b.stage_bytes + (size_t) b.cap_al * 8);
	fence_proxy_async_smem();
	mbar_arrive_expect_tx(&bars[s], cnt * 12u);
	bulk_g2s(sv, mt.vals + e0, cnt * 8u, &bars[s]);
	bulk_g2s(sc, mt.cols + e0, cnt * 4u, &bars[s]);
}

__global__ void __launch_bounds__(STAGED_MAX_THREADS) batch_kernel(BatchArgs b)
{
	extern __shared__ __align__(128) uint8_t smem[];
	__shared__ int64_t claim[8];
	double * xb = reinterpret_cast<double *>(smem + (size_t) b.stages * b.stage_bytes);
	uint64_t * bars = reinterpret_cast<uint64_t *>(smem + (size_t) b.stages * b.stage_bytes + (size_t) b.cap_al * 8);
	if (threadIdx.x == 0) {
		for (int s = 0; s < b.stages; s++)
			mbar_init(&bars[s], 1);
		mbar_fence_init();
	}
	__syncthreads();
	if (threadIdx.x == 0)
		for (int s = 0; s < b.stages; s++)
			batch_issue(b, (int64_t) atomicAdd(b.counter, 1ULL), s, smem, bars, claim);
	int s = 0;
	uint32_t parity = 0;
	for (;; ) {
		const bool ok = mbar_wait_bounded(&bars[s], parity, kWaitBudgetCycles);
		if (__syncthreads_or(!ok)) {
			if (threadIdx.x == 0) {
				dev_flag_error(b.err, DEV_ERR_TIMEOUT);
				drain_ring(bars, b.stages, s, parity, b.stages, kWaitBudgetCycles);   // every slot holds a claim
			}
			return;
		}
		const int64_t c = claim[s];
		if (c < 0)
			break;          // the queue is drained; every later slot of this ring is empty too
		const StagedBlock d = b.blocks[c];
		const BatchMat mt = b.mats[b.bmat[c]];
		StagedArgs a{};
		a.ptr = mt.ptr;
		a.cols = mt.cols;
		a.vals = mt.vals;
		a.ymap = mt.ymap;
		a.x = b.x + mt.x_off;
		a.y = b.y + mt.y_off;
		a.m = mt.m;
		a.V = mt.V;
		a.cap_al = b.cap_al;
		a.stages = b.stages;
		a.stage_bytes = b.stage_bytes;
		a.exact = b.exact;
		a.err = b.err;
		uint8_t * stage = smem + (size_t) s * b.stage_bytes;
		if (mt.kind == 0)
			staged_block<Kind::CSR, Arith::SEQ_SPLIT, 1, false>(a, d, stage, xb);
		else
			staged_block<Kind::SLICED, Arith::SEQ_FMA, 1, true>(a, d, stage, xb);
		__syncthreads();
		if (threadIdx.x == 0)
			batch_issue(b, (int64_t) atomicAdd(b.counter, 1ULL), s, smem, bars, claim);
		if (++s == b.stages) {
			s = 0;
			parity ^= 1u;
		}
	}
}

struct SlicedArgs {
	const int64_t * sptr;    // slice pointers (SELL-C-sigma) or nullptr
	const int32_t * rcp;     // row_cluster_ptr (SELL) or nullptr
	const int32_t * widths;  // slice widths (SELL-C-sigma) or nullptr
	const int32_t * cols;
	const double * vals;
	const int32_t * ymap;    // row_order / rev_permutation or nullptr
	const double * x;
	double * y;
	int64_t m;
	int64_t nslices;
	int C;
};

template <bool PTR64, bool YMAP>
__global__ void __launch_bounds__(256) sliced_kernel(SlicedArgs a)
{
	const int C = a.C;
	const int spc = blockDim.x / C;
	const int lane = threadIdx.x % C;
	const int sl = threadIdx.x / C;
	for (int64_t s = (int64_t) blockIdx.x * spc + sl; s < a.nslices; s += (int64_t) gridDim.x * spc) {
		const int64_t row = s * C + lane;
		if (row >= a.m)
			continue;
		int64_t p;
		int w;
		if (PTR64) {
			p = a.sptr[s];
			w = a.widths[s];
		} else {
			p = a.rcp[s];
			w = (a.rcp[s + 1] - a.rcp[s]) / C;
		}
		p += lane;
		const double * __restrict__ v = a.vals + p;
		const int32_t * __restrict__ c = a.cols + p;
		double acc = 0.0;
		int k = 0;
		for (; k + 4 <= w; k += 4) {
			const int64_t o = (int64_t) k * C;
			double v0 = v[o], v1 = v[o + C], v2 = v[o + 2 * C], v3 = v[o + 3 * C];
			int32_t c0 = c[o], c1 = c[o + C], c2 = c[o + 2 * C], c3 = c[o + 3 * C];
			double x0 = ldg(a.x + c0), x1 = ldg(a.x + c1), x2 = ldg(a.x + c2), x3 = ldg(a.x + c3);
			acc = __fma_rn(v0, x0, acc);
			acc = __fma_rn(v1, x1, acc);
			acc = __fma_rn(v2, x2, acc);
			acc = __fma_rn(v3, x3, acc);
		}
		for (; k < w; k++) {
			const int64_t o = (int64_t) k * C;
			acc = __fma_rn(v[o], ldg(a.x + c[o]), acc);
		}
		a.y[(YMAP && a.ymap) ? a.ymap[row] : row] = acc;
	}
}

using StagedFn = void (*)(StagedArgs);

template <bool OWNX>
StagedFn pick_staged_t(const Handle & h);

// The staged kernel instance of a handle's format / lane count (kernel 5: rows gather
// their own x).
StagedFn pick_staged(const Handle & h)
{
	return h.exec_kernel == 5 ? pick_staged_t<true>(h) : pick_staged_t<false>(h);
}

template <bool OWNX>
StagedFn pick_staged_t(const Handle & h)
{
	const int fmt = h.desc.format;
	if (fmt == SPMV_FMT_CSR_NAIVE)
		return staged_kernel<Kind::CSR, Arith::SEQ_SPLIT, 1, false, OWNX>;
	if (fmt == SPMV_FMT_CSR_VEC) {
		switch (h.desc.vec_len) {
		case 1: return staged_kernel<Kind::CSR, Arith::LANES_FMA, 1, false, OWNX>;
		case 2: return staged_kernel<Kind::CSR, Arith::LANES_FMA, 2, false, OWNX>;
		case 4: return staged_kernel<Kind::CSR, Arith::LANES_FMA, 4, false, OWNX>;
		case 8: return staged_kernel<Kind::CSR, Arith::LANES_FMA, 8, false, OWNX>;
		case 16: return staged_kernel<Kind::CSR, Arith::LANES_FMA, 16, false, OWNX>;
		}
		return nullptr;
	}
	if (fmt == SPMV_FMT_SELL_SORTED || fmt == SPMV_FMT_SELL_C_S)
		return staged_kernel<Kind::SLICED, Arith::SEQ_FMA, 1, true, OWNX>;
	if (fmt == SPMV_FMT_SELL)
		return staged_kernel<Kind::SLICED, Arith::SEQ_FMA, 1, false, OWNX>;
	return nullptr;
}

// The pipelined kernel instance of a handle's format / lane count.
StagedFn pick_pipe(const Handle & h)
{
	const int fmt = h.desc.format;
	if (fmt == SPMV_FMT_CSR_NAIVE)
		return pipe_kernel<Kind::CSR, Arith::SEQ_SPLIT, 1, false>;
	if (fmt == SPMV_FMT_CSR_VEC) {
		switch (h.desc.vec_len) {
		case 1: return pipe_kernel<Kind::CSR, Arith::LANES_FMA, 1, false>;
		case 2: return pipe_kernel<Kind::CSR, Arith::LANES_FMA, 2, false>;
		case 4: return pipe_kernel<Kind::CSR, Arith::LANES_FMA, 4, false>;
		case 8: return pipe_kernel<Kind::CSR, Arith::LANES_FMA, 8, false>;
		case 16: return pipe_kernel<Kind::CSR, Arith::LANES_FMA, 16, false>;
		}
		return nullptr;
	}
	if (fmt == SPMV_FMT_SELL_SORTED || fmt == SPMV_FMT_SELL_C_S)
		return pipe_kernel<Kind::SLICED, Arith::SEQ_FMA, 1, true>;
	if (fmt == SPMV_FMT_SELL)
		return pipe_kernel<Kind::SLICED, Arith::SEQ_FMA, 1, false>;
	return nullptr;
}

// The warp-specialised kernel instance of a handle's format / lane count.
StagedFn pick_ws(const Handle & h)
{
	const int fmt = h.desc.format;
	if (fmt == SPMV_FMT_CSR_NAIVE)
		return h.desc.pack_cols == 1 ? ws_kernel<Kind::CSR, Arith::SEQ_SPLIT, 1, false, false, true>
		                             : ws_kernel<Kind::CSR, Arith::SEQ_SPLIT, 1, false>;
	if (fmt == SPMV_FMT_CSR_VEC) {
		switch (h.desc.vec_len) {
		case 1: return ws_kernel<Kind::CSR, Arith::LANES_FMA, 1, false>;
		case 2: return ws_kernel<Kind::CSR, Arith::LANES_FMA, 2, false>;
		case 4: return ws_kernel<Kind::CSR, Arith::LANES_FMA, 4, false>;
		case 8: return ws_kernel<Kind::CSR, Arith::LANES_FMA, 8, false>;
		case 16: return ws_kernel<Kind::CSR, Arith::LANES_FMA, 16, false>;
		}
		return nullptr;
	}
	if (fmt == SPMV_FMT_SELL_SORTED || fmt == SPMV_FMT_SELL_C_S)
		return ws_kernel<Kind::SLICED, Arith::SEQ_FMA, 1, true>;
	if (fmt == SPMV_FMT_SELL)
		return ws_kernel<Kind::SLICED, Arith::SEQ_FMA, 1, false>;
	return nullptr;
}

// The tiled warp-specialised kernel instance (kernel 8) of a sliced format.
StagedFn pick_ws_tiled(const Handle & h)
{
	const int fmt = h.desc.format;
	if (fmt == SPMV_FMT_SELL_SORTED || fmt == SPMV_FMT_SELL_C_S)
		return ws_kernel<Kind::SLICED, Arith::SEQ_FMA, 1, true, true>;
	if (fmt == SPMV_FMT_SELL)
		return ws_kernel<Kind::SLICED, Arith::SEQ_FMA, 1, false, true>;
	return nullptr;
}

// Bytes of one stage of the pipelined kernel (values, columns, and gathered x unless the
// products are formed in place).
int pipe_stage_bytes(int format, int cap_al)
{
	const int per = (format == SPMV_FMT_CSR_NAIVE) ? 12 : 20;
	return (int) (ceil_div((int64_t) cap_al * per, 128) * 128);
}

// Stage of the warp-specialised kernels (4 and 8): csr_naive stages values and columns, the
// rounded products replacing the values (12 bytes an entry); the FMA formats stage values
// and an x buffer whose top holds the staged columns until the gather overwrites them (16
// bytes an entry; 17 with the tiled kernel's e + e / 8 buffer).  Returns the stage bytes and
// the columns' byte offset (a multiple of 16, as the bulk copy needs).
int ws_stage_layout(int format, int cap_al, bool tiled, int * cols_off)
{
	if (format == SPMV_FMT_CSR_NAIVE) {
		*cols_off = cap_al * 8;
		return (int) (ceil_div((int64_t) cap_al * 12, 128) * 128);
	}
	const int64_t xb = tiled ? ceil_div(8 * ((int64_t) cap_al + ceil_div((int64_t) cap_al, 8)), 16) * 16
	                         : (int64_t) cap_al * 8;
	*cols_off = (int) ((int64_t) cap_al * 8 + xb - (int64_t) cap_al * 4);
	return (int) (ceil_div((int64_t) cap_al * 8 + xb, 128) * 128);
}

}  // namespace

int batch_launch(const BatchArgs & b, int grid, int threads, size_t smem, cudaStream_t s)
{
	static bool configured = false;
	if (!configured) {
		SPMV_CUDA_TRY(cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
		configured = true;
	}
	batch_kernel<<<grid, threads, smem, s>>>(b);
	SPMV_CUDA_TRY(cudaGetLastError());
	return SPMV_OK;
}

int batch_occupancy(int threads, size_t smem, int * per_sm)
{
	SPMV_CUDA_TRY(cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
	SPMV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, batch_kernel, threads, smem));
	return SPMV_OK;
}

// Block-table order of the warp-specialised kernels.  A group is a block of whole units or
// the full run of chunk blocks of one long unit (a CTA keeps the unit's running sums in
// registers, so a group never splits).  CTA c walks the contiguous range [ranges[c],
// ranges[c + 1]) of the permuted table.  Groups are given to CTAs by their cost (entries
// plus a per-block overhead): groups above a quarter of the per-CTA share first, largest
// first, each to the least-loaded CTA (one 65,280-entry SELL-C-sigma slice is half a CTA's
// share on the 4M-row matrix); then the rest in matrix order, dealt round-robin over the
// CTAs still below the share, so CTAs running at the same time work on neighbouring rows.
// A CTA runs its large groups first.  The table is small (16 bytes a block) and is ordered
// once on the host at set-up.
int ws_order_blocks(Handle & h)
{
	cudaStream_t s = h.stream;
	const int64_t nb = h.num_blocks, G = h.grid;
	SPMV_TRY(h.alloc(&h.d_cta_ranges, G + 1));
	std::vector<StagedBlock> hb((size_t) nb);
	if (nb > 0)
		SPMV_CUDA_TRY(cudaMemcpyAsync(hb.data(), h.d_blocks, nb * sizeof(StagedBlock), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	constexpr int64_t BLOCK_OVERHEAD = 64;       // entries' worth of hand-off cost per block
	std::vector<int64_t> gs;                     // group starts, then nb
	std::vector<int64_t> cost;
	for (int64_t b = 0; b < nb; b++) {
		const StagedBlock & d = hb[(size_t) b];
		if (d.units >= 0 || ((-d.units - 1) & 1)) {
			gs.push_back(b);
			cost.push_back(0);
		}
		cost.back() += d.elems + BLOCK_OVERHEAD;
	}
	const int64_t ng = (int64_t) cost.size();
	gs.push_back(nb);
	int64_t total = 0;
	for (int64_t c : cost)
		total += c;
	const double share = (double) total / (double) G;
	std::vector<int64_t> load((size_t) G, 0);
	std::vector<int32_t> owner((size_t) ng, -1);
	std::vector<int64_t> big;
	for (int64_t g = 0; g < ng; g++)
		if ((double) cost[(size_t) g] > 0.25 * share)
			big.push_back(g);
	std::stable_sort(big.begin(), big.end(), [&](int64_t a, int64_t b) { return cost[(size_t) a] > cost[(size_t) b]; });
	auto least = [&]() {
		int64_t c = 0;
		for (int64_t k = 1; k < G; k++)
			if (load[(size_t) k] < load[(size_t) c])
				c = k;
		return c;
	};
	for (int64_t g : big) {
		const int64_t c = least();
		owner[(size_t) g] = (int32_t) c;
		load[(size_t) c] += cost[(size_t) g];
	}
	int64_t c = 0;
	for (int64_t g = 0; g < ng; g++) {
		if (owner[(size_t) g] >= 0)
			continue;
		int64_t tries = 0;
		while ((double) load[(size_t) c] >= share && tries < G) {
			c = (c + 1) % G;
			tries++;
		}
		if (tries == G)
			c = least();
		owner[(size_t) g] = (int32_t) c;
		load[(size_t) c] += cost[(size_t) g];
		c = (c + 1) % G;
	}
	// each CTA's blocks: its large groups (largest first), then its other groups in order
	std::vector<int64_t> ranges((size_t) G + 1, 0);
	for (int64_t g = 0; g < ng; g++)
		ranges[(size_t) owner[(size_t) g] + 1] += gs[(size_t) g + 1] - gs[(size_t) g];
	for (int64_t k = 0; k < G; k++)
		ranges[(size_t) k + 1] += ranges[(size_t) k];
	std::vector<int64_t> fill(ranges.begin(), ranges.end() - 1);
	std::vector<StagedBlock> out((size_t) nb);
	auto place = [&](int64_t g) {
		int64_t & f = fill[(size_t) owner[(size_t) g]];
		for (int64_t b = gs[(size_t) g]; b < gs[(size_t) g + 1]; b++)
			out[(size_t) f++] = hb[(size_t) b];
	};
	std::vector<char> is_big((size_t) ng, 0);
	for (int64_t g : big) {
		is_big[(size_t) g] = 1;
		place(g);
	}
	for (int64_t g = 0; g < ng; g++)
		if (!is_big[(size_t) g])
			place(g);
	if (nb > 0)
		SPMV_CUDA_TRY(cudaMemcpyAsync(h.d_blocks, out.data(), nb * sizeof(StagedBlock), cudaMemcpyHostToDevice, s));
	SPMV_CUDA_TRY(cudaMemcpyAsync(h.d_cta_ranges, ranges.data(), (G + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	return SPMV_OK;
}

// Grid / shared-memory geometry of the staged kernel for this handle.
int staged_geometry(Handle & h)
{
	if (h.exec_kernel == 4 || h.exec_kernel == 8) {
		const int cap_al = h.block_cap + 8;
		int cols_off = 0;
		const int stage_bytes = h.desc.values == SPMV_VALUES_F32 ? f32ws_stage_bytes(cap_al)
		                        : ws_stage_layout(h.desc.format, cap_al, h.exec_kernel == 8, &cols_off);
		const int max_stages = (220 * 1024 - 128) / stage_bytes;
		if (max_stages < 2) {
			set_error(SPMV_ERR_ARG, "warp-specialised kernel: staging block of %d entries exceeds shared memory",
					h.block_cap);
			return SPMV_ERR_ARG;
		}
		if (h.stages > max_stages)
			h.stages = max_stages;
		if (h.stages < 2)
			h.stages = 2;
		h.smem_bytes = (size_t) h.stages * stage_bytes + (size_t) h.stages * 16;
		// FP32-value handles run ws_f32_kernel (fp32.cu), whose stage is also 12 B per entry
		const void * kern = (h.desc.values == SPMV_VALUES_F32) ? ws_f32_kernel_fn(h.desc.pack_cols == 1)
		                    : (const void *) (h.exec_kernel == 8 ? pick_ws_tiled(h) : pick_ws(h));
		if (!kern) {
			set_error(SPMV_ERR_ARG, "no warp-specialised kernel for format %d with vec_len %d", h.desc.format,
					h.desc.vec_len);
			return SPMV_ERR_ARG;
		}
		SPMV_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) h.smem_bytes));
		int ctas = h.desc.ctas_per_sm > 0 ? h.desc.ctas_per_sm : 0;
		if (ctas == 0) {
			int per_sm = 0;
			SPMV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, h.threads, h.smem_bytes));
			ctas = per_sm > 0 ? per_sm : 1;
		}
		int64_t g = (int64_t) h.num_sms * ctas;
		if (g > h.num_blocks)
			g = h.num_blocks;
		h.grid = (int) (g > 0 ? g : 1);
		return ws_order_blocks(h);
	}
	if (h.exec_kernel == 3) {
		const int cap_al = h.block_cap + 8;
		if (h.block_cap > PIPE_G * h.threads) {
			set_error(SPMV_ERR_ARG, "pipelined kernel: %d staged entries exceed %d per thread x %d threads",
					h.block_cap, PIPE_G, h.threads);
			return SPMV_ERR_ARG;
		}
		const int stage_bytes = pipe_stage_bytes(h.desc.format, cap_al);
		const int max_stages = (220 * 1024 - 64) / stage_bytes;
		if (max_stages < 2) {
			set_error(SPMV_ERR_ARG, "pipelined kernel: staging block of %d entries exceeds shared memory", h.block_cap);
			return SPMV_ERR_ARG;
		}
		if (h.stages > max_stages)
			h.stages = max_stages;
		if (h.stages < 2)
			h.stages = 2;
		h.smem_bytes = (size_t) h.stages * stage_bytes + 64;
		StagedFn kern = pick_pipe(h);
		if (!kern) {
			set_error(SPMV_ERR_ARG, "no pipelined kernel for format %d with vec_len %d", h.desc.format, h.desc.vec_len);
			return SPMV_ERR_ARG;
		}
		SPMV_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) h.smem_bytes));
		int ctas = h.desc.ctas_per_sm > 0 ? h.desc.ctas_per_sm : 0;
		if (ctas == 0) {
			int per_sm = 0;
			SPMV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, h.threads, h.smem_bytes));
			ctas = per_sm > 0 ? per_sm : 1;
		}
		int64_t g = (int64_t) h.num_sms * ctas;
		if (g > h.num_blocks)
			g = h.num_blocks;
		h.grid = (int) (g > 0 ? g : 1);
		return SPMV_OK;
	}
	const int cap_al = h.block_cap + 8;
	const int stage_bytes = (int) (ceil_div((int64_t) cap_al * 12, 128) * 128);
	// keep the pipeline inside the 227 KB a CTA may use (fewer stages for large blocks)
	const int xbuf_bytes = cap_al * 8;
	const int max_stages = (int) ((220 * 1024 - 64 - xbuf_bytes) / stage_bytes);
	if (max_stages < 1) {
		set_error(SPMV_ERR_ARG, "staging block of %d entries exceeds shared memory", h.block_cap);
		return SPMV_ERR_ARG;
	}
	if (h.stages > max_stages)
		h.stages = max_stages;
	h.smem_bytes = (size_t) h.stages * stage_bytes + (size_t) xbuf_bytes + 64;
	StagedFn kern = pick_staged(h);
	if (!kern) {
		set_error(SPMV_ERR_ARG, "no staged kernel for format %d with vec_len %d", h.desc.format, h.desc.vec_len);
		return SPMV_ERR_ARG;
	}
	SPMV_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) h.smem_bytes));
	int ctas = h.desc.ctas_per_sm > 0 ? h.desc.ctas_per_sm : 0;
	if (ctas == 0) {
		int per_sm = 0;
		SPMV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, h.threads, h.smem_bytes));
		ctas = per_sm > 0 ? per_sm : 1;
	}
	int64_t g = (int64_t) h.num_sms * ctas;
	if (g > h.num_blocks)
		g = h.num_blocks;
	h.grid = (int) (g > 0 ? g : 1);
	return SPMV_OK;
}

int launch_spmv(Handle & h, const double * d_x, double * d_y, cudaStream_t s)
{
	const int fmt = h.desc.format;
	if (fmt == SPMV_FMT_DIV_RF)
		return launch_div(h, d_x, d_y, s);
	if (h.exec_kernel == 2 || h.exec_kernel == 6 || h.exec_kernel == 9 || h.exec_kernel == 10)
		return launch_warp(h, d_x, d_y, s);
	if (h.exec_kernel == 1) {
		SlicedArgs a{};
		a.x = d_x;
		a.y = d_y;
		a.m = h.m;
		if (fmt == SPMV_FMT_SELL_C_S) {
			a.sptr = h.d_sptr;
			a.widths = h.d_widths;
			a.cols = h.d_scols;
			a.vals = h.d_svals;
			a.ymap = h.d_order;
			a.nslices = h.nslices;
			a.C = h.desc.sellcs_c;
		} else {
			a.rcp = h.d_rcp;
			a.cols = h.d_ja;
			a.vals = h.d_a;
			a.ymap = (fmt == SPMV_FMT_SELL_SORTED) ? h.d_rev : nullptr;
			a.nslices = h.nclusters;
			a.C = h.desc.vec_len;
		}
		if (a.nslices == 0)
			return SPMV_OK;
		const int spc = 256 / a.C;
		int64_t grid = ceil_div(a.nslices, spc);
		const int64_t cap = (int64_t) h.num_sms * 16;
		if (grid > cap)
			grid = cap;
		if (a.sptr) {
			sliced_kernel<true, true><<<(unsigned) grid, 256, 0, s>>>(a);
		} else if (a.ymap) {
			sliced_kernel<false, true><<<(unsigned) grid, 256, 0, s>>>(a);
		} else {
			sliced_kernel<false, false><<<(unsigned) grid, 256, 0, s>>>(a);
		}
		SPMV_CUDA_TRY(cudaGetLastError());
		return SPMV_OK;
	}

	if (h.num_blocks == 0)
		return SPMV_OK;
	StagedArgs a{};
	a.blocks = h.d_blocks;
	a.nblocks = h.num_blocks;
	a.x = d_x;
	a.y = d_y;
	a.m = h.m;
	a.cap_al = h.block_cap + 8;
	a.stages = h.stages;
	a.stage_bytes = (int) (ceil_div((int64_t) a.cap_al * 12, 128) * 128);
	a.exact = h.desc.exact;
	a.err = h.d_err;
	a.wait_budget = wait_budget_cycles(h.desc.wait_limit_us);
	a.hold = (h.desc.debug_flags & SPMV_DEBUG_WITHHOLD_HANDOFF) != 0;
	if (fmt == SPMV_FMT_CSR_NAIVE || fmt == SPMV_FMT_CSR_VEC) {
		a.ptr = h.d_rp;
		a.cols = h.d_ci;
		a.vals = h.d_v;
	} else if (fmt == SPMV_FMT_SELL_C_S) {
		a.ptr = h.d_sptr32;
		a.cols = h.d_scols;
		a.vals = h.d_svals;
		a.V = h.desc.sellcs_c;
		a.ymap = h.d_order;
	} else {
		a.ptr = h.d_rcp;
		a.cols = h.d_ja;
		a.vals = h.d_a;
		a.V = h.desc.vec_len;
		a.ymap = (fmt == SPMV_FMT_SELL_SORTED) ? h.d_rev : nullptr;
	}
	StagedFn kern = pick_staged(h);
	if (h.exec_kernel == 3) {
		kern = pick_pipe(h);
		a.stage_bytes = pipe_stage_bytes(fmt, a.cap_al);
	} else if (h.exec_kernel == 4) {
		kern = pick_ws(h);
		a.stage_bytes = ws_stage_layout(fmt, a.cap_al, false, &a.cols_off);
		a.row_threads = h.row_threads;
		a.ranges = h.d_cta_ranges;
		a.pinfo = h.d_pinfo;
		a.pcols = h.d_pcols;
	} else if (h.exec_kernel == 8) {
		kern = pick_ws_tiled(h);
		a.cols = h.d_tcols;
		a.stage_bytes = ws_stage_layout(fmt, a.cap_al, true, &a.cols_off);
		a.row_threads = h.row_threads;
		a.ranges = h.d_cta_ranges;
	}
	kern<<<h.grid, h.threads, h.smem_bytes, s>>>(a);
	SPMV_CUDA_TRY(cudaGetLastError());
	return SPMV_OK;
}

}  // namespace spmv
