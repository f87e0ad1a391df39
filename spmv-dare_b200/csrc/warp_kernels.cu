// Warp-autonomous staged SpMV (kernels 2, 6 and 9; options beside the warp-specialised defaults).
//
// Every warp owns a contiguous run of "chunks" of the matrix and its own pipeline in
// shared memory: a ring of bulk-copy stages (cp.async.bulk global->shared, completion on a
// per-warp mbarrier), a gather buffer, and no CTA-wide barrier at all -- a warp waits only
// for its own copies and its own 32 rows.  Per chunk:
//   1. the chunk's stored entries (values, columns: one contiguous range) have landed;
//   2. the 32 lanes gather x for every entry (coalesced when a row's columns are clustered)
//      -- csr_naive stores the rounded product v*x in place, the FMA formats keep x;
//   3. lane r sums its row (or slice lane) from shared memory in the reference format's
//      own operation order, so y is bit-identical to the reference;
//   4. lane 0 refills the stage with the chunk `stages` ahead.
// A row / slice larger than one chunk spans consecutive chunks of the same warp and its
// accumulators live in registers across them (flags CONT_PREV / CONT_NEXT).
#include <algorithm>
#include <vector>

#include "internal.h"
#include "primitives.cuh"

namespace spmv {

namespace {

constexpr int WARP_CTA_THREADS = 128;         // 4 independent warps per CTA
constexpr uint32_t CONT_PREV = 1, CONT_NEXT = 2;

struct WarpArgs {
	const WarpChunk * chunks;
	const int32_t * warp_begin;    // chunk range of warp w: [warp_begin[w], warp_begin[w+1])
	int64_t nwarps;
	const int32_t * ptr;           // CSR row_ptr or slice pointer
	const int32_t * cols;
	const double * vals;
	const int32_t * ymap;
	const double * x;
	double * y;
	int64_t m;
	int V;
	int cap_al;                    // entries per stage buffer
	int stages;
	int stage_bytes;
	int warp_bytes;                // shared memory per warp
	int xbuf_bytes;                // gather buffer per warp (0 when products are stored in place)
	int * err;
};

template <int L>
__device__ __forceinline__ double lanes_reduce_w(const double * s)
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

__device__ __forceinline__ void warp_issue(const WarpArgs & a, int64_t c, uint8_t * wsm, uint64_t * bar, int s)
{
	const WarpChunk d = a.chunks[c];
	if (d.elems == 0) {
		mbar_arrive(bar);
		return;
	}
	const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
	const int64_t e1 = ((int64_t) d.elem0 + d.elems + 3) & ~(int64_t) 3;
	const uint32_t cnt = (uint32_t) (e1 - e0);
	double * sv = reinterpret_cast<double *>(wsm + (size_t) s * a.stage_bytes);
	int32_t * sc = reinterpret_cast<int32_t *>(wsm + (size_t) s * a.stage_bytes + (size_t) a.cap_al * 8);
	fence_proxy_async_smem();
	mbar_arrive_expect_tx(bar, cnt * 12u);
	bulk_g2s(sv, a.vals + e0, cnt * 8u, bar);
	bulk_g2s(sc, a.cols + e0, cnt * 4u, bar);
}

// OWNX (slices only): no gather pass and no x buffer -- each lane loads the x entries of
// its own slice row inside its FMA loop (8 independent loads in flight), so a warp's
// shared memory holds only its bulk-copy ring and more warps fit on an SM.
template <Kind K, Arith A, int L, bool YMAP, bool OWNX = false>
__global__ void __launch_bounds__(WARP_CTA_THREADS) warp_kernel(WarpArgs a)
{
	extern __shared__ __align__(128) uint8_t smem[];
	const int lane = threadIdx.x & 31;
	const int wib = threadIdx.x >> 5;
	const int64_t w = (int64_t) blockIdx.x * (blockDim.x >> 5) + wib;
	uint8_t * wsm = smem + (size_t) wib * a.warp_bytes;
	double * xb = reinterpret_cast<double *>(wsm + (size_t) a.stages * a.stage_bytes);
	uint64_t * bars = reinterpret_cast<uint64_t *>(wsm + (size_t) a.stages * a.stage_bytes + (size_t) a.xbuf_bytes);
	if (w >= a.nwarps)
		return;
	const int64_t cb = a.warp_begin[w], ce = a.warp_begin[w + 1];
	if (cb >= ce)
		return;
	if (lane == 0) {
		for (int s = 0; s < a.stages; s++)
			mbar_init(&bars[s], 1);
		mbar_fence_init();
	}
	__syncwarp();
	if (lane == 0)
		for (int s = 0; s < a.stages && cb + s < ce; s++)
			warp_issue(a, cb + s, wsm, &bars[s], s);

	double acc = 0.0;          // a lane's running sum across chunks of one long unit
	double ln[L];
	#pragma unroll
	for (int l = 0; l < L; l++)
		ln[l] = 0.0;
	int s = 0;
	uint32_t parity = 0;
	for (int64_t c = cb; c < ce; c++) {
		const WarpChunk d = a.chunks[c];
		bool ok = mbar_wait_bounded(&bars[s], parity, kWaitBudgetCycles);
		if (!__all_sync(0xffffffffu, ok)) {
			if (lane == 0) {
				dev_flag_error(a.err, DEV_ERR_TIMEOUT);
				// lane 0 issued the copies of chunks c .. c + stages - 1
				drain_ring(bars, a.stages, s, parity, (int) (ce - c < a.stages ? ce - c : a.stages), kWaitBudgetCycles);
			}
			return;
		}
		const int64_t e0 = (int64_t) d.elem0 & ~(int64_t) 3;
		const int off = (int) (d.elem0 - e0);
		double * sv = reinterpret_cast<double *>(wsm + (size_t) s * a.stage_bytes) + off;
		const int32_t * sc = reinterpret_cast<const int32_t *>(wsm + (size_t) s * a.stage_bytes + (size_t) a.cap_al * 8) + off;
		double * xs = xb + off;
		if (!OWNX) {
			// gather x for all entries of the chunk
			#pragma unroll 8
			for (int e = lane; e < d.elems; e += 32) {
				const double xv = ldg(a.x + sc[e]);
				if (A == Arith::SEQ_SPLIT)
					sv[e] = __dmul_rn(sv[e], xv);
				else
					xs[e] = xv;
			}
			__syncwarp();
		}
		const bool long_unit = (d.flags & (CONT_PREV | CONT_NEXT)) != 0;
		if (K == Kind::CSR) {
			if (!long_unit) {
				if (lane < d.units) {
					const int64_t r = (int64_t) d.unit0 + lane;
					const int js = a.ptr[r] - d.elem0, je = a.ptr[r + 1] - d.elem0;
					double sum = 0.0;
					if (A == Arith::SEQ_SPLIT) {
						#pragma unroll 4
						for (int j = js; j < je; j++)
							sum = __dadd_rn(sum, sv[j]);
					} else if (A == Arith::SEQ_FMA) {
						#pragma unroll 4
						for (int j = js; j < je; j++)
							sum = __fma_rn(sv[j], xs[j], sum);
					} else {
						double q[L];
						#pragma unroll
						for (int l = 0; l < L; l++)
							q[l] = 0.0;
						const int jv = js + ((je - js) & ~(L - 1));
						for (int j = js; j < jv; j += L) {
							#pragma unroll
							for (int l = 0; l < L; l++)
								q[l] = __fma_rn(sv[j + l], xs[j + l], q[l]);
						}
						sum = lanes_reduce_w<L>(q);
						for (int j = jv; j < je; j++)
							sum = __dadd_rn(sum, __dmul_rn(sv[j], xs[j]));
					}
					a.y[r] = sum;
				}
			} else if (A == Arith::LANES_FMA) {
				// one long row, csr_vec order: lane l < L keeps accumulator l (entries j with
				// (j - row start) % L == l below the vector bound), lane 0 adds the tail
				const int64_t r = d.unit0;
				const int64_t js = a.ptr[r], je = a.ptr[r + 1];
				const int64_t jv = js + ((je - js) & ~(int64_t) (L - 1));
				if (!(d.flags & CONT_PREV)) {
					acc = 0.0;
					ln[0] = 0.0;
				}
				if (lane < L) {
					for (int e = 0; e < d.elems; e++) {
						const int64_t j = (int64_t) d.elem0 + e;
						if (j < jv && (int) ((j - js) & (L - 1)) == lane)
							ln[0] = __fma_rn(sv[e], xs[e], ln[0]);
					}
				}
				if (!(d.flags & CONT_NEXT) || (int64_t) d.elem0 + d.elems > jv) {
					// the lane sums are final once the chunk passes the vector bound
					double q[L];
					#pragma unroll
					for (int l = 0; l < L; l++)
						q[l] = __shfl_sync(0xffffffffu, ln[0], l);
					if (lane == 0) {
						if ((int64_t) d.elem0 <= jv)
							acc = lanes_reduce_w<L>(q);
						for (int e = 0; e < d.elems; e++) {
							const int64_t j = (int64_t) d.elem0 + e;
							if (j >= jv)
								acc = __dadd_rn(acc, __dmul_rn(sv[e], xs[e]));
						}
						if (!(d.flags & CONT_NEXT))
							a.y[r] = acc;
					}
				}
			} else if (lane == 0) {
				// one long row: lane 0 continues the row's sum in the reference order
				const int64_t r = d.unit0;
				if (!(d.flags & CONT_PREV))
					acc = 0.0;
				for (int e = 0; e < d.elems; e++) {
					if (A == Arith::SEQ_SPLIT)
						acc = __dadd_rn(acc, sv[e]);
					else
						acc = __fma_rn(sv[e], xs[e], acc);
				}
				if (!(d.flags & CONT_NEXT))
					a.y[r] = acc;
			}
		} else {
			const int V = a.V;
			if (!long_unit) {
				if (lane < d.units * V) {
					const int64_t sl = (int64_t) d.unit0 + lane / V;
					const int r = lane % V;
					const int64_t row = sl * V + r;
					if (row < a.m) {
						const int ks = a.ptr[sl] - d.elem0 + r;
						const int wd = (a.ptr[sl + 1] - a.ptr[sl]) / V;
						double sum = 0.0;
						if (OWNX) {
							#pragma unroll 8
							for (int k = 0; k < wd; k++)
								sum = __fma_rn(sv[ks + k * V], ldg(a.x + sc[ks + k * V]), sum);
						} else {
							#pragma unroll 4
							for (int k = 0; k < wd; k++)
								sum = __fma_rn(sv[ks + k * V], xs[ks + k * V], sum);
						}
						a.y[YMAP ? a.ymap[row] : row] = sum;
					}
				}
			} else if (lane < V) {
				// one long slice in column chunks: lane r continues row r of the slice
				if (!(d.flags & CONT_PREV))
					acc = 0.0;
				const int kn = d.elems / V;
				if (OWNX) {
					#pragma unroll 8
					for (int k = 0; k < kn; k++)
						acc = __fma_rn(sv[k * V + lane], ldg(a.x + sc[k * V + lane]), acc);
				} else {
					for (int k = 0; k < kn; k++)
						acc = __fma_rn(sv[k * V + lane], xs[k * V + lane], acc);
				}
				if (!(d.flags & CONT_NEXT)) {
					const int64_t row = (int64_t) d.unit0 * V + lane;
					if (row < a.m)
						a.y[YMAP ? a.ymap[row] : row] = acc;
				}
			}
		}
		__syncwarp();
		if (lane == 0 && c + a.stages < ce)
			warp_issue(a, c + a.stages, wsm, &bars[s], s);
		if (++s == a.stages) {
			s = 0;
			parity ^= 1u;
		}
	}
}


// ------------------------------------------------------------------ tiled warp kernel (kernel 9)
// 32-row slices whose column indices are stored row-major in tiles of 8 slice columns
// (tile_cols_kernel).  A warp owns its slices as kernel 6 does, but loads x in the tiled
// order: load q of lane L is tile entry q * 32 + L, row 4q + L / 8, column L % 8, so a warp
// request covers 4 rows x 8 neighbouring columns (about 7 distinct sectors on the 4M-row
// matrix, against 24 for 32 rows x 1 column).  An 8 x 8 transpose between the lanes of
// each group of 8 and their registers (three shfl.xor stages) then leaves x(row, t8 + j) in
// register j of lane L, row = 4 (L % 8) + L / 8, which sums its row from the column-major
// values in the stage: no x buffer in shared memory.  The slice's narrower last tile
// (width tw < 8, rows at r * tw) is loaded row by row.
__device__ __forceinline__ void transpose8(double (&X)[8], int lane)
{
	#pragma unroll
	for (int b = 1; b < 8; b <<= 1) {
		const bool up = (lane & b) != 0;
		#pragma unroll
		for (int q = 0; q < 8; q++) {
			if (q & b)
				continue;
			const double send = up ? X[q] : X[q | b];
			const double recv = __shfl_xor_sync(0xffffffffu, send, b);
			if (up)
				X[q] = recv;
			else
				X[q | b] = recv;
		}
	}
}

template <bool YMAP>
__global__ void __launch_bounds__(WARP_CTA_THREADS) tiled_warp_kernel(WarpArgs a)
{
	extern __shared__ __align__(128) uint8_t smem[];
	const int lane = threadIdx.x & 31;
	const int wib = threadIdx.x >> 5;
	const int64_t w = (int64_t) blockIdx.x * (blockDim.x >> 5) + wib;
	uint8_t * wsm = smem + (size_t) wib * a.warp_bytes;
	uint64_t * bars = reinterpret_cast<uint64_t *>(wsm + (size_t) a.stages * a.stage_bytes);
	if (w >= a.nwarps)
		return;
	const int64_t cb = a.warp_begin[w], ce = a.warp_begin[w + 1];
	if (cb >= ce)
		return;
	if (lane == 0) {
		for (int s = 0; s < a.stages; s++)
			mbar_init(&bars[s], 1);
		mbar_fence_init();
	}
	__syncwarp();
	if (lane == 0)
		for (int s = 0; s < a.stages && cb + s < ce; s++)
			warp_issue(a, cb + s, wsm, &bars[s], s);
	const int R = 4 * (lane & 7) + (lane >> 3);     // this lane's slice row
	double acc = 0.0;
	int s = 0;
	uint32_t parity = 0;
	for (int64_t c = cb; c < ce; c++) {
		const WarpChunk d = a.chunks[c];
		const bool ok = mbar_wait_bounded(&bars[s], parity, kWaitBudgetCycles);
		if (!__all_sync(0xffffffffu, ok)) {
			if (lane == 0) {
				dev_flag_error(a.err, DEV_ERR_TIMEOUT);
				// lane 0 issued the copies of chunks c .. c + stages - 1
				drain_ring(bars, a.stages, s, parity, (int) (ce - c < a.stages ? ce - c : a.stages), kWaitBudgetCycles);
			}
			return;
		}
		// chunks start at slice starts or tile boundaries (multiples of 32 entries): off == 0
		const double * sv = reinterpret_cast<const double *>(wsm + (size_t) s * a.stage_bytes);
		const int32_t * sc = reinterpret_cast<const int32_t *>(wsm + (size_t) s * a.stage_bytes + (size_t) a.cap_al * 8);
		if (!(d.flags & CONT_PREV))
			acc = 0.0;
		const int wd = d.elems >> 5;
		const int full = wd & ~7;
		int t8 = 0;
		for (; t8 + 16 <= full; t8 += 16) {                 // two tiles' loads in flight
			double X[8], Y[8];
			#pragma unroll
			for (int q = 0; q < 8; q++) {
				X[q] = ldg(a.x + sc[t8 * 32 + q * 32 + lane]);
				Y[q] = ldg(a.x + sc[(t8 + 8) * 32 + q * 32 + lane]);
			}
			transpose8(X, lane);
			#pragma unroll
			for (int j = 0; j < 8; j++)
				acc = __fma_rn(sv[(t8 + j) * 32 + R], X[j], acc);
			transpose8(Y, lane);
			#pragma unroll
			for (int j = 0; j < 8; j++)
				acc = __fma_rn(sv[(t8 + 8 + j) * 32 + R], Y[j], acc);
		}
		if (t8 < full) {
			double X[8];
			#pragma unroll
			for (int q = 0; q < 8; q++)
				X[q] = ldg(a.x + sc[t8 * 32 + q * 32 + lane]);
			transpose8(X, lane);
			#pragma unroll
			for (int j = 0; j < 8; j++)
				acc = __fma_rn(sv[(t8 + j) * 32 + R], X[j], acc);
			t8 += 8;
		}
		if (t8 < wd) {                                      // the slice's narrower last tile
			const int tw = wd - t8;
			double X[8];
			#pragma unroll
			for (int j = 0; j < 8; j++)
				X[j] = j < tw ? ldg(a.x + sc[t8 * 32 + R * tw + j]) : 0.0;
			#pragma unroll
			for (int j = 0; j < 8; j++)
				if (j < tw)
					acc = __fma_rn(sv[(t8 + j) * 32 + R], X[j], acc);
		}
		if (!(d.flags & CONT_NEXT)) {
			const int64_t row = (int64_t) d.unit0 * 32 + R;
			if (row < a.m)
				a.y[YMAP ? a.ymap[row] : row] = acc;
		}
		__syncwarp();
		if (lane == 0 && c + a.stages < ce)
			warp_issue(a, c + a.stages, wsm, &bars[s], s);
		if (++s == a.stages) {
			s = 0;
			parity ^= 1u;
		}
	}
}

// ------------------------------------------------------------------ register-tiled slice kernel (kernel 10)
// 32-row slices (SELL-C-sigma with C = 32, or SELL with V = 32) over the same tiled column
// indices, without shared memory: a warp claims work items (runs of slices, the heaviest
// ones first) from a queue and sums each slice's 32 rows straight from global memory.  Per
// tile of 8 slice columns, lane L loads 8 tiled column indices (tile entry q * 32 + L: four
// 128-byte requests' worth of one contiguous 1 KB) and the 8 values of its row
// R = 4 (L % 8) + L / 8 (column-major: for each column the 32 lanes read one 256-byte
// segment), both with streaming loads (evict first, so x keeps its place in L2); the
// next tile's indices and values are requested before this tile's x, so DRAM latency
// overlaps the x gather and the FMA chain.  x is transposed between lanes as in kernel 9
// and each lane runs its row's FMA chain in column order, padding included: y is the
// reference's bit for bit.  No shared memory, so occupancy is set by registers alone.
struct TileRegArgs {
	const int2 * items;            // work items: slice ranges [x, y)
	int64_t nitems;
	const int32_t * sptr;          // slice pointers (32-bit)
	const int32_t * tcols;         // column indices, row-major in tiles of 8 slice columns
	const double * vals;           // values, column-major per slice
	const int32_t * ymap;          // row map (row_order / rev_permutation) or null
	const double * x;
	double * y;
	int64_t m;
	unsigned int * queue;          // [0] next item, [1] warps done: zero at launch, reset on exit
	unsigned int total_warps;
	int pf_dist;                   // line prefetch distance in entries (a multiple of 256)
	int64_t heavy_min;             // items of one slice this long prefetch 4 x pf_dist ahead
};

constexpr int TILE_REG_THREADS = 256;

__device__ __forceinline__ void tile_load(const TileRegArgs & a, int64_t t0, int lane, int R, int32_t (&c)[8],
		double (&v)[8])
{
	#pragma unroll
	for (int q = 0; q < 8; q++)
		c[q] = __ldcs(a.tcols + t0 + q * 32 + lane);
	#pragma unroll
	for (int j = 0; j < 8; j++)
		v[j] = __ldcs(a.vals + t0 + j * 32 + R);
}

// The prefetch forms of kernel 10 (template PF): 0 none; 1 / 2 the cache lines of the tile
// `dist` entries ahead (two tiles by default, eight in a heavy slice; across slice boundaries:
// an item's slices are contiguous; never past the item's end e_end) requested into L1 / L2 by
// one prefetch per lane (lanes 0-15 the 2 KB of values, 16-23 the 1 KB of columns), so that
// tile's register loads find them close; 3 / 4 the same into L1 / L2 with every item claimed
// one ahead and its first two tiles prefetched.  2 is the default.
template <int PF>
__device__ __forceinline__ void tile_prefetch(const TileRegArgs & a, int64_t t0, int64_t e_end, int lane, int dist)
{
	const int64_t p = t0 + dist;
	if (PF == 0 || lane >= 24 || p + 256 > e_end)
		return;
	const void * addr = lane < 16 ? (const void *) (a.vals + p + lane * 16) : (const void *) (a.tcols + p + (lane - 16) * 32);
	if (PF == 2 || PF == 4)
		asm volatile("prefetch.global.L2 [%0];" ::"l"(addr));
	else
		asm volatile("prefetch.global.L1 [%0];" ::"l"(addr));
}

// PF 3 / 4: the first two tiles of a claimed item asked of L1 / L2 (lanes 0-31: the 4 KB of
// values, 32 lines; lanes 0-15: the 2 KB of columns), for an item claimed one ahead of the one
// being summed.
template <int PF>
__device__ __forceinline__ void item_head_prefetch(const TileRegArgs & a, int64_t e0, int64_t e_end, int lane)
{
	if (e0 + 512 > e_end)
		return;
	if (PF == 4) {
		asm volatile("prefetch.global.L2 [%0];" ::"l"(a.vals + e0 + lane * 16));
		if (lane < 16)
			asm volatile("prefetch.global.L2 [%0];" ::"l"(a.tcols + e0 + lane * 32));
	} else {
		asm volatile("prefetch.global.L1 [%0];" ::"l"(a.vals + e0 + lane * 16));
		if (lane < 16)
			asm volatile("prefetch.global.L1 [%0];" ::"l"(a.tcols + e0 + lane * 32));
	}
}

template <int PF>
__device__ __forceinline__ void tile_reg_slice(const TileRegArgs & a, int64_t sl, int64_t e_end, int lane, int R,
		int dist)
{
	const int64_t b = a.sptr[sl];
	const int W = (int) (((int64_t) a.sptr[sl + 1] - b) >> 5);
	const int nt = W >> 3, rem = W & 7;
	double acc = 0.0;
	int32_t c[8], cn[8];
	double v[8], vn[8];
	if (nt > 0)
		tile_load(a, b, lane, R, c, v);
	for (int t = 0; t < nt; t++) {
		tile_prefetch<PF>(a, b + (int64_t) t * 256, e_end, lane, dist);
		if (t + 1 < nt)
			tile_load(a, b + (int64_t) (t + 1) * 256, lane, R, cn, vn);
		double X[8];
		#pragma unroll
		for (int q = 0; q < 8; q++)
			X[q] = __ldg(a.x + c[q]);
		transpose8(X, lane);
		#pragma unroll
		for (int j = 0; j < 8; j++)
			acc = __fma_rn(v[j], X[j], acc);
		#pragma unroll
		for (int j = 0; j < 8; j++) {
			c[j] = cn[j];
			v[j] = vn[j];
		}
	}
	if (rem > 0) {                               // the narrower last tile: rows at R * rem
		const int64_t t0 = b + (int64_t) nt * 256;
		double X[8], vv[8];
		#pragma unroll
		for (int j = 0; j < 8; j++) {
			if (j < rem) {
				X[j] = __ldg(a.x + __ldcs(a.tcols + t0 + R * rem + j));
				vv[j] = __ldcs(a.vals + t0 + j * 32 + R);
			}
		}
		#pragma unroll
		for (int j = 0; j < 8; j++)
			if (j < rem)
				acc = __fma_rn(vv[j], X[j], acc);
	}
	const int64_t row = sl * 32 + R;
	if (row < a.m)
		a.y[a.ymap ? (int64_t) a.ymap[row] : row] = acc;
}

template <int PF>
__global__ void __launch_bounds__(TILE_REG_THREADS, 2) tile_reg_kernel(TileRegArgs a)
{
	const int lane = threadIdx.x & 31;
	const int R = 4 * (lane & 7) + (lane >> 3);
	if (PF == 3 || PF == 4) {
		// the next item claimed while this one is summed, its head prefetched
		unsigned int it = 0;
		if (lane == 0)
			it = atomicAdd(&a.queue[0], 1u);
		it = __shfl_sync(0xffffffffu, it, 0);
		while ((int64_t) it < a.nitems) {
			unsigned int nx = 0;
			if (lane == 0)
				nx = atomicAdd(&a.queue[0], 1u);
			nx = __shfl_sync(0xffffffffu, nx, 0);
			if ((int64_t) nx < a.nitems) {
				const int2 q = a.items[nx];
				item_head_prefetch<PF>(a, a.sptr[q.x], a.sptr[q.y], lane);
			}
			const int2 r = a.items[it];
			const int64_t e_end = a.sptr[r.y];
			// a heavy slice is one warp's long sequential stream: its lines go four times as
			// far ahead (the SpMV waits on the last such item to finish)
			const int dist = (r.y - r.x == 1 && e_end - a.sptr[r.x] >= a.heavy_min) ? 4 * a.pf_dist : a.pf_dist;
			for (int64_t sl = r.x; sl < r.y; sl++)
				tile_reg_slice<PF>(a, sl, e_end, lane, R, dist);
			it = nx;
		}
	} else {
		for (;;) {
			unsigned int it = 0;
			if (lane == 0)
				it = atomicAdd(&a.queue[0], 1u);
			it = __shfl_sync(0xffffffffu, it, 0);
			if ((int64_t) it >= a.nitems)
				break;
			const int2 r = a.items[it];
			const int64_t e_end = a.sptr[r.y];
			// a heavy slice is one warp's long sequential stream: its lines go four times as
			// far ahead (the SpMV waits on the last such item to finish)
			const int dist = (r.y - r.x == 1 && e_end - a.sptr[r.x] >= a.heavy_min) ? 4 * a.pf_dist : a.pf_dist;
			for (int64_t sl = r.x; sl < r.y; sl++)
				tile_reg_slice<PF>(a, sl, e_end, lane, R, dist);
		}
	}
	// every warp has made its last claim before it counts itself done: the last one to
	// finish puts the queue back to zero for the next launch
	if (lane == 0 && atomicAdd(&a.queue[1], 1u) == a.total_warps - 1) {
		atomicExch(&a.queue[0], 0u);
		atomicExch(&a.queue[1], 0u);
	}
}

using WarpFn = void (*)(WarpArgs);

WarpFn pick_warp(const Handle & h)
{
	const int fmt = h.desc.format;
	if (fmt == SPMV_FMT_CSR_NAIVE)
		return warp_kernel<Kind::CSR, Arith::SEQ_SPLIT, 1, false>;
	if (fmt == SPMV_FMT_CSR_VEC) {
		switch (h.desc.vec_len) {
		case 1: return warp_kernel<Kind::CSR, Arith::LANES_FMA, 1, false>;
		case 2: return warp_kernel<Kind::CSR, Arith::LANES_FMA, 2, false>;
		case 4: return warp_kernel<Kind::CSR, Arith::LANES_FMA, 4, false>;
		case 8: return warp_kernel<Kind::CSR, Arith::LANES_FMA, 8, false>;
		case 16: return warp_kernel<Kind::CSR, Arith::LANES_FMA, 16, false>;
		}
		return nullptr;
	}
	if (h.exec_kernel == 9)
		return fmt == SPMV_FMT_SELL ? tiled_warp_kernel<false> : tiled_warp_kernel<true>;
	const bool own = h.exec_kernel == 6;
	if (fmt == SPMV_FMT_SELL)
		return own ? warp_kernel<Kind::SLICED, Arith::SEQ_FMA, 1, false, true>
		           : warp_kernel<Kind::SLICED, Arith::SEQ_FMA, 1, false>;
	if (fmt == SPMV_FMT_SELL_SORTED || fmt == SPMV_FMT_SELL_C_S)
		return own ? warp_kernel<Kind::SLICED, Arith::SEQ_FMA, 1, true, true>
		           : warp_kernel<Kind::SLICED, Arith::SEQ_FMA, 1, true>;
	return nullptr;
}

// ------------------------------------------------------------------ chunk table
constexpr int TILE_UNITS = 1024;

// Chunks of one tile of units: normal chunks pack whole units (at most 32 rows and `cap`
// entries); a unit larger than `cap` is cut into consecutive chunks (CSR: runs of entries;
// slices: runs of whole slice columns, in multiples of `gran` columns) flagged CONT_PREV /
// CONT_NEXT.
template <bool WRITE>
__global__ void warp_chunks_kernel(const int32_t * P, int64_t U, int V, int gran, int cap, int64_t * counts,
		const int64_t * offs, WarpChunk * out)
{
	int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	int64_t u = t * TILE_UNITS;
	if (u >= U)
		return;
	const int64_t end = u + TILE_UNITS < U ? u + TILE_UNITS : U;
	const int max_units = 32 / V;
	int64_t nb = 0;
	const int64_t o = WRITE ? offs[t] : 0;
	while (u < end) {
		const int64_t len = (int64_t) P[u + 1] - P[u];
		if (len > cap) {
			const int64_t step = (V == 1) ? cap : (int64_t) (cap / (V * gran)) * V * gran;
			for (int64_t c0 = 0; c0 < len; c0 += step) {
				const int64_t cl = (len - c0) < step ? (len - c0) : step;
				if (WRITE) {
					WarpChunk d;
					d.unit0 = (int32_t) u;
					d.units = 1;
					d.flags = (uint16_t) ((c0 > 0 ? CONT_PREV : 0) | (c0 + cl < len ? CONT_NEXT : 0));
					d.elem0 = (int32_t) (P[u] + c0);
					d.elems = (int32_t) cl;
					out[o + nb] = d;
				}
				nb++;
			}
			u++;
			continue;
		}
		const int64_t start = u;
		const int64_t e0 = P[u];
		while (u < end && u - start < max_units && (int64_t) P[u + 1] - e0 <= cap)
			u++;
		if (WRITE) {
			WarpChunk d;
			d.unit0 = (int32_t) start;
			d.units = (uint16_t) (u - start);
			d.flags = 0;
			d.elem0 = (int32_t) e0;
			d.elems = (int32_t) ((int64_t) P[u] - e0);
			out[o + nb] = d;
		}
		nb++;
	}
	if (!WRITE)
		counts[t] = nb;
}

// Work estimate of a chunk: the bytes it stages plus a fixed cost; a chunk of a long unit
// is summed by one lane (or the V lanes of a slice) in a dependent chain, so its entries
// cost as much as LONG_FACTOR parallel ones -- long rows are spread over many warps.
constexpr int64_t LONG_FACTOR = 24;

__global__ void chunk_weights_kernel(const WarpChunk * ch, int64_t n, int V, int64_t * wgt)
{
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const WarpChunk d = ch[i];
	int64_t w = (int64_t) d.elems * 12 + 64;
	if (d.flags & (CONT_PREV | CONT_NEXT))
		w = (int64_t) d.elems * 12 * LONG_FACTOR / (V < 32 ? V : 32) + 64;
	wgt[i] = w;
}

// Warp w starts at the first chunk whose weight prefix reaches w/W of the total and which
// does not continue a previous chunk (long units stay with one warp).
__global__ void warp_ranges_kernel(const WarpChunk * ch, const int64_t * prefix, int64_t n, int64_t W, int32_t * begin)
{
	int64_t w = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (w > W)
		return;
	if (w == 0) {
		begin[0] = 0;
		return;
	}
	if (w == W) {
		begin[W] = (int32_t) n;
		return;
	}
	const int64_t total = prefix[n];
	const int64_t target = (total * w) / W;
	int64_t lo = 0, hi = n;
	while (lo < hi) {
		int64_t mid = (lo + hi) >> 1;
		if (prefix[mid] < target)
			lo = mid + 1;
		else
			hi = mid;
	}
	while (lo < n && (ch[lo].flags & CONT_PREV))
		lo++;
	begin[w] = (int32_t) lo;
}

// Bytes of a warp's x gather buffer: none when csr_naive stores its products in place or
// when the slice rows load their own x (kernel 6).
int warp_xbuf_bytes(const Handle & h, int cap_al)
{
	const bool slices = h.desc.format == SPMV_FMT_SELL || h.desc.format == SPMV_FMT_SELL_SORTED ||
			h.desc.format == SPMV_FMT_SELL_C_S;
	return (h.desc.format == SPMV_FMT_CSR_NAIVE || ((h.exec_kernel == 6 || h.exec_kernel == 9) && slices)) ? 0
	                                                                                           : cap_al * 8;
}

}  // namespace

int warp_geometry(Handle & h)
{
	// fit 4 warps' pipelines in a CTA's shared memory: fewer stages, then a smaller chunk
	for (;;) {
		const int cap_al = h.block_cap + 8;
		const int stage_bytes = (int) (ceil_div((int64_t) cap_al * 12, 128) * 128);
		const int xbuf = warp_xbuf_bytes(h, cap_al);
		h.warp_bytes = (int) (ceil_div((int64_t) h.stages * stage_bytes + xbuf + 8 * h.stages, 128) * 128);
		h.smem_bytes = (size_t) h.warp_bytes * (WARP_CTA_THREADS / 32);
		if (h.smem_bytes <= 220 * 1024)
			break;
		if (h.stages > 2)
			h.stages--;
		else if (h.block_cap > 64)
			h.block_cap = ((h.block_cap / 2) + 7) & ~7;
		else {
			set_error(SPMV_ERR_ARG, "warp pipeline does not fit in shared memory");
			return SPMV_ERR_ARG;
		}
	}
	WarpFn kern = pick_warp(h);
	if (!kern) {
		set_error(SPMV_ERR_ARG, "no warp kernel for format %d", h.desc.format);
		return SPMV_ERR_ARG;
	}
	SPMV_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) h.smem_bytes));
	int per_sm = h.desc.ctas_per_sm;
	if (per_sm <= 0) {
		SPMV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARP_CTA_THREADS, h.smem_bytes));
		if (per_sm < 1)
			per_sm = 1;
	}
	h.grid = h.num_sms * per_sm;
	return SPMV_OK;
}

// Builds the chunk table over the unit pointer P (CSR row_ptr, V = 1; or slice pointer,
// V = slice height dividing 32) and the per-warp chunk ranges.
int build_warp_chunks(Handle & h, const int32_t * d_P, int64_t U, int V)
{
	cudaStream_t s = h.stream;
	// kernel 9 cuts long slices at 8-column tile boundaries
	const int gran = h.exec_kernel == 9 ? 8 : 1;
	h.block_cap = h.desc.block_nnz > 0 ? h.desc.block_nnz : 512;
	if (V > 1 && h.block_cap < V * gran)
		h.block_cap = V * gran;
	h.block_cap = (h.block_cap + 7) & ~7;
	h.stages = h.desc.stages > 0 ? h.desc.stages : (h.exec_kernel == 6 || h.exec_kernel == 9 ? 3 : 2);
	SPMV_TRY(warp_geometry(h));
	int64_t tiles = ceil_div(U, TILE_UNITS);
	int64_t nch = 0;
	if (tiles > 0) {
		DevBuf counts, offs;
		SPMV_TRY(counts.alloc(tiles * sizeof(int64_t), s));
		SPMV_TRY(offs.alloc((tiles + 1) * sizeof(int64_t), s));
		unsigned g = (unsigned) ceil_div(tiles, 128);
		warp_chunks_kernel<false><<<g, 128, 0, s>>>(d_P, U, V, gran, h.block_cap, counts.as<int64_t>(), nullptr, nullptr);
		SPMV_CUDA_TRY(cudaGetLastError());
		SPMV_TRY(scan_exclusive(counts.as<int64_t>(), offs.as<int64_t>(), tiles, s));
		SPMV_CUDA_TRY(cudaMemcpyAsync(&nch, offs.as<int64_t>() + tiles, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
		SPMV_CUDA_TRY(cudaStreamSynchronize(s));
		if (nch > INT32_MAX - 1) {
			set_error(SPMV_ERR_OVERFLOW, "too many chunks");
			return SPMV_ERR_OVERFLOW;
		}
		SPMV_TRY(h.alloc(&h.d_chunks, nch));
		warp_chunks_kernel<true><<<g, 128, 0, s>>>(d_P, U, V, gran, h.block_cap, nullptr, offs.as<int64_t>(), h.d_chunks);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	h.num_chunks = nch;
	int64_t W = (int64_t) h.grid * (WARP_CTA_THREADS / 32);
	h.num_warps = W;
	SPMV_TRY(h.alloc(&h.d_warp_begin, W + 1));
	if (nch == 0) {
		SPMV_CUDA_TRY(cudaMemsetAsync(h.d_warp_begin, 0, (W + 1) * sizeof(int32_t), s));
		return SPMV_OK;
	}
	DevBuf wgt, pre;
	SPMV_TRY(wgt.alloc(nch * sizeof(int64_t), s));
	SPMV_TRY(pre.alloc((nch + 1) * sizeof(int64_t), s));
	chunk_weights_kernel<<<(unsigned) ceil_div(nch, 256), 256, 0, s>>>(h.d_chunks, nch, V, wgt.as<int64_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(scan_exclusive(wgt.as<int64_t>(), pre.as<int64_t>(), nch, s));
	warp_ranges_kernel<<<(unsigned) ceil_div(W + 1, 256), 256, 0, s>>>(h.d_chunks, pre.as<int64_t>(), nch, W,
			h.d_warp_begin);
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	return SPMV_OK;
}

// Work items of kernel 10: slices of at least TILE_REG_HEAVY entries alone, the heaviest
// first; the others in matrix order, in runs of consecutive slices of about
// TILE_REG_ITEM entries (neighbouring rows keep x warm in L2; the line prefetch runs across
// the slices of an item); block_rows sets the item size in 256-entry tiles instead (the
// heavy threshold is twice the item size).  4,096 / 8,192 measured fastest on the 4M-row
// matrix with the L1 prefetch (0.213 ms; 2,048 / 4,096: 0.217, 8,192 / 16,384: 0.231).
constexpr int64_t TILE_REG_HEAVY = 8192, TILE_REG_ITEM = 4096;

int build_tile_reg(Handle & h, const int32_t * d_P, int64_t U, int V)
{
	if (V != 32) {
		set_error(SPMV_ERR_ARG, "kernel 10 takes slices of exactly 32 rows (got %d)", V);
		return SPMV_ERR_ARG;
	}
	cudaStream_t s = h.stream;
	std::vector<int32_t> P((size_t) U + 1);
	SPMV_CUDA_TRY(cudaMemcpyAsync(P.data(), d_P, (U + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	std::vector<int2> heavy, rest;
	const int64_t item = h.desc.block_rows > 0 ? (int64_t) h.desc.block_rows * 256 : TILE_REG_ITEM;
	const int64_t heavy_min = h.desc.block_rows > 0 ? 2 * item : TILE_REG_HEAVY;
	h.tile_heavy_min = heavy_min;
	int64_t u = 0;
	while (u < U) {
		const int64_t len = (int64_t) P[u + 1] - P[u];
		if (len >= heavy_min) {
			heavy.push_back(make_int2((int) u, (int) (u + 1)));
			u++;
			continue;
		}
		const int64_t u0 = u, e0 = P[u];
		while (u < U && (int64_t) P[u + 1] - P[u] < heavy_min && (int64_t) P[u] - e0 < item)
			u++;
		rest.push_back(make_int2((int) u0, (int) u));
	}
	std::stable_sort(heavy.begin(), heavy.end(), [&](const int2 & p, const int2 & q) {
		return P[p.x + 1] - P[p.x] > P[q.x + 1] - P[q.x];
	});
	heavy.insert(heavy.end(), rest.begin(), rest.end());
	h.num_items = (int64_t) heavy.size();
	SPMV_TRY(h.alloc(&h.d_items, h.num_items));
	if (h.num_items > 0)
		SPMV_CUDA_TRY(cudaMemcpyAsync(h.d_items, heavy.data(), h.num_items * sizeof(int2), cudaMemcpyHostToDevice, s));
	SPMV_TRY(h.alloc(&h.d_queue, 2));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_queue, 0, 2 * sizeof(unsigned int), s));
	int per_sm = h.desc.ctas_per_sm;
	if (per_sm <= 0) {
		SPMV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tile_reg_kernel<2>, TILE_REG_THREADS, 0));
		if (per_sm < 1)
			per_sm = 1;
	}
	h.grid = h.num_sms * per_sm;
	h.threads = TILE_REG_THREADS;
	h.smem_bytes = 0;
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	return SPMV_OK;
}

int launch_warp(Handle & h, const double * d_x, double * d_y, cudaStream_t s)
{
	if (h.exec_kernel == 10) {
		if (h.num_items == 0)
			return SPMV_OK;
		TileRegArgs a{};
		a.items = h.d_items;
		a.nitems = h.num_items;
		a.tcols = h.d_tcols;
		a.x = d_x;
		a.y = d_y;
		a.m = h.m;
		a.queue = h.d_queue;
		a.total_warps = (unsigned int) h.grid * (TILE_REG_THREADS / 32);
		// block_nnz: the line prefetch distance in entries (whole tiles; default two tiles)
		a.pf_dist = h.desc.block_nnz > 0 ? (int) (ceil_div(h.desc.block_nnz, 256) * 256) : 512;
		a.heavy_min = h.tile_heavy_min;
		if (h.desc.format == SPMV_FMT_SELL_C_S) {
			a.sptr = h.d_sptr32;
			a.vals = h.d_svals;
			a.ymap = h.d_order;
		} else {
			a.sptr = h.d_rcp;
			a.vals = h.d_a;
			a.ymap = h.desc.format == SPMV_FMT_SELL_SORTED ? h.d_rev : nullptr;
		}
		// default: the lines pf_dist entries ahead (4 x inside a heavy slice) prefetched into L2
		// (0.2109 ms on the 4M-row SELL-C-sigma matrix); stages 3: into L1 (0.2221); 5: into
		// L1, items claimed one ahead with their first two tiles prefetched (0.2130); 6: that
		// form into L2 (0.2130); 1: no prefetch (0.2350)
		if (h.desc.stages == 1)
			tile_reg_kernel<0><<<h.grid, TILE_REG_THREADS, 0, s>>>(a);
		else if (h.desc.stages == 3)
			tile_reg_kernel<1><<<h.grid, TILE_REG_THREADS, 0, s>>>(a);
		else if (h.desc.stages == 5)
			tile_reg_kernel<3><<<h.grid, TILE_REG_THREADS, 0, s>>>(a);
		else if (h.desc.stages == 6)
			tile_reg_kernel<4><<<h.grid, TILE_REG_THREADS, 0, s>>>(a);
		else
			tile_reg_kernel<2><<<h.grid, TILE_REG_THREADS, 0, s>>>(a);
		SPMV_CUDA_TRY(cudaGetLastError());
		return SPMV_OK;
	}
	if (h.num_chunks == 0)
		return SPMV_OK;
	const int fmt = h.desc.format;
	WarpArgs a{};
	a.chunks = h.d_chunks;
	a.warp_begin = h.d_warp_begin;
	a.nwarps = h.num_warps;
	a.x = d_x;
	a.y = d_y;
	a.m = h.m;
	a.cap_al = h.block_cap + 8;
	a.stages = h.stages;
	a.stage_bytes = (int) (ceil_div((int64_t) a.cap_al * 12, 128) * 128);
	a.warp_bytes = h.warp_bytes;
	a.xbuf_bytes = warp_xbuf_bytes(h, a.cap_al);
	a.err = h.d_err;
	if (fmt == SPMV_FMT_CSR_NAIVE || fmt == SPMV_FMT_CSR_VEC) {
		a.ptr = h.d_rp;
		a.cols = h.d_ci;
		a.vals = h.d_v;
		a.V = 1;
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
	if (h.exec_kernel == 9)
		a.cols = h.d_tcols;
	WarpFn kern = pick_warp(h);
	kern<<<h.grid, WARP_CTA_THREADS, h.smem_bytes, s>>>(a);
	SPMV_CUDA_TRY(cudaGetLastError());
	return SPMV_OK;
}

}  // namespace spmv
