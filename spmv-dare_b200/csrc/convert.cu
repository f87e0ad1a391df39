// GPU conversions from CSR to the reference's storage formats.  Every converted array is
// bit-identical to the reference's csr_to_format output for the same thread count T and
// slice height / lane count (checked array-for-array by the parity tests):
//
//   sell         src/spmv_kernels/sell.cpp:95-199
//   sell_sorted  src/spmv_kernels/sell_sorted.cpp:119-305
//   sell_c_s     src/spmv_kernels/sell-C-s/sellcs_format.c:137-224, radix_sort.c:36-122
//
// The sequential per-thread loops of the reference become data-parallel passes: segmented
// maxima and scans for the slice widths, the reference's nearest-index partitioner for the
// thread ranges, a stable radix sort for the per-range / per-window row orderings, and a
// max-scan that carries the "last column written in this thread range" used as padding.
#include "internal.h"
#include "primitives.cuh"

namespace spmv {

int staged_geometry(Handle & h);

namespace {

constexpr int BLOCK_TILE_UNITS = 1024;   // units (rows / slices) scanned by one builder thread

// ------------------------------------------------------------------ CSR validation
__global__ void validate_csr_kernel(const int32_t * rp, const int32_t * ci, int64_t m, int64_t n, int64_t nnz,
		int * flag)
{
	int64_t tid = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	int64_t stride = (int64_t) gridDim.x * blockDim.x;
	if (tid == 0 && (rp[0] != 0 || (int64_t) rp[m] != nnz))
		atomicOr(flag, 1);
	for (int64_t i = tid; i < m; i += stride)
		if (rp[i] > rp[i + 1])
			atomicOr(flag, 1);
	for (int64_t j = tid; j < nnz; j += stride)
		if (ci[j] < 0 || (int64_t) ci[j] >= n)
			atomicOr(flag, 2);
}

// ------------------------------------------------------------------ staged blocks
// Greedy packing of consecutive units into blocks of at most `cap` stored entries and
// `max_units` units, inside tiles of BLOCK_TILE_UNITS units (one thread per tile).
// A unit larger than `cap` becomes a block of its own, marked long (units = -1).
template <bool WRITE>
// chunk > 0: a unit longer than `cap` becomes consecutive chunk blocks of `chunk` entries
// (units = -1 - flags, flags bit 0 = first chunk, bit 1 = last chunk) instead of one long
// block (units = -1, elems = the unit's length).
__global__ void blocks_kernel(const int32_t * P, int64_t U, int cap, int max_units, int chunk, int64_t * counts,
		const int64_t * offs, StagedBlock * out)
{
	int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	int64_t u = t * BLOCK_TILE_UNITS;
	if (u >= U)
		return;
	int64_t end = u + BLOCK_TILE_UNITS < U ? u + BLOCK_TILE_UNITS : U;
	int64_t nb = 0;
	int64_t o = WRITE ? offs[t] : 0;
	while (u < end) {
		int64_t len = (int64_t) P[u + 1] - P[u];
		if (len > cap) {
			if (chunk > 0) {
				for (int64_t c0 = 0; c0 < len; c0 += chunk) {
					const int64_t cl = (len - c0) < chunk ? (len - c0) : chunk;
					const int flags = (c0 == 0 ? 1 : 0) | (c0 + cl == len ? 2 : 0);
					if (WRITE)
						out[o + nb] = StagedBlock{(int32_t) u, -1 - flags, (int32_t) (P[u] + c0), (int32_t) cl};
					nb++;
				}
			} else {
				if (WRITE)
					out[o + nb] = StagedBlock{(int32_t) u, -1, P[u], (int32_t) len};
				nb++;
			}
			u++;
			continue;
		}
		int64_t start = u;
		int64_t e0 = P[u];
		while (u < end && u - start < max_units && (int64_t) P[u + 1] - e0 <= cap)
			u++;
		if (WRITE)
			out[o + nb] = StagedBlock{(int32_t) start, (int32_t) (u - start), (int32_t) e0,
					(int32_t) ((int64_t) P[u] - e0)};
		nb++;
	}
	if (!WRITE)
		counts[t] = nb;
}

int build_blocks(Handle & h, const int32_t * d_P, int64_t U, int max_units, int chunk)
{
	cudaStream_t s = h.stream;
	int64_t tiles = ceil_div(U, BLOCK_TILE_UNITS);
	if (tiles == 0) {
		h.num_blocks = 0;
		return SPMV_OK;
	}
	DevBuf counts, offs;
	SPMV_TRY(counts.alloc(tiles * sizeof(int64_t), s));
	SPMV_TRY(offs.alloc((tiles + 1) * sizeof(int64_t), s));
	unsigned grid = (unsigned) ceil_div(tiles, 128);
	blocks_kernel<false><<<grid, 128, 0, s>>>(d_P, U, h.block_cap, max_units, chunk, counts.as<int64_t>(), nullptr, nullptr);
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(scan_exclusive(counts.as<int64_t>(), offs.as<int64_t>(), tiles, s));
	int64_t nb = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&nb, offs.as<int64_t>() + tiles, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	h.num_blocks = nb;
	SPMV_TRY(h.alloc(&h.d_blocks, nb));
	blocks_kernel<true><<<grid, 128, 0, s>>>(d_P, U, h.block_cap, max_units, chunk, nullptr, offs.as<int64_t>(), h.d_blocks);
	SPMV_CUDA_TRY(cudaGetLastError());
	return staged_geometry(h);
}

void staged_defaults(Handle & h)
{
	// defaults measured on B200 with the 4M-row configuration (staging capacity, CTA size)
	int cap = 1024, threads = 256;
	if (h.desc.format == SPMV_FMT_CSR_NAIVE)
		cap = 768;
	else if (h.desc.format == SPMV_FMT_SELL_C_S) {
		cap = 2048;
		threads = 512;
	}
	h.block_cap = h.desc.block_nnz > 0 ? h.desc.block_nnz : cap;
	h.block_cap = (h.block_cap + 7) & ~7;
	h.stages = h.desc.stages > 0 ? h.desc.stages : 2;
	h.threads = h.desc.threads > 0 ? h.desc.threads : threads;
}

// ------------------------------------------------------------------ SELL
__global__ void slice_width_kernel(const int32_t * rp, int64_t m, int V, int64_t nc, int64_t * W)
{
	int64_t c = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= nc)
		return;
	int64_t w = 0;
	int64_t e = (c + 1) * V < m ? (c + 1) * V : m;
	for (int64_t k = c * V; k < e; k++) {
		int64_t d = (int64_t) rp[k + 1] - rp[k];
		w = d > w ? d : w;
	}
	W[c] = (int64_t) V * w;
}

__global__ void i64_to_i32_kernel(const int64_t * in, int32_t * out, int64_t n)
{
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		out[i] = (int32_t) in[i];
}

// Index of the last non-empty row at or before each row (or -1).
__global__ void nonempty_index_kernel(const int32_t * rp, int64_t m, int32_t * out)
{
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < m)
		out[i] = (rp[i + 1] > rp[i]) ? (int32_t) i : -1;
}

// One thread per row slot of the slices: writes its column-major entries and the
// reference's padding (value 0, column = last column written in the thread range so far).
__global__ void sell_fill_kernel(const int32_t * rp, const int32_t * ci, const double * v, int64_t m, int V,
		int64_t nc, const int32_t * rcp, const int64_t * ranges, int T, const int32_t * last_nonempty,
		int32_t * ja, double * a)
{
	int64_t u = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (u >= nc * V)
		return;
	const int64_t sl = u / V;
	const int lane = (int) (u % V);
	const int64_t row = u;
	// thread range of this slice
	int64_t range_row0 = 0;
	for (int t = 0; t < T; t++)
		if (sl >= ranges[2 * t] && sl < ranges[2 * t + 1]) {
			range_row0 = ranges[2 * t] * V;
			break;
		}
	const int64_t base = rcp[sl];
	const int w = (rcp[sl + 1] - rcp[sl]) / V;
	int64_t len = 0, j0 = 0;
	if (row < m) {
		j0 = rp[row];
		len = (int64_t) rp[row + 1] - j0;
	}
	int32_t pad = 0;
	{
		int64_t g = last_nonempty[row < m ? row : m - 1];
		if (g >= range_row0 && g >= 0)
			pad = ci[rp[g + 1] - 1];
	}
	for (int k = 0; k < w; k++) {
		int64_t d = base + (int64_t) k * V + lane;
		if (k < len) {
			a[d] = v[j0 + k];
			ja[d] = ci[j0 + k];
		} else {
			a[d] = 0.0;
			ja[d] = pad;
		}
	}
}

// Builds SELL slices over (rp, ci, v) into h.d_rcp / d_ja / d_a.  `ranges_given` holds
// the thread ranges in slice units (sell_sorted) or is null (sell: balanced over the
// padded slice sizes, sell.cpp:161).
int sell_from_csr(Handle & h, const int32_t * rp, const int32_t * ci, const double * v, const int64_t * ranges_given)
{
	cudaStream_t s = h.stream;
	const int V = h.desc.vec_len;
	const int T = h.desc.num_threads;
	const int64_t m = h.m;
	const int64_t nc = ceil_div(m, V);
	h.nclusters = nc;
	DevBuf W, W_scan;
	SPMV_TRY(W.alloc((nc + 1) * sizeof(int64_t), s));
	SPMV_TRY(W_scan.alloc((nc + 2) * sizeof(int64_t), s));
	if (nc > 0) {
		slice_width_kernel<<<(unsigned) ceil_div(nc, 256), 256, 0, s>>>(rp, m, V, nc, W.as<int64_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	SPMV_TRY(scan_exclusive(W.as<int64_t>(), W_scan.as<int64_t>(), nc, s));
	int64_t total = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&total, W_scan.as<int64_t>() + nc, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	if (total > INT32_MAX - 64) {
		set_error(SPMV_ERR_OVERFLOW, "SELL stores %lld entries, beyond the 32-bit row_cluster_ptr", (long long) total);
		return SPMV_ERR_OVERFLOW;
	}
	h.nnz_ext = total;
	SPMV_TRY(h.alloc(&h.d_rcp, nc + 1));
	i64_to_i32_kernel<<<(unsigned) ceil_div(nc + 1, 256), 256, 0, s>>>(W_scan.as<int64_t>(), h.d_rcp, nc + 1);
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(h.alloc(&h.d_ranges, 2 * T));
	if (ranges_given) {
		SPMV_CUDA_TRY(cudaMemcpyAsync(h.d_ranges, ranges_given, 2 * T * sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
	} else if (nc > 0) {
		SPMV_TRY(partition_prefix_sums(h.d_rcp, nc, total, T, h.d_ranges, s));
	} else {
		SPMV_CUDA_TRY(cudaMemsetAsync(h.d_ranges, 0, 2 * T * sizeof(int64_t), s));
	}
	// stored arrays, padded by 8 entries for the 16-byte bulk-copy granularity
	SPMV_TRY(h.alloc(&h.d_ja, total + 8));
	SPMV_TRY(h.alloc(&h.d_a, total + 8));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_ja, 0, (total + 8) * sizeof(int32_t), s));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_a, 0, (total + 8) * sizeof(double), s));
	if (nc > 0) {
		DevBuf last;
		SPMV_TRY(last.alloc(m * sizeof(int32_t), s));
		nonempty_index_kernel<<<(unsigned) ceil_div(m, 256), 256, 0, s>>>(rp, m, last.as<int32_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
		SPMV_TRY(scan_inclusive_max(last.as<int32_t>(), last.as<int32_t>(), m, s));
		sell_fill_kernel<<<(unsigned) ceil_div(nc * V, 256), 256, 0, s>>>(rp, ci, v, m, V, nc, h.d_rcp, h.d_ranges, T,
				last.as<int32_t>(), h.d_ja, h.d_a);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	h.stored_elems = total;
	return SPMV_OK;
}

// ------------------------------------------------------------------ sell_sorted
__global__ void cluster_sums_kernel(const int32_t * rp, int64_t m, int V, int64_t nc, int32_t * S)
{
	int64_t c = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (c < nc)
		S[c] = rp[c * V];
	else if (c == nc)
		S[nc] = rp[m];
}

// Sort keys of the rows: (thread range, row length); values: row index.
__global__ void sorted_keys_kernel(const int32_t * rp, int64_t m, int V, const int64_t * ranges, int T, int len_bits,
		uint64_t * keys, uint32_t * vals)
{
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= m)
		return;
	int t = 0;
	for (int q = 0; q < T; q++) {
		int64_t i_s = ranges[2 * q] * V;
		int64_t i_e = (q == T - 1) ? m : ranges[2 * q + 1] * V;
		if (i >= i_s && i < i_e) {
			t = q;
			break;
		}
	}
	keys[i] = ((uint64_t) t << len_bits) | (uint64_t) (rp[i + 1] - rp[i]);
	vals[i] = (uint32_t) i;
}

__global__ void perm_kernel(const uint32_t * sorted_rows, int64_t m, int32_t * perm, int32_t * rev)
{
	int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= m)
		return;
	int32_t row = (int32_t) sorted_rows[p];
	rev[p] = row;
	perm[row] = (int32_t) p;
}

__global__ void reordered_len_kernel(const int32_t * rp, const int32_t * rev, int64_t m, int32_t * len)
{
	int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (p < m)
		len[p] = rp[rev[p] + 1] - rp[rev[p]];
}

__global__ void reordered_copy_kernel(const int32_t * rp, const int32_t * ci, const double * v, const int32_t * rev,
		const int64_t * rp2, int64_t m, int32_t * ci2, double * v2)
{
	int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= m)
		return;
	int64_t src = rp[rev[p]], len = (int64_t) rp[rev[p] + 1] - src, dst = rp2[p];
	for (int64_t k = 0; k < len; k++) {
		ci2[dst + k] = ci[src + k];
		v2[dst + k] = v[src + k];
	}
}


__global__ void i64_to_i32_rp_kernel(const int64_t * in, int32_t * out, int64_t n)
{
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		out[i] = (int32_t) in[i];
}

static int bits_for(int64_t v)
{
	int b = 0;
	while (v) {
		b++;
		v >>= 1;
	}
	return b;
}

// ------------------------------------------------------------------ SELL-C-sigma
__global__ void sellcs_keys_kernel(const int32_t * rp, int64_t m, int64_t sigma, int32_t maxlen, int len_bits,
		uint64_t * keys, uint32_t * vals)
{
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= m)
		return;
	uint64_t win = (uint64_t) (i / sigma);
	uint64_t len = (uint64_t) (rp[i + 1] - rp[i]);
	keys[i] = (win << len_bits) | ((uint64_t) maxlen - len);   // descending length inside the window
	vals[i] = (uint32_t) i;
}

__global__ void sellcs_widths_kernel(const int32_t * rp, const uint32_t * order, int64_t m, int C, int64_t ns,
		int32_t * order_out, int32_t * widths, int64_t * W)
{
	int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (p < m)
		order_out[p] = (int32_t) order[p];
	if (p < ns) {
		int32_t r = (int32_t) order[p * C];
		int32_t w = rp[r + 1] - rp[r];
		widths[p] = w;
		W[p] = (int64_t) w * C;
	}
}

__global__ void sellcs_fill_kernel(const int32_t * rp, const int32_t * ci, const double * v, const int32_t * order,
		int64_t m, int C, int64_t ns, const int32_t * widths, const int64_t * sptr, int32_t * cols, double * vals)
{
	int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= ns * C)
		return;
	const int64_t sl = p / C;
	const int lane = (int) (p % C);
	const int w = widths[sl];
	int64_t len = 0, j0 = 0;
	if (p < m) {
		int32_t r = order[p];
		j0 = rp[r];
		len = (int64_t) rp[r + 1] - j0;
	}
	const int64_t base = sptr[sl] + lane;
	for (int k = 0; k < w; k++) {
		int64_t d = base + (int64_t) k * C;
		if (k < len) {
			vals[d] = v[j0 + k];
			cols[d] = ci[j0 + k];
		} else {
			vals[d] = 0.0;
			cols[d] = 0;
		}
	}
}

}  // namespace

int validate_csr(Handle & h)
{
	cudaStream_t s = h.stream;
	DevBuf flag;
	SPMV_TRY(flag.alloc(sizeof(int), s));
	SPMV_CUDA_TRY(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
	int64_t work = h.m > h.nnz ? h.m : h.nnz;
	int64_t grid = ceil_div(work > 0 ? work : 1, 256);
	if (grid > 8192)
		grid = 8192;
	validate_csr_kernel<<<(unsigned) grid, 256, 0, s>>>(h.d_rp, h.d_ci, h.m, h.n, h.nnz, flag.as<int>());
	SPMV_CUDA_TRY(cudaGetLastError());
	int f = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&f, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	if (f & 1) {
		set_error(SPMV_ERR_CSR, "row_ptr is not a valid CSR row pointer (row_ptr[0] != 0, decreasing, or row_ptr[m] != nnz)");
		return SPMV_ERR_CSR;
	}
	if (f & 2) {
		set_error(SPMV_ERR_CSR, "a column index is outside [0, n)");
		return SPMV_ERR_CSR;
	}
	return SPMV_OK;
}

// Column indices of the slices in row-major tiles of 8 slice columns (kernel 8).  Entry
// (row r, column k) of slice s, width W = (P[s + 1] - P[s]) / V, moves from
// P[s] + k * V + r to P[s] + k8 * V + r * tw + (k - k8), k8 = k & ~7, tw = min(8, W - k8):
// a permutation inside every slice, so blocks of whole slices and chunks of whole tiles
// are contiguous ranges of the tiled array too.  One thread per slice row.
__global__ void tile_cols_kernel(const int32_t * P, int64_t ns, int V, const int32_t * cols, int32_t * out)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= ns * V)
		return;
	const int64_t sl = i / V;
	const int r = (int) (i % V);
	const int64_t b = P[sl];
	const int W = (int) (((int64_t) P[sl + 1] - b) / V);
	for (int k = 0; k < W; k++) {
		const int k8 = k & ~7;
		const int tw = W - k8 < 8 ? W - k8 : 8;
		out[b + (int64_t) k8 * V + (int64_t) r * tw + (k - k8)] = cols[b + (int64_t) k * V + r];
	}
}

// The tiled copy of a sliced format's column indices (kernels 8 and 9).
static int build_tiled_cols(Handle & h, const int32_t * d_P, int64_t U, int V)
{
	const int32_t * cols = h.desc.format == SPMV_FMT_SELL_C_S ? h.d_scols : h.d_ja;
	SPMV_TRY(h.alloc(&h.d_tcols, h.stored_elems + 8));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_tcols, 0, (h.stored_elems + 8) * sizeof(int32_t), h.stream));
	if (U > 0) {
		tile_cols_kernel<<<(unsigned) ceil_div(U * V, 256), 256, 0, h.stream>>>(d_P, U, V, cols, h.d_tcols);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	return SPMV_OK;
}

// Kernel choice: -1 = the format's default (the register-tiled warp kernel for slices of 32
// rows, the tiled warp-specialised kernel for wider SELL-C-sigma slices, the warp-specialised
// kernel otherwise: the fastest of each on the 4M-row configuration); 0 = CTA
// staged kernel; 1 = direct column-major kernel (slices of >= 32 rows only); 2 =
// warp-autonomous staged kernel (slices of <= 32 rows); 3 = CTA staged kernel with the next
// block's gather overlapping this block's rows; 4 = warp-specialised staged kernel; 5 = CTA
// staged kernel whose row threads load their own x (no separate gather phase); 6 =
// warp-autonomous kernel whose slice rows load their own x (slices of <= 32 rows); 8 =
// warp-specialised kernel over the column indices in row-major 8-column tiles (slices of
// >= 8 rows); 9 = warp-autonomous kernel over the same tiles, x transposed between lanes
// (slices of exactly 32 rows); 10 = warps that claim runs of 32-row slices from a queue and
// sum them from registers, tiles one ahead, x transposed between lanes (no shared memory).
int build_exec(Handle & h, const int32_t * d_P, int64_t U, int V)
{
	int k = h.desc.kernel;
	if (k < 0) {
		// measured on the 4M-row matrix: kernel 4 is the fastest for csr_naive (0.193 ms),
		// csr_vec, and sell / sell_sorted with slices of up to 16 rows; kernel 10 for slices of
		// exactly 32 rows (SELL-C-sigma 0.213 ms against kernel 8's 0.255-0.266, sell 0.197,
		// sell_sorted 0.217); kernel 8 for SELL-C-sigma with wider slices.  A requested staging
		// block selects the staged kernels.
		const bool sliced = h.desc.format == SPMV_FMT_SELL_C_S || h.desc.format == SPMV_FMT_SELL ||
				h.desc.format == SPMV_FMT_SELL_SORTED;
		if (sliced && V == 32 && h.desc.block_nnz == 0)
			k = 10;
		else
			k = h.desc.format == SPMV_FMT_SELL_C_S ? 8 : 4;
		// a requested staging block too large for their two-stage pipeline (about 220 KB of
		// shared memory per CTA at 12, 16 or 17 bytes an entry) goes to the CTA staged kernel,
		// which stages fewer blocks at once
		const int per = k == 8 ? 17 : (h.desc.format == SPMV_FMT_CSR_NAIVE ? 12 : 16);
		if (h.desc.block_nnz > 0 && 2 * ((int64_t) h.desc.block_nnz + 16) * per > 220 * 1024 - 256)
			k = 0;
	}
	if (k == 1 && V < 32)
		k = 0;
	if ((k == 2 || k == 6) && V > 32)
		k = 0;
	if (k == 6 && V == 1)
		k = 2;                      // CSR: the warp kernel's own path
	if (k == 8 && V < 8)
		k = 4;                      // narrower slices already give a warp 8 neighbouring columns
	if ((k == 9 || k == 10) && V != 32)
		k = V >= 8 ? 8 : 4;         // kernels 9 and 10's lane transpose takes slices of exactly 32 rows
	if (k == 10 && V == 1)
		k = 4;
	h.exec_kernel = k;
	if (k == 1)
		return SPMV_OK;
	if (k == 2 || k == 6)
		return build_warp_chunks(h, d_P, U, V);
	if (k == 9) {
		SPMV_TRY(build_tiled_cols(h, d_P, U, V));
		return build_warp_chunks(h, d_P, U, V);
	}
	if (k == 10) {
		SPMV_TRY(build_tiled_cols(h, d_P, U, V));
		return build_tile_reg(h, d_P, U, V);
	}
	staged_defaults(h);
	if (k == 3 && h.desc.stages == 0)
		h.stages = 3;
	if (k == 4) {
		// defaults measured on the 4M-row matrix: 2 stages, 3 gather warps and 2 row warps;
		// 768-entry blocks for csr_naive (0.195-0.207 ms; 3 stages 0.202 ms), 1280 for the FMA
		// formats, whose stages take 16 bytes an entry (csr_vec 0.316 ms, sell 0.285 ms; 768-entry
		// blocks 0.334 / 0.291)
		if (h.desc.block_nnz == 0)
			h.block_cap = h.desc.format == SPMV_FMT_CSR_NAIVE ? 768 : 1280;
		if (h.desc.stages == 0)
			h.stages = 2;
		if (h.desc.threads == 0)
			h.threads = 160;
		h.row_threads = h.desc.block_rows > 0 ? h.desc.block_rows : 64;
	}
	if (k == 8) {
		// defaults measured on the 4M-row matrix with C = 32: one row warp per slice, 2 gather
		// warps, 512-entry blocks, 2 stages (0.255-0.264 ms; 640-entry blocks 0.28-0.31 ms,
		// 3 stages 0.38 ms: the CTAs an SM holds set the pace)
		const int rows = V > 32 ? ((V + 31) / 32) * 32 : 32;
		if (h.desc.block_nnz == 0)
			h.block_cap = (8 * V > 512 ? 8 * V : 512);
		if (h.desc.stages == 0)
			h.stages = 2;
		h.row_threads = h.desc.block_rows > 0 ? h.desc.block_rows : rows;
		if (h.desc.threads == 0)
			h.threads = h.row_threads + 64;
	}
	if (k == 4 || k == 8) {
		// row warps: block_rows threads; at least one gather warp besides them
		if (h.row_threads % 32 != 0 || h.row_threads + 32 > h.threads || h.row_threads < V) {
			set_error(SPMV_ERR_ARG, "warp-specialised kernel: block_rows %d must be a multiple of 32, at least the "
					"slice height %d and leave a gather warp of %d threads", h.row_threads, V, h.threads);
			return SPMV_ERR_ARG;
		}
		if (h.block_cap < V) {
			set_error(SPMV_ERR_ARG, "warp-specialised kernel: block_nnz %d below the slice height %d", h.block_cap, V);
			return SPMV_ERR_ARG;
		}
		if (k == 8) {
			// chunks of whole 8-column tiles, and the tiled copy of the column indices
			if (h.block_cap < 8 * V) {
				set_error(SPMV_ERR_ARG, "tiled kernel: block_nnz %d below one tile of 8 x %d entries", h.block_cap, V);
				return SPMV_ERR_ARG;
			}
			SPMV_TRY(build_tiled_cols(h, d_P, U, V));
			return build_blocks(h, d_P, U, h.row_threads / V, (h.block_cap / (8 * V)) * 8 * V);
		}
		// units longer than a block: chunks of whole slice columns, summed in order by one CTA
		return build_blocks(h, d_P, U, h.row_threads / V, (h.block_cap / V) * V);
	}
	int max_units = (h.desc.block_rows > 0 ? h.desc.block_rows : h.threads) / V;
	if (max_units < 1)
		max_units = 1;
	return build_blocks(h, d_P, U, max_units, 0);
}

int convert_csr(Handle & h)
{
	SPMV_TRY(build_exec(h, h.d_rp, h.m, 1));
	if (h.desc.pack_cols == 1) {
		if (h.exec_kernel != 4) {
			set_error(SPMV_ERR_ARG, "pack_cols: FP64 csr_naive packs columns for kernel 4 only (got kernel %d)",
					h.exec_kernel);
			return SPMV_ERR_ARG;
		}
		SPMV_TRY(build_packed_cols(h));
	}
	return SPMV_OK;
}

int convert_sell(Handle & h, bool sorted)
{
	cudaStream_t s = h.stream;
	const int V = h.desc.vec_len;
	const int T = h.desc.num_threads;
	const int64_t m = h.m;
	const int64_t nc = ceil_div(m, V);
	if (!sorted) {
		SPMV_TRY(sell_from_csr(h, h.d_rp, h.d_ci, h.d_v, nullptr));
	} else {
		// thread ranges over whole slices, balanced by nnz (sell_sorted.cpp:146-166)
		DevBuf S, ranges;
		SPMV_TRY(S.alloc((nc + 1) * sizeof(int32_t), s));
		SPMV_TRY(ranges.alloc(2 * T * sizeof(int64_t), s));
		cluster_sums_kernel<<<(unsigned) ceil_div(nc + 1, 256), 256, 0, s>>>(h.d_rp, m, V, nc, S.as<int32_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
		if (nc > 0) {
			SPMV_TRY(partition_prefix_sums(S.as<int32_t>(), nc, h.nnz, T, ranges.as<int64_t>(), s));
		} else {
			SPMV_CUDA_TRY(cudaMemsetAsync(ranges.p, 0, 2 * T * sizeof(int64_t), s));
		}
		// stable ascending sort of row lengths inside each range (sell_sorted.cpp:182-196)
		DevBuf d_max;
		SPMV_TRY(d_max.alloc(sizeof(int32_t), s));
		SPMV_TRY(max_row_length(h.d_rp, m, d_max.as<int32_t>(), s));
		int32_t maxlen = 0;
		SPMV_CUDA_TRY(cudaMemcpyAsync(&maxlen, d_max.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
		SPMV_CUDA_TRY(cudaStreamSynchronize(s));
		const int len_bits = bits_for(maxlen) > 0 ? bits_for(maxlen) : 1;
		const int key_bits = len_bits + bits_for(T);
		SPMV_TRY(h.alloc(&h.d_perm, m));
		SPMV_TRY(h.alloc(&h.d_rev, m));
		DevBuf keys, vals, rlen, rp2_64, rp2, ci2, v2;
		SPMV_TRY(keys.alloc(m * sizeof(uint64_t), s));
		SPMV_TRY(vals.alloc(m * sizeof(uint32_t), s));
		if (m > 0) {
			sorted_keys_kernel<<<(unsigned) ceil_div(m, 256), 256, 0, s>>>(h.d_rp, m, V, ranges.as<int64_t>(), T,
					len_bits, keys.as<uint64_t>(), vals.as<uint32_t>());
			SPMV_CUDA_TRY(cudaGetLastError());
			SPMV_TRY(radix_sort_pairs(keys.as<uint64_t>(), vals.as<uint32_t>(), m, key_bits, s));
			perm_kernel<<<(unsigned) ceil_div(m, 256), 256, 0, s>>>(vals.as<uint32_t>(), m, h.d_perm, h.d_rev);
			SPMV_CUDA_TRY(cudaGetLastError());
		}
		// reordered CSR (sell_sorted.cpp:198-225)
		SPMV_TRY(rlen.alloc(m * sizeof(int32_t), s));
		SPMV_TRY(rp2_64.alloc((m + 1) * sizeof(int64_t), s));
		SPMV_TRY(rp2.alloc((m + 1) * sizeof(int32_t), s));
		SPMV_TRY(ci2.alloc((h.nnz + 1) * sizeof(int32_t), s));
		SPMV_TRY(v2.alloc((h.nnz + 1) * sizeof(double), s));
		if (m > 0) {
			reordered_len_kernel<<<(unsigned) ceil_div(m, 256), 256, 0, s>>>(h.d_rp, h.d_rev, m, rlen.as<int32_t>());
			SPMV_CUDA_TRY(cudaGetLastError());
		}
		SPMV_TRY(scan_exclusive(rlen.as<int32_t>(), rp2_64.as<int64_t>(), m, s));
		i64_to_i32_rp_kernel<<<(unsigned) ceil_div(m + 1, 256), 256, 0, s>>>(rp2_64.as<int64_t>(), rp2.as<int32_t>(), m + 1);
		SPMV_CUDA_TRY(cudaGetLastError());
		if (m > 0) {
			reordered_copy_kernel<<<(unsigned) ceil_div(m, 256), 256, 0, s>>>(h.d_rp, h.d_ci, h.d_v, h.d_rev,
					rp2_64.as<int64_t>(), m, ci2.as<int32_t>(), v2.as<double>());
			SPMV_CUDA_TRY(cudaGetLastError());
		}
		SPMV_TRY(sell_from_csr(h, rp2.as<int32_t>(), ci2.as<int32_t>(), v2.as<double>(), ranges.as<int64_t>()));
		SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	}
	return build_exec(h, h.d_rcp, nc, V);
}

int convert_sellcs(Handle & h)
{
	cudaStream_t s = h.stream;
	const int C = h.desc.sellcs_c;
	const int64_t sigma = h.desc.sellcs_sigma;
	const int64_t m = h.m;
	const int64_t ns = ceil_div(m, C);
	h.nslices = ns;
	DevBuf d_max, keys, vals, W;
	SPMV_TRY(d_max.alloc(sizeof(int32_t), s));
	SPMV_TRY(max_row_length(h.d_rp, m, d_max.as<int32_t>(), s));
	int32_t maxlen = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&maxlen, d_max.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	const int len_bits = bits_for(maxlen) > 0 ? bits_for(maxlen) : 1;
	const int key_bits = len_bits + bits_for(m > 0 ? (m - 1) / sigma : 0);
	SPMV_TRY(keys.alloc(m * sizeof(uint64_t), s));
	SPMV_TRY(vals.alloc(m * sizeof(uint32_t), s));
	SPMV_TRY(W.alloc((ns + 1) * sizeof(int64_t), s));
	SPMV_TRY(h.alloc(&h.d_order, m));
	SPMV_TRY(h.alloc(&h.d_widths, ns));
	SPMV_TRY(h.alloc(&h.d_sptr, ns + 1));
	if (m > 0) {
		sellcs_keys_kernel<<<(unsigned) ceil_div(m, 256), 256, 0, s>>>(h.d_rp, m, sigma, maxlen, len_bits,
				keys.as<uint64_t>(), vals.as<uint32_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
		SPMV_TRY(radix_sort_pairs(keys.as<uint64_t>(), vals.as<uint32_t>(), m, key_bits, s));
		int64_t cnt = m > ns ? m : ns;
		sellcs_widths_kernel<<<(unsigned) ceil_div(cnt, 256), 256, 0, s>>>(h.d_rp, vals.as<uint32_t>(), m, C, ns,
				h.d_order, h.d_widths, W.as<int64_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	SPMV_TRY(scan_exclusive(W.as<int64_t>(), h.d_sptr, ns, s));
	int64_t total = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&total, h.d_sptr + ns, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	h.sellcs_size = total;
	h.stored_elems = total;
	SPMV_TRY(h.alloc(&h.d_scols, total + 8));
	SPMV_TRY(h.alloc(&h.d_svals, total + 8));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_scols, 0, (total + 8) * sizeof(int32_t), s));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_svals, 0, (total + 8) * sizeof(double), s));
	if (total > INT32_MAX - 64) {
		set_error(SPMV_ERR_OVERFLOW, "SELL-C-sigma stores %lld entries, beyond the 32-bit range", (long long) total);
		return SPMV_ERR_OVERFLOW;
	}
	SPMV_TRY(h.alloc(&h.d_sptr32, ns + 1));
	i64_to_i32_kernel<<<(unsigned) ceil_div(ns + 1, 256), 256, 0, s>>>(h.d_sptr, h.d_sptr32, ns + 1);
	SPMV_CUDA_TRY(cudaGetLastError());
	if (ns > 0) {
		sellcs_fill_kernel<<<(unsigned) ceil_div(ns * C, 256), 256, 0, s>>>(h.d_rp, h.d_ci, h.d_v, h.d_order, m, C, ns,
				h.d_widths, h.d_sptr, h.d_scols, h.d_svals);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	if (h.desc.values == SPMV_VALUES_F32)
		return build_sliced_f32(h);      // the FP32 variant over the same slices (fp32.cu)
	return build_exec(h, h.d_sptr32, ns, C);
}

}  // namespace spmv
