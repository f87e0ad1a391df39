// Internal state of a converted matrix (the GPU counterpart of one Matrix_Format object).
#pragma once

#include <chrono>
#include <string>
#include <vector>

#include "common.cuh"

namespace spmv {

// A staged block: rows (or slices) [unit0, unit0 + units) whose stored entries
// [elem0, elem0 + elems) are copied to shared memory in one bulk transfer.  units < 0
// marks a long unit (one row / one slice larger than the staging capacity), processed
// straight from global memory.
// Zero entries after the last nonzero of every device copy of the CSR arrays.
constexpr int64_t SPMV_ENTRY_PAD = 256;

struct StagedBlock {
	int32_t unit0;
	int32_t units;
	int32_t elem0;
	int32_t elems;
};

// A chunk of the warp-autonomous kernel: units [unit0, unit0 + units) (rows, or slices of
// V rows) whose entries [elem0, elem0 + elems) are staged together.  A unit larger than
// one chunk spans consecutive chunks with flags 1 (continues the previous chunk) and
// 2 (continues in the next chunk).
struct WarpChunk {
	int32_t unit0;
	uint16_t units;
	uint16_t flags;
	int32_t elem0;
	int32_t elems;
};

enum class Kind { CSR = 0, SLICED = 1 };

// One matrix of a batch (device table).
struct BatchMat {
	int32_t kind;                  // 0: csr_naive order; 1: slices, one FMA per column
	int32_t V;                     // slice height (kind 1)
	int64_t m;
	const int32_t * ptr;           // row_ptr or slice pointer
	const int32_t * cols;
	const double * vals;
	const int32_t * ymap;          // row map of sorted slices, or null
	int64_t x_off, y_off;          // offsets into the batch's concatenated x and y
};

struct BatchArgs {
	const StagedBlock * blocks;
	const int32_t * bmat;          // matrix of each block
	int64_t nblocks;
	const BatchMat * mats;
	const double * x;
	double * y;
	int cap_al;
	int stages;
	int stage_bytes;
	int exact;
	unsigned long long * counter;  // work-queue head, zero at launch
	int * err;
};

int batch_launch(const BatchArgs & b, int grid, int threads, size_t smem, cudaStream_t s);
int batch_occupancy(int threads, size_t smem, int * per_sm);
enum class Arith { SEQ_SPLIT = 0, SEQ_FMA = 1, LANES_FMA = 2 };

struct Handle {
	spmv_format_desc desc{};
	int64_t m = 0, n = 0, nnz = 0;
	int device = 0;
	int num_sms = 0;
	cudaStream_t stream = nullptr;
	int * d_err = nullptr;       // device error word

	// CSR (csr_naive, csr_vec) -- also kept for sell/sell_sorted/sell_c_s conversions
	int32_t * d_rp = nullptr;
	int32_t * d_ci = nullptr;
	double * d_v = nullptr;
	float * d_vf = nullptr;      // FP32 variant values
	// FP32 segmented kernel (kernel 7): first row of every 256-entry chunk, the rows that
	// cross a chunk boundary, the empty rows, per-chunk partial sums (head, tail)
	int32_t * d_chunk_row = nullptr;
	int32_t * d_cross_rows = nullptr;
	int32_t * d_empty_rows = nullptr;
	float2 * d_chunk_head = nullptr;
	float2 * d_chunk_tail = nullptr;
	int64_t num_seg_chunks = 0, num_cross_rows = 0, num_empty_rows = 0;

	// staged kernel
	StagedBlock * d_blocks = nullptr;
	int64_t * d_cta_ranges = nullptr;  // kernel 4: first block of each CTA's contiguous range (grid + 1)
	int64_t num_blocks = 0;
	int grid = 0;
	int block_cap = 0;           // staging capacity in entries
	int stages = 0;
	int threads = 256;           // threads per CTA of the staged kernel
	size_t smem_bytes = 0;
	int exec_kernel = 0;         // 0 CTA staged, 1 direct sliced, 2 warp-autonomous, 3 pipelined,
	                             // 4 warp-specialised (gather warps + row warps), 5 CTA staged
	                             // own-gather, 6 warp-autonomous own-gather, 7 FP32 segmented,
	                             // 8 warp-specialised over tiled slice columns
	int row_threads = 0;         // kernels 4 and 8: threads of the row warps (the rest gather)
	int32_t * d_tcols = nullptr; // kernels 8-10: slice column indices, row-major in 8-column tiles
	int2 * d_items = nullptr;    // kernel 10: work items (slice ranges), heaviest first
	int64_t num_items = 0;
	int64_t tile_heavy_min = 0;  // kernel 10: slices at least this long are items of their own
	unsigned int * d_queue = nullptr;  // kernel 10: work-queue head and finished-warp count
	uint16_t * d_rassign = nullptr;  // FP32 kernel 4, row_assign 1: local row of each row thread
	int4 * d_pinfo = nullptr;    // packed columns: per block {16-byte offset, base, bits, bytes}
	uint32_t * d_pcols = nullptr;  // packed columns: the block streams
	int64_t packed_bytes = 0;

	// warp-autonomous kernel
	WarpChunk * d_chunks = nullptr;
	int64_t num_chunks = 0;
	int32_t * d_warp_begin = nullptr;
	int64_t num_warps = 0;
	int warp_bytes = 0;

	// SELL / sell_sorted (slice height V)
	int64_t nclusters = 0;
	int64_t nnz_ext = 0;
	int32_t * d_rcp = nullptr;   // row_cluster_ptr[nclusters+1]
	int32_t * d_ja = nullptr;
	double * d_a = nullptr;
	int32_t * d_perm = nullptr;
	int32_t * d_rev = nullptr;
	int64_t * d_ranges = nullptr; // 2T thread ranges

	// SELL-C-sigma
	int64_t nslices = 0;
	int64_t sellcs_size = 0;
	int32_t * d_order = nullptr;
	int32_t * d_widths = nullptr;
	int64_t * d_sptr = nullptr;
	int32_t * d_sptr32 = nullptr;   // the same slice pointers, 32-bit, for the staged kernel
	int32_t * d_scols = nullptr;
	double * d_svals = nullptr;
	// FP32 variant over 32-row slices: FP32 values, row lengths, first tile of each slice,
	// per-tile headers {first word, high bits, base, bit width} and the packed offsets
	float * d_svals_f = nullptr;
	int32_t * d_srlen = nullptr;
	int32_t * d_stptr = nullptr;
	int4 * d_sthdr = nullptr;
	uint32_t * d_swords = nullptr;
	int64_t swords = 0;

	// DIV-RF
	int64_t div_bytes = 0;
	int64_t num_packets = 0;
	uint8_t * d_div = nullptr;
	int64_t * d_pkt = nullptr;          // packet byte offsets [num_packets+1]
	int4 * d_pkt_meta = nullptr;        // per packet: {y row start, y row end, flags, 0}
	int64_t * d_groups = nullptr;       // per-thread group offsets (concatenated)
	int64_t num_group_entries = 0;
	int64_t * d_thread_bytes = nullptr;
	int64_t * d_thread_groups = nullptr;
	int32_t * d_zero_rows = nullptr;    // rows not covered by any packet (zeroed each run)
	int64_t num_zero_rows = 0;
	double * d_split_part = nullptr;    // partial sums of rows split across packets
	int32_t * d_split_rows = nullptr;
	int64_t num_split = 0;

	// host-buffer path staging
	double * d_x = nullptr;
	double * d_y = nullptr;
	float * d_xf = nullptr;
	float * d_yf = nullptr;

	std::vector<void *> allocations;    // everything above, freed by destroy
	double mem_footprint = 0;
	double csr_mem_footprint = 0;
	int64_t stored_elems = 0;
	int64_t device_bytes = 0;
	double convert_ms = 0;
	double alloc_ms = 0;        // host time inside cudaMalloc during the conversion
	double copy_in_ms = 0;      // the CSR arrays' copy to the device (until it completed)
	int64_t x_lo = 0, x_hi = -1;  // span of the format's columns above 0 (inclusive; empty if hi < lo)
	int64_t x_col0 = 0;           // column 0 occurs (SELL-C-sigma pads with it)
	int kernels_per_run = 0;
	std::string name;

	template <typename T>
	int alloc(T ** p, int64_t count)
	{
		size_t bytes = (size_t) (count > 0 ? count : 1) * sizeof(T);
		const auto t0 = std::chrono::steady_clock::now();
		cudaError_t e = cudaMalloc((void **) p, bytes);
		alloc_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
		if (e != cudaSuccess) {
			*p = nullptr;
			set_error(SPMV_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
			return SPMV_ERR_NOMEM;
		}
		allocations.push_back((void *) *p);
		device_bytes += (int64_t) bytes;
		return SPMV_OK;
	}
};

// ---- conversions (each fills the format's device arrays from d_rp/d_ci/d_v)
int convert_csr(Handle & h);
int convert_sell(Handle & h, bool sorted);
int convert_sellcs(Handle & h);
int convert_div(Handle & h);
int convert_f32(Handle & h);
int build_sliced_f32(Handle & h);
const void * ws_f32_kernel_fn(bool packed);   // the FP32 warp-specialised kernel (geometry queries)
int build_packed_cols(Handle & h);  // packed column streams of the staged blocks (pack.cu)
int f32ws_stage_bytes(int cap_al);  // its stage size: 8 bytes per staged entry
int run_mixed_noalloc(Handle & h, const double * d_x, double * d_y, cudaStream_t s);
int convert_vector_d2f(const double * in, float * out, int64_t n, cudaStream_t s);
int convert_vector_f2d(const float * in, double * out, int64_t n, cudaStream_t s);


// Builds the execution schedule of the chosen kernel over the unit pointer P (CSR row_ptr
// with V = 1, or a slice pointer with slice height V).
int build_exec(Handle & h, const int32_t * d_P, int64_t U, int V);
int build_warp_chunks(Handle & h, const int32_t * d_P, int64_t U, int V);
int build_tile_reg(Handle & h, const int32_t * d_P, int64_t U, int V);
int launch_warp(Handle & h, const double * d_x, double * d_y, cudaStream_t s);

// ---- SpMV launches
int launch_spmv(Handle & h, const double * d_x, double * d_y, cudaStream_t s);
int launch_spmv_f32(Handle & h, const float * d_x, float * d_y, cudaStream_t s);
int launch_div(Handle & h, const double * d_x, double * d_y, cudaStream_t s);

// Validates a device CSR: row_ptr[0] == 0, monotone, row_ptr[m] == nnz, 0 <= col < n.
int validate_csr(Handle & h);

}  // namespace spmv
