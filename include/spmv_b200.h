/*
 * spmv_b200.h -- C ABI of the B200-native SpMV engine (libspmv_b200.so).
 *
 * This is the drop-in boundary for the reference's format plugin API:
 *
 *   struct Matrix_Format * csr_to_format(INT_T * row_ptr, INT_T * col_ind,
 *           ValueTypeReference * values, long m, long n, long nnz,
 *           long symmetric, long symmetry_expanded);           src/spmv_kernels/spmv_kernel.h:28
 *   virtual void Matrix_Format::spmv(ValueType * x, ValueType * y);   spmv_kernel.h:17
 *   double Matrix_Format::mem_footprint / csr_mem_footprint;         spmv_kernel.h:13-14,23
 *   char * Matrix_Format::format_name;                                spmv_kernel.h:10
 *   int statistics_print_labels(char * buf, long buf_n);              spmv_kernel.h:29
 *   int Matrix_Format::statistics_print_data(char * buf, long buf_n); spmv_kernel.h:19
 *
 * spmv_create() replaces csr_to_format() (the conversion runs on the GPU); spmv_run()
 * replaces Matrix_Format::spmv() for host buffers; spmv_run_device() is the
 * device-resident variant.  All entry points are plain C: pointers, sizes and status
 * codes, no CUDA or torch types.  Streams are passed as `void *` (a cudaStream_t).
 *
 * Errors: every entry point returns (or writes through `status`) one of SPMV_OK /
 * SPMV_ERR_*; spmv_last_error() gives the message of the calling thread's last error.
 * The reference instead prints and exits (error(), e.g. csr.cpp:131-132); the C++
 * plugin shim maps a non-zero status back to that behaviour.
 */
#ifndef SPMV_B200_H
#define SPMV_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
#define SPMV_OK                0
#define SPMV_ERR_ARG           1   /* invalid argument or parameter combination             */
#define SPMV_ERR_CSR           2   /* malformed CSR: row_ptr not monotone / col out of range */
#define SPMV_ERR_CUDA          3   /* CUDA runtime error                                     */
#define SPMV_ERR_NOMEM         4   /* device allocation failed                               */
#define SPMV_ERR_UNSUPPORTED   5   /* e.g. symmetric input that is not expanded (csr.cpp:131) */
#define SPMV_ERR_TIMEOUT       6   /* a bounded device wait gave up                          */
#define SPMV_ERR_BOUNDS        7   /* a device-side bounds check fired                       */
#define SPMV_ERR_NO_DEVICE     8   /* no CUDA device                                         */
#define SPMV_ERR_OVERFLOW      9   /* a converted array exceeds the 32-bit index range       */

/* ---------------------------------------------------------------- formats */
/* One id per reference format executable (src/Makefile_in:47-74, config.sh:183-196). */
#define SPMV_FMT_CSR_NAIVE     0   /* src/spmv_kernels/csr.cpp                    */
#define SPMV_FMT_CSR_VEC       1   /* src/spmv_kernels/csr_vec.cpp                */
#define SPMV_FMT_SELL          2   /* src/spmv_kernels/sell.cpp                   */
#define SPMV_FMT_SELL_SORTED   3   /* src/spmv_kernels/sell_sorted.cpp            */
#define SPMV_FMT_SELL_C_S      4   /* src/spmv_kernels/sell_c_s.cpp + sell-C-s/   */
#define SPMV_FMT_DIV_RF        5   /* src/spmv_kernels/DIV/div.cpp, DIV_TYPE_RF   */
#define SPMV_NUM_FORMATS       6

/* Value storage of a handle. */
#define SPMV_VALUES_F64        0   /* FP64 values and arithmetic: the drop-in                 */
#define SPMV_VALUES_F32        1   /* FP32 values, FP32 products, TwoSum-compensated row sums */

/*
 * Conversion parameters.  spmv_format_desc_init() fills the reference's defaults; the
 * layout-defining ones are those of the reference's x86 AVX2 build:
 *   num_threads      T   the OpenMP thread count the reference converts with; it defines
 *                        the thread ranges that sell / sell_sorted / div_rf layouts depend on
 *                        (sell.cpp:161, sell_sorted.cpp:164-180, div.cpp:263).   default 8
 *   vec_len          V/L csr_vec lanes, SELL slice height, DIV-RF lanes (VEC_LEN;
 *                        vectorization_x86_avx256_f64.h:22).                     default 4
 *   sellcs_c         C   SELL-C-sigma slice height, a power of two <= 256.       default 32
 *   sellcs_sigma     s   SELL-C-sigma sorting window, a multiple of C.           default 512
 *                        (the reference hard-codes C=256, s=16384 at sell_c_s.cpp:58-60)
 *   div_packet_vals      CSRCV_NUM_PACKET_VALS (config.sh:150).                  default 16384
 *   div_tolerance        DIV_VC_TOLERANCE, lossy value rounding (config.sh:123). default 0
 *   div_packet_reordering DIV_PACKET_REORDERING (config.sh:133): each thread's packet
 *                        groups stored in ascending order of a median column
 *                        (div.cpp:377-395, :455-498).                            default 0
 *   pack_cols            csr_naive (FP64 on kernel 4, and the FP32 variant): 1 = the kernel
 *                        reads a device copy of the column indices packed per staged block
 *                        (smallest column + a fixed bit width), 0 = plain int32 columns.
 *                        Values, y and the exported arrays are unchanged.        default 0
 *   row_assign           FP32 variant on its warp-specialised kernel: 1 = the row threads of
 *                        a staged block take its rows longest first, so a row warp's 32
 *                        rows have similar lengths; 0 = in row order.  y is unchanged.
 *                                                                                default 0
 *   exact                1: every row is summed in the reference format's own order
 *                        (bit-identical y); 0: rows longer than one staged block are
 *                        reduced in parallel (tolerance parity; kernels 0 and 3 only,
 *                        the others always sum in order).                          default 1
 *   values               SPMV_VALUES_F64 or SPMV_VALUES_F32.                       default F64
 *   block_nnz, block_rows, stages, ctas_per_sm, threads: kernel tuning knobs (entries
 *                    staged per block, rows per block, pipeline depth, CTAs per SM,
 *                    threads per CTA), 0 = default.
 *   wait_limit_us    bound of every device-side wait (a bulk copy landing, a stage hand-off):
 *                    a kernel whose wait runs out records SPMV_ERR_TIMEOUT (reported by the
 *                    next spmv_sync() / spmv_run()), waits for its own copies in flight and
 *                    leaves.  0 = about 2 s.                                   default 0
 *   debug_flags      SPMV_DEBUG_WITHHOLD_HANDOFF: the gather warps of the warp-specialised
 *                    kernels (4, 8 and the FP32 default) never hand a stage to the row
 *                    warps, so the row warps' wait runs out: a test of the timeout path
 *                    that faults nothing.                                      default 0
 *   kernel          -1: the format's default (10 for slices of 32 rows -- SELL-C-sigma
 *                       with C = 32, sell / sell_sorted with vec_len 32 -- without a
 *                       block_nnz, 8 for other SELL-C-sigma, 2 for DIV-RF with 32
 *                       lanes, 4 for the others);
 *                    0: CTA staged kernel (bulk copy + shared-memory gather, every format);
 *                    1: direct column-major kernel for slices of >= 32 rows;
 *                    2: warp-autonomous staged kernel (CSR, slices of <= 32 rows);
 *                    3: CTA staged kernel whose next-block x gather overlaps this block's
 *                       rows (every format but DIV-RF; block_nnz <= 8 * threads);
 *                    4: warp-specialised staged kernel: gather warps and block_rows row
 *                       threads (default 64 of 160) work on consecutive blocks at once
 *                       (every format but DIV-RF);
 *                    5: CTA staged kernel whose row threads load their own x, no gather
 *                       phase (every format but DIV-RF);
 *                    6: warp-autonomous kernel whose slice rows load their own x, no x
 *                       buffer (sell, sell_sorted, SELL-C-sigma with C <= 32);
 *                    7: FP32 variant only: segmented kernel, 256-entry chunks with Dot2
 *                       per lane and compensated merges across lanes and chunks (spreads
 *                       a single very long row over the whole GPU);
 *                    8: FP64 slices of >= 8 rows: kernel 4 over a copy of
 *                       the column indices laid out row-major in tiles of 8 slice
 *                       columns, so a gather warp reads 4 rows x 8 columns (the exported
 *                       arrays keep the reference layout);
 *                    9: FP64 slices of exactly 32 rows: kernel 6's warp-owned slices over
 *                       the same tiles; each warp loads x tile by tile and transposes it
 *                       between lanes (no x buffer);
 *                   10: FP64 slices of exactly 32 rows: warps claim runs of slices from a
 *                       queue (the heaviest slices first) and sum them from registers, the
 *                       next tile's columns and values loaded while this tile is summed and
 *                       the lines two tiles on prefetched into L2, x transposed between
 *                       lanes (no shared memory).  Its knobs: stages 1 = no prefetch,
 *                       3 = prefetch into L1, 5 / 6 = into L1 / L2 with items claimed one
 *                       ahead; block_nnz = prefetch distance (entries); block_rows =
 *                       work-item size in 256-entry tiles.
 *                    DIV-RF: 0 = one CTA per packet (any lane count), 2 = one warp per
 *                    packet, one lane per lane stream (32 lanes).             default -1
 */
typedef struct spmv_format_desc {
	int32_t format;
	int32_t num_threads;
	int32_t vec_len;
	int32_t sellcs_c;
	int32_t sellcs_sigma;
	int32_t div_packet_vals;
	double  div_tolerance;
	int32_t exact;
	int32_t values;
	int32_t block_nnz;
	int32_t block_rows;
	int32_t stages;
	int32_t ctas_per_sm;
	int32_t kernel;
	int32_t threads;
	int32_t wait_limit_us;
	int32_t debug_flags;
	int32_t div_packet_reordering;
	int32_t pack_cols;
	int32_t row_assign;
	int32_t reserved;
} spmv_format_desc;

#define SPMV_DEBUG_WITHHOLD_HANDOFF 1

typedef struct spmv_handle spmv_handle;

/* Per-handle information (Matrix_Format's public fields plus GPU facts). */
typedef struct spmv_info {
	int64_t m, n, nnz;
	double  mem_footprint;       /* bytes of the converted format (format-specific, as the reference) */
	double  csr_mem_footprint;   /* nnz*(sizeof(value)+4) + (m+1)*4  (spmv_kernel.h:23)          */
	int64_t stored_elems;        /* stored (padded) entries for sliced formats; nnz otherwise    */
	int64_t device_bytes;        /* device memory held by the handle                             */
	double  convert_ms;          /* GPU conversion time (host->device copy included)             */
	int32_t kernels_per_run;     /* kernel launches one spmv_run_device() makes                  */
	int32_t format;
	char    format_name[64];     /* the reference's format_name, e.g. "Naive_CSR_CPU" -> "Naive_CSR_GPU" */
	double  alloc_ms;            /* part of convert_ms spent in cudaMalloc                         */
	double  copy_in_ms;          /* part of convert_ms spent copying the CSR arrays to the device  */
	int64_t x_lo, x_hi;          /* span of x the converted format reads: its stored columns other
	                                than 0, padding included (empty if x_hi < x_lo)              */
	int64_t x_col0;              /* 1 if a stored column (or a padding entry) is 0.  spmv_run /
	                                spmv_run_f32 copy only x[0] (if x_col0) and x[x_lo..x_hi]   */
} spmv_info;

/* Fill *desc with the defaults above for `format`. */
void spmv_format_desc_init(spmv_format_desc * desc, int32_t format);

/*
 * csr_to_format: validate and convert a HOST CSR matrix (borrowed: it is copied, as every
 * reference format deep-copies, csr.cpp:55-66) into the requested GPU format on the
 * current CUDA device.  symmetric && !symmetry_expanded is rejected with
 * SPMV_ERR_UNSUPPORTED, as every reference format rejects it (csr.cpp:131).
 * Returns NULL on error with *status set.
 */
spmv_handle * spmv_create(const int32_t * row_ptr, const int32_t * col_ind, const double * values,
		int64_t m, int64_t n, int64_t nnz, int64_t symmetric, int64_t symmetry_expanded,
		const spmv_format_desc * desc, int * status);

/* As spmv_create, with the CSR arrays already in device memory (read-only, borrowed). */
spmv_handle * spmv_create_device(const int32_t * d_row_ptr, const int32_t * d_col_ind, const double * d_values,
		int64_t m, int64_t n, int64_t nnz, const spmv_format_desc * desc, void * stream, int * status);

/* Matrix_Format::spmv(x, y) with HOST buffers: x -> device (only x[x_lo..x_hi], the span the
 * converted matrix reads, see spmv_info), y[m] <- device, synchronous.
 * Rows without entries get 0 (the reference's y=1.0 probe, bench_spmv.cpp:561-564). */
int spmv_run(spmv_handle * h, const double * x, double * y);

/* Device-resident SpMV: d_x[n], d_y[m] in device memory, enqueued on `stream` (NULL =
 * the handle's stream); returns after the launch.  Errors raised by device-side checks
 * are reported by the next spmv_sync() / spmv_run(). */
int spmv_run_device(spmv_handle * h, const double * d_x, double * d_y, void * stream);

/* FP32 variant (handle created with values = SPMV_VALUES_F32): float x / y, device-resident
 * or host buffers (the reference's `_f` executables, ValueType = float, make.sh:148).
 * spmv_run() also accepts an FP32 handle: x is rounded to FP32 once and y widened. */
int spmv_run_device_f32(spmv_handle * h, const float * d_x, float * d_y, void * stream);
int spmv_run_f32(spmv_handle * h, const float * x, float * y);

/*
 * Allocation-free FP32-storage SpMV with FP64 vectors on the device.  No counterpart in
 * the reference.  For callers that cannot call cudaMalloc while they run: a host program
 * that owns all device memory through its own pool or arena and gives libraries none of
 * their own, or a loop with a deadline that cannot take the device-wide synchronisation a
 * cudaMalloc / cudaFree may cause.
 * Does what spmv_run() does with an FP32 handle and FP64 buffers (x rounded to FP32 once,
 * the Dot2-compensated FP32 SpMV, y widened to FP64), but on device vectors, enqueued on
 * `stream` (NULL: the handle's stream), and with its two temporaries (the FP32 x and the
 * FP32 y) in a fixed array that the library reserves statically on every GPU that loads
 * it, for as long as the process lives.
 *   - Limit: n + m <= SPMV_NOALLOC_MAX_ELEMS (262144 FP32 elements, 1 MiB); larger
 *     matrices get SPMV_ERR_ARG and nothing is launched.
 *   - The handle's device must be the current device (SPMV_ERR_ARG otherwise).
 *   - The first call on a device looks the array's device address up (once per device,
 *     with that device current): make that first call before any stream capture.  The
 *     address is not looked up again after a cudaDeviceReset(): do not use the entry point
 *     across one.
 *   - All calls on a device share the array, and it keeps what the last call wrote.  Every
 *     element a call reads it first writes, so nothing has to start at zero.  Calls whose
 *     executions overlap on the GPU (other streams, other host threads) race on it:
 *     serialise them.
 * Calls no cudaMalloc, cudaFree or other allocating routine.
 */
#define SPMV_NOALLOC_MAX_ELEMS 262144
int spmv_run_device_mixed_noalloc(spmv_handle * h, const double * d_x, double * d_y, void * stream);

/* ------------------------------------------------------------------ learned selector
 * No counterpart in the reference's SpMV path: its generator computes the same statistics on
 * the host (artificial-matrix-generator/artificial_matrix_generation.c:529-570, matrix_util.h).
 *
 * spmv_features(_device): the 10 structural features of a CSR matrix, computed on the GPU:
 *   [0] log2(m+1)  [1] log2(nnz+1)  [2] avg nnz/row  [3] std/avg nnz/row  [4] skew (max-avg)/avg
 *   [5] mean row bandwidth / n  [6] mean row scatter (degree / bandwidth)
 *   [7] avg neighbours (2 x entries within +1 column after each entry, per nnz)
 *   [8] cross-row similarity with the next non-empty row (window 1)
 *   [9] mean groups of consecutive columns / degree
 * Host arrays (copied) or device arrays on `stream`; out10 is host memory.
 */
int spmv_features(const int32_t * row_ptr, const int32_t * col_ind, int64_t m, int64_t n, int64_t nnz, double * out10);
int spmv_features_device(const int32_t * d_row_ptr, const int32_t * d_col_ind, int64_t m, int64_t n, int64_t nnz,
		double * out10, void * stream);

/* FP32 MLP in -> h1 -> h2 -> out (ReLU hidden layers, softmax cross-entropy on the logits),
 * trained and run by hand-written kernels.  Parameters are contiguous: W1[h1][in], b1[h1],
 * W2[h2][h1], b2[h2], W3[out][h2], b3[out] (spmv_mlp_num_params floats); init_params gives
 * their initial values (host).  spmv_mlp_get copies (0) parameters, (1) gradients of the
 * last spmv_mlp_loss_grad, (2) / (3) Adam first / second moments to host; spmv_mlp_set loads
 * parameters.  Batches are row-major [batch][in] device arrays; labels int32 class indices;
 * spmv_mlp_loss_grad writes the batch-mean loss to *loss_out (host) when given. */
typedef struct spmv_mlp spmv_mlp;
spmv_mlp * spmv_mlp_create(int32_t in, int32_t h1, int32_t h2, int32_t out, const float * init_params, int * status);
int32_t spmv_mlp_num_params(const spmv_mlp * mlp);
int spmv_mlp_get(const spmv_mlp * mlp, int32_t which, float * host_out);
int spmv_mlp_set(spmv_mlp * mlp, const float * host_params);
int spmv_mlp_forward(spmv_mlp * mlp, const float * d_x, int32_t batch, float * d_logits, void * stream);
/* Host-buffer inference: copies [batch][in] inputs in, runs the forward pass, copies the
 * [batch][out] logits back and waits (the selector's per-matrix query). */
int spmv_mlp_forward_host(spmv_mlp * mlp, const float * x_host, int32_t batch, float * logits_host);
int spmv_mlp_loss_grad(spmv_mlp * mlp, const float * d_x, const int32_t * d_labels, int32_t batch, float * loss_out,
		void * stream);
int spmv_mlp_adam_step(spmv_mlp * mlp, float lr, float beta1, float beta2, float eps, float weight_decay, void * stream);
void spmv_mlp_destroy(spmv_mlp * mlp);

/* Waits for the handle's stream and returns the first device-side error, if any. */
int spmv_sync(spmv_handle * h);

int spmv_get_info(const spmv_handle * h, spmv_info * out);

/*
 * Copies one converted array to host memory, for array-for-array parity with the
 * reference's csr_to_format.  If dst is NULL only *count (elements) is written.
 * Array ids and element types:
 */
#define SPMV_ARR_ROW_PTR          0   /* int32[m+1]           CSR                                */
#define SPMV_ARR_COL_IND          1   /* int32[nnz]           CSR                                */
#define SPMV_ARR_VALUES           2   /* f64[nnz] / f32[nnz]  CSR                                */
#define SPMV_ARR_SELL_PTR        10   /* int32[clusters+1]    sell, sell_sorted: row_cluster_ptr  */
#define SPMV_ARR_SELL_JA         11   /* int32[nnz_ext]       ja                                 */
#define SPMV_ARR_SELL_A          12   /* f64[nnz_ext]         a                                  */
#define SPMV_ARR_SELL_PERM       13   /* int32[m]             sell_sorted: permutation           */
#define SPMV_ARR_SELL_REV_PERM   14   /* int32[m]             sell_sorted: rev_permutation       */
#define SPMV_ARR_THREAD_RANGES   15   /* int64[2T]            per-thread [start, end)            */
#define SPMV_ARR_SELLCS_ORDER    20   /* int32[m]             row_order                          */
#define SPMV_ARR_SELLCS_WIDTHS   21   /* int32[slices]        slice_widths                       */
#define SPMV_ARR_SELLCS_PTR      22   /* int64[slices+1]      slice_pointers                     */
#define SPMV_ARR_SELLCS_COLS     23   /* int32[size]          column_indices                     */
#define SPMV_ARR_SELLCS_VALS     24   /* f64[size]            values                             */
#define SPMV_ARR_DIV_DATA        30   /* uint8[bytes]         all threads' packet streams, in thread order */
#define SPMV_ARR_DIV_PACKETS     31   /* int64[packets+1]     packet byte offsets                */
#define SPMV_ARR_DIV_GROUPS      32   /* int64[...]           each thread's packet-group offsets (groups+1 each) */
#define SPMV_ARR_DIV_THREAD_BYTES 33  /* int64[T]             bytes per thread                   */
#define SPMV_ARR_DIV_THREAD_GROUPS 34 /* int64[T]             packet groups per thread           */
int spmv_export(const spmv_handle * h, int32_t array_id, void * dst, int64_t * count);

void spmv_destroy(spmv_handle * h);

/* Message of the calling thread's last error ("" if none). */
const char * spmv_last_error(void);

/* Matrix_Format statistics hooks (spmv_kernel.h:18-19,29): CSV labels / values of the GPU
 * run (launches, stored entries, bytes moved per SpMV).  Return the characters written. */
int spmv_statistics_print_labels(char * buf, int64_t buf_n);
int spmv_statistics_print_data(const spmv_handle * h, char * buf, int64_t buf_n);

/* ---------------------------------------------------------------- batched SpMV */
/*
 * Many matrices, one persistent launch.  Each matrix is converted with its own descriptor
 * (an autotuner's pick: csr_naive, sell, sell_sorted or sell_c_s with its slice
 * parameters; the staging geometry -- block_nnz, stages, threads, exact -- of descs[0]
 * applies to the whole batch).  The staged blocks of all matrices form one work queue that
 * the kernel's CTAs drain through an atomic counter.  x and y are the matrices' vectors
 * concatenated in order (offsets from spmv_batch_info).  No reference counterpart: the
 * reference runs one matrix per process (src/bench.cpp:470-663).
 */
typedef struct spmv_batch spmv_batch;
spmv_batch * spmv_batch_create(int32_t count, const int32_t * const * row_ptrs, const int32_t * const * col_inds,
		const double * const * values, const int64_t * ms, const int64_t * ns, const spmv_format_desc * descs,
		int * status);
/* One launch (work-queue reset + persistent kernel) on `stream` (NULL: the batch's stream). */
int spmv_batch_run_device(spmv_batch * b, const double * d_x, double * d_y, void * stream);
/* The same two operations captured once into a CUDA graph (per (d_x, d_y) pair) and replayed. */
int spmv_batch_run_graph(spmv_batch * b, const double * d_x, double * d_y, void * stream);
int spmv_batch_sync(spmv_batch * b);
int spmv_batch_info(const spmv_batch * b, int64_t * total_x, int64_t * total_y, int64_t * total_nnz,
		int64_t * x_offsets, int64_t * y_offsets, int64_t * num_blocks);
void spmv_batch_destroy(spmv_batch * b);

/* ---------------------------------------------------------------- artificial matrices */
/*
 * The reference's artificial matrix generator, restated natively on the host
 * (artificial-matrix-generator/artificial_matrix_generation.c:163-579, argv order of
 * src/bench.cpp:564-578).  Output is independent of the thread count.  Two calls:
 * spmv_artgen_create() generates and returns an opaque result (NULL + *status on error);
 * spmv_artgen_get() copies its arrays (row_ptr int32[rows+1], col int32[nnz],
 * values f64[nnz], any may be NULL) and 37 structural statistics (may be NULL).
 */
typedef struct spmv_artgen spmv_artgen;
spmv_artgen * spmv_artgen_create(int64_t rows, int64_t cols, double avg_nnz_per_row, double std_nnz_per_row,
		const char * distribution, const char * placement, double bw, double skew,
		double avg_num_neighbours, double cross_row_similarity, uint32_t seed, int num_threads, int * status);
int64_t spmv_artgen_nnz(const spmv_artgen * g);
int spmv_artgen_get(const spmv_artgen * g, int32_t * row_ptr, int32_t * col_ind, double * values, double * stats);
void spmv_artgen_destroy(spmv_artgen * g);

/* ---------------------------------------------------------------- Matrix-Market import */
/*
 * The reference's real-matrix path (src/bench.cpp:127-238): mtx_read(filename,
 * expand_symmetry, pattern values 1.0) + mtx_values_convert_to_real
 * (lib/storage_formats/matrix_market/matrix_market.c:258-331, :421-463) + coo_to_csr with
 * sorted columns (lib/storage_formats/csr/csr_gen.c:178-210).  The text is parsed on the
 * host (strtol / strtod); COO -> CSR runs on the GPU.  expand_symmetry = 0 keeps a
 * symmetric file's stored triangle (the reference's KEEP_SYMMETRY build); its CSR is then
 * flagged symmetric and not expanded, which spmv_create() rejects as the reference's formats
 * do (csr.cpp:131).  Coordinate files only (the reference's import has no path for the
 * dense array format).  spmv_mtx_read returns NULL + *status on error (message in
 * spmv_last_error()).
 */
typedef struct spmv_mtx spmv_mtx;
spmv_mtx * spmv_mtx_read(const char * filename, int32_t expand_symmetry, int * status);
int spmv_mtx_info(const spmv_mtx * mtx, int64_t * m, int64_t * n, int64_t * nnz, int32_t * symmetric,
		int32_t * symmetry_expanded, int64_t * nnz_diag, int64_t * nnz_non_diag);
/* Copies row_ptr int32[m+1], col_ind int32[nnz], values f64[nnz] (any may be NULL). */
int spmv_mtx_get(const spmv_mtx * mtx, int32_t * row_ptr, int32_t * col_ind, double * values);
void spmv_mtx_destroy(spmv_mtx * mtx);

/* coo_to_csr(R, C, V, m, n, nnz, row_ptr, col_idx, values, sort_columns = 1, transpose = 0)
 * (csr_gen.c:178-210) on device arrays, enqueued on `stream`; d_vals may be NULL (values
 * 1.0).  Every row's entries come out sorted by column; entries repeated at one coordinate
 * keep their input order.  SPMV_ERR_CSR if a coordinate lies outside m x n. */
int spmv_coo_to_csr_device(const int32_t * d_rows, const int32_t * d_cols, const double * d_vals, int64_t m,
		int64_t n, int64_t nnz, int32_t * d_row_ptr, int32_t * d_col_ind, double * d_values, void * stream);

/* ---------------------------------------------------------------- symmetric matrices, RCM */
/*
 * The bench's symmetric transforms on the GPU (host CSR in, host CSR out through an opaque
 * result; NULL + *status on error):
 *   spmv_expand_symmetric  csr_expand_symmetric (lib/storage_formats/csr/csr_gen.c:256-336)
 *                          with sorted columns: a stored lower triangle to the full matrix
 *                          (an entry above the diagonal is SPMV_ERR_CSR, as the reference
 *                          stops on it);
 *   spmv_drop_upper        csr_drop_upper (csr_gen.c:344-420) with sorted columns;
 *   spmv_rcm               the bench's rcm() (src/bench.cpp:280-358): reverse Cuthill-McKee
 *                          (lib/rcm/rcm_gen.c:96-410) with sorted columns, of the full matrix
 *                          (symmetry_expanded = 1) or of a stored triangle (0: expanded first,
 *                          its upper triangle dropped after).  permutation[old row] = new row.
 * RCM ordering: the degree <= 1 vertices first in vertex order, then frontier by frontier
 * ordered by (earliest visited neighbour, degree, index), new components at the unvisited
 * vertex of least (degree, index); the reference places the degree <= 1 vertices through an
 * atomic counter, so the permutations agree with its one-thread run.
 */
typedef struct spmv_csr_out spmv_csr_out;
spmv_csr_out * spmv_expand_symmetric(const int32_t * row_ptr, const int32_t * col_ind, const double * values,
		int64_t m, int64_t n, int64_t nnz, int * status);
spmv_csr_out * spmv_drop_upper(const int32_t * row_ptr, const int32_t * col_ind, const double * values, int64_t m,
		int64_t n, int64_t nnz, int * status);
spmv_csr_out * spmv_rcm(const int32_t * row_ptr, const int32_t * col_ind, const double * values, int64_t m, int64_t n,
		int64_t nnz, int32_t symmetry_expanded, int * status);
int spmv_csr_out_info(const spmv_csr_out * out, int64_t * m, int64_t * n, int64_t * nnz, int64_t * nnz_diag);
/* row_ptr int32[m+1], col_ind int32[nnz], values f64[nnz], permutation int32[m] (RCM only);
 * any may be NULL. */
int spmv_csr_out_get(const spmv_csr_out * out, int32_t * row_ptr, int32_t * col_ind, double * values,
		int32_t * permutation);
void spmv_csr_out_destroy(spmv_csr_out * out);

/* ---------------------------------------------------------------- artificial matrices on the GPU */
/*
 * The same generator on the GPU (one thread per anchor segment: the reference reseeds with
 * seed + row at every anchor row, so segments are independent), into device memory on
 * `stream`.  The steps and the random stream are the host generator's; CUDA's log, cos,
 * exp, pow and sqrt may differ from glibc's in the last bit, so a value that lands on a
 * rounding or rejection boundary can differ: the matrices follow the reference's
 * distribution, and nearly always match it entry for entry.  Values are U[0,1).
 * spmv_gen_copy_device copies row_ptr int32[rows+1], col_ind int32[nnz], values f64[nnz]
 * (any may be NULL) into caller device arrays.
 */
typedef struct spmv_gen spmv_gen;
spmv_gen * spmv_gen_create_device(int64_t rows, int64_t cols, double avg_nnz_per_row, double std_nnz_per_row,
		const char * distribution, const char * placement, double bw, double skew, double avg_num_neighbours,
		double cross_row_similarity, uint32_t seed, void * stream, int * status);
int spmv_gen_info(const spmv_gen * gen, int64_t * m, int64_t * n, int64_t * nnz);
int spmv_gen_copy_device(const spmv_gen * gen, int32_t * d_row_ptr, int32_t * d_col_ind, double * d_values, void * stream);
void spmv_gen_destroy(spmv_gen * gen);
/* The GPU generator's per-segment code run on the host (host libm) into host arrays
 * (row_ptr[rows+1]; col_ind / values of cap entries); returns nnz or -1.  It checks that
 * code against spmv_artgen_create without a GPU. */
int64_t spmv_gen_host_check(int64_t rows, int64_t cols, double avg_nnz_per_row, double std_nnz_per_row,
		const char * distribution, const char * placement, double bw, double skew, double avg_num_neighbours,
		double cross_row_similarity, uint32_t seed, int32_t * row_ptr, int32_t * col_ind, double * values, int64_t cap);

/* Library version string. */
const char * spmv_version(void);

/* sizeof(spmv_format_desc) and sizeof(spmv_info) as built into the library.  A caller
 * compiled against another revision of this header compares them with its own sizeof and
 * stops, instead of the library reading or writing past the caller's structs. */
size_t spmv_format_desc_size(void);
size_t spmv_info_size(void);

#ifdef __cplusplus
}
#endif

#endif /* SPMV_B200_H */
