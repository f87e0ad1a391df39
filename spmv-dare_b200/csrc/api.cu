// C ABI of libspmv_b200 (include/spmv_b200.h): handle lifetime, dispatch, export.
#include <stdarg.h>
#include <string.h>

#include <chrono>
#include <string>

#include "hostcopy.h"
#include "internal.h"
#include "primitives.cuh"

namespace spmv {

static thread_local int g_status = SPMV_OK;
static thread_local char g_msg[512] = "";

void set_error(int code, const char * fmt, ...)
{
	g_status = code;
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
	va_end(ap);
}

int last_status()
{
	return g_status;
}

void clear_error()
{
	g_status = SPMV_OK;
	g_msg[0] = 0;
}

static const char * kNames[SPMV_NUM_FORMATS] = {
	"Naive_CSR_B200", "Custom_CSR_VEC_B200", "SELL_B200", "SELL_SORTED_B200", "SELL_C_s_B200", "DIV_RF_B200",
};

static int check_desc(const spmv_format_desc & d)
{
	if (d.format < 0 || d.format >= SPMV_NUM_FORMATS) {
		set_error(SPMV_ERR_ARG, "unknown format id %d", d.format);
		return SPMV_ERR_ARG;
	}
	if (d.num_threads < 1 || d.num_threads > 4096) {
		set_error(SPMV_ERR_ARG, "num_threads must be in [1, 4096] (got %d)", d.num_threads);
		return SPMV_ERR_ARG;
	}
	if (d.vec_len < 1 || d.vec_len > 256 || (d.vec_len & (d.vec_len - 1))) {
		set_error(SPMV_ERR_ARG, "vec_len must be a power of two in [1, 256] (got %d)", d.vec_len);
		return SPMV_ERR_ARG;
	}
	if (d.format == SPMV_FMT_CSR_VEC && d.vec_len > 16) {
		set_error(SPMV_ERR_ARG, "csr_vec supports vec_len up to 16 (got %d)", d.vec_len);
		return SPMV_ERR_ARG;
	}
	if (d.format == SPMV_FMT_SELL_C_S) {
		int C = d.sellcs_c;
		if (C < 32 || C > 256 || (C & (C - 1))) {
			set_error(SPMV_ERR_ARG, "SELL-C-sigma: C must be a power of two in [32, 256] (got %d)", C);
			return SPMV_ERR_ARG;
		}
		if (d.sellcs_sigma < C || d.sellcs_sigma % C) {
			set_error(SPMV_ERR_ARG, "SELL-C-sigma: sigma must be a positive multiple of C (got C=%d sigma=%d)", C,
					d.sellcs_sigma);
			return SPMV_ERR_ARG;
		}
	}
	if (d.format == SPMV_FMT_DIV_RF) {
		if (d.div_packet_vals < 1 || d.div_packet_vals > (1 << 20)) {
			set_error(SPMV_ERR_ARG, "DIV-RF: packet values must be in [1, 2^20] (got %d)", d.div_packet_vals);
			return SPMV_ERR_ARG;
		}
		if (!(d.div_tolerance >= 0.0 && d.div_tolerance < 1.0)) {
			set_error(SPMV_ERR_ARG, "DIV-RF: tolerance must be in [0, 1) (got %g)", d.div_tolerance);
			return SPMV_ERR_ARG;
		}
	}
	if (d.wait_limit_us < 0 || d.wait_limit_us > 60000000) {
		set_error(SPMV_ERR_ARG, "wait_limit_us must be in [0, 60e6] (got %d)", d.wait_limit_us);
		return SPMV_ERR_ARG;
	}
	if (d.pack_cols != 0 && d.pack_cols != 1) {
		set_error(SPMV_ERR_ARG, "pack_cols must be 0 or 1 (got %d)", d.pack_cols);
		return SPMV_ERR_ARG;
	}
	if (d.pack_cols == 1 && d.format != SPMV_FMT_CSR_NAIVE) {
		set_error(SPMV_ERR_ARG, "pack_cols applies to csr_naive (FP64) and the FP32 variant");
		return SPMV_ERR_ARG;
	}
	if (d.row_assign != 0 && d.row_assign != 1) {
		set_error(SPMV_ERR_ARG, "row_assign must be 0 or 1 (got %d)", d.row_assign);
		return SPMV_ERR_ARG;
	}
	if (d.row_assign == 1 && (d.values != SPMV_VALUES_F32 || d.format != SPMV_FMT_CSR_NAIVE)) {
		set_error(SPMV_ERR_ARG, "row_assign applies to the FP32 variant on CSR");
		return SPMV_ERR_ARG;
	}
	if (d.div_packet_reordering != 0 && d.div_packet_reordering != 1) {
		set_error(SPMV_ERR_ARG, "div_packet_reordering must be 0 or 1 (got %d)", d.div_packet_reordering);
		return SPMV_ERR_ARG;
	}
	if (d.debug_flags & ~SPMV_DEBUG_WITHHOLD_HANDOFF) {
		set_error(SPMV_ERR_ARG, "unknown debug_flags bits 0x%x", d.debug_flags);
		return SPMV_ERR_ARG;
	}
	if (d.values != SPMV_VALUES_F64 && d.values != SPMV_VALUES_F32) {
		set_error(SPMV_ERR_ARG, "values must be SPMV_VALUES_F64 or SPMV_VALUES_F32");
		return SPMV_ERR_ARG;
	}
	if (d.values == SPMV_VALUES_F32 && d.format != SPMV_FMT_CSR_NAIVE &&
			!(d.format == SPMV_FMT_SELL_C_S && d.sellcs_c == 32)) {
		set_error(SPMV_ERR_ARG, "the FP32 variant stores CSR (format csr_naive) or SELL-C-sigma slices of 32 rows");
		return SPMV_ERR_ARG;
	}
	if (d.values == SPMV_VALUES_F32 && d.format == SPMV_FMT_SELL_C_S && d.kernel != -1) {
		set_error(SPMV_ERR_ARG, "the FP32 variant on 32-row slices has one kernel (kernel -1)");
		return SPMV_ERR_ARG;
	}
	if (d.block_nnz < 0 || d.block_nnz > 16384 || d.stages < 0 || d.stages > 8 || d.block_rows < 0 ||
			d.block_rows > 4096 || d.ctas_per_sm < 0 || d.ctas_per_sm > 32 || d.kernel < -1 || d.kernel > 10 ||
			!(d.threads == 0 || (d.threads % 32 == 0 && d.threads >= 64 && d.threads <= 512))) {
		set_error(SPMV_ERR_ARG, "tuning knob out of range");
		return SPMV_ERR_ARG;
	}
	if (d.kernel == 7 && d.values != SPMV_VALUES_F32) {
		set_error(SPMV_ERR_ARG, "kernel 7 (segmented) is the FP32 variant's kernel");
		return SPMV_ERR_ARG;
	}
	if ((d.kernel == 8 || d.kernel == 9 || d.kernel == 10) && d.values != SPMV_VALUES_F64) {
		set_error(SPMV_ERR_ARG, "kernels 8, 9 and 10 (tiled slices) run FP64 values");
		return SPMV_ERR_ARG;
	}
	return SPMV_OK;
}

// Releases every device resource of a handle (the Handle object itself is owned by the caller).
static void release_handle(Handle & h)
{
	if (h.stream)
		cudaStreamSynchronize(h.stream);
	for (void * p : h.allocations)
		cudaFree(p);
	h.allocations.clear();
	if (h.stream)
		cudaStreamDestroy(h.stream);
	h.stream = nullptr;
}

// Reference mem_footprint of each format (bytes).
static void set_footprints(Handle & h)
{
	const double vs = (h.desc.values == SPMV_VALUES_F32) ? 4.0 : 8.0;
	h.csr_mem_footprint = (double) h.nnz * (vs + 4.0) + (double) (h.m + 1) * 4.0;   // spmv_kernel.h:23
	switch (h.desc.format) {
	case SPMV_FMT_CSR_NAIVE:
	case SPMV_FMT_CSR_VEC:
		h.mem_footprint = h.csr_mem_footprint;                                       // csr.cpp:130
		h.stored_elems = h.nnz;
		break;
	case SPMV_FMT_SELL:
		h.mem_footprint = (double) (h.nclusters + 1) * 4.0 + (double) h.nnz_ext * 12.0;   // sell.cpp:197
		break;
	case SPMV_FMT_SELL_SORTED:
		h.mem_footprint = (double) (h.nclusters + 1) * 4.0 + (double) h.nnz_ext * 12.0 + (double) h.m * 4.0;
		break;
	case SPMV_FMT_SELL_C_S:
		h.mem_footprint = h.csr_mem_footprint;   // the reference reports the CSR size (sell_c_s.cpp:113)
		break;
	case SPMV_FMT_DIV_RF:
		h.mem_footprint = (double) h.div_bytes + (double) h.num_group_entries * 8.0;   // div.cpp:458-466
		h.stored_elems = h.nnz;
		break;
	}
}

static int init_device(Handle & h)
{
	int dev_count = 0;
	cudaError_t e = cudaGetDeviceCount(&dev_count);
	if (e != cudaSuccess || dev_count == 0) {
		set_error(SPMV_ERR_NO_DEVICE, "no CUDA device: %s", e != cudaSuccess ? cudaGetErrorString(e) : "count = 0");
		return SPMV_ERR_NO_DEVICE;
	}
	SPMV_CUDA_TRY(cudaGetDevice(&h.device));
	SPMV_CUDA_TRY(cudaDeviceGetAttribute(&h.num_sms, cudaDevAttrMultiProcessorCount, h.device));
	SPMV_CUDA_TRY(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
	SPMV_TRY(h.alloc(&h.d_err, 1));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_err, 0, sizeof(int), h.stream));
	return SPMV_OK;
}

// Over a stored column array (padding included): the smallest column other than 0, the
// largest column, and whether column 0 occurs (the padding column of SELL-C-sigma).
__global__ void col_span_kernel(const int32_t * c, int64_t n, int * lo_hi_zero)
{
	int lo = INT32_MAX, hi = -1, zero = 0;
	for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
		const int ci = c[i];
		if (ci == 0)
			zero = 1;
		else
			lo = min(lo, ci);
		hi = max(hi, ci);
	}
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
		hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
		zero |= __shfl_xor_sync(0xffffffffu, zero, o);
	}
	if ((threadIdx.x & 31) == 0) {
		atomicMin(&lo_hi_zero[0], lo);
		atomicMax(&lo_hi_zero[1], hi);
		if (zero)
			atomicOr(&lo_hi_zero[2], 1);
	}
}

// The parts of x the converted format reads, from the stored column array of the format
// (SELL's and SELL-C-sigma's padding columns included; DIV-RF reads the CSR columns):
// x[0] if column 0 occurs, and x[x_lo..x_hi] over the other columns.  spmv_run copies only
// those parts of a host x to the device.
static int set_x_span(Handle & h)
{
	const int32_t * c = h.d_ci;
	int64_t cnt = h.nnz;
	if (h.desc.format == SPMV_FMT_SELL || h.desc.format == SPMV_FMT_SELL_SORTED) {
		c = h.d_ja;
		cnt = h.nnz_ext;
	} else if (h.desc.format == SPMV_FMT_SELL_C_S) {
		c = h.d_scols;
		cnt = h.sellcs_size;
	}
	h.x_lo = 0;
	h.x_hi = -1;
	h.x_col0 = 0;
	if (cnt <= 0 || h.n <= 0)
		return SPMV_OK;
	int * d = nullptr;
	SPMV_TRY(h.alloc(&d, 3));
	const int init[3] = {INT32_MAX, -1, 0};
	SPMV_CUDA_TRY(cudaMemcpyAsync(d, init, sizeof(init), cudaMemcpyHostToDevice, h.stream));
	col_span_kernel<<<(unsigned) (cnt < 256 * 148 * 4 ? ceil_div(cnt, 256) : 148 * 4), 256, 0, h.stream>>>(c, cnt, d);
	SPMV_CUDA_TRY(cudaGetLastError());
	int lh[3];
	SPMV_CUDA_TRY(cudaMemcpyAsync(lh, d, sizeof(lh), cudaMemcpyDeviceToHost, h.stream));
	SPMV_CUDA_TRY(cudaStreamSynchronize(h.stream));
	h.x_col0 = lh[2];
	if (lh[0] != INT32_MAX) {          // some column above 0
		h.x_lo = lh[0];
		h.x_hi = lh[1];
	}
	return SPMV_OK;
}

// Host x -> device: x[0] when column 0 occurs, and x[x_lo..x_hi].
template <typename T>
static int copy_x_parts(const Handle & h, T * d_x, const T * x, cudaStream_t s)
{
	if (h.x_col0)
		SPMV_CUDA_TRY(cudaMemcpyAsync(d_x, x, sizeof(T), cudaMemcpyHostToDevice, s));
	if (h.x_hi >= h.x_lo)
		SPMV_CUDA_TRY(cudaMemcpyAsync(d_x + h.x_lo, x + h.x_lo, (h.x_hi - h.x_lo + 1) * sizeof(T),
				cudaMemcpyHostToDevice, s));
	return SPMV_OK;
}

static int convert_all(Handle & h)
{
	SPMV_TRY(validate_csr(h));
	switch (h.desc.format) {
	case SPMV_FMT_CSR_NAIVE:
	case SPMV_FMT_CSR_VEC:
		if (h.desc.values == SPMV_VALUES_F32) {
			SPMV_TRY(convert_f32(h));
			break;
		}
		SPMV_TRY(convert_csr(h));
		h.kernels_per_run = (h.num_blocks > 0 || h.num_chunks > 0) ? 1 : 0;
		break;
	case SPMV_FMT_SELL:
	case SPMV_FMT_SELL_SORTED:
		SPMV_TRY(convert_sell(h, h.desc.format == SPMV_FMT_SELL_SORTED));
		h.kernels_per_run = h.nclusters > 0 ? 1 : 0;
		break;
	case SPMV_FMT_SELL_C_S:
		SPMV_TRY(convert_sellcs(h));
		h.kernels_per_run = h.nslices > 0 ? 1 : 0;
		break;
	case SPMV_FMT_DIV_RF:
		SPMV_TRY(convert_div(h));
		break;
	}
	SPMV_CUDA_TRY(cudaStreamSynchronize(h.stream));
	set_footprints(h);
	SPMV_TRY(set_x_span(h));
	h.name = kNames[h.desc.format];
	if (h.desc.values == SPMV_VALUES_F32)
		h.name = h.desc.format == SPMV_FMT_SELL_C_S ? "SELL_C_s_F32_Dot2_B200" : "Naive_CSR_F32_Dot2_B200";
	return SPMV_OK;
}

static int create_common(Handle & h, const int32_t * rp, const int32_t * ci, const double * v, int64_t m, int64_t n,
		int64_t nnz, bool host, cudaStream_t user_stream)
{
	auto t0 = std::chrono::steady_clock::now();
	if (m < 0 || n < 0 || nnz < 0 || m > INT32_MAX - 1 || n > INT32_MAX || nnz > INT32_MAX - 64) {
		set_error(SPMV_ERR_ARG, "sizes out of the 32-bit index range (m=%lld n=%lld nnz=%lld)", (long long) m,
				(long long) n, (long long) nnz);
		return SPMV_ERR_ARG;
	}
	if ((m > 0 && !rp) || (nnz > 0 && (!ci || !v)) || (m == 0 && !rp)) {
		set_error(SPMV_ERR_ARG, "null CSR array");
		return SPMV_ERR_ARG;
	}
	h.m = m;
	h.n = n;
	h.nnz = nnz;
	SPMV_TRY(init_device(h));
	cudaStream_t s = h.stream;
	// device copies padded by SPMV_ENTRY_PAD zero entries (column 0, value 0): the staged
	// kernels copy whole 16-byte units, the FP32 segmented kernel whole 256-entry chunks
	SPMV_TRY(h.alloc(&h.d_rp, m + 1));
	SPMV_TRY(h.alloc(&h.d_ci, nnz + SPMV_ENTRY_PAD));
	SPMV_TRY(h.alloc(&h.d_v, nnz + SPMV_ENTRY_PAD));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_ci + nnz, 0, SPMV_ENTRY_PAD * sizeof(int32_t), s));
	SPMV_CUDA_TRY(cudaMemsetAsync(h.d_v + nnz, 0, SPMV_ENTRY_PAD * sizeof(double), s));
	const auto tc = std::chrono::steady_clock::now();
	if (host) {
		// pageable host arrays: large ones go through the pinned staging copy
		SPMV_CUDA_TRY(spmv_h2d_pageable(h.d_rp, rp, (m + 1) * sizeof(int32_t), s));
		if (nnz > 0) {
			SPMV_CUDA_TRY(spmv_h2d_pageable(h.d_ci, ci, nnz * sizeof(int32_t), s));
			SPMV_CUDA_TRY(spmv_h2d_pageable(h.d_v, v, nnz * sizeof(double), s));
		}
	} else {
		if (user_stream) {
			cudaEvent_t ev;
			SPMV_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
			SPMV_CUDA_TRY(cudaEventRecord(ev, user_stream));
			SPMV_CUDA_TRY(cudaStreamWaitEvent(s, ev, 0));
			cudaEventDestroy(ev);
		}
		SPMV_CUDA_TRY(cudaMemcpyAsync(h.d_rp, rp, (m + 1) * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
		if (nnz > 0) {
			SPMV_CUDA_TRY(cudaMemcpyAsync(h.d_ci, ci, nnz * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
			SPMV_CUDA_TRY(cudaMemcpyAsync(h.d_v, v, nnz * sizeof(double), cudaMemcpyDeviceToDevice, s));
		}
	}
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	h.copy_in_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tc).count();
	SPMV_TRY(convert_all(h));
	auto t1 = std::chrono::steady_clock::now();
	h.convert_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
	return SPMV_OK;
}

static int check_device_error(Handle & h)
{
	int e = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&e, h.d_err, sizeof(int), cudaMemcpyDeviceToHost, h.stream));
	SPMV_CUDA_TRY(cudaStreamSynchronize(h.stream));
	if (e == DEV_ERR_TIMEOUT) {
		set_error(SPMV_ERR_TIMEOUT, "a device-side wait ran out of its budget");
		return SPMV_ERR_TIMEOUT;
	}
	if (e != 0) {
		set_error(SPMV_ERR_BOUNDS, "a device-side check failed (code %d)", e);
		return SPMV_ERR_BOUNDS;
	}
	return SPMV_OK;
}

}  // namespace spmv

using spmv::Handle;

struct spmv_handle {
	Handle h;
};

namespace spmv {
Handle * handle_of(spmv_handle * H)
{
	return &H->h;
}
}  // namespace spmv

extern "C" {

void spmv_format_desc_init(spmv_format_desc * d, int32_t format)
{
	if (!d)
		return;
	memset(d, 0, sizeof(*d));
	d->format = format;
	d->num_threads = 8;
	d->vec_len = 4;
	d->sellcs_c = 32;
	d->sellcs_sigma = 512;
	d->div_packet_vals = 16384;
	d->div_tolerance = 0.0;
	d->exact = 1;
	d->values = SPMV_VALUES_F64;
	d->kernel = -1;
}

spmv_handle * spmv_create(const int32_t * row_ptr, const int32_t * col_ind, const double * values, int64_t m, int64_t n,
		int64_t nnz, int64_t symmetric, int64_t symmetry_expanded, const spmv_format_desc * desc, int * status)
{
	spmv::clear_error();
	int st = SPMV_OK;
	spmv_handle * H = nullptr;
	if (!desc) {
		spmv::set_error(SPMV_ERR_ARG, "null format descriptor");
		st = SPMV_ERR_ARG;
	} else if (symmetric && !symmetry_expanded) {
		spmv::set_error(SPMV_ERR_UNSUPPORTED, "symmetric matrices have to be expanded to be supported by this format");
		st = SPMV_ERR_UNSUPPORTED;
	} else if ((st = spmv::check_desc(*desc)) == SPMV_OK) {
		H = new spmv_handle();
		H->h.desc = *desc;
		st = spmv::create_common(H->h, row_ptr, col_ind, values, m, n, nnz, true, nullptr);
		if (st != SPMV_OK) {
			spmv::release_handle(H->h);
			delete H;
			H = nullptr;
		}
	}
	if (status)
		*status = st;
	return H;
}

spmv_handle * spmv_create_device(const int32_t * d_row_ptr, const int32_t * d_col_ind, const double * d_values,
		int64_t m, int64_t n, int64_t nnz, const spmv_format_desc * desc, void * stream, int * status)
{
	spmv::clear_error();
	int st = SPMV_OK;
	spmv_handle * H = nullptr;
	if (!desc) {
		spmv::set_error(SPMV_ERR_ARG, "null format descriptor");
		st = SPMV_ERR_ARG;
	} else if ((st = spmv::check_desc(*desc)) == SPMV_OK) {
		H = new spmv_handle();
		H->h.desc = *desc;
		st = spmv::create_common(H->h, d_row_ptr, d_col_ind, d_values, m, n, nnz, false, (cudaStream_t) stream);
		if (st != SPMV_OK) {
			spmv::release_handle(H->h);
			delete H;
			H = nullptr;
		}
	}
	if (status)
		*status = st;
	return H;
}

int spmv_run_device(spmv_handle * H, const double * d_x, double * d_y, void * stream)
{
	spmv::clear_error();
	if (!H || (!d_x && H->h.n > 0) || (!d_y && H->h.m > 0)) {
		spmv::set_error(SPMV_ERR_ARG, "null handle or vector");
		return SPMV_ERR_ARG;
	}
	Handle & h = H->h;
	if (h.desc.values != SPMV_VALUES_F64) {
		spmv::set_error(SPMV_ERR_ARG, "handle stores FP32 values: use spmv_run_device_f32");
		return SPMV_ERR_ARG;
	}
	cudaStream_t s = stream ? (cudaStream_t) stream : h.stream;
	return spmv::launch_spmv(h, d_x, d_y, s);
}

int spmv_run_device_f32(spmv_handle * H, const float * d_x, float * d_y, void * stream)
{
	spmv::clear_error();
	if (!H || (!d_x && H->h.n > 0) || (!d_y && H->h.m > 0)) {
		spmv::set_error(SPMV_ERR_ARG, "null handle or vector");
		return SPMV_ERR_ARG;
	}
	Handle & h = H->h;
	if (h.desc.values != SPMV_VALUES_F32) {
		spmv::set_error(SPMV_ERR_ARG, "handle stores FP64 values: use spmv_run_device");
		return SPMV_ERR_ARG;
	}
	cudaStream_t s = stream ? (cudaStream_t) stream : h.stream;
	return spmv::launch_spmv_f32(h, d_x, d_y, s);
}

int spmv_run(spmv_handle * H, const double * x, double * y)
{
	spmv::clear_error();
	if (!H || (!x && H->h.n > 0) || (!y && H->h.m > 0)) {
		spmv::set_error(SPMV_ERR_ARG, "null handle or vector");
		return SPMV_ERR_ARG;
	}
	Handle & h = H->h;
	if (!h.d_x) {
		SPMV_TRY(h.alloc(&h.d_x, h.n + 1));
		SPMV_TRY(h.alloc(&h.d_y, h.m + 1));
	}
	cudaStream_t s = h.stream;
	SPMV_TRY(copy_x_parts(h, h.d_x, x, s));       // only the parts of x the matrix reads
	if (h.desc.values == SPMV_VALUES_F32) {
		// FP32 handle driven with FP64 buffers: round x once, widen y
		if (!h.d_xf) {
			SPMV_TRY(h.alloc(&h.d_xf, h.n + 1));
			SPMV_TRY(h.alloc(&h.d_yf, h.m + 1));
		}
		SPMV_TRY(spmv::convert_vector_d2f(h.d_x, h.d_xf, h.n, s));
		SPMV_TRY(spmv::launch_spmv_f32(h, h.d_xf, h.d_yf, s));
		SPMV_TRY(spmv::convert_vector_f2d(h.d_yf, h.d_y, h.m, s));
	} else {
		SPMV_TRY(spmv::launch_spmv(h, h.d_x, h.d_y, s));
	}
	if (h.m > 0)
		SPMV_CUDA_TRY(cudaMemcpyAsync(y, h.d_y, h.m * sizeof(double), cudaMemcpyDeviceToHost, s));
	return spmv::check_device_error(h);
}

int spmv_run_f32(spmv_handle * H, const float * x, float * y)
{
	spmv::clear_error();
	if (!H || (!x && H->h.n > 0) || (!y && H->h.m > 0)) {
		spmv::set_error(SPMV_ERR_ARG, "null handle or vector");
		return SPMV_ERR_ARG;
	}
	Handle & h = H->h;
	if (h.desc.values != SPMV_VALUES_F32) {
		spmv::set_error(SPMV_ERR_ARG, "handle stores FP64 values: use spmv_run");
		return SPMV_ERR_ARG;
	}
	if (!h.d_xf) {
		SPMV_TRY(h.alloc(&h.d_xf, h.n + 1));
		SPMV_TRY(h.alloc(&h.d_yf, h.m + 1));
	}
	cudaStream_t s = h.stream;
	SPMV_TRY(copy_x_parts(h, h.d_xf, x, s));
	SPMV_TRY(spmv::launch_spmv_f32(h, h.d_xf, h.d_yf, s));
	if (h.m > 0)
		SPMV_CUDA_TRY(cudaMemcpyAsync(y, h.d_yf, h.m * sizeof(float), cudaMemcpyDeviceToHost, s));
	return spmv::check_device_error(h);
}

int spmv_run_device_mixed_noalloc(spmv_handle * H, const double * d_x, double * d_y, void * stream)
{
	spmv::clear_error();
	if (!H || (!d_x && H->h.n > 0) || (!d_y && H->h.m > 0)) {
		spmv::set_error(SPMV_ERR_ARG, "null handle or vector");
		return SPMV_ERR_ARG;
	}
	Handle & h = H->h;
	return spmv::run_mixed_noalloc(h, d_x, d_y, stream ? (cudaStream_t) stream : h.stream);
}

int spmv_sync(spmv_handle * H)
{
	spmv::clear_error();
	if (!H) {
		spmv::set_error(SPMV_ERR_ARG, "null handle");
		return SPMV_ERR_ARG;
	}
	SPMV_CUDA_TRY(cudaDeviceSynchronize());
	return spmv::check_device_error(H->h);
}

int spmv_get_info(const spmv_handle * H, spmv_info * out)
{
	if (!H || !out) {
		spmv::set_error(SPMV_ERR_ARG, "null handle or info");
		return SPMV_ERR_ARG;
	}
	const Handle & h = H->h;
	memset(out, 0, sizeof(*out));
	out->m = h.m;
	out->n = h.n;
	out->nnz = h.nnz;
	out->mem_footprint = h.mem_footprint;
	out->csr_mem_footprint = h.csr_mem_footprint;
	out->stored_elems = h.stored_elems;
	out->device_bytes = h.device_bytes;
	out->convert_ms = h.convert_ms;
	out->alloc_ms = h.alloc_ms;
	out->copy_in_ms = h.copy_in_ms;
	out->x_lo = h.x_lo;
	out->x_hi = h.x_hi;
	out->x_col0 = h.x_col0;
	out->kernels_per_run = h.kernels_per_run;
	out->format = h.desc.format;
	snprintf(out->format_name, sizeof(out->format_name), "%s", h.name.c_str());
	return SPMV_OK;
}

static int export_copy(const void * src, int64_t count, size_t elem, void * dst, int64_t * cnt)
{
	if (cnt)
		*cnt = count;
	if (!dst || count <= 0)
		return SPMV_OK;
	SPMV_CUDA_TRY(cudaMemcpy(dst, src, (size_t) count * elem, cudaMemcpyDeviceToHost));
	return SPMV_OK;
}

int spmv_export(const spmv_handle * H, int32_t id, void * dst, int64_t * count)
{
	spmv::clear_error();
	if (!H) {
		spmv::set_error(SPMV_ERR_ARG, "null handle");
		return SPMV_ERR_ARG;
	}
	const Handle & h = H->h;
	cudaStreamSynchronize(h.stream);
	const int fmt = h.desc.format;
	const bool sell = (fmt == SPMV_FMT_SELL || fmt == SPMV_FMT_SELL_SORTED);
	switch (id) {
	case SPMV_ARR_ROW_PTR: return export_copy(h.d_rp, h.m + 1, 4, dst, count);
	case SPMV_ARR_COL_IND: return export_copy(h.d_ci, h.nnz, 4, dst, count);
	case SPMV_ARR_VALUES:
		if (h.desc.values == SPMV_VALUES_F32 && fmt == SPMV_FMT_SELL_C_S)   // FP32 slices, column-major
			return export_copy(h.d_svals_f, h.sellcs_size, 4, dst, count);
		if (h.desc.values == SPMV_VALUES_F32)
			return export_copy(h.d_vf, h.nnz, 4, dst, count);
		return export_copy(h.d_v, h.nnz, 8, dst, count);
	case SPMV_ARR_SELL_PTR: if (sell) return export_copy(h.d_rcp, h.nclusters + 1, 4, dst, count); break;
	case SPMV_ARR_SELL_JA: if (sell) return export_copy(h.d_ja, h.nnz_ext, 4, dst, count); break;
	case SPMV_ARR_SELL_A: if (sell) return export_copy(h.d_a, h.nnz_ext, 8, dst, count); break;
	case SPMV_ARR_SELL_PERM: if (fmt == SPMV_FMT_SELL_SORTED) return export_copy(h.d_perm, h.m, 4, dst, count); break;
	case SPMV_ARR_SELL_REV_PERM: if (fmt == SPMV_FMT_SELL_SORTED) return export_copy(h.d_rev, h.m, 4, dst, count); break;
	case SPMV_ARR_THREAD_RANGES:
		if (h.d_ranges)
			return export_copy(h.d_ranges, 2 * (int64_t) h.desc.num_threads, 8, dst, count);
		break;
	case SPMV_ARR_SELLCS_ORDER: if (fmt == SPMV_FMT_SELL_C_S) return export_copy(h.d_order, h.m, 4, dst, count); break;
	case SPMV_ARR_SELLCS_WIDTHS: if (fmt == SPMV_FMT_SELL_C_S) return export_copy(h.d_widths, h.nslices, 4, dst, count); break;
	case SPMV_ARR_SELLCS_PTR: if (fmt == SPMV_FMT_SELL_C_S) return export_copy(h.d_sptr, h.nslices + 1, 8, dst, count); break;
	case SPMV_ARR_SELLCS_COLS: if (fmt == SPMV_FMT_SELL_C_S) return export_copy(h.d_scols, h.sellcs_size, 4, dst, count); break;
	case SPMV_ARR_SELLCS_VALS: if (fmt == SPMV_FMT_SELL_C_S) return export_copy(h.d_svals, h.sellcs_size, 8, dst, count); break;
	case SPMV_ARR_DIV_DATA: if (fmt == SPMV_FMT_DIV_RF) return export_copy(h.d_div, h.div_bytes, 1, dst, count); break;
	case SPMV_ARR_DIV_PACKETS: if (fmt == SPMV_FMT_DIV_RF) return export_copy(h.d_pkt, h.num_packets + 1, 8, dst, count); break;
	case SPMV_ARR_DIV_GROUPS: if (fmt == SPMV_FMT_DIV_RF) return export_copy(h.d_groups, h.num_group_entries, 8, dst, count); break;
	case SPMV_ARR_DIV_THREAD_BYTES: if (fmt == SPMV_FMT_DIV_RF) return export_copy(h.d_thread_bytes, h.desc.num_threads, 8, dst, count); break;
	case SPMV_ARR_DIV_THREAD_GROUPS: if (fmt == SPMV_FMT_DIV_RF) return export_copy(h.d_thread_groups, h.desc.num_threads, 8, dst, count); break;
	}
	spmv::set_error(SPMV_ERR_ARG, "array id %d is not part of format %d", id, fmt);
	return SPMV_ERR_ARG;
}

void spmv_destroy(spmv_handle * H)
{
	if (!H)
		return;
	spmv::release_handle(H->h);
	delete H;
}

const char * spmv_last_error(void)
{
	return spmv::g_msg;
}

int spmv_statistics_print_labels(char * buf, int64_t buf_n)
{
	if (!buf || buf_n <= 0)
		return 0;
	return snprintf(buf, (size_t) buf_n, ",gpu_format,gpu_stored_entries,gpu_mem_footprint_bytes,gpu_convert_ms,gpu_kernels_per_spmv");
}

int spmv_statistics_print_data(const spmv_handle * H, char * buf, int64_t buf_n)
{
	if (!H || !buf || buf_n <= 0)
		return 0;
	const Handle & h = H->h;
	return snprintf(buf, (size_t) buf_n, ",%s,%lld,%.0f,%.3f,%d", h.name.c_str(), (long long) h.stored_elems,
			h.mem_footprint, h.convert_ms, h.kernels_per_run);
}

struct artgen_result;
struct artgen_result * spmv_artgen_run(long nr_rows, long nr_cols, double avg_nnz_per_row, double std_nnz_per_row,
		const char * distribution, unsigned int seed, const char * placement, double bw_scaled, double skew,
		double avg_num_neighbours, double cross_row_similarity, int num_threads);
void spmv_artgen_free_result(struct artgen_result * R);

}  // extern "C"

// Layout of the generator result (artgen.c).
struct artgen_result_view {
	long rows, cols, nnz;
	int * row_ptr;
	int * col;
	double * val;
	double stats[37];
	int status;
};

struct spmv_artgen {
	artgen_result * r;
};

extern "C" {

spmv_artgen * spmv_artgen_create(int64_t rows, int64_t cols, double avg, double std, const char * distribution,
		const char * placement, double bw, double skew, double neigh, double cross, uint32_t seed, int num_threads,
		int * status)
{
	spmv::clear_error();
	int st = SPMV_OK;
	spmv_artgen * g = nullptr;
	if (rows < 1 || cols < 1 || rows > INT32_MAX - 1 || cols > INT32_MAX || !distribution || !placement) {
		spmv::set_error(SPMV_ERR_ARG, "artificial matrix: invalid sizes or null strings");
		st = SPMV_ERR_ARG;
	} else {
		artgen_result * r = spmv_artgen_run((long) rows, (long) cols, avg, std, distribution, seed, placement, bw, skew,
				neigh, cross, num_threads);
		if (!r) {
			spmv::set_error(SPMV_ERR_NOMEM, "artificial matrix: host allocation failed");
			st = SPMV_ERR_NOMEM;
		} else {
			int rs = reinterpret_cast<artgen_result_view *>(r)->status;
			if (rs != 0) {
				const char * why = rs == 2 ? "host allocation failed" : rs == 3 ? "nnz exceeds the 32-bit range"
						: rs == 4 ? "cross-row copy hit an occupied column (the reference exits here)" : "invalid arguments";
				spmv::set_error(rs == 2 ? SPMV_ERR_NOMEM : SPMV_ERR_ARG, "artificial matrix: %s", why);
				st = rs == 2 ? SPMV_ERR_NOMEM : SPMV_ERR_ARG;
				spmv_artgen_free_result(r);
			} else {
				g = new spmv_artgen{r};
			}
		}
	}
	if (status)
		*status = st;
	return g;
}

int64_t spmv_artgen_nnz(const spmv_artgen * g)
{
	return g ? reinterpret_cast<const artgen_result_view *>(g->r)->nnz : -1;
}

int spmv_artgen_get(const spmv_artgen * g, int32_t * row_ptr, int32_t * col_ind, double * values, double * stats)
{
	if (!g) {
		spmv::set_error(SPMV_ERR_ARG, "null generator result");
		return SPMV_ERR_ARG;
	}
	const artgen_result_view * r = reinterpret_cast<const artgen_result_view *>(g->r);
	if (row_ptr)
		memcpy(row_ptr, r->row_ptr, (r->rows + 1) * sizeof(int32_t));
	if (col_ind && r->nnz)
		memcpy(col_ind, r->col, r->nnz * sizeof(int32_t));
	if (values && r->nnz)
		memcpy(values, r->val, r->nnz * sizeof(double));
	if (stats)
		memcpy(stats, r->stats, sizeof(r->stats));
	return SPMV_OK;
}

void spmv_artgen_destroy(spmv_artgen * g)
{
	if (!g)
		return;
	spmv_artgen_free_result(g->r);
	delete g;
}

const char * spmv_version(void)
{
	return "spmv_b200 1.0 (sm_100a)";
}

size_t spmv_format_desc_size(void)
{
	return sizeof(spmv_format_desc);
}

size_t spmv_info_size(void)
{
	return sizeof(spmv_info);
}

}  // extern "C"
