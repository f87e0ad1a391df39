// Batched SpMV: hundreds of uneven matrices in one persistent launch (and one CUDA graph).
//
// spmv_batch_create converts every matrix with its own format descriptor (the autotuner's
// pick per matrix: csr_naive, sell, sell_sorted or sell_c_s with their slice parameters),
// then merges their staged-block tables into one work queue (long units first, so the
// dependent chains of huge rows start early) with a matrix id per block.  One launch of
// batch_kernel (spmv_kernels.cu) drains the queue: CTAs claim blocks through an atomic
// counter, so the load balances across matrices of any size.  x and y of all matrices are
// concatenated (offsets in spmv_batch_info).
//
// A batch whose matrices are all csr_naive is one SpMV of their block-diagonal matrix over
// the concatenated x and y: the batch then builds that merged CSR on the device (row
// pointers and columns shifted by the matrix offsets, each matrix's columns checked against
// its own n) and runs it as one csr_naive handle -- one launch of the warp-specialised
// kernel, whose blocks never straddle two matrices' rows.  Every row is still summed in the
// csr_naive order, so y is bit-identical to the matrices' own handles.
#include <string.h>

#include <algorithm>
#include <vector>

#include "internal.h"
#include "primitives.cuh"

struct spmv_handle;   // C ABI handle (api.cu)

namespace spmv {
Handle * handle_of(spmv_handle * H);
}

using spmv::Handle;

struct spmv_batch {
	std::vector<spmv_handle *> mats;
	std::vector<int64_t> x_off, y_off;
	int64_t total_x = 0, total_y = 0, total_nnz = 0;
	int device = 0;
	cudaStream_t stream = nullptr;
	spmv::StagedBlock * d_blocks = nullptr;
	int32_t * d_bmat = nullptr;
	spmv::BatchMat * d_mats = nullptr;
	unsigned long long * d_counter = nullptr;
	int * d_err = nullptr;
	int64_t nblocks = 0;
	int cap = 0, stages = 0, threads = 0, grid = 0;
	size_t smem = 0;
	int exact = 1;
	spmv_handle * merged = nullptr;    // all-csr_naive batches: the block-diagonal matrix
	// cached CUDA graph of (counter reset + kernel) for one (x, y) pair
	cudaGraphExec_t graph = nullptr;
	const double * graph_x = nullptr;
	double * graph_y = nullptr;
	std::vector<void *> allocs;
};

namespace {

template <typename T>
int balloc(spmv_batch * b, T ** p, int64_t count)
{
	cudaError_t e = cudaMalloc((void **) p, (size_t) (count > 0 ? count : 1) * sizeof(T));
	if (e != cudaSuccess) {
		spmv::set_error(SPMV_ERR_NOMEM, "batch allocation failed: %s", cudaGetErrorString(e));
		return SPMV_ERR_NOMEM;
	}
	b->allocs.push_back((void *) *p);
	return SPMV_OK;
}

void release(spmv_batch * b)
{
	if (b->graph)
		cudaGraphExecDestroy(b->graph);
	if (b->merged)
		spmv_destroy(b->merged);
	for (spmv_handle * h : b->mats)
		spmv_destroy(h);
	for (void * p : b->allocs)
		cudaFree(p);
	if (b->stream)
		cudaStreamDestroy(b->stream);
	delete b;
}

__global__ void merge_rows_kernel(const int32_t * rp, int64_t m, int64_t row_off, int64_t nnz_off, int32_t * out)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < m)
		out[row_off + i] = (int32_t) (rp[i] + nnz_off);
}

// Shifts one matrix's columns by its x offset, flagging any column outside [0, n).
__global__ void merge_cols_kernel(int32_t * ci, int64_t nnz, int64_t n, int64_t x_off, int * bad)
{
	const int64_t j = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= nnz)
		return;
	const int32_t c = ci[j];
	if (c < 0 || (int64_t) c >= n)
		atomicOr(bad, 1);
	ci[j] = (int32_t) (c + x_off);
}

// The block-diagonal csr_naive handle of an all-csr_naive batch.
int build_merged(spmv_batch * b, int32_t count, const int32_t * const * row_ptrs, const int32_t * const * col_inds,
		const double * const * values, const int64_t * ms, const int64_t * ns, const spmv_format_desc & d0)
{
	int64_t M = 0, N = 0, NNZ = 0, maxm = 0;
	for (int32_t i = 0; i < count; i++) {
		if (ms[i] < 0 || ns[i] < 0 || !row_ptrs[i] || row_ptrs[i][0] != 0) {
			spmv::set_error(SPMV_ERR_CSR, "batch: matrix %d: row_ptr[0] must be 0", i);
			return SPMV_ERR_CSR;
		}
		b->x_off.push_back(N);
		b->y_off.push_back(M);
		M += ms[i];
		N += ns[i];
		NNZ += row_ptrs[i][ms[i]];
		maxm = ms[i] > maxm ? ms[i] : maxm;
	}
	if (M >= INT32_MAX || N >= INT32_MAX || NNZ >= (int64_t) INT32_MAX - 16) {
		spmv::set_error(SPMV_ERR_OVERFLOW, "batch: the merged matrix exceeds 32-bit indices");
		return SPMV_ERR_OVERFLOW;
	}
	cudaStream_t s = b->stream;
	int32_t *rp = nullptr, *ci = nullptr, *tmp = nullptr;
	double * v = nullptr;
	int * bad = nullptr;
	int st = SPMV_OK;
	auto fail = [&](cudaError_t e) {
		if (e != cudaSuccess && st == SPMV_OK) {
			spmv::set_error(e == cudaErrorMemoryAllocation ? SPMV_ERR_NOMEM : SPMV_ERR_CUDA, "batch merge: %s",
					cudaGetErrorString(e));
			st = e == cudaErrorMemoryAllocation ? SPMV_ERR_NOMEM : SPMV_ERR_CUDA;
		}
	};
	fail(cudaMalloc((void **) &rp, (M + 1) * sizeof(int32_t)));
	fail(cudaMalloc((void **) &ci, (NNZ + 1) * sizeof(int32_t)));
	fail(cudaMalloc((void **) &v, (NNZ + 1) * sizeof(double)));
	fail(cudaMalloc((void **) &tmp, (maxm + 1) * sizeof(int32_t)));
	fail(cudaMalloc((void **) &bad, sizeof(int)));
	if (st == SPMV_OK)
		fail(cudaMemsetAsync(bad, 0, sizeof(int), s));
	int64_t nnz_off = 0;
	for (int32_t i = 0; i < count && st == SPMV_OK; i++) {
		const int64_t nnz = row_ptrs[i][ms[i]];
		if (ms[i] > 0) {
			fail(cudaMemcpyAsync(tmp, row_ptrs[i], ms[i] * sizeof(int32_t), cudaMemcpyHostToDevice, s));
			merge_rows_kernel<<<(unsigned) spmv::ceil_div(ms[i], 256), 256, 0, s>>>(tmp, ms[i], b->y_off[i], nnz_off, rp);
			fail(cudaGetLastError());
		}
		if (nnz > 0) {
			fail(cudaMemcpyAsync(ci + nnz_off, col_inds[i], nnz * sizeof(int32_t), cudaMemcpyHostToDevice, s));
			fail(cudaMemcpyAsync(v + nnz_off, values[i], nnz * sizeof(double), cudaMemcpyHostToDevice, s));
			merge_cols_kernel<<<(unsigned) spmv::ceil_div(nnz, 256), 256, 0, s>>>(ci + nnz_off, nnz, ns[i], b->x_off[i], bad);
			fail(cudaGetLastError());
		}
		// a pageable source is copied before the call returns, so tmp may be refilled
		fail(cudaStreamSynchronize(s));
		nnz_off += nnz;
	}
	if (st == SPMV_OK) {
		const int32_t last = (int32_t) NNZ;
		fail(cudaMemcpyAsync(rp + M, &last, sizeof(int32_t), cudaMemcpyHostToDevice, s));
		int hbad = 0;
		fail(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
		fail(cudaStreamSynchronize(s));
		if (st == SPMV_OK && hbad) {
			spmv::set_error(SPMV_ERR_CSR, "batch: a column index is outside its matrix's [0, n)");
			st = SPMV_ERR_CSR;
		}
	}
	if (st == SPMV_OK) {
		spmv_format_desc d;
		spmv_format_desc_init(&d, SPMV_FMT_CSR_NAIVE);
		d.exact = d0.exact;
		b->merged = spmv_create_device(rp, ci, v, M, N, NNZ, &d, b->stream, &st);
	}
	for (void * p : {(void *) rp, (void *) ci, (void *) v, (void *) tmp, (void *) bad})
		if (p)
			cudaFree(p);
	if (st != SPMV_OK)
		return st;
	b->total_x = N;
	b->total_y = M;
	b->total_nnz = NNZ;
	b->nblocks = spmv::handle_of(b->merged)->num_blocks;
	return SPMV_OK;
}

int enqueue(spmv_batch * b, const double * d_x, double * d_y, cudaStream_t s)
{
	if (b->merged)
		return spmv_run_device(b->merged, d_x, d_y, s);
	SPMV_CUDA_TRY(cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), s));
	if (b->nblocks == 0)
		return SPMV_OK;
	spmv::BatchArgs a{};
	a.blocks = b->d_blocks;
	a.bmat = b->d_bmat;
	a.nblocks = b->nblocks;
	a.mats = b->d_mats;
	a.x = d_x;
	a.y = d_y;
	a.cap_al = b->cap + 8;
	a.stages = b->stages;
	a.stage_bytes = (int) (spmv::ceil_div((int64_t) a.cap_al * 12, 128) * 128);
	a.exact = b->exact;
	a.counter = b->d_counter;
	a.err = b->d_err;
	return spmv::batch_launch(a, b->grid, b->threads, b->smem, s);
}

}  // namespace

extern "C" {

spmv_batch * spmv_batch_create(int32_t count, const int32_t * const * row_ptrs, const int32_t * const * col_inds,
		const double * const * values, const int64_t * ms, const int64_t * ns, const spmv_format_desc * descs,
		int * status)
{
	int st = SPMV_OK;
	if (count < 0 || (count > 0 && (!row_ptrs || !col_inds || !values || !ms || !ns || !descs))) {
		spmv::set_error(SPMV_ERR_ARG, "batch: null arrays");
		if (status)
			*status = SPMV_ERR_ARG;
		return nullptr;
	}
	spmv_batch * b = new spmv_batch();
	bool all_csr = count > 0;
	for (int32_t i = 0; i < count; i++)
		all_csr = all_csr && descs[i].format == SPMV_FMT_CSR_NAIVE && descs[i].values == SPMV_VALUES_F64;
	if (all_csr) {
		cudaGetDevice(&b->device);
		if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
			spmv::set_error(SPMV_ERR_CUDA, "batch: stream creation failed");
			st = SPMV_ERR_CUDA;
		}
		if (st == SPMV_OK)
			st = build_merged(b, count, row_ptrs, col_inds, values, ms, ns, descs[0]);
		if (st == SPMV_OK)
			st = balloc(b, &b->d_err, 1);
		if (st == SPMV_OK && cudaMemset(b->d_err, 0, sizeof(int)) != cudaSuccess)
			st = SPMV_ERR_CUDA;
		if (st != SPMV_OK) {
			release(b);
			b = nullptr;
		}
		if (status)
			*status = st;
		return b;
	}
	// one staging geometry for the whole batch (that of the first descriptor)
	b->cap = (count > 0 && descs[0].block_nnz > 0) ? descs[0].block_nnz : 1024;
	b->cap = (b->cap + 7) & ~7;
	b->stages = (count > 0 && descs[0].stages > 0) ? descs[0].stages : 2;
	b->threads = (count > 0 && descs[0].threads > 0) ? descs[0].threads : 256;
	b->exact = count > 0 ? descs[0].exact : 1;
	std::vector<spmv::BatchMat> hm(count);
	std::vector<spmv::StagedBlock> blocks;
	std::vector<int32_t> bmat;
	std::vector<int64_t> order_long, order_rest;
	for (int32_t i = 0; i < count && st == SPMV_OK; i++) {
		spmv_format_desc d = descs[i];
		if (!(d.format == SPMV_FMT_CSR_NAIVE || d.format == SPMV_FMT_SELL || d.format == SPMV_FMT_SELL_SORTED ||
				d.format == SPMV_FMT_SELL_C_S)) {
			spmv::set_error(SPMV_ERR_ARG, "batch: matrix %d: format %d is not batchable "
					"(csr_naive, sell, sell_sorted, sell_c_s)", i, d.format);
			st = SPMV_ERR_ARG;
			break;
		}
		d.kernel = 0;
		d.block_nnz = b->cap;
		d.stages = b->stages;
		d.threads = b->threads;
		d.exact = b->exact;
		d.values = SPMV_VALUES_F64;
		const int64_t nnz = row_ptrs[i][ms[i]];
		spmv_handle * H = spmv_create(row_ptrs[i], col_inds[i], values[i], ms[i], ns[i], nnz, 0, 1, &d, &st);
		if (!H)
			break;
		b->mats.push_back(H);
		Handle & h = *spmv::handle_of(H);
		spmv::BatchMat & mt = hm[i];
		mt.m = h.m;
		mt.x_off = b->total_x;
		mt.y_off = b->total_y;
		b->x_off.push_back(b->total_x);
		b->y_off.push_back(b->total_y);
		b->total_x += h.n;
		b->total_y += h.m;
		b->total_nnz += h.nnz;
		if (d.format == SPMV_FMT_CSR_NAIVE) {
			mt.kind = 0;
			mt.V = 1;
			mt.ptr = h.d_rp;
			mt.cols = h.d_ci;
			mt.vals = h.d_v;
			mt.ymap = nullptr;
		} else if (d.format == SPMV_FMT_SELL_C_S) {
			mt.kind = 1;
			mt.V = d.sellcs_c;
			mt.ptr = h.d_sptr32;
			mt.cols = h.d_scols;
			mt.vals = h.d_svals;
			mt.ymap = h.d_order;
		} else {
			mt.kind = 1;
			mt.V = d.vec_len;
			mt.ptr = h.d_rcp;
			mt.cols = h.d_ja;
			mt.vals = h.d_a;
			mt.ymap = (d.format == SPMV_FMT_SELL_SORTED) ? h.d_rev : nullptr;
		}
		std::vector<spmv::StagedBlock> hb(h.num_blocks);
		if (h.num_blocks > 0 && cudaMemcpy(hb.data(), h.d_blocks, h.num_blocks * sizeof(spmv::StagedBlock),
					cudaMemcpyDeviceToHost) != cudaSuccess) {
			spmv::set_error(SPMV_ERR_CUDA, "batch: block table copy failed");
			st = SPMV_ERR_CUDA;
			break;
		}
		for (const spmv::StagedBlock & sb : hb) {
			blocks.push_back(sb);
			bmat.push_back(i);
			(sb.units < 0 ? order_long : order_rest).push_back((int64_t) blocks.size() - 1);
		}
	}
	if (st == SPMV_OK) {
		// long units first: their serial chains start while the short blocks stream
		std::vector<spmv::StagedBlock> ob;
		std::vector<int32_t> om;
		ob.reserve(blocks.size());
		om.reserve(blocks.size());
		for (int64_t k : order_long) {
			ob.push_back(blocks[k]);
			om.push_back(bmat[k]);
		}
		for (int64_t k : order_rest) {
			ob.push_back(blocks[k]);
			om.push_back(bmat[k]);
		}
		b->nblocks = (int64_t) ob.size();
		cudaGetDevice(&b->device);
		if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
			spmv::set_error(SPMV_ERR_CUDA, "batch: stream creation failed");
			st = SPMV_ERR_CUDA;
		}
		if (st == SPMV_OK)
			st = balloc(b, &b->d_blocks, b->nblocks);
		if (st == SPMV_OK)
			st = balloc(b, &b->d_bmat, b->nblocks);
		if (st == SPMV_OK)
			st = balloc(b, &b->d_mats, count);
		if (st == SPMV_OK)
			st = balloc(b, &b->d_counter, 1);
		if (st == SPMV_OK)
			st = balloc(b, &b->d_err, 1);
		if (st == SPMV_OK) {
			cudaMemcpy(b->d_blocks, ob.data(), ob.size() * sizeof(spmv::StagedBlock), cudaMemcpyHostToDevice);
			cudaMemcpy(b->d_bmat, om.data(), om.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
			cudaMemcpy(b->d_mats, hm.data(), hm.size() * sizeof(spmv::BatchMat), cudaMemcpyHostToDevice);
			cudaMemset(b->d_err, 0, sizeof(int));
			const int cap_al = b->cap + 8;
			const int stage_bytes = (int) (spmv::ceil_div((int64_t) cap_al * 12, 128) * 128);
			const int max_stages = (int) ((220 * 1024 - 64 - cap_al * 8) / stage_bytes);
			if (b->stages > max_stages)
				b->stages = max_stages > 0 ? max_stages : 1;
			b->smem = (size_t) b->stages * stage_bytes + (size_t) cap_al * 8 + 64;
			int per_sm = 0, sms = 0;
			st = spmv::batch_occupancy(b->threads, b->smem, &per_sm);
			cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
			b->grid = sms * (per_sm > 0 ? per_sm : 1);
		}
	}
	if (st != SPMV_OK) {
		release(b);
		b = nullptr;
	}
	if (status)
		*status = st;
	return b;
}

int spmv_batch_run_device(spmv_batch * b, const double * d_x, double * d_y, void * stream)
{
	if (!b || (!d_x && b->total_x > 0) || (!d_y && b->total_y > 0)) {
		spmv::set_error(SPMV_ERR_ARG, "batch: null argument");
		return SPMV_ERR_ARG;
	}
	return enqueue(b, d_x, d_y, stream ? (cudaStream_t) stream : b->stream);
}

int spmv_batch_run_graph(spmv_batch * b, const double * d_x, double * d_y, void * stream)
{
	if (!b || (!d_x && b->total_x > 0) || (!d_y && b->total_y > 0)) {
		spmv::set_error(SPMV_ERR_ARG, "batch: null argument");
		return SPMV_ERR_ARG;
	}
	cudaStream_t s = stream ? (cudaStream_t) stream : b->stream;
	if (!b->graph || b->graph_x != d_x || b->graph_y != d_y) {
		if (b->graph) {
			cudaGraphExecDestroy(b->graph);
			b->graph = nullptr;
		}
		cudaGraph_t g;
		SPMV_CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
		int st = enqueue(b, d_x, d_y, b->stream);
		cudaError_t e = cudaStreamEndCapture(b->stream, &g);
		if (st != SPMV_OK)
			return st;
		SPMV_CUDA_TRY(e);
		SPMV_CUDA_TRY(cudaGraphInstantiate(&b->graph, g, 0));
		cudaGraphDestroy(g);
		b->graph_x = d_x;
		b->graph_y = d_y;
	}
	SPMV_CUDA_TRY(cudaGraphLaunch(b->graph, s));
	return SPMV_OK;
}

int spmv_batch_sync(spmv_batch * b)
{
	if (!b) {
		spmv::set_error(SPMV_ERR_ARG, "batch: null handle");
		return SPMV_ERR_ARG;
	}
	SPMV_CUDA_TRY(cudaDeviceSynchronize());
	if (b->merged)
		return spmv_sync(b->merged);
	int e = 0;
	SPMV_CUDA_TRY(cudaMemcpy(&e, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
	if (e == DEV_ERR_TIMEOUT) {
		spmv::set_error(SPMV_ERR_TIMEOUT, "batch: a device-side wait ran out of its budget");
		return SPMV_ERR_TIMEOUT;
	}
	return SPMV_OK;
}

int spmv_batch_info(const spmv_batch * b, int64_t * total_x, int64_t * total_y, int64_t * total_nnz,
		int64_t * x_offsets, int64_t * y_offsets, int64_t * num_blocks)
{
	if (!b) {
		spmv::set_error(SPMV_ERR_ARG, "batch: null handle");
		return SPMV_ERR_ARG;
	}
	if (total_x)
		*total_x = b->total_x;
	if (total_y)
		*total_y = b->total_y;
	if (total_nnz)
		*total_nnz = b->total_nnz;
	if (num_blocks)
		*num_blocks = b->nblocks;
	if (x_offsets)
		memcpy(x_offsets, b->x_off.data(), b->x_off.size() * sizeof(int64_t));
	if (y_offsets)
		memcpy(y_offsets, b->y_off.data(), b->y_off.size() * sizeof(int64_t));
	return SPMV_OK;
}

void spmv_batch_destroy(spmv_batch * b)
{
	if (b)
		release(b);
}

}  // extern "C"
