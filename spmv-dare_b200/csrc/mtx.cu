// Matrix-Market import: COO -> CSR on the GPU (the reference's coo_to_csr with sorted
// columns, lib/storage_formats/csr/csr_gen.c:178-210, as src/bench.cpp:218 calls it), and
// the C ABI of the reader (spmv_mtx_*; the text itself is parsed on the host, mtx_parse.c).
//
// coo_to_csr buckets the entries by row, then sorts each row by column
// (csr_sort_columns, csr_gen.c:96-171).  Here that is one stable LSD radix sort of the key
// (row, column) carrying the entry index, a gather of columns and values, and row
// pointers from a row histogram and a scan.  For coordinates that occur once each -- every
// Matrix-Market file the reference's readers accept -- this is exactly the reference's
// CSR; entries repeated at one coordinate keep their file order here, whereas the
// reference's per-row quicksort leaves their order to its pivoting.
#include <string.h>

#include <string>
#include <vector>

#include "internal.h"
#include "mtx_parse.h"
#include "primitives.cuh"

namespace spmv {

namespace {

int bits_of(int64_t v)
{
	int b = 0;
	while (v > 0) {
		b++;
		v >>= 1;
	}
	return b;
}

__global__ void coo_keys_kernel(const int32_t * R, const int32_t * C, int64_t nnz, int64_t m, int64_t n, int cbits,
		uint64_t * keys, uint32_t * idx, int32_t * counts, int * err)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nnz)
		return;
	const int32_t r = R[i], c = C[i];
	if (r < 0 || r >= m || c < 0 || c >= n) {
		atomicCAS(err, 0, 1);
		keys[i] = 0;
		idx[i] = (uint32_t) i;
		return;
	}
	keys[i] = ((uint64_t) r << cbits) | (uint64_t) c;
	idx[i] = (uint32_t) i;
	atomicAdd(&counts[r], 1);
}

__global__ void coo_gather_kernel(const uint64_t * keys, const uint32_t * idx, const double * V, int64_t nnz,
		uint64_t cmask, int32_t * col, double * val)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nnz)
		return;
	col[i] = (int32_t) (keys[i] & cmask);
	val[i] = V ? V[idx[i]] : 1.0;
}

__global__ void narrow_kernel(const int64_t * in, int32_t * out, int64_t n)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		out[i] = (int32_t) in[i];
}

}  // namespace

// COO -> CSR of device arrays on stream s (row_ptr[m+1], col[nnz], val[nnz] preallocated).
int coo_to_csr_device(const int32_t * R, const int32_t * C, const double * V, int64_t m, int64_t n, int64_t nnz,
		int32_t * row_ptr, int32_t * col, double * val, cudaStream_t s)
{
	if (m < 0 || n < 0 || nnz < 0 || m > INT32_MAX - 1 || n > INT32_MAX || nnz > INT32_MAX - 1) {
		set_error(SPMV_ERR_ARG, "coo_to_csr: sizes out of the 32-bit index range");
		return SPMV_ERR_ARG;
	}
	DevBuf keys, idx, counts, offs, err;
	SPMV_TRY(counts.alloc((m + 1) * sizeof(int32_t), s));
	SPMV_TRY(offs.alloc((m + 1) * sizeof(int64_t), s));
	SPMV_TRY(err.alloc(sizeof(int), s));
	SPMV_CUDA_TRY(cudaMemsetAsync(counts.p, 0, (m + 1) * sizeof(int32_t), s));
	SPMV_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(int), s));
	const int cbits = bits_of(n > 0 ? n - 1 : 0);
	const int rbits = bits_of(m > 0 ? m - 1 : 0);
	if (nnz > 0) {
		SPMV_TRY(keys.alloc(nnz * sizeof(uint64_t), s));
		SPMV_TRY(idx.alloc(nnz * sizeof(uint32_t), s));
		const unsigned g = (unsigned) ceil_div(nnz, 256);
		coo_keys_kernel<<<g, 256, 0, s>>>(R, C, nnz, m, n, cbits, keys.as<uint64_t>(), idx.as<uint32_t>(),
				counts.as<int32_t>(), err.as<int>());
		SPMV_CUDA_TRY(cudaGetLastError());
		int bad = 0;
		SPMV_CUDA_TRY(cudaMemcpyAsync(&bad, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
		SPMV_CUDA_TRY(cudaStreamSynchronize(s));
		if (bad) {
			set_error(SPMV_ERR_CSR, "coo_to_csr: a coordinate lies outside the %lld x %lld matrix", (long long) m,
					(long long) n);
			return SPMV_ERR_CSR;
		}
		SPMV_TRY(radix_sort_pairs(keys.as<uint64_t>(), idx.as<uint32_t>(), nnz, cbits + rbits, s));
		coo_gather_kernel<<<g, 256, 0, s>>>(keys.as<uint64_t>(), idx.as<uint32_t>(), V, nnz,
				cbits >= 64 ? ~0ULL : ((1ULL << cbits) - 1), col, val);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	SPMV_TRY(scan_exclusive(counts.as<int32_t>(), offs.as<int64_t>(), m, s));
	narrow_kernel<<<(unsigned) ceil_div(m + 1, 256), 256, 0, s>>>(offs.as<int64_t>(), row_ptr, m + 1);
	SPMV_CUDA_TRY(cudaGetLastError());
	return SPMV_OK;
}

}  // namespace spmv

struct spmv_mtx {
	int64_t m = 0, n = 0, nnz = 0, nnz_diag = 0, nnz_non_diag = 0;
	int32_t symmetric = 0, expanded = 0;
	std::vector<int32_t> row_ptr, col;
	std::vector<double> val;
};

extern "C" {

int spmv_coo_to_csr_device(const int32_t * d_rows, const int32_t * d_cols, const double * d_vals, int64_t m,
		int64_t n, int64_t nnz, int32_t * d_row_ptr, int32_t * d_col_ind, double * d_values, void * stream)
{
	spmv::clear_error();
	if (!d_row_ptr || (nnz > 0 && (!d_rows || !d_cols || !d_col_ind || !d_values))) {
		spmv::set_error(SPMV_ERR_ARG, "null array");
		return SPMV_ERR_ARG;
	}
	return spmv::coo_to_csr_device(d_rows, d_cols, d_vals, m, n, nnz, d_row_ptr, d_col_ind, d_values,
			(cudaStream_t) stream);
}

spmv_mtx * spmv_mtx_read(const char * filename, int32_t expand_symmetry, int * status)
{
	spmv::clear_error();
	int st = SPMV_OK;
	spmv_mtx * X = nullptr;
	mtx_coo coo;
	if (!filename) {
		spmv::set_error(SPMV_ERR_ARG, "null file name");
		st = SPMV_ERR_ARG;
	} else if (mtx_parse_file(filename, expand_symmetry, &coo) != 0) {
		spmv::set_error(SPMV_ERR_ARG, "Matrix-Market import: %s", coo.err);
		st = SPMV_ERR_ARG;
	} else {
		X = new spmv_mtx();
		X->m = coo.m;
		X->n = coo.n;
		X->nnz = coo.nnz;
		X->nnz_diag = coo.nnz_diag;
		X->nnz_non_diag = coo.nnz_non_diag;
		X->symmetric = coo.symmetric;
		X->expanded = coo.expanded;
		X->row_ptr.resize((size_t) coo.m + 1);
		X->col.resize((size_t) coo.nnz);
		X->val.resize((size_t) coo.nnz);
		cudaStream_t s = nullptr;
		int32_t * dR = nullptr, * dC = nullptr, * drp = nullptr, * dcol = nullptr;
		double * dV = nullptr, * dval = nullptr;
		const size_t nz = (size_t) (coo.nnz > 0 ? coo.nnz : 1);
		auto run = [&]() -> int {
			SPMV_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
			SPMV_CUDA_TRY(cudaMallocAsync((void **) &dR, nz * sizeof(int32_t), s));
			SPMV_CUDA_TRY(cudaMallocAsync((void **) &dC, nz * sizeof(int32_t), s));
			SPMV_CUDA_TRY(cudaMallocAsync((void **) &dV, nz * sizeof(double), s));
			SPMV_CUDA_TRY(cudaMallocAsync((void **) &drp, ((size_t) coo.m + 1) * sizeof(int32_t), s));
			SPMV_CUDA_TRY(cudaMallocAsync((void **) &dcol, nz * sizeof(int32_t), s));
			SPMV_CUDA_TRY(cudaMallocAsync((void **) &dval, nz * sizeof(double), s));
			if (coo.nnz > 0) {
				SPMV_CUDA_TRY(cudaMemcpyAsync(dR, coo.R, coo.nnz * sizeof(int32_t), cudaMemcpyHostToDevice, s));
				SPMV_CUDA_TRY(cudaMemcpyAsync(dC, coo.C, coo.nnz * sizeof(int32_t), cudaMemcpyHostToDevice, s));
				SPMV_CUDA_TRY(cudaMemcpyAsync(dV, coo.V, coo.nnz * sizeof(double), cudaMemcpyHostToDevice, s));
			}
			SPMV_TRY(spmv::coo_to_csr_device(dR, dC, dV, coo.m, coo.n, coo.nnz, drp, dcol, dval, s));
			SPMV_CUDA_TRY(cudaMemcpyAsync(X->row_ptr.data(), drp, ((size_t) coo.m + 1) * sizeof(int32_t),
					cudaMemcpyDeviceToHost, s));
			if (coo.nnz > 0) {
				SPMV_CUDA_TRY(cudaMemcpyAsync(X->col.data(), dcol, coo.nnz * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
				SPMV_CUDA_TRY(cudaMemcpyAsync(X->val.data(), dval, coo.nnz * sizeof(double), cudaMemcpyDeviceToHost, s));
			}
			SPMV_CUDA_TRY(cudaStreamSynchronize(s));
			return SPMV_OK;
		};
		st = run();
		for (void * p : {(void *) dR, (void *) dC, (void *) dV, (void *) drp, (void *) dcol, (void *) dval})
			if (p)
				cudaFreeAsync(p, s);
		if (s) {
			cudaStreamSynchronize(s);
			cudaStreamDestroy(s);
		}
		mtx_coo_free(&coo);
		if (st != SPMV_OK) {
			delete X;
			X = nullptr;
		}
	}
	if (status)
		*status = st;
	return X;
}

int spmv_mtx_info(const spmv_mtx * X, int64_t * m, int64_t * n, int64_t * nnz, int32_t * symmetric,
		int32_t * expanded, int64_t * nnz_diag, int64_t * nnz_non_diag)
{
	spmv::clear_error();
	if (!X) {
		spmv::set_error(SPMV_ERR_ARG, "null matrix");
		return SPMV_ERR_ARG;
	}
	if (m) *m = X->m;
	if (n) *n = X->n;
	if (nnz) *nnz = X->nnz;
	if (symmetric) *symmetric = X->symmetric;
	if (expanded) *expanded = X->expanded;
	if (nnz_diag) *nnz_diag = X->nnz_diag;
	if (nnz_non_diag) *nnz_non_diag = X->nnz_non_diag;
	return SPMV_OK;
}

int spmv_mtx_get(const spmv_mtx * X, int32_t * row_ptr, int32_t * col_ind, double * values)
{
	spmv::clear_error();
	if (!X) {
		spmv::set_error(SPMV_ERR_ARG, "null matrix");
		return SPMV_ERR_ARG;
	}
	if (row_ptr)
		memcpy(row_ptr, X->row_ptr.data(), X->row_ptr.size() * sizeof(int32_t));
	if (col_ind && X->nnz)
		memcpy(col_ind, X->col.data(), X->col.size() * sizeof(int32_t));
	if (values && X->nnz)
		memcpy(values, X->val.data(), X->val.size() * sizeof(double));
	return SPMV_OK;
}

void spmv_mtx_destroy(spmv_mtx * X)
{
	delete X;
}

}  // extern "C"
