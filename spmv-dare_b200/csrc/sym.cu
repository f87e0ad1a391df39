// Symmetric-matrix transforms of the reference's bench on the GPU: csr_expand_symmetric and
// csr_drop_upper (lib/storage_formats/csr/csr_gen.c:256-420, sorted columns) and the RCM
// reordering of src/bench.cpp:280-358 (rcm(): expand a stored triangle, reverse Cuthill-McKee
// with sorted columns, drop the upper triangle again), whose ordering follows
// reverse_cuthill_mckee (lib/rcm/rcm_gen.c:96-410):
//   1. every vertex of degree <= 1 first, in vertex order;
//   2. while vertices remain: if the last frontier found no new vertex, start a new component
//      at the unvisited vertex of least (degree, index); the next frontier is every unvisited
//      neighbour of the vertices added since the previous step (the first step: of all vertices
//      placed so far), ordered by (earliest position of a visited neighbour, degree, index);
//   3. permutation[R[i]] = m - 1 - i; row i moves to row permutation[i], columns are mapped
//      through the permutation and sorted.
// Each frontier is one pass of GPU kernels (mark, compact, earliest-neighbour positions, a
// stable radix sort, insert); the host only reads the frontier size.  The reference runs
// step 1 with an atomic counter across threads, so its order of the degree <= 1 vertices is
// that of a one-thread run; with one thread its permutation and ours are the same.
#include <string.h>

#include <vector>

#include "internal.h"
#include "primitives.cuh"

namespace spmv {

int coo_to_csr_device(const int32_t * R, const int32_t * C, const double * V, int64_t m, int64_t n, int64_t nnz,
		int32_t * row_ptr, int32_t * col, double * val, cudaStream_t s);

namespace {

__global__ void row_of_entry_kernel(const int32_t * rp, int64_t m, int32_t * row)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= m)
		return;
	for (int64_t j = rp[i]; j < rp[i + 1]; j++)
		row[j] = (int32_t) i;
}

// kind 0: expand a lower triangle (entry + mirror); kind 1: keep col <= row.  Counts first
// (pass 0), then writes COO at the scanned positions (pass 1).
__global__ void sym_entries_kernel(const int32_t * row, const int32_t * ci, const double * v, int64_t nnz, int kind,
		int pass, int64_t * cnt, const int64_t * pos, int32_t * R, int32_t * C, double * V, int * err,
		unsigned long long * ndiag)
{
	const int64_t j = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= nnz)
		return;
	const int32_t r = row[j], c = ci[j];
	int k;
	if (kind == 0) {
		if (c > r) {
			atomicCAS(err, 0, 1);
			k = 0;
		} else {
			k = (c == r) ? 1 : 2;
		}
	} else {
		k = (c <= r) ? 1 : 0;
	}
	if (pass == 0) {
		cnt[j] = k;
		if (k > 0 && c == r)
			atomicAdd(ndiag, 1ULL);
		return;
	}
	const int64_t p = pos[j];
	if (k >= 1) {
		R[p] = r;
		C[p] = c;
		V[p] = v[j];
	}
	if (k == 2) {
		R[p + 1] = c;
		C[p + 1] = r;
		V[p + 1] = v[j];
	}
}

// ---- RCM
__global__ void rcm_init_kernel(const int32_t * rp, int64_t m, int32_t * pos, int32_t * lowdeg)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= m)
		return;
	pos[i] = (int32_t) m;
	lowdeg[i] = (rp[i + 1] - rp[i] <= 1) ? 1 : 0;
}

__global__ void rcm_place_lowdeg_kernel(const int32_t * lowdeg, const int64_t * ex, int64_t m, int32_t * R, int32_t * pos)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= m || !lowdeg[i])
		return;
	R[ex[i]] = (int32_t) i;
	pos[i] = (int32_t) ex[i];
}

// least (degree, index) among the unvisited vertices
__global__ void rcm_start_kernel(const int32_t * rp, const int32_t * pos, int64_t m, unsigned long long * best)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long key = ~0ULL;
	if (i < m && pos[i] >= m)
		key = ((unsigned long long) (uint32_t) (rp[i + 1] - rp[i]) << 32) | (unsigned long long) i;
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		const unsigned long long k2 = __shfl_xor_sync(0xffffffffu, key, o);
		key = k2 < key ? k2 : key;
	}
	if ((threadIdx.x & 31) == 0 && key != ~0ULL)
		atomicMin(best, key);
}

__global__ void rcm_append_kernel(unsigned long long * best, int32_t * R, int32_t * pos, int64_t at)
{
	const int32_t v = (int32_t) (*best & 0xffffffffULL);
	R[at] = v;
	pos[v] = (int32_t) at;
	*best = ~0ULL;
}

__global__ void rcm_mark_kernel(const int32_t * rp, const int32_t * ci, const int32_t * R, int64_t f0, int64_t f1,
		const int32_t * pos, int64_t m, int32_t * flag)
{
	const int64_t t = (int64_t) blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
	if (f0 + t >= f1)
		return;
	const int32_t v = R[f0 + t];
	for (int64_t j = rp[v] + (threadIdx.x & 31); j < rp[v + 1]; j += 32) {
		const int32_t c = ci[j];
		if (pos[c] >= m)
			flag[c] = 1;
	}
}

__global__ void rcm_compact_kernel(const int32_t * flag, const int64_t * ex, int64_t m, uint32_t * A)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < m && flag[i])
		A[ex[i]] = (uint32_t) i;
}

// key of frontier vertex A[k]: (earliest position of a visited neighbour, degree)
__global__ void rcm_key_kernel(const int32_t * rp, const int32_t * ci, const uint32_t * A, int64_t na, const int32_t * pos,
		int64_t m, uint64_t * key)
{
	const int64_t k = (int64_t) blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
	if (k >= na)
		return;
	const int32_t v = (int32_t) A[k];
	int32_t best = (int32_t) m;
	for (int64_t j = rp[v] + (threadIdx.x & 31); j < rp[v + 1]; j += 32) {
		const int32_t p = pos[ci[j]];
		best = p < best ? p : best;
	}
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		const int32_t b2 = __shfl_xor_sync(0xffffffffu, best, o);
		best = b2 < best ? b2 : best;
	}
	if ((threadIdx.x & 31) == 0)
		key[k] = ((uint64_t) (uint32_t) best << 31) | (uint64_t) (uint32_t) (rp[v + 1] - rp[v]);
}

__global__ void rcm_insert_kernel(const uint32_t * A, int64_t na, int64_t at, int32_t * R, int32_t * pos)
{
	const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= na)
		return;
	R[at + k] = (int32_t) A[k];
	pos[A[k]] = (int32_t) (at + k);
}

__global__ void rcm_perm_kernel(const int32_t * R, int64_t m, int32_t * perm)
{
	const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < m)
		perm[R[i]] = (int32_t) (m - 1 - i);
}

__global__ void permute_coo_kernel(const int32_t * row, const int32_t * ci, int64_t nnz, const int32_t * perm,
		int32_t * R, int32_t * C)
{
	const int64_t j = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= nnz)
		return;
	R[j] = perm[row[j]];
	C[j] = perm[ci[j]];
}

int bits64(int64_t v)
{
	int b = 0;
	while (v > 0) {
		b++;
		v >>= 1;
	}
	return b;
}

}  // namespace

// A device CSR (owning) produced by a transform.
struct DevCsr {
	int64_t m = 0, n = 0, nnz = 0, nnz_diag = 0;
	DevBuf rp, ci, v;
};

// kind 0: csr_expand_symmetric; kind 1: csr_drop_upper (both with sorted columns)
static int sym_transform(const int32_t * rp, const int32_t * ci, const double * v, int64_t m, int64_t n, int64_t nnz,
		int kind, DevCsr & out, cudaStream_t s)
{
	DevBuf row, cnt, ex, R, C, V, err, nd;
	SPMV_TRY(row.alloc((nnz > 0 ? nnz : 1) * 4, s));
	SPMV_TRY(cnt.alloc((nnz > 0 ? nnz : 1) * 8, s));
	SPMV_TRY(ex.alloc((nnz + 1) * 8, s));
	SPMV_TRY(err.alloc(4, s));
	SPMV_TRY(nd.alloc(8, s));
	SPMV_CUDA_TRY(cudaMemsetAsync(err.p, 0, 4, s));
	SPMV_CUDA_TRY(cudaMemsetAsync(nd.p, 0, 8, s));
	if (m > 0) {
		row_of_entry_kernel<<<(unsigned) ceil_div(m, 256), 256, 0, s>>>(rp, m, row.as<int32_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	const unsigned g = (unsigned) ceil_div(nnz > 0 ? nnz : 1, 256);
	if (nnz > 0) {
		sym_entries_kernel<<<g, 256, 0, s>>>(row.as<int32_t>(), ci, v, nnz, kind, 0, cnt.as<int64_t>(), nullptr, nullptr,
				nullptr, nullptr, err.as<int>(), nd.as<unsigned long long>());
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	SPMV_TRY(scan_exclusive(cnt.as<int64_t>(), ex.as<int64_t>(), nnz, s));
	int64_t total = 0;
	int bad = 0;
	unsigned long long ndiag = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&total, ex.as<int64_t>() + nnz, 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaMemcpyAsync(&bad, err.p, 4, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaMemcpyAsync(&ndiag, nd.p, 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	if (bad) {
		set_error(SPMV_ERR_CSR, "csr_expand_symmetric: an entry above the diagonal (expected a lower triangle)");
		return SPMV_ERR_CSR;
	}
	if (total > INT32_MAX - 1) {
		set_error(SPMV_ERR_OVERFLOW, "symmetric expansion: %lld entries beyond the 32-bit range", (long long) total);
		return SPMV_ERR_OVERFLOW;
	}
	SPMV_TRY(R.alloc((total > 0 ? total : 1) * 4, s));
	SPMV_TRY(C.alloc((total > 0 ? total : 1) * 4, s));
	SPMV_TRY(V.alloc((total > 0 ? total : 1) * 8, s));
	if (nnz > 0) {
		sym_entries_kernel<<<g, 256, 0, s>>>(row.as<int32_t>(), ci, v, nnz, kind, 1, nullptr, ex.as<int64_t>(),
				R.as<int32_t>(), C.as<int32_t>(), V.as<double>(), err.as<int>(), nd.as<unsigned long long>());
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	out.m = m;
	out.n = n;
	out.nnz = total;
	out.nnz_diag = (int64_t) ndiag;
	SPMV_TRY(out.rp.alloc((m + 1) * 4, s));
	SPMV_TRY(out.ci.alloc((total > 0 ? total : 1) * 4, s));
	SPMV_TRY(out.v.alloc((total > 0 ? total : 1) * 8, s));
	SPMV_TRY(coo_to_csr_device(R.as<int32_t>(), C.as<int32_t>(), V.as<double>(), m, n, total, out.rp.as<int32_t>(),
			out.ci.as<int32_t>(), out.v.as<double>(), s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	return SPMV_OK;
}

// reverse_cuthill_mckee on a full (expanded) square CSR: the permutation and the reordered CSR
static int rcm_full(const int32_t * rp, const int32_t * ci, const double * v, int64_t m, int64_t nnz, DevBuf & perm,
		DevCsr & out, cudaStream_t s)
{
	DevBuf R, pos, flag, ex, A, key, best;
	SPMV_TRY(R.alloc(m * 4, s));
	SPMV_TRY(pos.alloc(m * 4, s));
	SPMV_TRY(flag.alloc(m * 4, s));
	SPMV_TRY(ex.alloc((m + 1) * 8, s));
	SPMV_TRY(A.alloc(m * 4, s));
	SPMV_TRY(key.alloc(m * 8, s));
	SPMV_TRY(best.alloc(8, s));
	SPMV_CUDA_TRY(cudaMemsetAsync(best.p, 0xff, 8, s));
	const unsigned gm = (unsigned) ceil_div(m, 256);
	rcm_init_kernel<<<gm, 256, 0, s>>>(rp, m, pos.as<int32_t>(), flag.as<int32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(scan_exclusive(flag.as<int32_t>(), ex.as<int64_t>(), m, s));
	rcm_place_lowdeg_kernel<<<gm, 256, 0, s>>>(flag.as<int32_t>(), ex.as<int64_t>(), m, R.as<int32_t>(), pos.as<int32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	int64_t Rn = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&Rn, ex.as<int64_t>() + m, 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	int64_t Rprev = 0, nv = 0;
	const int kb = 31 + bits64(m);
	while (Rn < m) {
		if (nv == 0) {
			rcm_start_kernel<<<gm, 256, 0, s>>>(rp, pos.as<int32_t>(), m, best.as<unsigned long long>());
			SPMV_CUDA_TRY(cudaGetLastError());
			rcm_append_kernel<<<1, 1, 0, s>>>(best.as<unsigned long long>(), R.as<int32_t>(), pos.as<int32_t>(), Rn);
			SPMV_CUDA_TRY(cudaGetLastError());
			Rn++;
		}
		SPMV_CUDA_TRY(cudaMemsetAsync(flag.p, 0, m * 4, s));
		const int64_t nf = Rn - Rprev;
		rcm_mark_kernel<<<(unsigned) ceil_div(nf, 8), 256, 0, s>>>(rp, ci, R.as<int32_t>(), Rprev, Rn, pos.as<int32_t>(), m,
				flag.as<int32_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
		SPMV_TRY(scan_exclusive(flag.as<int32_t>(), ex.as<int64_t>(), m, s));
		SPMV_CUDA_TRY(cudaMemcpyAsync(&nv, ex.as<int64_t>() + m, 8, cudaMemcpyDeviceToHost, s));
		SPMV_CUDA_TRY(cudaStreamSynchronize(s));
		if (nv == 0) {
			Rprev = Rn;
			continue;
		}
		rcm_compact_kernel<<<gm, 256, 0, s>>>(flag.as<int32_t>(), ex.as<int64_t>(), m, A.as<uint32_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
		rcm_key_kernel<<<(unsigned) ceil_div(nv, 8), 256, 0, s>>>(rp, ci, A.as<uint32_t>(), nv, pos.as<int32_t>(), m,
				key.as<uint64_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
		SPMV_TRY(radix_sort_pairs(key.as<uint64_t>(), A.as<uint32_t>(), nv, kb, s));   // stable: ties keep index order
		rcm_insert_kernel<<<(unsigned) ceil_div(nv, 256), 256, 0, s>>>(A.as<uint32_t>(), nv, Rn, R.as<int32_t>(),
				pos.as<int32_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
		Rprev = Rn;
		Rn += nv;
	}
	SPMV_TRY(perm.alloc(m * 4, s));
	rcm_perm_kernel<<<gm, 256, 0, s>>>(R.as<int32_t>(), m, perm.as<int32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	DevBuf row, Rr, Cc;
	SPMV_TRY(row.alloc((nnz > 0 ? nnz : 1) * 4, s));
	SPMV_TRY(Rr.alloc((nnz > 0 ? nnz : 1) * 4, s));
	SPMV_TRY(Cc.alloc((nnz > 0 ? nnz : 1) * 4, s));
	row_of_entry_kernel<<<gm, 256, 0, s>>>(rp, m, row.as<int32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	if (nnz > 0) {
		permute_coo_kernel<<<(unsigned) ceil_div(nnz, 256), 256, 0, s>>>(row.as<int32_t>(), ci, nnz, perm.as<int32_t>(),
				Rr.as<int32_t>(), Cc.as<int32_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	out.m = out.n = m;
	out.nnz = nnz;
	SPMV_TRY(out.rp.alloc((m + 1) * 4, s));
	SPMV_TRY(out.ci.alloc((nnz > 0 ? nnz : 1) * 4, s));
	SPMV_TRY(out.v.alloc((nnz > 0 ? nnz : 1) * 8, s));
	SPMV_TRY(coo_to_csr_device(Rr.as<int32_t>(), Cc.as<int32_t>(), v, m, m, nnz, out.rp.as<int32_t>(), out.ci.as<int32_t>(),
			out.v.as<double>(), s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	return SPMV_OK;
}

}  // namespace spmv

// Host-side result of a transform (the CSR arrays, nnz_diag and, for RCM, the permutation).
struct spmv_csr_out {
	int64_t m = 0, n = 0, nnz = 0, nnz_diag = 0;
	std::vector<int32_t> rp, ci, perm;
	std::vector<double> v;
};

namespace {

using spmv::DevBuf;
using spmv::DevCsr;

int upload_csr(const int32_t * rp, const int32_t * ci, const double * v, int64_t m, int64_t nnz, DevBuf & drp,
		DevBuf & dci, DevBuf & dv, cudaStream_t s)
{
	SPMV_TRY(drp.alloc((m + 1) * 4, s));
	SPMV_TRY(dci.alloc((nnz > 0 ? nnz : 1) * 4, s));
	SPMV_TRY(dv.alloc((nnz > 0 ? nnz : 1) * 8, s));
	SPMV_CUDA_TRY(cudaMemcpyAsync(drp.p, rp, (m + 1) * 4, cudaMemcpyHostToDevice, s));
	if (nnz > 0) {
		SPMV_CUDA_TRY(cudaMemcpyAsync(dci.p, ci, nnz * 4, cudaMemcpyHostToDevice, s));
		SPMV_CUDA_TRY(cudaMemcpyAsync(dv.p, v, nnz * 8, cudaMemcpyHostToDevice, s));
	}
	return SPMV_OK;
}

int download(const DevCsr & c, spmv_csr_out * o, cudaStream_t s)
{
	o->m = c.m;
	o->n = c.n;
	o->nnz = c.nnz;
	o->nnz_diag = c.nnz_diag;
	o->rp.resize((size_t) c.m + 1);
	o->ci.resize((size_t) c.nnz);
	o->v.resize((size_t) c.nnz);
	SPMV_CUDA_TRY(cudaMemcpyAsync(o->rp.data(), c.rp.p, (c.m + 1) * 4, cudaMemcpyDeviceToHost, s));
	if (c.nnz > 0) {
		SPMV_CUDA_TRY(cudaMemcpyAsync(o->ci.data(), c.ci.p, c.nnz * 4, cudaMemcpyDeviceToHost, s));
		SPMV_CUDA_TRY(cudaMemcpyAsync(o->v.data(), c.v.p, c.nnz * 8, cudaMemcpyDeviceToHost, s));
	}
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	return SPMV_OK;
}

int check_sizes(const int32_t * rp, int64_t m, int64_t n, int64_t nnz, const int32_t * ci, const double * v)
{
	if (!rp || m < 0 || n < 0 || nnz < 0 || m > INT32_MAX - 1 || n > INT32_MAX || nnz > INT32_MAX / 2 ||
			(nnz > 0 && (!ci || !v))) {
		spmv::set_error(SPMV_ERR_ARG, "bad CSR arguments");
		return SPMV_ERR_ARG;
	}
	if (rp[m] != nnz) {
		spmv::set_error(SPMV_ERR_CSR, "row_ptr[m] = %d differs from nnz = %lld", rp[m], (long long) nnz);
		return SPMV_ERR_CSR;
	}
	return SPMV_OK;
}

// kind 0 expand, 1 drop upper, 2 rcm (symmetry_expanded tells whether rp/ci hold the full matrix)
spmv_csr_out * run_transform(int kind, const int32_t * rp, const int32_t * ci, const double * v, int64_t m, int64_t n,
		int64_t nnz, int32_t symmetry_expanded, int * status)
{
	spmv::clear_error();
	int st = check_sizes(rp, m, n, nnz, ci, v);
	if (st == SPMV_OK && kind == 2 && (m != n || m == 0)) {
		spmv::set_error(SPMV_ERR_ARG, "RCM needs a non-empty square matrix (m=%lld n=%lld)", (long long) m, (long long) n);
		st = SPMV_ERR_ARG;
	}
	spmv_csr_out * o = nullptr;
	if (st == SPMV_OK) {
		cudaStream_t s = nullptr;
		o = new spmv_csr_out();
		auto body = [&]() -> int {
			SPMV_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
			DevBuf drp, dci, dv;
			SPMV_TRY(upload_csr(rp, ci, v, m, nnz, drp, dci, dv, s));
			if (kind < 2) {
				DevCsr c;
				SPMV_TRY(spmv::sym_transform(drp.as<int32_t>(), dci.as<int32_t>(), dv.as<double>(), m, n, nnz, kind, c, s));
				return download(c, o, s);
			}
			// rcm(): a stored triangle is expanded first and dropped again afterwards
			DevCsr full, reord;
			const int32_t * frp = drp.as<int32_t>(), * fci = dci.as<int32_t>();
			const double * fv = dv.as<double>();
			int64_t fnnz = nnz;
			if (!symmetry_expanded) {
				SPMV_TRY(spmv::sym_transform(frp, fci, fv, m, n, nnz, 0, full, s));
				frp = full.rp.as<int32_t>();
				fci = full.ci.as<int32_t>();
				fv = full.v.as<double>();
				fnnz = full.nnz;
			}
			DevBuf perm;
			SPMV_TRY(spmv::rcm_full(frp, fci, fv, m, fnnz, perm, reord, s));
			o->perm.resize((size_t) m);
			SPMV_CUDA_TRY(cudaMemcpyAsync(o->perm.data(), perm.p, m * 4, cudaMemcpyDeviceToHost, s));
			if (!symmetry_expanded) {
				DevCsr low;
				SPMV_TRY(spmv::sym_transform(reord.rp.as<int32_t>(), reord.ci.as<int32_t>(), reord.v.as<double>(), m, n,
						reord.nnz, 1, low, s));
				return download(low, o, s);
			}
			return download(reord, o, s);
		};
		st = body();
		if (s) {
			cudaStreamSynchronize(s);
			cudaStreamDestroy(s);
		}
		if (st != SPMV_OK) {
			delete o;
			o = nullptr;
		}
	}
	if (status)
		*status = st;
	return o;
}

}  // namespace

extern "C" {

spmv_csr_out * spmv_expand_symmetric(const int32_t * row_ptr, const int32_t * col_ind, const double * values,
		int64_t m, int64_t n, int64_t nnz, int * status)
{
	return run_transform(0, row_ptr, col_ind, values, m, n, nnz, 0, status);
}

spmv_csr_out * spmv_drop_upper(const int32_t * row_ptr, const int32_t * col_ind, const double * values, int64_t m,
		int64_t n, int64_t nnz, int * status)
{
	return run_transform(1, row_ptr, col_ind, values, m, n, nnz, 0, status);
}

spmv_csr_out * spmv_rcm(const int32_t * row_ptr, const int32_t * col_ind, const double * values, int64_t m, int64_t n,
		int64_t nnz, int32_t symmetry_expanded, int * status)
{
	return run_transform(2, row_ptr, col_ind, values, m, n, nnz, symmetry_expanded, status);
}

int spmv_csr_out_info(const spmv_csr_out * o, int64_t * m, int64_t * n, int64_t * nnz, int64_t * nnz_diag)
{
	spmv::clear_error();
	if (!o) {
		spmv::set_error(SPMV_ERR_ARG, "null result");
		return SPMV_ERR_ARG;
	}
	if (m) *m = o->m;
	if (n) *n = o->n;
	if (nnz) *nnz = o->nnz;
	if (nnz_diag) *nnz_diag = o->nnz_diag;
	return SPMV_OK;
}

int spmv_csr_out_get(const spmv_csr_out * o, int32_t * row_ptr, int32_t * col_ind, double * values, int32_t * permutation)
{
	spmv::clear_error();
	if (!o) {
		spmv::set_error(SPMV_ERR_ARG, "null result");
		return SPMV_ERR_ARG;
	}
	if (row_ptr)
		memcpy(row_ptr, o->rp.data(), o->rp.size() * 4);
	if (col_ind && o->nnz)
		memcpy(col_ind, o->ci.data(), o->ci.size() * 4);
	if (values && o->nnz)
		memcpy(values, o->v.data(), o->v.size() * 8);
	if (permutation && !o->perm.empty())
		memcpy(permutation, o->perm.data(), o->perm.size() * 4);
	return SPMV_OK;
}

void spmv_csr_out_destroy(spmv_csr_out * o)
{
	delete o;
}

}  // extern "C"
