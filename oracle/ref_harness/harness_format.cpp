/*
 * Test-infrastructure harness (oracle only; never linked into the product).
 *
 * Compiles ONE of the reference's format translation units in place (selected by
 * -DREF_FMT_*) and exposes its csr_to_format / spmv pair and its converted arrays
 * through a small C ABI, so the parity tests can compare the GPU conversions
 * array-for-array with the reference's own csr_to_format output.
 *
 * The reference sources are included from the reference checkout by the recipe in
 * oracle/Makefile; nothing of them is copied here.  Interfaces followed:
 *   src/spmv_kernels/spmv_kernel.h:8-29   (Matrix_Format, csr_to_format)
 *   src/spmv_kernels/csr.cpp:42-139       (CSRArrays)
 *   src/spmv_kernels/csr_vec.cpp:75-172   (CSR, nnz-balanced ranges)
 *   src/spmv_kernels/sell.cpp:95-199      (SELLArray)
 *   src/spmv_kernels/sell_sorted.cpp:119-305 (SELLArray with permutations)
 *   src/spmv_kernels/DIV/div.cpp:236-604  (DIVArray, per-thread packet streams)
 */
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#if defined(REF_FMT_CSR_NAIVE)
#  include "spmv_kernels/csr.cpp"
#elif defined(REF_FMT_CSR_VEC)
#  include "spmv_kernels/csr_vec.cpp"
#elif defined(REF_FMT_SELL)
#  include "spmv_kernels/sell.cpp"
#elif defined(REF_FMT_SELL_SORTED)
#  include "spmv_kernels/sell_sorted.cpp"
#elif defined(REF_FMT_DIV_RF)
#  include "spmv_kernels/DIV/div.cpp"
#else
#  error "select a reference format with -DREF_FMT_*"
#endif

#define EXPORT extern "C" __attribute__((visibility("default")))

#if !defined(REF_FMT_DIV_RF)
/* Defined by src/bench_spmv.cpp:53 in the reference build. */
long num_loops_out = 1;
#else
long num_loops_out = 1;
#endif
int prefetch_distance = 0;

static void ref_default_env(void)
{
	/* Environment contract of config.sh:67-159; defaults as shipped. */
	setenv("USE_PROCESSES", "0", 0);
	setenv("DIV_VC_TOLERANCE", "0", 0);
	setenv("DIV_STEALING_ENABLED", "1", 0);
	setenv("DIV_PACKET_REORDERING", "0", 0);
	setenv("CSRCV_NUM_PACKET_VALS", "16384", 0);
	setenv("USE_ARTIFICIAL_MATRICES", "1", 0);
	setenv("GPU_KERNEL", "0", 0);
}

EXPORT void * ref_convert(int32_t * row_ptr, int32_t * col, double * val, long m, long n, long nnz, int num_threads)
{
	ref_default_env();
	omp_set_num_threads(num_threads);
	return (void *) csr_to_format(row_ptr, col, val, m, n, nnz, 0, 1);
}

EXPORT void ref_spmv(void * mf, double * x, double * y)
{
	((struct Matrix_Format *) mf)->spmv(x, y);
}

/* Destroys a converted matrix.  The reference's formats keep per-thread state in file-scope
 * globals (e.g. thread_i_s / thread_i_e, src/spmv_kernels/csr.cpp:21-22), so only one
 * converted matrix may be alive at a time: free it before converting the next. */
EXPORT void ref_free(void * mf)
{
	delete (struct Matrix_Format *) mf;
}

EXPORT double ref_mem_footprint(void * mf)
{
	return ((struct Matrix_Format *) mf)->mem_footprint;
}

EXPORT const char * ref_format_name(void * mf)
{
	return ((struct Matrix_Format *) mf)->format_name;
}

EXPORT int ref_vec_len(void)
{
#if defined(VEC_LEN)
	return VEC_LEN;
#else
	return 1;
#endif
}

#if defined(REF_FMT_SELL) || defined(REF_FMT_SELL_SORTED)
/* what: 0 row_cluster_ptr (int32, clusters+1), 1 ja (int32, nnz_ext), 2 a (f64, nnz_ext),
 *       3 permutation (int32, m), 4 rev_permutation (int32, m), 5 thread ranges (int64 pairs). */
EXPORT long ref_export(void * mf, int what, void * dst)
{
	SELLArray * s = (SELLArray *) mf;
	long cnt = 0;
	switch (what) {
	case 0: cnt = s->num_row_clusters + 1; if (dst) memcpy(dst, s->row_cluster_ptr, cnt * sizeof(INT_T)); break;
	case 1: cnt = s->nnz_ext; if (dst) memcpy(dst, s->ja, cnt * sizeof(INT_T)); break;
	case 2: cnt = s->nnz_ext; if (dst) memcpy(dst, s->a, cnt * sizeof(ValueType)); break;
#if defined(REF_FMT_SELL_SORTED)
	case 3: cnt = s->m; if (dst) memcpy(dst, s->permutation, cnt * sizeof(int)); break;
	case 4: cnt = s->m; if (dst) memcpy(dst, s->rev_permutation, cnt * sizeof(int)); break;
#endif
	case 5: {
		long t, T = omp_get_max_threads();
		cnt = 2 * T;
		if (dst)
			for (t = 0; t < T; t++) {
				((int64_t *) dst)[2*t] = tds[t]->ii_s;
				((int64_t *) dst)[2*t+1] = tds[t]->ii_e;
			}
		break;
	}
	default: cnt = -1;
	}
	return cnt;
}
#elif defined(REF_FMT_DIV_RF)
/* what: 10 number of threads; per thread t (what = 100 + t): compressed bytes;
 *       (what = 200 + t): packet group offsets (int64, groups+1);
 *       (what = 300 + t): row range [i_s, i_e) (int64 pair). */
EXPORT long ref_export(void * mf, int what, void * dst)
{
	(void) mf;
	long T = omp_get_max_threads();
	if (what == 10)
		return T;
	if (what >= 100 && what < 100 + T) {
		struct thread_data * td = tds[what - 100];
		if (dst)
			memcpy(dst, td->compr_data_stealable, td->compr_data_size_stealable);
		return td->compr_data_size_stealable;
	}
	if (what >= 200 && what < 200 + T) {
		struct thread_data * td = tds[what - 200];
		long cnt = td->num_packet_groups + 1;
		if (dst)
			memcpy(dst, td->packet_group_pos, cnt * sizeof(long));
		return cnt;
	}
	if (what >= 300 && what < 300 + T) {
		struct thread_data * td = tds[what - 300];
		if (dst) {
			((int64_t *) dst)[0] = td->i_s;
			((int64_t *) dst)[1] = td->i_e;
		}
		return 2;
	}
	return -1;
}
EXPORT long ref_div_header_size(void)
{
	return sizeof(struct packet_header);
}
#else
EXPORT long ref_export(void * mf, int what, void * dst)
{
	(void) mf; (void) what; (void) dst;
	return -1;
}
#endif
