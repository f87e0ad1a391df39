/*
 * Test-infrastructure harness (oracle only).  The reference's own Matrix-Market import,
 * step for step as src/bench.cpp:127-238 (import_file) runs it: mtx_read(filename,
 * expand_symmetry, pattern_dummy_vals = 1), mtx_values_convert_to_real, then coo_to_csr
 * with sorted columns (lib/storage_formats/csr/csr_gen.c:178-210) into CSR arrays, so
 * spmv_mtx_read can be compared with it array for array.  The reference exits on a
 * malformed file, so only well-formed files are given to it.
 */
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <omp.h>

#include "storage_formats/matrix_market/matrix_market.h"
#include "aux/csr_converter_reference.h"

#define EXPORT __attribute__((visibility("default")))

struct ref_mtx {
	long m, n, nnz, nnz_diag, nnz_non_diag, symmetric, expanded;
	int32_t * ia, * ja;
	double * a;
};

EXPORT void * ref_mtx_import(const char * path, long expand_symmetry, int num_threads)
{
	omp_set_num_threads(num_threads);
	struct ref_mtx * r = (struct ref_mtx *) calloc(1, sizeof(*r));
	struct Matrix_Market * MTX = mtx_read((char *) path, expand_symmetry, 1);
	int32_t * R = MTX->R, * C = MTX->C;
	r->m = MTX->m;
	r->n = MTX->n;
	r->nnz_diag = MTX->nnz_diag;
	r->nnz_non_diag = MTX->nnz_non_diag;
	r->symmetric = MTX->symmetric;
	r->expanded = expand_symmetry;
	r->nnz = MTX->nnz_stored;
	mtx_values_convert_to_real(MTX);
	double * V = (double *) MTX->V;
	MTX->R = NULL;
	MTX->C = NULL;
	MTX->V = NULL;
	mtx_destroy(&MTX);
	r->ia = (int32_t *) calloc(r->m + 1, sizeof(int32_t));
	r->ja = (int32_t *) calloc(r->nnz > 0 ? r->nnz : 1, sizeof(int32_t));
	r->a = (double *) calloc(r->nnz > 0 ? r->nnz : 1, sizeof(double));
	coo_to_csr(R, C, V, r->m, r->n, r->nnz, r->ia, r->ja, r->a, 1, 0);
	free(R);
	free(C);
	free(V);
	return r;
}

/* m, n, nnz, nnz_diag, nnz_non_diag, symmetric, expanded */
EXPORT void ref_mtx_info(void * p, long * out7)
{
	struct ref_mtx * r = (struct ref_mtx *) p;
	long v[7] = {r->m, r->n, r->nnz, r->nnz_diag, r->nnz_non_diag, r->symmetric, r->expanded};
	memcpy(out7, v, sizeof(v));
}

EXPORT void ref_mtx_arrays(void * p, int32_t * ia, int32_t * ja, double * a)
{
	struct ref_mtx * r = (struct ref_mtx *) p;
	memcpy(ia, r->ia, (r->m + 1) * sizeof(int32_t));
	memcpy(ja, r->ja, r->nnz * sizeof(int32_t));
	memcpy(a, r->a, r->nnz * sizeof(double));
}

EXPORT void ref_mtx_free(void * p)
{
	struct ref_mtx * r = (struct ref_mtx *) p;
	free(r->ia);
	free(r->ja);
	free(r->a);
	free(r);
}
