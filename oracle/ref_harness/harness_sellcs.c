/*
 * Test-infrastructure harness (oracle only).  Runs the reference's SELL-C-sigma
 * conversion (src/spmv_kernels/sell-C-s/sellcs_format.c:32-51, :137-224 and
 * radix_sort.c:36-122, built with INDEX64 as src/Makefile_in:62-65 does) and exports
 * its arrays.  The reference SpMV kernel for this format is RVV-only
 * (sellcs_mv_kernels_epi.c:176) and cannot be built on x86; its CPU restatement lives
 * in oracle/spmv_oracle.c.
 */
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#include "sellcs-spmv.h"

#define EXPORT __attribute__((visibility("default")))

EXPORT void * ref_sellcs_convert(const int32_t * row_ptr, const int32_t * col, const double * val,
		long m, long n, long nnz, long C, long sigma)
{
	sellcs_matrix_t * s = (sellcs_matrix_t *) calloc(1, sizeof(*s));
	index_t * rp = (index_t *) malloc((m + 1) * sizeof(index_t));
	index_t * ci = (index_t *) malloc((nnz > 0 ? nnz : 1) * sizeof(index_t));
	long i;
	for (i = 0; i < m + 1; i++)
		rp[i] = row_ptr[i];
	for (i = 0; i < nnz; i++)
		ci[i] = col[i];
	sellcs_init_params(C, sigma, s);
	sellcs_create_matrix_from_CSR_rd(m, n, rp, ci, val, 0, 0, s);
	free(rp);
	free(ci);
	return s;
}

EXPORT long ref_sellcs_nslices(void * p)
{
	return ((sellcs_matrix_t *) p)->nslices;
}

EXPORT long ref_sellcs_size(void * p)
{
	sellcs_matrix_t * s = (sellcs_matrix_t *) p;
	return s->slice_pointers[s->nslices];
}

/* Exports as int64: row_order[m], slice_widths[nslices], slice_pointers[nslices+1],
 * column_indices[size]; values[size] as f64. */
EXPORT void ref_sellcs_export(void * p, int64_t * row_order, int64_t * slice_widths, int64_t * slice_pointers,
		int64_t * column_indices, double * values)
{
	sellcs_matrix_t * s = (sellcs_matrix_t *) p;
	long i, size = s->slice_pointers[s->nslices];
	for (i = 0; i < s->nrows; i++)
		row_order[i] = s->row_order[i];
	for (i = 0; i < s->nslices; i++)
		slice_widths[i] = s->slice_widths[i];
	for (i = 0; i < s->nslices + 1; i++)
		slice_pointers[i] = s->slice_pointers[i];
	for (i = 0; i < size; i++) {
		column_indices[i] = s->column_indices[i];
		values[i] = s->values[i];
	}
}

EXPORT void ref_sellcs_free(void * p)
{
	sellcs_matrix_t * s = (sellcs_matrix_t *) p;
	free(s->row_order);
	free(s->slice_widths);
	free(s->slice_pointers);
	free(s->column_indices);
	free(s->values);
	free(s);
}
