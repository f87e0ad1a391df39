/*
 * Test-infrastructure harness (oracle only).  Exposes the reference's own artificial
 * matrix generator (artificial-matrix-generator/artificial_matrix_generation.c:163-579)
 * through a C ABI, so the product's generator can be pinned against it and the parity
 * tests can feed both sides identical CSR arrays.
 */
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <omp.h>

#include "artificial_matrix_generation.h"

#define EXPORT __attribute__((visibility("default")))

EXPORT void * ref_gen(long rows, long cols, double avg, double std, const char * distribution, unsigned int seed,
		const char * placement, double bw, double skew, double neigh, double cross, int num_threads)
{
	omp_set_num_threads(num_threads);
	return artificial_matrix_generation(rows, cols, avg, std, (char *) distribution, seed, (char *) placement,
			bw, skew, neigh, cross);
}

EXPORT long ref_gen_nnz(void * p)
{
	return ((struct csr_matrix *) p)->nr_nzeros;
}

EXPORT void ref_gen_arrays(void * p, int32_t * row_ptr, int32_t * col, double * val)
{
	struct csr_matrix * c = (struct csr_matrix *) p;
	long m = c->nr_rows, nnz = c->nr_nzeros;
	memcpy(row_ptr, c->row_ptr, (m + 1) * sizeof(int32_t));
	memcpy(col, c->col_ind, nnz * sizeof(int32_t));
	memcpy(val, c->values, nnz * sizeof(double));
}

/* Structural statistics in a fixed order (artificial_matrix_generation.c:529-570). */
EXPORT void ref_gen_stats(void * p, double * out)
{
	struct csr_matrix * c = (struct csr_matrix *) p;
	double v[] = {
		c->avg_nnz_per_row, c->std_nnz_per_row, c->min_nnz_per_row, c->max_nnz_per_row, c->skew,
		c->avg_bw, c->std_bw, c->min_bw, c->max_bw,
		c->avg_sc, c->std_sc, c->min_sc, c->max_sc,
		c->avg_num_neighbours, c->std_num_neighbours, c->min_num_neighbours, c->max_num_neighbours,
		c->cross_row_similarity, c->std_cross_row_similarity, c->min_cross_row_similarity, c->max_cross_row_similarity,
		c->avg_clustering, c->std_clustering, c->min_clustering, c->max_clustering,
		c->avg_ngroups, c->std_ngroups, c->min_ngroups, c->max_ngroups,
		c->avg_dis, c->std_dis, c->min_dis, c->max_dis,
		c->avg_ngroups_size, c->std_ngroups_size, c->min_ngroups_size, c->max_ngroups_size,
	};
	memcpy(out, v, sizeof(v));
}

EXPORT int ref_gen_num_stats(void)
{
	return 37;
}

EXPORT void ref_gen_free(void * p)
{
	free_csr_matrix((struct csr_matrix *) p);
}

/* The reference's cross-row similarity over non-empty rows (matrix_util.h:269-328, window
 * 1), called directly: the generator's own value (csr_cross_row_similarity2) averages over
 * a partly uninitialised buffer, so the selector's feature is pinned on this one. */
#include "matrix_util.h"

EXPORT double ref_cross_row_similarity(int32_t * row_ptr, int32_t * col, long m, long n, long nnz, int num_threads)
{
	omp_set_num_threads(num_threads);
	return csr_cross_row_similarity((int *) row_ptr, (int *) col, m, n, nnz, 1);
}
