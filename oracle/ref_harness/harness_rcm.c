/*
 * Test-infrastructure harness (oracle only).  The reference's symmetric transforms as
 * src/bench.cpp:280-358 (rcm()) calls them: csr_expand_symmetric / csr_drop_upper
 * (lib/storage_formats/csr/csr_gen.c:256-420, sorted columns) and
 * reverse_cuthill_mckee (lib/rcm/rcm_gen.c:96-410) with sorted columns.  kind 0: expand a
 * stored lower triangle; 1: drop the upper triangle; 2: rcm() on a matrix whose triangle is
 * stored (expanded = 0) or which is already full (expanded = 1).
 */
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <omp.h>

#include "aux/csr_converter_reference.h"
#include "aux/rcm.h"

#define EXPORT __attribute__((visibility("default")))

struct ref_csr {
	long m, nnz, nnz_diag;
	int32_t * ia, * ja, * perm;
	double * a;
};

EXPORT void * ref_sym_transform(int kind, int32_t * ia, int32_t * ja, double * a, long m, long n, long nnz, long expanded,
		int num_threads)
{
	omp_set_num_threads(num_threads);
	struct ref_csr * r = (struct ref_csr *) calloc(1, sizeof(*r));
	int32_t * rp = NULL, * ci = NULL, * perm = NULL;
	double * v = NULL;
	long nnz_new = nnz, nnz_diag = 0;
	r->m = m;
	if (kind == 0) {
		csr_expand_symmetric(ia, ja, a, m, n, nnz, &rp, &ci, &v, &nnz_new, &nnz_diag, 1);
	} else if (kind == 1) {
		csr_drop_upper(ia, ja, a, m, n, nnz, &rp, &ci, &v, &nnz_new, &nnz_diag, 1);
	} else {
		int32_t * frp = ia, * fci = ja;
		double * fv = a;
		long fnnz = nnz;
		if (!expanded)
			csr_expand_symmetric(ia, ja, a, m, n, nnz, &frp, &fci, &fv, &fnnz, &nnz_diag, 1);
		reverse_cuthill_mckee(frp, fci, fv, m, n, fnnz, 1, &rp, &ci, &v, &perm);
		nnz_new = fnnz;
		if (!expanded) {
			int32_t * rp2, * ci2;
			double * v2;
			csr_drop_upper(rp, ci, v, m, n, fnnz, &rp2, &ci2, &v2, &nnz_new, &nnz_diag, 1);
			free(rp);
			free(ci);
			free(v);
			free(frp);
			free(fci);
			free(fv);
			rp = rp2;
			ci = ci2;
			v = v2;
		}
	}
	r->ia = rp;
	r->ja = ci;
	r->a = v;
	r->perm = perm;
	r->nnz = nnz_new;
	r->nnz_diag = nnz_diag;
	return r;
}

EXPORT long ref_sym_nnz(void * p)
{
	return ((struct ref_csr *) p)->nnz;
}

EXPORT long ref_sym_nnz_diag(void * p)
{
	return ((struct ref_csr *) p)->nnz_diag;
}

EXPORT void ref_sym_arrays(void * p, int32_t * ia, int32_t * ja, double * a, int32_t * perm)
{
	struct ref_csr * r = (struct ref_csr *) p;
	memcpy(ia, r->ia, (r->m + 1) * sizeof(int32_t));
	memcpy(ja, r->ja, r->nnz * sizeof(int32_t));
	memcpy(a, r->a, r->nnz * sizeof(double));
	if (perm && r->perm)
		memcpy(perm, r->perm, r->m * sizeof(int32_t));
}

EXPORT void ref_sym_free(void * p)
{
	struct ref_csr * r = (struct ref_csr *) p;
	free(r->ia);
	free(r->ja);
	free(r->a);
	free(r->perm);
	free(r);
}
