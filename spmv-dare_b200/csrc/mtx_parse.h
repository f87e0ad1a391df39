/* Host Matrix-Market parser of spmv_mtx_read (mtx_parse.c). */
#ifndef SPMV_MTX_PARSE_H
#define SPMV_MTX_PARSE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

struct mtx_coo {
	long m, n;
	long nnz;                 /* entries in R, C, V (after the symmetric expansion, if any) */
	long nnz_diag, nnz_non_diag;   /* of the stored entries */
	int symmetric, skew;
	int expanded;             /* expand_symmetry as requested (the reference's csr->expanded_symmetry) */
	int32_t * R, * C;         /* 0-based coordinates */
	double * V;               /* real values */
	char err[256];
};

/* 0 on success; -1 with out->err set. */
int mtx_parse_file(const char * path, int expand_symmetry, struct mtx_coo * out);
void mtx_coo_free(struct mtx_coo * c);

#ifdef __cplusplus
}
#endif

#endif
