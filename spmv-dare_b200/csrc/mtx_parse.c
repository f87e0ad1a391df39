/*
 * Matrix-Market reader (host side of spmv_mtx_read): the text is parsed here, the COO ->
 * CSR conversion runs on the GPU (mtx.cu).
 *
 * Follows the reference's import path (src/bench.cpp:127-238):
 *   mtx_read(filename, expand_symmetry, pattern_dummy_vals = 1)
 *       (lib/storage_formats/matrix_market/matrix_market.c:152-331, matrix_market_gen.c)
 *   mtx_values_convert_to_real (matrix_market.c:421-463).
 * Rules restated:
 *   - lines are split at '\n' and empty lines dropped; a file that does not start with
 *     "%%MatrixMarket" is read as "coordinate real general" from its first line on;
 *   - the banner is "%%MatrixMarket matrix coordinate <field> <symmetry>", field real,
 *     integer, complex or pattern, symmetry general, symmetric, skew-symmetric or Hermitian;
 *     the dense "array" format is refused (the reference's import has no COO for it);
 *   - comment lines (leading '%') follow the banner; then "M N NNZ"; then exactly NNZ entry
 *     lines "row col [value [imag]]", 1-based;
 *   - numbers are parsed with strtol / strtod, as the reference's gen_strtonum does, and a
 *     number that sets errno (out of range, a subnormal value) is an error there and here;
 *   - with symmetry and expand_symmetry, the mirror (col, row) of every off-diagonal entry
 *     is appended after all stored entries, in their order, its value negated for
 *     skew-symmetric files (matrix_market_gen.c:62-127), in the type the field is read
 *     into: a real 0 becomes -0.0, an integer 0 stays 0 (integers are read as int,
 *     matrix_market.c:23-27, 288-293);
 *   - values become real: integer -> double, complex -> cabs(value) (the conjugate of a
 *     Hermitian mirror has the same modulus), pattern -> 1.0.
 */
#include <complex.h>
#include <errno.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mtx_parse.h"

static int fail(struct mtx_coo * out, const char * fmt, const char * a, long b)
{
	snprintf(out->err, sizeof(out->err), fmt, a, b);
	return -1;
}

/* next whitespace-separated token of [*p, end) into buf (at most n - 1 characters) */
static int next_token(const char ** p, const char * end, char * buf, int n)
{
	const char * s = *p;
	while (s < end && (*s == ' ' || *s == '\t' || *s == '\r'))
		s++;
	int k = 0;
	while (s < end && *s != ' ' && *s != '\t' && *s != '\r' && k < n - 1)
		buf[k++] = *s++;
	buf[k] = 0;
	*p = s;
	return k;
}

/* strtol / strtod over [p, end) without running past the line: the number is copied out */
static int parse_long(const char ** p, const char * end, long * v)
{
	char buf[64];
	if (next_token(p, end, buf, sizeof(buf)) == 0)
		return 0;
	char * e;
	errno = 0;
	*v = strtol(buf, &e, 10);
	return *e == 0 && errno == 0;
}

static int parse_double(const char ** p, const char * end, double * v)
{
	char buf[128];
	if (next_token(p, end, buf, sizeof(buf)) == 0)
		return 0;
	char * e;
	errno = 0;
	*v = strtod(buf, &e);
	return *e == 0 && errno == 0;      /* the reference stops on any strtod error, ERANGE included */
}

int mtx_parse_file(const char * path, int expand_symmetry, struct mtx_coo * out)
{
	memset(out, 0, sizeof(*out));
	FILE * f = fopen(path, "rb");
	if (!f)
		return fail(out, "cannot open %s (%ld)", path, (long) errno);
	fseek(f, 0, SEEK_END);
	long size = ftell(f);
	fseek(f, 0, SEEK_SET);
	char * text = (char *) malloc((size_t) size + 1);
	if (!text || fread(text, 1, (size_t) size, f) != (size_t) size) {
		fclose(f);
		free(text);
		return fail(out, "cannot read %s (%ld bytes)", path, size);
	}
	fclose(f);
	text[size] = 0;

	/* non-empty lines */
	long nlines = 0, cap = 1024;
	long * ls = (long *) malloc(cap * sizeof(long)), * le = (long *) malloc(cap * sizeof(long));
	for (long i = 0; i < size;) {
		long j = i;
		while (j < size && text[j] != '\n')
			j++;
		if (j > i) {
			if (nlines == cap) {
				cap *= 2;
				ls = (long *) realloc(ls, cap * sizeof(long));
				le = (long *) realloc(le, cap * sizeof(long));
			}
			ls[nlines] = i;
			le[nlines] = j;
			nlines++;
		}
		i = j + 1;
	}
	int rc = -1;
	long li = 0;
	char tok[5][64];
	int field = 0;            /* 0 real, 1 integer, 2 complex, 3 pattern */
	int symmetric = 0, skew = 0;
	if (nlines == 0) {
		fail(out, "%s: empty file%ld", path, 0);
		goto done;
	}
	{
		const char * p = text + ls[0], * e = text + le[0];
		next_token(&p, e, tok[0], 64);
		if (strcmp(tok[0], "%%MatrixMarket") == 0) {
			for (int t = 1; t < 5; t++)
				next_token(&p, e, tok[t], 64);
			if (strcmp(tok[1], "matrix") || strcmp(tok[2], "coordinate")) {
				fail(out, "%s: only 'matrix coordinate' files are imported%ld", path, 0);
				goto done;
			}
			if (!strcmp(tok[3], "real"))
				field = 0;
			else if (!strcmp(tok[3], "integer"))
				field = 1;
			else if (!strcmp(tok[3], "complex"))
				field = 2;
			else if (!strcmp(tok[3], "pattern"))
				field = 3;
			else {
				fail(out, "unrecognized field type: %s%ld", tok[3], 0);
				goto done;
			}
			if (!strcmp(tok[4], "symmetric"))
				symmetric = 1;
			else if (!strcmp(tok[4], "skew-symmetric"))
				symmetric = skew = 1;
			else if (!strcmp(tok[4], "Hermitian"))
				symmetric = 1;
			else if (strcmp(tok[4], "general")) {
				fail(out, "unsupported symmetry type: %s%ld", tok[4], 0);
				goto done;
			}
			li = 1;
		}
	}
	while (li < nlines && text[ls[li]] == '%')
		li++;
	if (li >= nlines) {
		fail(out, "%s: missing matrix sizes%ld", path, 0);
		goto done;
	}
	long M, N, NNZ;
	{
		const char * p = text + ls[li], * e = text + le[li];
		if (!parse_long(&p, e, &M) || !parse_long(&p, e, &N) || !parse_long(&p, e, &NNZ) || M < 0 || N < 0 ||
				NNZ < 0) {
			fail(out, "%s: invalid/missing matrix sizes (line %ld)", path, li + 1);
			goto done;
		}
		li++;
	}
	if (NNZ != nlines - li) {
		fail(out, "%s: the remaining lines don't match the number of non-zeros (%ld)", path, NNZ);
		goto done;
	}
	if (M > INT32_MAX || N > INT32_MAX) {
		fail(out, "%s: dimensions beyond the 32-bit index range%ld", path, 0);
		goto done;
	}
	long cap_e = symmetric && expand_symmetry ? 2 * NNZ : NNZ;
	out->R = (int32_t *) malloc((size_t) (cap_e > 0 ? cap_e : 1) * sizeof(int32_t));
	out->C = (int32_t *) malloc((size_t) (cap_e > 0 ? cap_e : 1) * sizeof(int32_t));
	out->V = (double *) malloc((size_t) (cap_e > 0 ? cap_e : 1) * sizeof(double));
	long bad = -1, diag = 0;
	#pragma omp parallel for reduction(+ : diag) schedule(static)
	for (long k = 0; k < NNZ; k++) {
		const char * p = text + ls[li + k], * e = text + le[li + k];
		long r, c;
		double v = 1.0;
		int ok = parse_long(&p, e, &r) && parse_long(&p, e, &c);
		if (ok && field == 0)
			ok = parse_double(&p, e, &v);
		else if (ok && field == 1) {
			long iv;
			ok = parse_long(&p, e, &iv);
			v = (double) (int) iv;
		} else if (ok && field == 2) {
			double re, im;
			ok = parse_double(&p, e, &re) && parse_double(&p, e, &im);
			v = cabs(re + im * I);
		}
		if (!ok || r < 1 || r > M || c < 1 || c > N) {
			#pragma omp critical
			{
				if (bad < 0 || k < bad)
					bad = k;
			}
			continue;
		}
		out->R[k] = (int32_t) (r - 1);
		out->C[k] = (int32_t) (c - 1);
		out->V[k] = v;
		diag += (r == c);
	}
	if (bad >= 0) {
		fail(out, "%s: badly formed or out-of-range entry on entry line %ld", path, bad + 1);
		goto done;
	}
	out->m = M;
	out->n = N;
	out->nnz_diag = diag;
	out->nnz_non_diag = NNZ - diag;
	out->symmetric = symmetric;
	out->skew = skew;
	out->nnz = NNZ;
	out->expanded = expand_symmetry ? 1 : 0;     /* the flag the bench passes on (bench.cpp:206) */
	if (symmetric && expand_symmetry) {
		long j = NNZ;
		for (long k = 0; k < NNZ; k++) {
			if (out->R[k] != out->C[k]) {
				out->R[j] = out->C[k];
				out->C[j] = out->R[k];
				/* a complex value is already its modulus: |-conj(z)| = |z|; an integer value
				 * is negated as the int it was read into (0 stays +0.0, INT_MIN wraps) */
				if (!skew || field == 2)
					out->V[j] = out->V[k];
				else if (field == 1)
					out->V[j] = (double) (int32_t) (0u - (uint32_t) (int32_t) out->V[k]);
				else
					out->V[j] = -out->V[k];
				j++;
			}
		}
		out->nnz = j;
	}
	rc = 0;
done:
	free(ls);
	free(le);
	free(text);
	if (rc != 0)
		mtx_coo_free(out);
	return rc;
}

void mtx_coo_free(struct mtx_coo * c)
{
	free(c->R);
	free(c->C);
	free(c->V);
	c->R = c->C = NULL;
	c->V = NULL;
}
