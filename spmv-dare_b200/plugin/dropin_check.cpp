/*
 * y check of the drop-in: drives one format through the reference's plugin interface
 * (src/spmv_kernels/spmv_kernel.h:17,28) exactly as the reference's bench does, and writes
 * the y it gets for a comparison with the reference format's own y.
 *
 *   dropin_check_<fmt>_d.exe <matrix.bin> <x.bin> <y_out.bin>
 *
 * matrix.bin: int64 m, n, nnz; int32 row_ptr[m+1]; int32 col_ind[nnz]; f64 values[nnz].
 * x.bin: f64 x[n].  y_out.bin: f64 y[m+64] of the second call.
 *
 * Buffer handling follows the bench (src/bench.cpp:622-651, src/bench_spmv.cpp:546-564):
 *   - csr_to_format() gets the CSR arrays, which are then overwritten and freed, so a
 *     format that kept a pointer to them reads garbage;
 *   - x and y are pageable aligned_alloc(64) buffers, y has m + 64 elements and its first
 *     m are 1.0 before every call (the probe for rows without entries);
 *   - the 64 elements past m are filled with a NaN pattern that no SpMV produces, so
 *     the output shows whether the format wrote past row m - 1.
 * Two calls are made (the bench's warm-up and timed calls reuse the format object); the
 * second call's y is written.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "macros/cpp_defines.h"

#include "spmv_kernel.h"

#ifdef __cplusplus
extern "C" {
#endif
	#include "macros/macrolib.h"
#ifdef __cplusplus
}
#endif

static void * read_exact(FILE * f, size_t bytes)
{
	void * p = aligned_alloc(64, bytes ? (bytes + 63) / 64 * 64 : 64);
	if (p == NULL || fread(p, 1, bytes, f) != bytes) {
		fprintf(stderr, "dropin_check: short read of %zu bytes\n", bytes);
		exit(2);
	}
	return p;
}

int main(int argc, char ** argv)
{
	if (argc != 4) {
		fprintf(stderr, "usage: %s matrix.bin x.bin y_out.bin\n", argv[0]);
		return 2;
	}
	FILE * f = fopen(argv[1], "rb");
	if (f == NULL) {
		perror(argv[1]);
		return 2;
	}
	int64_t hdr[3];
	if (fread(hdr, sizeof(hdr), 1, f) != 1) {
		fprintf(stderr, "dropin_check: bad header\n");
		return 2;
	}
	const long m = (long) hdr[0], n = (long) hdr[1], nnz = (long) hdr[2];
	INT_T * ia = (INT_T *) read_exact(f, (size_t) (m + 1) * sizeof(INT_T));
	INT_T * ja = (INT_T *) read_exact(f, (size_t) nnz * sizeof(INT_T));
	ValueTypeReference * a = (ValueTypeReference *) read_exact(f, (size_t) nnz * sizeof(ValueTypeReference));
	fclose(f);

	struct Matrix_Format * MF = csr_to_format(ia, ja, a, m, n, nnz, 0, 0);
	// The bench reallocates its CSR right after the conversion (bench.cpp:627-651).
	memset(ia, 0xff, (size_t) (m + 1) * sizeof(INT_T));
	memset(ja, 0xff, (size_t) nnz * sizeof(INT_T));
	memset(a, 0xff, (size_t) nnz * sizeof(ValueTypeReference));
	free(ia);
	free(ja);
	free(a);

	f = fopen(argv[2], "rb");
	if (f == NULL) {
		perror(argv[2]);
		return 2;
	}
	ValueType * x = (ValueType *) read_exact(f, (size_t) n * sizeof(ValueType));
	fclose(f);
	ValueType * y = (ValueType *) aligned_alloc(64, (size_t) (m + 64) * sizeof(ValueType));
	const uint64_t sentinel = 0x7ff8dead0000beefULL;
	for (int call = 0; call < 2; call++) {
		for (long i = 0; i < m; i++)
			y[i] = 1.0;
		for (long i = m; i < m + 64; i++)
			memcpy(&y[i], &sentinel, sizeof(sentinel));
		MF->spmv(x, y);
	}
	char buf[1000];
	statistics_print_labels(buf, sizeof(buf));
	printf("labels: %s\n", buf);
	MF->statistics_print_data(buf, sizeof(buf));
	printf("data: %s\n", buf);
	printf("format_name: %s mem_footprint: %.17g\n", MF->format_name, MF->mem_footprint);

	f = fopen(argv[3], "wb");
	if (f == NULL || fwrite(y, sizeof(ValueType), (size_t) (m + 64), f) != (size_t) (m + 64)) {
		fprintf(stderr, "dropin_check: cannot write %s\n", argv[3]);
		return 2;
	}
	fclose(f);
	// Matrix_Format has no virtual destructor and the bench never deletes its format object.
	free(x);
	free(y);
	return 0;
}
