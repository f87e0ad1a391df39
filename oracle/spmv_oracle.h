/*
 * CPU restatement of the reference's SpMV hot path (TEST INFRASTRUCTURE ONLY).
 *
 * This library is the oracle the GPU product is checked against.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  The product never
 * links, calls or falls back to it.
 *
 * Each function restates one reference routine in plain C (file:line cited at the
 * definition).  The restatement is pinned against the reference itself, compiled from
 * its own sources into oracle/_ref/ (see oracle/Makefile and tests/test_oracle_pin.py).
 */
#ifndef SPMV_ORACLE_H
#define SPMV_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- partitioners (lib/parallel_util.h, lib/macros/macrolib.h) ---- */
long orc_nearest_index(const int32_t * A, long lo, long hi, long target);
void orc_partition_prefix_sums(long T, long t, const int32_t * sums, long N, long total, long * s, long * e);
void orc_partition_iterations(long T, long t, long start, long end, long * s, long * e);

/* ---- CSR (src/spmv_kernels/csr.cpp, csr_vec.cpp) ---- */
void orc_csr_spmv(const int32_t * rp, const int32_t * ci, const double * v, long m, const double * x, double * y);
void orc_csr_vec_spmv(const int32_t * rp, const int32_t * ci, const double * v, long m, long L, const double * x, double * y);
/* Kahan-compensated long-double row sums: a high-accuracy gold used by the tolerance tests,
 * after src/bench_spmv.cpp:150-172 (which uses _Float128). Also returns sum_j |a_ij x_j|. */
void orc_csr_gold(const int32_t * rp, const int32_t * ci, const double * v, long m, const double * x, double * y, double * absy);

/* FP32 storage variant: compensated (Dot2) FP32 row sums. */
void orc_csr_f32_dot2(const int32_t * rp, const int32_t * ci, const float * v, long m, const float * x, float * y);

/* ---- SELL (src/spmv_kernels/sell.cpp) ---- */
long orc_sell_size(const int32_t * rp, long m, long V);
void orc_sell_convert(const int32_t * rp, const int32_t * ci, const double * v, long m, long V, long T,
		int32_t * rcp, int32_t * ja, double * a, int64_t * ranges);
void orc_sell_spmv(const int32_t * rcp, const int32_t * ja, const double * a, long m, long V, const double * x, double * y);

/* ---- sell_sorted (src/spmv_kernels/sell_sorted.cpp) ---- */
long orc_sell_sorted_size(const int32_t * rp, long m, long V, long T);
void orc_sell_sorted_convert(const int32_t * rp, const int32_t * ci, const double * v, long m, long V, long T,
		int32_t * rcp, int32_t * ja, double * a, int32_t * perm, int32_t * rev_perm, int64_t * ranges);
void orc_sell_sorted_spmv(const int32_t * rcp, const int32_t * ja, const double * a, const int32_t * rev_perm,
		long m, long V, const double * x, double * y);

/* ---- SELL-C-sigma (src/spmv_kernels/sell-C-s/) ---- */
long orc_sellcs_size(const int32_t * rp, long m, long C, long sigma);
int orc_sellcs_convert(const int32_t * rp, const int32_t * ci, const double * v, long m, long C, long sigma,
		int32_t * row_order, int32_t * widths, int64_t * ptrs, int32_t * cols, double * vals);
void orc_sellcs_spmv(const int32_t * row_order, const int32_t * widths, const int64_t * ptrs, const int32_t * cols,
		const double * vals, long m, long C, const double * x, double * y);

/* ---- DIV-RF (src/spmv_kernels/DIV/div.cpp, div_kernels_rf.h) ---- */
/* Builds the compressed packet streams of all T thread ranges (div.cpp:236-453).
 * Returns an opaque handle (NULL on error); query it with orc_div_get. */
void * orc_div_build(const int32_t * rp, const int32_t * ci, const double * v, long m, long n, long T, long L,
		long packet_vals, double tolerance);
/* what: 0 total bytes (dst: uint8 stream, threads concatenated in thread order),
 *       1 number of packets (dst: int64 packet byte offsets, num_packets+1 entries),
 *       2 per-thread byte counts (dst: int64[T]),
 *       3 per-thread packet-group counts (dst: int64[T]),
 *       4 packet-group offsets, each thread's groups+1 entries concatenated (dst: int64),
 *       5 row ranges (dst: int64[2T]).  Returns the element count of dst. */
long orc_div_get(void * h, int what, void * dst);
void orc_div_free(void * h);
long orc_div_header_size(long L);
/* Decodes every packet in order and accumulates y, the rows of every range zeroed first,
 * following compute_div (div.cpp:1201-1316) and the decoder (div_kernels_rf.h:948-1162).
 * fused != 0 uses fma() for the multiply-add. */
int orc_div_spmv(const uint8_t * data, long total_bytes, const int64_t * ranges, long T, long L,
		const double * x, double * y, int fused);
/* Decodes every packet back to COO in packet order; returns the nnz decoded or -1. */
long orc_div_decode_coo(const uint8_t * data, long total_bytes, long L, int32_t * rows, int32_t * cols, double * vals);

#ifdef __cplusplus
}
#endif

#endif
