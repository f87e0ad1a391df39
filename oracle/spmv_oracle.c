/*
 * CPU restatement of the reference's SpMV hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * The GPU product is checked against this file; the product never links, calls or
 * falls back to it.  Each routine restates the reference routine cited beside it, in
 * plain C, with the reference's integer/byte layouts and its floating-point operation
 * order (multiply-add fused where the reference's x86 build fuses it, split where it
 * does not).  Build: `make -C oracle` (compiled with -ffp-contract=off so every fused
 * multiply-add here is an explicit fma()).
 */
#define _GNU_SOURCE
#include <stdlib.h>
#include <stdio.h>
#include <string.h>
#include <math.h>
#include <omp.h>

#include "spmv_oracle.h"

#define MAXV(a, b) ((a) > (b) ? (a) : (b))
#define MINV(a, b) ((a) < (b) ? (a) : (b))

/* ======================================================================================
 * Partitioners
 * ====================================================================================== */

/* Nearest-index binary search over an ascending array, inclusive bounds [lo, hi]
 * (lib/macros/macrolib.h:537-588 with the default compare/distance at :506-514):
 * an exact match returns its index; otherwise the closer neighbour, ties to the upper. */
long orc_nearest_index(const int32_t * A, long lo, long hi, long target)
{
	long s = lo, e = hi, mid;
	if (target < (long) A[s])
		return s;
	if (target > (long) A[e])
		return e;
	for (;;) {
		mid = (s + e) / 2;
		if (mid == s || mid == e)
			break;
		if (target > (long) A[mid])
			s = mid;
		else
			e = mid;
	}
	if (target == (long) A[s])
		return s;
	if (target == (long) A[e])
		return e;
	return (labs(target - (long) A[s]) < labs(target - (long) A[e])) ? s : e;
}

/* loop_partitioner_balance_prefix_sums (lib/parallel_util.h:156-181), ascending order. */
void orc_partition_prefix_sums(long T, long t, const int32_t * sums, long N, long total, long * s, long * e)
{
	long target = (long) sums[0] + (total * t) / T;
	long target_next = (long) sums[0] + (total * (t + 1)) / T;
	*s = (t == 0) ? 0 : orc_nearest_index(sums, 0, N - 1, target);
	*e = (t == T - 1) ? N : orc_nearest_index(sums, 0, N - 1, target_next);
}

/* loop_partitioner_balance_iterations_base with increment 1 (lib/parallel_util.h:50-85). */
void orc_partition_iterations(long T, long t, long start, long end, long * s, long * e)
{
	long len = end - start;
	if (1 > len) {
		*s = (t == 0) ? start : end;
		*e = end;
		return;
	}
	long per = len / T, rem = len % T;
	if (rem != 0 && t < rem) {
		per += 1;
		rem = 0;
	}
	*s = start + per * t + rem;
	*e = (t == T - 1) ? end : *s + per;
}

/* ======================================================================================
 * CSR
 * ====================================================================================== */

/* subkernel_csr_scalar (src/spmv_kernels/csr.cpp:167-182): the reference's x86 build
 * evaluates `sum += a[j] * x[ja[j]]` as a rounded product followed by a rounded add. */
void orc_csr_spmv(const int32_t * rp, const int32_t * ci, const double * v, long m, const double * x, double * y)
{
	#pragma omp parallel for schedule(static)
	for (long i = 0; i < m; i++) {
		double sum = 0;
		for (long j = rp[i]; j < rp[i + 1]; j++) {
			double p = v[j] * x[ci[j]];
			sum = sum + p;
		}
		y[i] = sum;
	}
}

/* subkernel_row_csr_vec (src/spmv_kernels/csr_vec.cpp:183-211): L lanes of fused
 * multiply-adds over the first (len & ~(L-1)) entries, the AVX2 horizontal reduction
 * (lib/vectorization/x86/avx256/vectorization_x86_avx256_f64.h:169-177: (s0+s2)+(s1+s3)
 * for L = 4; L = 8 reduces each 4-wide half and adds them, :167), then an unfused tail. */
static double csr_vec_reduce(const double * s, long L)
{
	if (L == 1)
		return s[0];
	if (L == 2)
		return s[0] + s[1];
	if (L == 4)
		return (s[0] + s[2]) + (s[1] + s[3]);
	double tot = 0;
	for (long h = 0; h < L; h += 4)
		tot += (s[h] + s[h + 2]) + (s[h + 1] + s[h + 3]);
	return tot;
}

void orc_csr_vec_spmv(const int32_t * rp, const int32_t * ci, const double * v, long m, long L, const double * x, double * y)
{
	#pragma omp parallel for schedule(static)
	for (long i = 0; i < m; i++) {
		long js = rp[i], je = rp[i + 1];
		if (js == je) {
			y[i] = 0;
			continue;
		}
		double lanes[64];
		long jv = js + ((je - js) & ~(L - 1));
		for (long l = 0; l < L; l++)
			lanes[l] = 0;
		for (long j = js; j < jv; j += L)
			for (long l = 0; l < L; l++)
				lanes[l] = fma(v[j + l], x[ci[j + l]], lanes[l]);
		double sum = csr_vec_reduce(lanes, L);
		for (long j = jv; j < je; j++) {
			double p = v[j] * x[ci[j]];
			sum = sum + p;
		}
		y[i] = sum;
	}
}

/* High-accuracy row sums in binary128 (after check_accuracy's _Float128 gold,
 * src/bench_spmv.cpp:150-172), and sum_j |a_ij x_j| for condition-aware tolerances. */
void orc_csr_gold(const int32_t * rp, const int32_t * ci, const double * v, long m, const double * x, double * y, double * absy)
{
	#pragma omp parallel for schedule(static)
	for (long i = 0; i < m; i++) {
		__float128 sum = 0, asum = 0;
		for (long j = rp[i]; j < rp[i + 1]; j++) {
			__float128 p = (__float128) v[j] * (__float128) x[ci[j]];
			sum += p;
			asum += (p < 0) ? -p : p;
		}
		y[i] = (double) sum;
		if (absy)
			absy[i] = (double) asum;
	}
}

/* FP32 variant: values and x rounded to FP32, each row summed with the compensated dot
 * product Dot2 (Ogita, Rump, Oishi, SIAM J. Sci. Comput. 26(6), 2005): TwoProduct by
 * fmaf, Knuth's TwoSum, errors accumulated in a second FP32 sum; y = s + c.  The GPU's
 * FP32 kernel sums rows in the same sequential order. */
void orc_csr_f32_dot2(const int32_t * rp, const int32_t * ci, const float * v, long m, const float * x, float * y)
{
	#pragma omp parallel for schedule(static)
	for (long i = 0; i < m; i++) {
		float s = 0.0f, c = 0.0f;
		for (long j = rp[i]; j < rp[i + 1]; j++) {
			float a = v[j], b = x[ci[j]];
			float p = a * b;
			float pe = fmaf(a, b, -p);
			float t = s + p;
			float z = t - s;
			float e = (s - (t - z)) + (p - z);
			s = t;
			c = c + (e + pe);
		}
		y[i] = s + c;
	}
}

/* ======================================================================================
 * SELL (slice height V, column-major slices)
 * ====================================================================================== */

static long exclusive_scan_i32(int32_t * A, long N)
{
	long acc = 0;
	for (long i = 0; i < N; i++) {
		long t = A[i];
		A[i] = (int32_t) acc;
		acc += t;
	}
	return acc;
}

static void slice_widths_to_ptr(const int32_t * rp, long m, long V, int32_t * rcp)
{
	long nc = (m + V - 1) / V;
	for (long c = 0; c < nc; c++) {
		long w = 0;
		for (long k = c * V; k < MINV(c * V + V, m); k++)
			w = MAXV(w, (long) rp[k + 1] - rp[k]);
		rcp[c] = (int32_t) (V * w);
	}
	rcp[nc] = 0;
	exclusive_scan_i32(rcp, nc + 1);
}

long orc_sell_size(const int32_t * rp, long m, long V)
{
	long nc = (m + V - 1) / V, tot = 0;
	for (long c = 0; c < nc; c++) {
		long w = 0;
		for (long k = c * V; k < MINV(c * V + V, m); k++)
			w = MAXV(w, (long) rp[k + 1] - rp[k]);
		tot += V * w;
	}
	return tot;
}

/* Fill the slices [ii_s, ii_e) of one thread range from a CSR (rp, ci, v): rows padded to
 * the slice width and missing rows of the last slice padded, value 0 and column = the
 * last column written in this range (0 at its start), then each slice transposed to
 * column-major (src/spmv_kernels/sell.cpp:163-197; also sell_sorted.cpp:262-301). */
static void sell_fill_range(const int32_t * rp, const int32_t * ci, const double * v, long m, long V,
		const int32_t * rcp, long ii_s, long ii_e, int32_t * ja, double * a)
{
	long col = 0;
	for (long ii = ii_s; ii < ii_e; ii++) {
		long width = (rcp[ii + 1] - rcp[ii]) / V;
		long i_s = V * ii, i_e = MINV(i_s + V, m);
		long base = rcp[ii];
		long jj = 0;
		/* row-major staging: row r of the slice at [r * width, (r+1) * width) */
		int32_t * tja = (int32_t *) malloc(MAXV(1, V * width) * sizeof(int32_t));
		double * ta = (double *) malloc(MAXV(1, V * width) * sizeof(double));
		for (long i = i_s; i < i_e; i++) {
			long j = rp[i];
			for (; j < rp[i + 1]; j++, jj++) {
				ta[jj] = v[j];
				col = ci[j];
				tja[jj] = (int32_t) col;
			}
			for (; j < rp[i] + width; j++, jj++) {
				ta[jj] = 0;
				tja[jj] = (int32_t) col;
			}
		}
		for (; jj < V * width; jj++) {
			ta[jj] = 0;
			tja[jj] = (int32_t) col;
		}
		for (long r = 0; r < V; r++)
			for (long k = 0; k < width; k++) {
				a[base + k * V + r] = ta[r * width + k];
				ja[base + k * V + r] = tja[r * width + k];
			}
		free(tja);
		free(ta);
	}
}

/* SELLArray constructor (src/spmv_kernels/sell.cpp:95-199): slice widths, exclusive scan,
 * thread ranges balanced over the padded sizes (:161), per-range fill. */
void orc_sell_convert(const int32_t * rp, const int32_t * ci, const double * v, long m, long V, long T,
		int32_t * rcp, int32_t * ja, double * a, int64_t * ranges)
{
	long nc = (m + V - 1) / V;
	slice_widths_to_ptr(rp, m, V, rcp);
	long nnz_ext = rcp[nc];
	for (long t = 0; t < T; t++) {
		long s, e;
		orc_partition_prefix_sums(T, t, rcp, nc, nnz_ext, &s, &e);
		if (ranges) {
			ranges[2 * t] = s;
			ranges[2 * t + 1] = e;
		}
		sell_fill_range(rp, ci, v, m, V, rcp, s, e, ja, a);
	}
}

/* compute_sell (src/spmv_kernels/sell.cpp:240-280): per slice, per lane, fused
 * multiply-adds over the slice width; rows >= m are not stored here (the reference
 * writes them into y's 64-element tail). */
void orc_sell_spmv(const int32_t * rcp, const int32_t * ja, const double * a, long m, long V, const double * x, double * y)
{
	long nc = (m + V - 1) / V;
	#pragma omp parallel for schedule(static)
	for (long ii = 0; ii < nc; ii++) {
		for (long r = 0; r < V; r++) {
			long i = ii * V + r;
			if (i >= m)
				break;
			double sum = 0;
			for (long jj = rcp[ii] + r; jj < rcp[ii + 1]; jj += V)
				sum = fma(a[jj], x[ja[jj]], sum);
			y[i] = sum;
		}
	}
}

/* ======================================================================================
 * sell_sorted
 * ====================================================================================== */

static void sell_sorted_ranges(const int32_t * rp, long m, long V, long T, long t, long * ii_s, long * ii_e, long * i_s, long * i_e)
{
	long nc = (m + V - 1) / V;
	int32_t * rcp = (int32_t *) malloc((nc + 1) * sizeof(int32_t));
	for (long c = 0; c < nc; c++)
		rcp[c] = rp[c * V];
	rcp[nc] = rp[m];
	orc_partition_prefix_sums(T, t, rcp, nc, rp[m], ii_s, ii_e);
	*i_s = *ii_s * V;
	*i_e = *ii_e * V;
	if (t == T - 1)
		*i_e = m;
	free(rcp);
}

/* Stable counting sort of the row lengths of [i_s, i_e), ascending
 * (bucketsort_stable_recalculate_bucket_serial, lib/sort/bucketsort/bucketsort_gen.c:168-193,
 * bucket = row length, src/spmv_kernels/sell_sorted.cpp:82-87, used at :183-196). */
static void sell_sorted_permutation(const int32_t * rp, long i_s, long i_e, int32_t * perm, int32_t * rev_perm)
{
	long dmax = 0;
	for (long i = i_s; i < i_e; i++)
		dmax = MAXV(dmax, (long) rp[i + 1] - rp[i]);
	long * off = (long *) calloc(dmax + 2, sizeof(long));
	for (long i = i_s; i < i_e; i++)
		off[rp[i + 1] - rp[i]]++;
	long acc = 0;
	for (long b = 0; b <= dmax + 1; b++) {
		acc += off[b];
		off[b] = acc;
	}
	for (long i = i_e - 1; i >= i_s; i--) {
		long b = rp[i + 1] - rp[i];
		off[b]--;
		perm[i] = (int32_t) (i_s + off[b]);
	}
	for (long i = i_s; i < i_e; i++)
		rev_perm[perm[i]] = (int32_t) i;
	free(off);
}

long orc_sell_sorted_size(const int32_t * rp, long m, long V, long T)
{
	int32_t * perm = (int32_t *) malloc(MAXV(1, m) * sizeof(int32_t));
	int32_t * rev = (int32_t *) malloc(MAXV(1, m) * sizeof(int32_t));
	int32_t * deg = (int32_t *) malloc((m + 1) * sizeof(int32_t));
	for (long t = 0; t < T; t++) {
		long ii_s, ii_e, i_s, i_e;
		sell_sorted_ranges(rp, m, V, T, t, &ii_s, &ii_e, &i_s, &i_e);
		sell_sorted_permutation(rp, i_s, i_e, perm, rev);
	}
	for (long i = 0; i < m; i++)
		deg[perm[i]] = rp[i + 1] - rp[i];
	deg[m] = 0;
	exclusive_scan_i32(deg, m + 1);
	long tot = orc_sell_size(deg, m, V);
	free(perm);
	free(rev);
	free(deg);
	return tot;
}

/* SELLArray constructor of src/spmv_kernels/sell_sorted.cpp:119-305: nnz-balanced ranges
 * of whole slices, a stable ascending sort of row lengths inside each range, the reordered
 * CSR, then SELL slices over it with per-range padding columns. */
void orc_sell_sorted_convert(const int32_t * rp, const int32_t * ci, const double * v, long m, long V, long T,
		int32_t * rcp, int32_t * ja, double * a, int32_t * perm, int32_t * rev_perm, int64_t * ranges)
{
	long nc = (m + V - 1) / V;
	long nnz = rp[m];
	int32_t * rp2 = (int32_t *) malloc((m + 1) * sizeof(int32_t));
	int32_t * ci2 = (int32_t *) malloc(MAXV(1, nnz) * sizeof(int32_t));
	double * v2 = (double *) malloc(MAXV(1, nnz) * sizeof(double));
	long (*rg)[4] = malloc(T * sizeof(*rg));
	for (long t = 0; t < T; t++) {
		sell_sorted_ranges(rp, m, V, T, t, &rg[t][0], &rg[t][1], &rg[t][2], &rg[t][3]);
		if (ranges) {
			ranges[2 * t] = rg[t][0];
			ranges[2 * t + 1] = rg[t][1];
		}
		sell_sorted_permutation(rp, rg[t][2], rg[t][3], perm, rev_perm);
	}
	for (long i = 0; i < m; i++)
		rp2[perm[i]] = rp[i + 1] - rp[i];
	rp2[m] = 0;
	exclusive_scan_i32(rp2, m + 1);
	for (long t = 0; t < T; t++) {
		long k = rp[rg[t][2]];
		for (long i = rg[t][2]; i < rg[t][3]; i++)
			for (long j = rp[rev_perm[i]]; j < rp[rev_perm[i] + 1]; j++, k++) {
				ci2[k] = ci[j];
				v2[k] = v[j];
			}
	}
	slice_widths_to_ptr(rp2, m, V, rcp);
	(void) nc;
	for (long t = 0; t < T; t++)
		sell_fill_range(rp2, ci2, v2, m, V, rcp, rg[t][0], rg[t][1], ja, a);
	free(rp2);
	free(ci2);
	free(v2);
	free(rg);
}

/* compute_sell of sell_sorted (src/spmv_kernels/sell_sorted.cpp:346-427): slot i of the
 * reordered rows is row rev_perm[i]. */
void orc_sell_sorted_spmv(const int32_t * rcp, const int32_t * ja, const double * a, const int32_t * rev_perm,
		long m, long V, const double * x, double * y)
{
	long nc = (m + V - 1) / V;
	#pragma omp parallel for schedule(static)
	for (long ii = 0; ii < nc; ii++) {
		for (long r = 0; r < V; r++) {
			long i = ii * V + r;
			if (i >= m)
				break;
			double sum = 0;
			for (long jj = rcp[ii] + r; jj < rcp[ii + 1]; jj += V)
				sum = fma(a[jj], x[ja[jj]], sum);
			y[rev_perm[i]] = sum;
		}
	}
}

/* ======================================================================================
 * SELL-C-sigma
 * ====================================================================================== */

/* get_order_by_row_size (src/spmv_kernels/sell-C-s/radix_sort.c:103-122) with
 * radix_sort_paired_descending / count_sort_paired_reversed (:36-101): per sigma window a
 * 4-bit LSD radix sort whose passes place larger digits first and keep equal digits in
 * their input order -- a stable descending sort of the row lengths. */
static void sellcs_order(const int32_t * rp, long m, long sigma, int32_t * sizes, int32_t * order)
{
	for (long i = 0; i < m; i++) {
		sizes[i] = rp[i + 1] - rp[i];
		order[i] = (int32_t) i;
	}
	for (long k = 0; k < m; k += sigma) {
		long e = MINV(k + sigma, m), len = e - k;
		int32_t * ts = (int32_t *) malloc(len * sizeof(int32_t));
		int32_t * to = (int32_t *) malloc(len * sizeof(int32_t));
		long maxv = 0;
		for (long i = k; i < e; i++)
			maxv = MAXV(maxv, (long) sizes[i]);
		long digits = 0;
		while (maxv) {
			digits++;
			maxv >>= 4;
		}
		for (long d = 0, sh = 0; d < digits; d++, sh += 4) {
			long cnt[16] = {0};
			for (long i = k; i < e; i++)
				cnt[(sizes[i] >> sh) & 15]++;
			long pos[16], acc = 0;
			for (long b = 15; b >= 0; b--) {     /* larger digits first */
				pos[b] = acc;
				acc += cnt[b];
			}
			for (long i = k; i < e; i++) {
				long b = (sizes[i] >> sh) & 15;
				ts[pos[b]] = sizes[i];
				to[pos[b]] = order[i];
				pos[b]++;
			}
			memcpy(&sizes[k], ts, len * sizeof(int32_t));
			memcpy(&order[k], to, len * sizeof(int32_t));
		}
		free(ts);
		free(to);
	}
}

long orc_sellcs_size(const int32_t * rp, long m, long C, long sigma)
{
	int32_t * sizes = (int32_t *) malloc(MAXV(1, m) * sizeof(int32_t));
	int32_t * order = (int32_t *) malloc(MAXV(1, m) * sizeof(int32_t));
	sellcs_order(rp, m, sigma, sizes, order);
	long ns = (m + C - 1) / C, tot = 0;
	for (long s = 0; s < ns; s++)
		tot += (long) sizes[s * C] * C;
	free(sizes);
	free(order);
	return tot;
}

/* csr_to_sellcs (src/spmv_kernels/sell-C-s/sellcs_format.c:137-200): slice width = the
 * length of the slice's first (sorted) row, slice pointers = exclusive scan of C * width,
 * column-major slices with zero padding (column 0, value 0).  C must be a power of two
 * (the kernel shifts by log2 C, sellcs_format.c:40-47) and sigma a multiple of C, so
 * no slice straddles two windows. */
int orc_sellcs_convert(const int32_t * rp, const int32_t * ci, const double * v, long m, long C, long sigma,
		int32_t * row_order, int32_t * widths, int64_t * ptrs, int32_t * cols, double * vals)
{
	if (C <= 0 || (C & (C - 1)) || sigma <= 0 || sigma % C)
		return -1;
	int32_t * sizes = (int32_t *) malloc(MAXV(1, m) * sizeof(int32_t));
	sellcs_order(rp, m, sigma, sizes, row_order);
	long ns = (m + C - 1) / C, tot = 0;
	for (long s = 0; s < ns; s++) {
		widths[s] = sizes[s * C];
		ptrs[s] = tot;
		tot += (long) sizes[s * C] * C;
	}
	ptrs[ns] = tot;
	memset(cols, 0, tot * sizeof(int32_t));
	memset(vals, 0, tot * sizeof(double));
	for (long r = 0; r < m; r++) {
		long w = ptrs[r / C] + (r % C);
		for (long j = rp[row_order[r]]; j < rp[row_order[r] + 1]; j++, w += C) {
			vals[w] = v[j];
			cols[w] = ci[j];
		}
	}
	free(sizes);
	return 0;
}

/* sellcs_mv_d (src/spmv_kernels/sell-C-s/sellcs_mv_kernels_epi.c:178-318, RVV): per slice,
 * lanes = min(C, m - first row); fused multiply-accumulate over the slice width (vfmacc);
 * scatter to y[row_order[...]]. */
void orc_sellcs_spmv(const int32_t * row_order, const int32_t * widths, const int64_t * ptrs, const int32_t * cols,
		const double * vals, long m, long C, const double * x, double * y)
{
	long ns = (m + C - 1) / C;
	#pragma omp parallel for schedule(static)
	for (long s = 0; s < ns; s++) {
		long lanes = MINV(C, m - s * C);
		for (long l = 0; l < lanes; l++) {
			double acc = 0;
			for (long k = 0; k < widths[s]; k++) {
				long w = ptrs[s] + k * C + l;
				acc = fma(x[cols[w]], vals[w], acc);
			}
			y[row_order[s * C + l]] = acc;
		}
	}
}

/* ======================================================================================
 * DIV-RF
 * ====================================================================================== */

/* packet_header (src/spmv_kernels/DIV/div_kernels_rf.h:65-79) with its natural C layout:
 * u32 num_vals @0, num_vals_unique @4, num_rows @8, row_min @12, col_min @16,
 * u8 row_bits @20, col_bits @21, (2 pad bytes), u32 num_rfs @24, u32 lane_sizes[L] @28. */
long orc_div_header_size(long L)
{
	return 28 + 4 * L;
}

static int bits_required(uint64_t v)
{
	return v ? 64 - __builtin_clzll(v) : 0;
}

/* reduce_precision (div_kernels_rf.h:467-510): round the mantissa to the requested
 * relative tolerance, down or up, whichever leaves more trailing zero bits. */
static double div_reduce_precision(double d, double tol)
{
	union { double d; uint64_t u; } val, lo, hi;
	val.d = d;
	if (tol == 0 || val.u == 0)
		return d;
	if (__builtin_ctzll(val.u) >= 53)
		return d;
	uint64_t prec = (uint64_t) ceil(fabs(log2(tol)));
	if (prec >= 52)
		return d;
	uint64_t drop = 52 - prec, p2 = 1ULL << drop, mask = p2 - 1;
	lo.u = val.u & ~mask;
	hi.u = (val.u + mask) & ~mask;
	uint64_t tzl = lo.u ? __builtin_ctzll(lo.u) : 64;
	uint64_t tzh = hi.u ? __builtin_ctzll(hi.u) : 64;
	return (tzl > tzh) ? lo.d : hi.d;
}

/* select_num_vals_complete_last_row (div_kernels_rf.h:437-464), rows capped at 255. */
static long div_select_num_vals(const int32_t * rp, long i_s, long j_s, long nv)
{
	long j_e = j_s + nv, i_e = i_s;
	while (rp[i_e] < j_e)
		i_e++;
	if (j_e != rp[i_e] && i_e - 1 > i_s) {
		i_e--;
		j_e = rp[i_e];
	}
	if (i_e - i_s > 255)
		i_e = i_s + 255;
	long r = rp[i_e] - j_s;
	return r > nv ? nv : r;
}

struct div_entry { uint64_t val; uint32_t row, col; };

static int div_entry_cmp(const void * pa, const void * pb)
{
	const struct div_entry * a = pa, * b = pb;
	if (a->val != b->val) return a->val < b->val ? -1 : 1;
	if (a->row != b->row) return a->row < b->row ? -1 : 1;
	if (a->col != b->col) return a->col < b->col ? -1 : 1;
	return 0;
}

/* permutation_interleave(in, out, N, S, U, 0, 1) (lib/macros/permutation.h:47-115): the
 * N elements are cut into S contiguous segments of whole units of U elements; the main
 * part interleaves element-wise over the segments, the remainder takes whole units. */
#define DEFINE_INTERLEAVE(NAME, TYPE)                                                        \
static void NAME(const TYPE * in, TYPE * out, long N, long S, long U)                        \
{                                                                                            \
	long nu = N / U, rem_u = N - nu * U, dv = nu / S, md = nu % S, mul = dv * U * S;     \
	long * seg = (long *) malloc(S * sizeof(long));                                      \
	for (long i = 0; i < S; i++) {                                                       \
		seg[i] = U * (i * dv + (i < md ? i : md));                                   \
		if (i > md)                                                                  \
			seg[i] += rem_u;                                                     \
	}                                                                                    \
	for (long j = 0; j < mul; j++)                                                       \
		out[j] = in[seg[j % S] + j / S];                                             \
	for (long j = mul; j < N; j++) {                                                     \
		long sg = (j / U) % S, pos = U * (j / (U * S)) + j % U;                      \
		out[j] = in[seg[sg] + pos];                                                  \
	}                                                                                    \
	free(seg);                                                                           \
}
DEFINE_INTERLEAVE(interleave_u64, uint64_t)
DEFINE_INTERLEAVE(interleave_entry, struct div_entry)

static inline void put_u32(uint8_t * p, uint32_t v) { memcpy(p, &v, 4); }
static inline uint32_t get_u32(const uint8_t * p) { uint32_t v; memcpy(&v, p, 4); return v; }

/* Delta-length code of one lane value difference (div_kernels_rf.h:824-892): the
 * significant bits of diff are stored in `len` bytes after shifting out a multiple of 4
 * trailing zeros; the code byte holds len (low nibble) and shift/4 (high nibble). */
static void div_encode_diff(uint64_t diff, uint8_t * code, uint64_t * payload, int * nbytes)
{
	if (diff == 0) {
		*code = 0;
		*payload = 0;
		*nbytes = 0;
		return;
	}
	uint64_t lz = __builtin_clzll(diff), tz = __builtin_ctzll(diff);
	uint64_t rem_tz = tz & 3;
	uint64_t len_bits = 64 - lz - tz;
	uint64_t len = (len_bits + 7) >> 3;
	uint64_t rem = (len << 3) - len_bits;
	if (rem >= rem_tz) {
		rem -= rem_tz;
		tz -= rem_tz;
	}
	if (rem <= lz) {
		lz -= rem;
		rem = 0;
	} else {
		rem -= lz;
		lz = 0;
	}
	tz -= rem;
	uint64_t tz4 = tz >> 2;
	tz = tz4 << 2;
	len_bits = 64 - lz - tz;
	len = (len_bits + 7) >> 3;
	*payload = diff >> tz;
	*nbytes = (int) len;
	*code = (uint8_t) (len | (tz4 << 4));
}

/* compress_kernel_div (div_kernels_rf.h:538-919): one packet starting at nnz j_s of row
 * i_s.  Returns the packet size in bytes, sets *nv_out. */
static long div_compress_packet(const int32_t * rp, const int32_t * ci, const double * v, long i_s, long j_s,
		long nv_max, long L, double tol, uint8_t * out, long * nv_out)
{
	long nv = div_select_num_vals(rp, i_s, j_s, nv_max);
	*nv_out = nv;
	struct div_entry * e = (struct div_entry *) malloc(nv * sizeof(*e));
	struct div_entry * e2 = (struct div_entry *) malloc(nv * sizeof(*e2));
	long row_min = i_s, col_min = ci[j_s], col_max = ci[j_s];
	long i = i_s;
	for (long k = 0, j = j_s; k < nv; k++, j++) {
		while (j >= rp[i + 1])
			i++;
		union { double d; uint64_t u; } u;
		u.d = (tol > 0) ? div_reduce_precision(v[j], tol) : v[j];
		long c = ci[j];
		col_min = MINV(col_min, c);
		col_max = MAXV(col_max, c);
		e[k].val = u.u;
		e[k].row = (uint32_t) i;
		e[k].col = (uint32_t) c;
	}
	long row_max = i;
	long row_bits = bits_required(row_max - row_min);
	long col_bits = bits_required(col_max - col_min);
	long cbytes = (row_bits + col_bits + 7) >> 3;
	if (row_bits % 8) {
		long cmpl = 8 - row_bits % 8;
		if (((row_bits + cmpl + col_bits + 7) >> 3) == cbytes)
			row_bits += cmpl;
	}
	col_bits = cbytes * 8 - row_bits;

	qsort(e, nv, sizeof(*e), div_entry_cmp);

	/* replication factor = multiplicity of each value (:671-700) */
	int32_t * rf = (int32_t *) malloc(nv * sizeof(int32_t));
	long max_rf = 1, nuniq = 0;
	for (long k = 0; k < nv;) {
		long kk = k + 1;
		while (kk < nv && e[kk].val == e[kk - 1].val)
			kk++;
		for (long t = k; t < kk; t++)
			rf[t] = (int32_t) (kk - k);
		max_rf = MAXV(max_rf, kk - k);
		nuniq++;
		k = kk;
	}
	/* stable bucket sort by rf (:703-712) */
	long * off = (long *) calloc(max_rf + 2, sizeof(long));
	for (long k = 0; k < nv; k++)
		off[rf[k]]++;
	long acc = 0;
	for (long b = 0; b <= max_rf + 1; b++) {
		long t = off[b];
		off[b] = acc;
		acc += t;
	}
	long * start = (long *) malloc((max_rf + 2) * sizeof(long));
	memcpy(start, off, (max_rf + 2) * sizeof(long));
	for (long k = 0; k < nv; k++)
		e2[off[rf[k]]++] = e[k];
	/* unique values in rf-group order (:714-729), then per rf group interleave (:731-756) */
	uint64_t * uq = (uint64_t *) malloc(MAXV(1, nuniq) * sizeof(uint64_t));
	uint64_t * uq2 = (uint64_t *) malloc(MAXV(1, nuniq) * sizeof(uint64_t));
	long * rfs = (long *) malloc((max_rf + 1) * sizeof(long));
	long * nu_rf = (long *) malloc((max_rf + 1) * sizeof(long));
	long num_rfs = 0, ku = 0;
	for (long r = 1; r <= max_rf; r++) {
		long ls = start[r], le = start[r + 1], cnt = le - ls;
		if (cnt == 0)
			continue;
		long u = cnt / r;
		rfs[num_rfs] = r;
		nu_rf[num_rfs] = u;
		num_rfs++;
		for (long q = 0; q < u; q++)
			uq[ku + q] = e2[ls + q * r].val;
		interleave_u64(uq + ku, uq2 + ku, u, L, 1);
		interleave_entry(e2 + ls, e + ls, cnt, L, r);
		ku += u;
	}
	/* layout (:758-917) */
	long hsz = orc_div_header_size(L);
	memset(out, 0, hsz);
	put_u32(out + 0, (uint32_t) nv);
	put_u32(out + 4, (uint32_t) nuniq);
	put_u32(out + 8, (uint32_t) (row_max - row_min + 1));
	put_u32(out + 12, (uint32_t) row_min);
	put_u32(out + 16, (uint32_t) col_min);
	out[20] = (uint8_t) row_bits;
	out[21] = (uint8_t) col_bits;
	put_u32(out + 24, (uint32_t) num_rfs);
	uint8_t * p = out + hsz;
	for (long q = 0; q < num_rfs; q++)
		put_u32(p + 4 * q, (uint32_t) rfs[q]);
	p += 4 * num_rfs;
	for (long q = 0; q < num_rfs; q++)
		put_u32(p + 4 * q, (uint32_t) nu_rf[q]);
	p += 4 * num_rfs;
	for (long k = 0; k < nv; k++) {
		uint64_t c = (uint64_t) (e[k].row - row_min) | ((uint64_t) (e[k].col - col_min) << row_bits);
		memcpy(p + k * cbytes, &c, cbytes);
	}
	p += cbytes * nv;
	uint8_t * codes = p;
	p += nuniq;
	/* lane streams: lane l's bytes are contiguous, lanes in order */
	long * lane_len = (long *) calloc(L, sizeof(long));
	uint8_t ** lane_buf = (uint8_t **) malloc(L * sizeof(uint8_t *));
	for (long l = 0; l < L; l++)
		lane_buf[l] = (uint8_t *) malloc(8 * (nuniq / L + num_rfs + 1));   /* ceil per rf group */
	uint64_t * prev = (uint64_t *) malloc(L * sizeof(uint64_t));
	long ks = 0;
	for (long g = 0; g < num_rfs; g++) {
		for (long l = 0; l < L; l++)
			prev[l] = 0;
		for (long q = 0; q < nu_rf[g]; q++) {
			long k = ks + q, lane = q % L;
			uint64_t diff = uq2[k] - prev[lane];
			prev[lane] += diff;
			uint64_t pay;
			int nb;
			div_encode_diff(diff, &codes[k], &pay, &nb);
			memcpy(lane_buf[lane] + lane_len[lane], &pay, nb);
			lane_len[lane] += nb;
		}
		ks += nu_rf[g];
	}
	for (long l = 0; l < L; l++) {
		put_u32(out + 28 + 4 * l, (uint32_t) lane_len[l]);
		memcpy(p, lane_buf[l], lane_len[l]);
		p += lane_len[l];
		free(lane_buf[l]);
	}
	long size = p - out;
	free(lane_buf); free(lane_len); free(prev);
	free(e); free(e2); free(rf); free(off); free(start); free(uq); free(uq2); free(rfs); free(nu_rf);
	return size;
}

struct div_thread {
	uint8_t * data;
	long bytes, cap;
	long * pkt;          /* packet start offsets within this thread's stream */
	long npkt, pkt_cap;
	long * grp;          /* group start offsets (+ end) */
	long ngrp, grp_cap;
	long i_s, i_e;
	int err;
};

struct div_handle {
	long T, L;
	struct div_thread * th;
};

static void * grow(void * p, long * cap, long need, long elem)
{
	if (need <= *cap)
		return p;
	long c = MAXV(need, 2 * *cap + 16);
	*cap = c;
	return realloc(p, c * elem);
}

/* DIVArray constructor, packetisation loop (src/spmv_kernels/DIV/div.cpp:236-453):
 * nnz-balanced row ranges per thread; in each range a chain of packets; a packet group
 * starts whenever a packet starts at a row start. */
void * orc_div_build(const int32_t * rp, const int32_t * ci, const double * v, long m, long n, long T, long L,
		long packet_vals, double tol)
{
	(void) n;
	if (T < 1 || L < 1 || packet_vals < 1 || tol < 0 || tol >= 1.0)
		return NULL;
	long nnz = rp[m];
	struct div_handle * h = (struct div_handle *) calloc(1, sizeof(*h));
	h->T = T;
	h->L = L;
	h->th = (struct div_thread *) calloc(T, sizeof(struct div_thread));
	long pbuf = orc_div_header_size(L) + packet_vals * 24 + 64;
	#pragma omp parallel for schedule(dynamic, 1)
	for (long t = 0; t < T; t++) {
		struct div_thread * td = &h->th[t];
		long i_s, i_e;
		orc_partition_prefix_sums(T, t, rp, m, nnz, &i_s, &i_e);
		td->i_s = i_s;
		td->i_e = i_e;
		uint8_t * buf = (uint8_t *) malloc(pbuf);
		long i = i_s, j = rp[i_s], j_e = rp[i_e];
		long grp_acc = -1;
		while (j < j_e) {
			while (rp[i] < j)
				i++;
			if (rp[i] != j)
				i--;
			while (rp[i] == rp[i + 1])
				i++;
			long nv_max = (j + packet_vals <= j_e) ? packet_vals : j_e - j;
			long nv;
			long sz = div_compress_packet(rp, ci, v, i, j, nv_max, L, tol, buf, &nv);
			td->data = (uint8_t *) grow(td->data, &td->cap, td->bytes + sz, 1);
			td->pkt = (long *) grow(td->pkt, &td->pkt_cap, td->npkt + 1, sizeof(long));
			td->pkt[td->npkt++] = td->bytes;
			if (j == rp[i]) {
				td->grp = (long *) grow(td->grp, &td->grp_cap, td->ngrp + 2, sizeof(long));
				td->grp[td->ngrp++] = td->bytes;
				grp_acc = 0;
			}
			if (grp_acc < 0)
				td->err = 1;           /* first packet must open a group */
			memcpy(td->data + td->bytes, buf, sz);
			td->bytes += sz;
			j += nv;
		}
		td->grp = (long *) grow(td->grp, &td->grp_cap, td->ngrp + 1, sizeof(long));
		td->grp[td->ngrp] = td->bytes;
		free(buf);
	}
	return h;
}

long orc_div_get(void * hp, int what, void * dst)
{
	struct div_handle * h = (struct div_handle *) hp;
	long T = h->T, cnt = 0, base = 0;
	switch (what) {
	case 0:
		for (long t = 0; t < T; t++) {
			if (dst)
				memcpy((uint8_t *) dst + cnt, h->th[t].data, h->th[t].bytes);
			cnt += h->th[t].bytes;
		}
		return cnt;
	case 1:
		for (long t = 0; t < T; t++) {
			for (long p = 0; p < h->th[t].npkt; p++) {
				if (dst)
					((int64_t *) dst)[cnt] = base + h->th[t].pkt[p];
				cnt++;
			}
			base += h->th[t].bytes;
		}
		if (dst)
			((int64_t *) dst)[cnt] = base;
		return cnt + 1;
	case 2:
		for (long t = 0; t < T; t++)
			if (dst)
				((int64_t *) dst)[t] = h->th[t].bytes;
		return T;
	case 3:
		for (long t = 0; t < T; t++)
			if (dst)
				((int64_t *) dst)[t] = h->th[t].ngrp;
		return T;
	case 4:
		for (long t = 0; t < T; t++)
			for (long g = 0; g <= h->th[t].ngrp; g++) {
				if (dst)
					((int64_t *) dst)[cnt] = h->th[t].grp[g];
				cnt++;
			}
		return cnt;
	case 5:
		for (long t = 0; t < T; t++)
			if (dst) {
				((int64_t *) dst)[2 * t] = h->th[t].i_s;
				((int64_t *) dst)[2 * t + 1] = h->th[t].i_e;
			}
		return 2 * T;
	case 6:
		for (long t = 0; t < T; t++)
			cnt += h->th[t].err;
		return cnt;
	}
	return -1;
}

void orc_div_free(void * hp)
{
	struct div_handle * h = (struct div_handle *) hp;
	if (!h)
		return;
	for (long t = 0; t < h->T; t++) {
		free(h->th[t].data);
		free(h->th[t].pkt);
		free(h->th[t].grp);
	}
	free(h->th);
	free(h);
}

/* Decoder of one packet (div_kernels_rf.h:948-1162): per rf group, each lane's value is the
 * running sum of its decoded differences (reset per group); the vector part visits blocks
 * of L unique values and, for each of the rf replicas, the L lanes in order; the
 * remaining values are visited one by one.  Calls emit(row, col, value) in that order. */
typedef void (*div_emit_fn)(void * ctx, long row, long col, double val, int single_row);

static long div_decode_packet(const uint8_t * buf, long L, div_emit_fn emit, void * ctx, long * nv_out)
{
	long nv = get_u32(buf + 0), nu = get_u32(buf + 4);
	long row_min = get_u32(buf + 12), col_min = get_u32(buf + 16);
	long row_bits = buf[20], col_bits = buf[21];
	long num_rfs = get_u32(buf + 24);
	long hsz = orc_div_header_size(L);
	const uint8_t * rfs = buf + hsz;
	const uint8_t * nurf = rfs + 4 * num_rfs;
	const uint8_t * coords = nurf + 4 * num_rfs;
	long cbytes = (row_bits + col_bits + 7) >> 3;
	const uint8_t * codes = coords + cbytes * nv;
	const uint8_t * lanes0 = codes + nu;
	const uint8_t ** lp = (const uint8_t **) malloc(L * sizeof(*lp));
	uint64_t * val = (uint64_t *) malloc(L * sizeof(uint64_t));
	long lanes_total = 0;
	lp[0] = lanes0;
	for (long l = 0; l < L; l++) {
		long sz = get_u32(buf + 28 + 4 * l);
		if (l + 1 < L)
			lp[l + 1] = lp[l] + sz;
		lanes_total += sz;
	}
	uint64_t rmask = row_bits ? ((1ULL << row_bits) - 1) : 0;
	uint64_t cmask = (col_bits >= 64) ? ~0ULL : ((1ULL << col_bits) - 1);
	for (long g = 0; g < num_rfs; g++) {
		long rf = get_u32(rfs + 4 * g), u = get_u32(nurf + 4 * g);
		for (long l = 0; l < L; l++)
			val[l] = 0;
		long mult = (u / L) * L;
		for (long q = 0; q < u; q++) {
			long lane = q % L;
			uint8_t code = codes[q];
			long len = code & 15, tz = (code >> 2) & ~3;
			uint64_t d = 0;
			memcpy(&d, lp[lane], len);
			lp[lane] += len;
			val[lane] += d << tz;
			if (q < mult && lane != L - 1)
				continue;
			/* emit: a full block of L values (vector part) or a single remainder value */
			if (q < mult) {
				long qb = q - (L - 1);
				for (long j = 0; j < rf; j++)
					for (long ln = 0; ln < L; ln++) {
						long k = qb * rf + L * j + ln;
						uint64_t c = 0;
						memcpy(&c, coords + k * cbytes, cbytes);
						union { uint64_t u; double d; } vv;
						vv.u = val[ln];
						emit(ctx, row_min + (long) (c & rmask), col_min + (long) ((c >> row_bits) & cmask), vv.d, row_bits == 0);
					}
			} else {
				for (long j = 0; j < rf; j++) {
					long k = q * rf + j;
					uint64_t c = 0;
					memcpy(&c, coords + k * cbytes, cbytes);
					union { uint64_t u; double d; } vv;
					vv.u = val[lane];
					emit(ctx, row_min + (long) (c & rmask), col_min + (long) ((c >> row_bits) & cmask), vv.d, row_bits == 0);
				}
			}
		}
		codes += u;
		coords += cbytes * rf * u;
	}
	free(lp);
	free(val);
	*nv_out = nv;
	return hsz + 8 * num_rfs + cbytes * nv + nu + lanes_total;
}

struct spmv_ctx { const double * x; double * y; int fused; };

/* The reference's x86 build fuses the multiply-add of packets that span several rows, but
 * for single-row packets (row_bits == 0, the gather returns row 0 for every lane) the
 * compiler turns the lane updates of y[row_min] into rounded products followed by
 * rounded adds; both are reproduced here. */
static void emit_spmv(void * c, long row, long col, double val, int single_row)
{
	struct spmv_ctx * s = (struct spmv_ctx *) c;
	if (s->fused && !single_row)
		s->y[row] = fma(val, s->x[col], s->y[row]);
	else {
		double p = val * s->x[col];
		s->y[row] = s->y[row] + p;
	}
}

int orc_div_spmv(const uint8_t * data, long total, const int64_t * ranges, long T, long L,
		const double * x, double * y, int fused)
{
	for (long t = 0; t < T; t++)
		for (long i = ranges[2 * t]; i < ranges[2 * t + 1]; i++)
			y[i] = 0;
	struct spmv_ctx c = { x, y, fused };
	long pos = 0;
	while (pos < total) {
		long nv;
		long sz = div_decode_packet(data + pos, L, emit_spmv, &c, &nv);
		if (sz <= 0)
			return -1;
		pos += sz;
	}
	return pos == total ? 0 : -1;
}

struct coo_ctx { int32_t * r; int32_t * c; double * v; long k; };

static void emit_coo(void * cp, long row, long col, double val, int single_row)
{
	(void) single_row;
	struct coo_ctx * s = (struct coo_ctx *) cp;
	s->r[s->k] = (int32_t) row;
	s->c[s->k] = (int32_t) col;
	s->v[s->k] = val;
	s->k++;
}

long orc_div_decode_coo(const uint8_t * data, long total, long L, int32_t * rows, int32_t * cols, double * vals)
{
	struct coo_ctx c = { rows, cols, vals, 0 };
	long pos = 0;
	while (pos < total) {
		long nv;
		long sz = div_decode_packet(data + pos, L, emit_coo, &c, &nv);
		if (sz <= 0)
			return -1;
		pos += sz;
	}
	return pos == total ? c.k : -1;
}
