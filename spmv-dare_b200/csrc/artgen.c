/*
 * Host restatement of the reference's artificial sparse-matrix generator
 * (artificial-matrix-generator/artificial_matrix_generation.c:163-579, random.h:119-307),
 * the input source of the benchmark (bench.cpp:243-290, argv order bench.cpp:564-578).
 *
 * The output must be the reference's matrix bit for bit, so the random streams and the
 * floating-point expressions follow the reference exactly:
 *   - glibc random_r with a 256-byte state (initstate_r / srandom_r), reseeded with
 *     seed + row at every anchor row, so the matrix does not depend on the thread count;
 *   - degrees: an exponentially decaying skew term plus a normal (Box-Muller) or gamma
 *     (Marsaglia-Tsang) term, rounded half up;
 *   - columns: an ordered set per row filled by cross-row copying, bounded random draws
 *     with 20 retries then deterministic bound scanning, and geometric clustering of right
 *     neighbours; values are U[0,1) draws in insertion order.
 * It is compiled as GNU C with the reference's optimisation flags so that the compiler
 * contracts the same multiply-adds.  The one deviation: fewer than 100 rows make the
 * reference divide by zero (anchors_num = rows / 100 = 0); here one anchor is used.
 */
#define _GNU_SOURCE
#include <stdlib.h>
#include <stdint.h>
#include <string.h>
#include <math.h>
#include <float.h>
#include <omp.h>

#define ART_RANDOM_MAX     0x7FFFFFFFL
#define ART_RANDOM_MAX_64  0x3FFFFFFFFFFFFFFFL

struct art_rng {
	struct random_data buf;
	char state[256];
};

static void rng_init(struct art_rng * r, unsigned int seed)
{
	memset(r, 0, sizeof(*r));
	r->buf.state = NULL;
	initstate_r(seed, r->state, sizeof(r->state), &r->buf);
	srandom_r(seed, &r->buf);
}

static inline void rng_reseed(struct art_rng * r, unsigned int seed)
{
	srandom_r(seed, &r->buf);
}

/* uniform double in [lo, hi) */
static inline double rng_uniform(struct art_rng * r, double lo, double hi)
{
	int32_t v;
	double res;
	random_r(&r->buf, &v);
	res = ((double) v) / ((double) (ART_RANDOM_MAX + 1L));
	res = (hi - lo) * res + lo;
	return res;
}

/* uniform integer in [lo, hi), rejection of the modulo-biased tail */
static inline long rng_uniform_int(struct art_rng * r, long lo, long hi)
{
	int64_t range = hi - lo;
	if (range >= ART_RANDOM_MAX) {
		int64_t lim = ART_RANDOM_MAX_64 - ART_RANDOM_MAX_64 % range;
		int32_t v;
		int64_t res;
		do {
			random_r(&r->buf, &v);
			res = v;
			res <<= 31;
			random_r(&r->buf, &v);
			res |= v;
		} while (res >= lim);
		return (long) (res % range + lo);
	} else {
		int64_t lim = ART_RANDOM_MAX - ART_RANDOM_MAX % range;
		int32_t v;
		do {
			random_r(&r->buf, &v);
		} while (v >= lim);
		return (long) (v % range + lo);
	}
}

static inline double rng_normal(struct art_rng * r, double mean, double std)
{
	double u1, u2;
	u1 = rng_uniform(r, 2 * DBL_EPSILON, 1);
	u2 = rng_uniform(r, 0, 1);
	double magnitude = std * sqrt(-2.0 * log(u1));
	double z0 = magnitude * cos(2.0 * M_PI * u2) + mean;
	return z0;
}

static double rng_gamma(struct art_rng * r, double k, double theta)
{
	if (k < 1) {
		double u = rng_uniform(r, 2 * DBL_EPSILON, 1);
		return rng_gamma(r, 1.0 + k, theta) * pow(u, 1.0 / k);
	}
	double x, v, u;
	double d = k - 1.0 / 3.0;
	double c = (1.0 / 3.0) / sqrt(d);
	while (1) {
		do {
			x = rng_normal(r, 0, 1);
			v = 1.0 + c * x;
		} while (v <= 0);
		v = v * v * v;
		u = rng_uniform(r, 2 * DBL_EPSILON, 1);
		if (u < 1 - 0.0331 * x * x * x * x)
			break;
		if (log(u) < 0.5 * x * x + d * (1 - v + log(v)))
			break;
	}
	return theta * d * v;
}

/* ---- bandwidth correction (artificial_matrix_generation.c:64-147) ---- */
static double expected_bandwidth(double B, double n)
{
	double E, a, b, b_e, x;
	long i;
	b_e = 0;
	for (i = 0; i < (long) n; i++)
		b_e += log2(n - i) - log2(B - i);
	b = pow(2, b_e);
	E = 0;
	for (i = n; i <= (long) B; i++) {
		x = i;
		a = (B - x + 1) * n / x * (n - 1) / (x - 1);
		E += a * b * (double) i;
		b_e += log2(x + 1) - log2(x + 1 - n);
		b = pow(2, b_e);
	}
	return E;
}

static double corrected_bandwidth(double B, double n)
{
	double E, ratio;
	n = floor(n + 0.5);
	if (n < 2)
		n = 2;
	E = expected_bandwidth(B, n);
	if (E == 0)
		return n;
	ratio = B / E;
	return B * ratio;
}

/* ---- ordered set of column indices of one row (sorted, no duplicates) ---- */
struct colset {
	int * v;
	long n, cap;
};

/* returns 1 if inserted, 0 if already present */
static inline int colset_insert(struct colset * s, int k)
{
	long lo = 0, hi = s->n;
	while (lo < hi) {
		long mid = (lo + hi) >> 1;
		if (s->v[mid] < k)
			lo = mid + 1;
		else
			hi = mid;
	}
	if (lo < s->n && s->v[lo] == k)
		return 0;
	memmove(&s->v[lo + 1], &s->v[lo], (s->n - lo) * sizeof(int));
	s->v[lo] = k;
	s->n++;
	return 1;
}

struct artgen_result {
	long rows, cols, nnz;
	int * row_ptr;
	int * col;
	double * val;
	double stats[37];
	int status;
};

static double mean_of(const double * a, long n)
{
	double s = 0;
	for (long i = 0; i < n; i++)
		s += a[i];
	return n ? s / n : 0;
}

static double std_of(const double * a, long n, double mean)
{
	double s = 0;
	for (long i = 0; i < n; i++)
		s += (a[i] - mean) * (a[i] - mean);
	return n ? sqrt(s / n) : 0;
}

static void min_max_of(const double * a, long n, double * mn, double * mx)
{
	*mn = n ? a[0] : 0;
	*mx = n ? a[0] : 0;
	for (long i = 0; i < n; i++) {
		if (a[i] < *mn) *mn = a[i];
		if (a[i] > *mx) *mx = a[i];
	}
}

/* Generates; returns NULL only on allocation failure (status in res->status otherwise). */
__attribute__((visibility("hidden"))) struct artgen_result * spmv_artgen_run(long nr_rows, long nr_cols, double avg_nnz_per_row, double std_nnz_per_row,
		const char * distribution, unsigned int seed, const char * placement, double bw_scaled, double skew,
		double avg_num_neighbours, double cross_row_similarity, int num_threads)
{
	struct artgen_result * R = (struct artgen_result *) calloc(1, sizeof(*R));
	if (!R)
		return NULL;
	R->rows = nr_rows;
	R->cols = nr_cols;
	if (nr_rows < 1 || nr_cols < 1 || !distribution || !placement) {
		R->status = 1;
		return R;
	}
	if (num_threads < 1)
		num_threads = 1;
	const char dist = distribution[0], plac = placement[0];
	double p_right_neigh = avg_num_neighbours / 2;
	double expected_cluster_size = 1 / (1 - p_right_neigh);
	if (bw_scaled > 1)
		bw_scaled = 1;

	double MAX, C, c_bound1, c_bound2, avg_exp, std_exp, avg_distr, std_distr;
	MAX = avg_nnz_per_row * (1 + skew);
	c_bound1 = MAX / avg_nnz_per_row;
	c_bound2 = (std_nnz_per_row > 0) ? MAX * MAX / (2 * std_nnz_per_row * std_nnz_per_row) : 0;
	C = (c_bound1 > c_bound2) ? c_bound1 : c_bound2;
	if (C <= 2 || skew < 1) {
		MAX = 0;
		C = 0;
		avg_exp = 0;
		std_exp = 0;
		avg_distr = avg_nnz_per_row;
		std_distr = std_nnz_per_row;
	} else {
		avg_exp = MAX / C;
		std_exp = sqrt(avg_exp * avg_exp * (C / 2 - 1));
		avg_distr = avg_nnz_per_row - MAX / C;
		std_distr = sqrt(std_nnz_per_row * std_nnz_per_row - std_exp * std_exp);
		if (dist == 'n')
			if (std_distr > avg_distr / 3)
				std_distr = avg_distr / 3;
	}
	(void) std_exp;

	long anchors_num = nr_rows / 100;
	if (anchors_num < 1)
		anchors_num = 1;
	else if (anchors_num > 1 << 12)
		anchors_num = 1 << 12;
	long period = nr_rows / anchors_num;
	long nseg = (nr_rows + period - 1) / period;

	double * degrees = (double *) malloc(nr_rows * sizeof(double));
	int * offsets = (int *) malloc((nr_rows + 1) * sizeof(int));
	double * bw = (double *) calloc(nr_rows, sizeof(double));
	double * sc = (double *) calloc(nr_rows, sizeof(double));
	double * ngr = (double *) calloc(nr_rows, sizeof(double));
	double * clu = (double *) calloc(nr_rows, sizeof(double));
	long * seg_nnz = (long *) calloc(nseg + 1, sizeof(long));
	if (!degrees || !offsets || !bw || !sc || !ngr || !clu || !seg_nnz) {
		R->status = 2;
		goto out;
	}

	/* pass 1: row degrees, one anchor segment at a time */
	#pragma omp parallel for schedule(dynamic, 1) num_threads(num_threads)
	for (long sg = 0; sg < nseg; sg++) {
		struct art_rng rs;
		rng_init(&rs, (unsigned int) sg);
		long i_s = sg * period, i_e = (sg + 1) * period < nr_rows ? (sg + 1) * period : nr_rows;
		long sum = 0;
		for (long i = i_s; i < i_e; i++) {
			if (i % period == 0)
				rng_reseed(&rs, seed + i);
			double degree_exp = MAX * exp(-C / nr_rows * (double) i);
			double degree_distr;
			if (std_distr > 0) {
				if (dist == 'n')
					degree_distr = rng_normal(&rs, avg_distr, std_distr);
				else {
					double k = (avg_distr * avg_distr) / (std_distr * std_distr);
					double theta = (avg_distr > 0) ? (std_distr * std_distr) / avg_distr : 1;
					degree_distr = rng_gamma(&rs, k, theta);
				}
			} else
				degree_distr = avg_distr;
			double degree = degree_exp + degree_distr;
			degree = (degree > 0) ? floor(degree + 0.5) : 0;
			if (degree > nr_cols)
				degree = nr_cols;
			degrees[i] = degree;
			sum += (long) degree;
		}
		seg_nnz[sg] = sum;
	}
	long nnz = 0;
	for (long sg = 0; sg < nseg; sg++) {
		long t = seg_nnz[sg];
		seg_nnz[sg] = nnz;
		nnz += t;
	}
	if (nnz > 0x7FFFFFFF - 64) {
		R->status = 3;
		goto out;
	}
	R->nnz = nnz;
	R->row_ptr = offsets;
	offsets[nr_rows] = (int) nnz;
	R->col = (int *) malloc((nnz ? nnz : 1) * sizeof(int));
	R->val = (double *) malloc((nnz ? nnz : 1) * sizeof(double));
	if (!R->col || !R->val) {
		R->status = 2;
		goto out;
	}
	double bw_corrected = corrected_bandwidth(bw_scaled * nr_cols, ((double) nnz) / nr_rows / expected_cluster_size);
	long max_degree = 0;
	for (long i = 0; i < nr_rows; i++)
		if (degrees[i] > max_degree)
			max_degree = (long) degrees[i];

	int failed = 0;
	/* pass 2: column placement and values */
	#pragma omp parallel num_threads(num_threads)
	{
		struct colset os;
		os.cap = max_degree > 0 ? max_degree : 1;
		os.v = (int *) malloc(os.cap * sizeof(int));
		os.n = 0;
		#pragma omp for schedule(dynamic, 1)
		for (long sg = 0; sg < nseg; sg++) {
			struct art_rng rs;
			rng_init(&rs, (unsigned int) sg);
			long i_s = sg * period, i_e = (sg + 1) * period < nr_rows ? (sg + 1) * period : nr_rows;
			long j_s = seg_nnz[sg];
			int * col_ind = R->col;
			double * values = R->val;
			for (long i = i_s; i < i_e; i++) {
				if (i % period == 0)
					rng_reseed(&rs, seed + i);
				long degree = (long) degrees[i];
				long j_e = j_s + degree;
				long j, k;
				offsets[i] = (int) j_s;
				if (degree == 0)
					continue;
				os.n = 0;
				long range = (long) floor(bw_corrected + 0.5);
				if (range < degree)
					range = degree;
				long half_range = range / 2;
				long bound_relaxed_l, bound_relaxed_r, bound_l, bound_r;
				if (plac == 's') {
					for (j = j_s; j < j_e; j++) {
						col_ind[j] = (int) (j - j_s);
						values[j] = rng_uniform(&rs, 0, 1);
					}
					goto placed;
				} else if (plac == 'd') {
					bound_relaxed_l = i - half_range;
					bound_relaxed_r = i + half_range + range % 2;
				} else {
					bound_relaxed_l = nr_cols / 2 - half_range;
					bound_relaxed_r = nr_cols / 2 + half_range + range % 2;
				}
				bound_l = bound_relaxed_l;
				bound_r = bound_relaxed_r;
				if (bound_l < 0) {
					bound_l = 0;
					if (bound_r < degree)
						bound_r = degree;
				}
				if (bound_r > nr_cols) {
					bound_r = nr_cols;
					if (bound_l > nr_cols - degree)
						bound_l = nr_cols - degree;
				}
				j = j_s;
				if ((cross_row_similarity > 0) && (i % period != 0) && (rng_uniform(&rs, 0, 1) <= cross_row_similarity)) {
					long degree_prev = (long) degrees[i - 1];
					long degree_min = degree < degree_prev ? degree : degree_prev;
					long jp = j_s - degree_prev, jp_e = jp + degree_min;
					while (jp < jp_e) {
						k = col_ind[jp];
						if (k >= bound_r)
							k = bound_l;
						if (!colset_insert(&os, (int) k)) {
							failed = 1;   /* the reference exits here (artificial_matrix_generation.c:425-429) */
							break;
						}
						values[j] = rng_uniform(&rs, 0, 1);
						j++;
						jp++;
					}
				}
				long d1 = 0, d2 = 0;
				for (; j < j_e;) {
					long retries = 0;
					do {
						if (retries < 20) {
							k = rng_uniform_int(&rs, bound_relaxed_l, bound_relaxed_r);
							if (k >= bound_r)
								k = bound_r - 1;
							else if (k < bound_l)
								k = bound_l;
							retries++;
						} else {
							if (d1 < d2) {
								k = bound_l + d1;
								d1++;
							} else {
								k = bound_r - d2 - 1;
								d2++;
							}
						}
					} while (!colset_insert(&os, (int) k));
					values[j] = rng_uniform(&rs, 0, 1);
					j++;
					if (p_right_neigh > 0) {
						while (j < j_e) {
							if (rng_uniform(&rs, 0, 1) > p_right_neigh)
								break;
							k++;
							if (k >= bound_r)
								k = bound_l;
							if (colset_insert(&os, (int) k)) {
								values[j] = rng_uniform(&rs, 0, 1);
								j++;
							}
						}
					}
				}
				memcpy(&col_ind[j_s], os.v, degree * sizeof(int));
			placed:
				{
					double b = col_ind[j_e - 1] - col_ind[j_s] + 1;
					bw[i] = b;
					sc[i] = degree / b;
					long groups = 1;
					for (long jj = j_s + 1; jj < j_e; jj++)
						if (col_ind[jj] > col_ind[jj - 1] + 1)
							groups++;
					ngr[i] = (double) groups;
					clu[i] = (double) groups / degree;
				}
				j_s = j_e;
			}
		}
		free(os.v);
	}
	if (failed) {
		R->status = 4;
		goto out;
	}

	/* structural statistics (artificial_matrix_generation.c:529-570), serial sums */
	{
		double * st = R->stats;
		for (int q = 0; q < 37; q++)
			st[q] = NAN;
		double avg = ((double) nnz) / nr_rows;
		st[0] = avg;
		st[1] = std_of(degrees, nr_rows, avg);
		min_max_of(degrees, nr_rows, &st[2], &st[3]);
		st[4] = (st[3] - avg) / avg;
		st[5] = mean_of(bw, nr_rows);
		st[6] = std_of(bw, nr_rows, st[5]);
		min_max_of(bw, nr_rows, &st[7], &st[8]);
		st[9] = mean_of(sc, nr_rows);
		st[10] = std_of(sc, nr_rows, st[9]);
		min_max_of(sc, nr_rows, &st[11], &st[12]);
		/* neighbours within column distance 1 (matrix_util.h:235-263) */
		double nsum = 0, nsq = 0, nmin = 1e300, nmax = -1e300;
		for (long i = 0; i < nr_rows; i++)
			for (long j = offsets[i]; j < offsets[i + 1]; j++) {
				long c = 0;
				for (long q = j + 1; q < offsets[i + 1]; q++) {
					if (R->col[q] - R->col[j] > 1)
						break;
					c += 2;
				}
				nsum += c;
				nmin = c < nmin ? c : nmin;
				nmax = c > nmax ? c : nmax;
			}
		st[13] = nnz ? nsum / nnz : 0;
		for (long i = 0; i < nr_rows; i++)
			for (long j = offsets[i]; j < offsets[i + 1]; j++) {
				long c = 0;
				for (long q = j + 1; q < offsets[i + 1]; q++) {
					if (R->col[q] - R->col[j] > 1)
						break;
					c += 2;
				}
				nsq += (c - st[13]) * (c - st[13]);
			}
		st[14] = nnz ? sqrt(nsq / nnz) : 0;
		st[15] = nnz ? nmin : 0;
		st[16] = nnz ? nmax : 0;
		/* cross-row similarity with the next non-empty row (matrix_util.h:332-405) */
		double * crs = (double *) calloc(nr_rows, sizeof(double));
		long nonempty = 0;
		for (long i = 0; i < nr_rows; i++) {
			long degree = offsets[i + 1] - offsets[i];
			if (degree <= 0)
				continue;
			long l;
			for (l = i + 1; l < nr_rows; l++)
				if (offsets[l + 1] - offsets[l] > 0)
					break;
			nonempty++;
			if (l < nr_rows) {
				long ks = offsets[l], ke = offsets[l + 1], kk = ks, sim = 0;
				for (long j = offsets[i]; j < offsets[i + 1]; j++) {
					while (kk < ke) {
						long diff = R->col[kk] - R->col[j];
						if (labs(diff) <= 1) {
							sim++;
							break;
						}
						if (diff <= 0)
							kk++;
						else
							break;
					}
				}
				crs[i] = ((double) sim) / degree;
			}
		}
		{
			double s = 0;
			for (long i = 0; i < nr_rows; i++)
				s += crs[i];
			st[17] = nonempty ? s / nonempty : 0;
			double q = 0;
			for (long i = 0; i < nr_rows; i++)
				if (offsets[i + 1] > offsets[i])
					q += (crs[i] - st[17]) * (crs[i] - st[17]);
			st[18] = nonempty ? sqrt(q / nonempty) : 0;
			min_max_of(crs, nr_rows, &st[19], &st[20]);
		}
		free(crs);
		st[21] = mean_of(clu, nr_rows);
		st[22] = std_of(clu, nr_rows, st[21]);
		min_max_of(clu, nr_rows, &st[23], &st[24]);
		st[25] = mean_of(ngr, nr_rows);
		st[26] = std_of(ngr, nr_rows, st[25]);
		min_max_of(ngr, nr_rows, &st[27], &st[28]);
	}
	free(degrees); free(bw); free(sc); free(ngr); free(clu); free(seg_nnz);
	return R;
out:
	free(degrees); free(bw); free(sc); free(ngr); free(clu); free(seg_nnz);
	if (R->row_ptr != offsets)
		free(offsets);
	return R;
}

__attribute__((visibility("hidden"))) void spmv_artgen_free_result(struct artgen_result * R)
{
	if (!R)
		return;
	free(R->row_ptr);
	free(R->col);
	free(R->val);
	free(R);
}
