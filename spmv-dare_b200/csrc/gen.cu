// The reference's artificial matrix generator on the GPU
// (artificial-matrix-generator/artificial_matrix_generation.c:163-579): one thread per anchor
// segment (the reference reseeds its stream with seed + row at every anchor row, so the
// segments are independent), each running the segment's rows in order exactly as the host
// restatement (artgen.c) does -- glibc's random_r with a 256-byte state (TYPE_4: 63 words,
// separation 1, restated below), Box-Muller normals, Marsaglia-Tsang gammas, ordered-set
// column placement with cross-row copying, retries and right-neighbour clustering.
//
// The per-segment code is __host__ __device__: spmv_gen_host_check runs it on the host
// against the bit-exact host generator.  On the GPU the same steps call CUDA's log, cos,
// exp, pow and sqrt, whose last bits may differ from glibc's, so a degree that rounds at
// exactly .5 or a rejection test on its boundary can go the other way: the GPU matrices
// follow the reference's distribution, nearly always entry for entry (the GPU tests
// measure how nearly).
#include <math.h>
#include <string.h>

#include <vector>

#include "internal.h"
#include "primitives.cuh"

#define HD __host__ __device__ __forceinline__

namespace spmv {

namespace {

constexpr int RNG_DEG = 63;   // glibc random_r TYPE_4 (a 256-byte state)
constexpr double RNG_DBL_EPS = 2.220446049250313080847e-16;
constexpr double RNG_PI = 3.14159265358979323846;

struct Rng {
	int32_t st[RNG_DEG];
	int f, r;
};

// glibc srandom_r for TYPE_4: state[i] = 16807 * state[i-1] mod (2^31 - 1) by Schrage's
// method, front pointer at state[1], rear at state[0], then 630 outputs discarded.
HD int32_t rng_next(Rng & g)
{
	const uint32_t val = (uint32_t) g.st[g.f] + (uint32_t) g.st[g.r];
	g.st[g.f] = (int32_t) val;
	if (++g.f >= RNG_DEG) {
		g.f = 0;
		++g.r;
	} else if (++g.r >= RNG_DEG) {
		g.r = 0;
	}
	return (int32_t) (val >> 1);
}

HD void rng_seed(Rng & g, unsigned int seed)
{
	if (seed == 0)
		seed = 1;
	g.st[0] = (int32_t) seed;
	int32_t word = (int32_t) seed;
	for (int i = 1; i < RNG_DEG; i++) {
		const long long hi = word / 127773, lo = word % 127773;
		long long w = 16807 * lo - 2836 * hi;
		if (w < 0)
			w += 2147483647;
		word = (int32_t) w;
		g.st[i] = word;
	}
	g.f = 1;
	g.r = 0;
	for (int k = 0; k < RNG_DEG * 10; k++)
		(void) rng_next(g);
}

HD double rng_uniform(Rng & g, double lo, double hi)
{
	const double res = (double) rng_next(g) / (double) (0x7FFFFFFFLL + 1LL);
	return (hi - lo) * res + lo;
}

HD long long rng_uniform_int(Rng & g, long long lo, long long hi)
{
	const long long range = hi - lo;
	if (range >= 0x7FFFFFFFLL) {
		const long long max64 = 0x3FFFFFFFFFFFFFFFLL;
		const long long lim = max64 - max64 % range;
		long long res;
		do {
			res = (long long) rng_next(g) << 31;
			res |= (long long) rng_next(g);
		} while (res >= lim);
		return res % range + lo;
	}
	const long long lim = 0x7FFFFFFFLL - 0x7FFFFFFFLL % range;
	long long v;
	do {
		v = rng_next(g);
	} while (v >= lim);
	return v % range + lo;
}

HD double rng_normal(Rng & g, double mean, double std)
{
	const double u1 = rng_uniform(g, 2 * RNG_DBL_EPS, 1);
	const double u2 = rng_uniform(g, 0, 1);
	const double magnitude = std * sqrt(-2.0 * log(u1));
	return magnitude * cos(2.0 * RNG_PI * u2) + mean;
}

// Marsaglia-Tsang for k >= 1; below 1 the k + 1 draw scaled by u^(1/k) (u drawn first)
HD double rng_gamma(Rng & g, double k, double theta)
{
	double scale = 1.0;
	if (k < 1) {
		const double u = rng_uniform(g, 2 * RNG_DBL_EPS, 1);
		scale = pow(u, 1.0 / k);
		k = 1.0 + k;
	}
	double x, v, u;
	const double d = k - 1.0 / 3.0;
	const double c = (1.0 / 3.0) / sqrt(d);
	while (true) {
		do {
			x = rng_normal(g, 0, 1);
			v = 1.0 + c * x;
		} while (v <= 0);
		v = v * v * v;
		u = rng_uniform(g, 2 * RNG_DBL_EPS, 1);
		if (u < 1 - 0.0331 * x * x * x * x)
			break;
		if (log(u) < 0.5 * x * x + d * (1 - v + log(v)))
			break;
	}
	return theta * d * v * scale;
}

struct GenParams {
	long long rows, cols;
	double MAX, C, avg_distr, std_distr;
	char dist, plac;
	double p_right, bw_corrected, cross;
	unsigned int seed;
	long long period, nseg;
};

// Degrees of segment sg (pass 1 of the generator), their sum.
HD long long seg_degrees(const GenParams & P, long long sg, int32_t * degrees)
{
	Rng g;
	const long long i_s = sg * P.period, i_e = (sg + 1) * P.period < P.rows ? (sg + 1) * P.period : P.rows;
	long long sum = 0;
	for (long long i = i_s; i < i_e; i++) {
		if (i % P.period == 0)
			rng_seed(g, P.seed + (unsigned int) i);
		const double degree_exp = P.MAX * exp(-P.C / P.rows * (double) i);
		double degree_distr;
		if (P.std_distr > 0) {
			if (P.dist == 'n') {
				degree_distr = rng_normal(g, P.avg_distr, P.std_distr);
			} else {
				const double k = (P.avg_distr * P.avg_distr) / (P.std_distr * P.std_distr);
				const double theta = (P.avg_distr > 0) ? (P.std_distr * P.std_distr) / P.avg_distr : 1;
				degree_distr = rng_gamma(g, k, theta);
			}
		} else {
			degree_distr = P.avg_distr;
		}
		double degree = degree_exp + degree_distr;
		degree = (degree > 0) ? floor(degree + 0.5) : 0;
		if (degree > P.cols)
			degree = (double) P.cols;
		degrees[i] = (int32_t) degree;
		sum += (long long) degree;
	}
	return sum;
}

// sorted insert into set[0..n); returns false if k is present
HD bool set_insert(int32_t * set, long long & n, int32_t k)
{
	long long lo = 0, hi = n;
	while (lo < hi) {
		const long long mid = (lo + hi) >> 1;
		if (set[mid] < k)
			lo = mid + 1;
		else
			hi = mid;
	}
	if (lo < n && set[lo] == k)
		return false;
	for (long long q = n; q > lo; q--)
		set[q] = set[q - 1];
	set[lo] = k;
	n++;
	return true;
}

// Columns and values of segment sg (pass 2); returns false where the reference stops
// (a copied column already present).
HD bool seg_place(const GenParams & P, long long sg, const int32_t * degrees, long long j0, int32_t * set,
		int32_t * row_ptr, int32_t * col, double * val)
{
	Rng g;
	const long long i_s = sg * P.period, i_e = (sg + 1) * P.period < P.rows ? (sg + 1) * P.period : P.rows;
	long long j_s = j0;
	for (long long i = i_s; i < i_e; i++) {
		if (i % P.period == 0)
			rng_seed(g, P.seed + (unsigned int) i);
		const long long degree = degrees[i];
		const long long j_e = j_s + degree;
		row_ptr[i] = (int32_t) j_s;
		if (degree == 0)
			continue;
		long long ns = 0;
		long long range = (long long) floor(P.bw_corrected + 0.5);
		if (range < degree)
			range = degree;
		const long long half = range / 2;
		long long brl, brr, bl, br, j, k;
		if (P.plac == 's') {
			for (j = j_s; j < j_e; j++) {
				col[j] = (int32_t) (j - j_s);
				val[j] = rng_uniform(g, 0, 1);
			}
			j_s = j_e;
			continue;
		} else if (P.plac == 'd') {
			brl = i - half;
			brr = i + half + range % 2;
		} else {
			brl = P.cols / 2 - half;
			brr = P.cols / 2 + half + range % 2;
		}
		bl = brl;
		br = brr;
		if (bl < 0) {
			bl = 0;
			if (br < degree)
				br = degree;
		}
		if (br > P.cols) {
			br = P.cols;
			if (bl > P.cols - degree)
				bl = P.cols - degree;
		}
		j = j_s;
		if ((P.cross > 0) && (i % P.period != 0) && (rng_uniform(g, 0, 1) <= P.cross)) {
			const long long dprev = degrees[i - 1];
			const long long dmin = degree < dprev ? degree : dprev;
			long long jp = j_s - dprev;
			const long long jp_e = jp + dmin;
			while (jp < jp_e) {
				k = col[jp];
				if (k >= br)
					k = bl;
				if (!set_insert(set, ns, (int32_t) k))
					return false;
				val[j] = rng_uniform(g, 0, 1);
				j++;
				jp++;
			}
		}
		long long d1 = 0, d2 = 0;
		while (j < j_e) {
			long long retries = 0;
			do {
				if (retries < 20) {
					k = rng_uniform_int(g, brl, brr);
					if (k >= br)
						k = br - 1;
					else if (k < bl)
						k = bl;
					retries++;
				} else if (d1 < d2) {
					k = bl + d1;
					d1++;
				} else {
					k = br - d2 - 1;
					d2++;
				}
			} while (!set_insert(set, ns, (int32_t) k));
			val[j] = rng_uniform(g, 0, 1);
			j++;
			if (P.p_right > 0) {
				while (j < j_e) {
					if (rng_uniform(g, 0, 1) > P.p_right)
						break;
					k++;
					if (k >= br)
						k = bl;
					if (set_insert(set, ns, (int32_t) k)) {
						val[j] = rng_uniform(g, 0, 1);
						j++;
					}
				}
			}
		}
		for (long long q = 0; q < degree; q++)
			col[j_s + q] = set[q];
		j_s = j_e;
	}
	return true;
}

__global__ void gen_degrees_kernel(GenParams P, int32_t * degrees, long long * seg_sum)
{
	const long long sg = (long long) blockIdx.x * blockDim.x + threadIdx.x;
	if (sg < P.nseg)
		seg_sum[sg] = seg_degrees(P, sg, degrees);
}

__global__ void gen_place_kernel(GenParams P, const int32_t * degrees, const long long * seg_off, int32_t * sets,
		long long set_cap, int32_t * row_ptr, int32_t * col, double * val, int * err)
{
	const long long sg = (long long) blockIdx.x * blockDim.x + threadIdx.x;
	if (sg >= P.nseg)
		return;
	if (!seg_place(P, sg, degrees, seg_off[sg], sets + sg * set_cap, row_ptr, col, val))
		atomicCAS(err, 0, 1);
}

__global__ void gen_max_kernel(const int32_t * d, long long n, int * out)
{
	const long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		atomicMax(out, d[i]);
}

// bandwidth correction (artificial_matrix_generation.c:64-147), on the host
double expected_bandwidth(double B, double n)
{
	double E, a, b, b_e, x;
	long i;
	b_e = 0;
	for (i = 0; i < (long) n; i++)
		b_e += log2(n - i) - log2(B - i);
	b = pow(2, b_e);
	E = 0;
	for (i = (long) n; i <= (long) B; i++) {
		x = (double) i;
		a = (B - x + 1) * n / x * (n - 1) / (x - 1);
		E += a * b * (double) i;
		b_e += log2(x + 1) - log2(x + 1 - n);
		b = pow(2, b_e);
	}
	return E;
}

double corrected_bandwidth(double B, double n)
{
	n = floor(n + 0.5);
	if (n < 2)
		n = 2;
	const double E = expected_bandwidth(B, n);
	if (E == 0)
		return n;
	return B * (B / E);
}

int gen_params(long long rows, long long cols, double avg, double std, const char * distribution, const char * placement,
		double bw_scaled, double skew, double neigh, double cross, unsigned int seed, GenParams & P)
{
	if (rows < 1 || cols < 1 || !distribution || !placement || rows > INT32_MAX - 1 || cols > INT32_MAX) {
		set_error(SPMV_ERR_ARG, "generator: bad sizes or parameters");
		return SPMV_ERR_ARG;
	}
	memset(&P, 0, sizeof(P));
	P.rows = rows;
	P.cols = cols;
	P.dist = distribution[0];
	P.plac = placement[0];
	P.seed = seed;
	P.p_right = neigh / 2;
	P.cross = cross;
	if (bw_scaled > 1)
		bw_scaled = 1;
	double MAX = avg * (1 + skew);
	const double cb1 = MAX / avg;
	const double cb2 = (std > 0) ? MAX * MAX / (2 * std * std) : 0;
	double C = cb1 > cb2 ? cb1 : cb2;
	double avg_distr, std_distr;
	if (C <= 2 || skew < 1) {
		MAX = 0;
		C = 0;
		avg_distr = avg;
		std_distr = std;
	} else {
		const double avg_exp = MAX / C;
		const double std_exp = sqrt(avg_exp * avg_exp * (C / 2 - 1));
		avg_distr = avg - MAX / C;
		std_distr = sqrt(std * std - std_exp * std_exp);
		if (P.dist == 'n' && std_distr > avg_distr / 3)
			std_distr = avg_distr / 3;
	}
	P.MAX = MAX;
	P.C = C;
	P.avg_distr = avg_distr;
	P.std_distr = std_distr;
	long long anchors = rows / 100;
	if (anchors < 1)
		anchors = 1;
	else if (anchors > 1 << 12)
		anchors = 1 << 12;
	P.period = rows / anchors;
	P.nseg = (rows + P.period - 1) / P.period;
	P.bw_corrected = 0;      // set once nnz is known
	(void) bw_scaled;
	return SPMV_OK;
}

}  // namespace

}  // namespace spmv

struct spmv_gen {
	int64_t m = 0, n = 0, nnz = 0;
	spmv::DevBuf rp, ci, v;
};

extern "C" {

spmv_gen * spmv_gen_create_device(int64_t rows, int64_t cols, double avg_nnz_per_row, double std_nnz_per_row,
		const char * distribution, const char * placement, double bw, double skew, double avg_num_neighbours,
		double cross_row_similarity, uint32_t seed, void * stream, int * status)
{
	spmv::clear_error();
	spmv::GenParams P;
	int st = spmv::gen_params(rows, cols, avg_nnz_per_row, std_nnz_per_row, distribution, placement, bw, skew,
			avg_num_neighbours, cross_row_similarity, seed, P);
	spmv_gen * G = nullptr;
	if (st == SPMV_OK) {
		G = new spmv_gen();
		cudaStream_t s = (cudaStream_t) stream;
		auto body = [&]() -> int {
			spmv::DevBuf deg, sums, offs, mx, err, sets;
			SPMV_TRY(deg.alloc(rows * sizeof(int32_t), s));
			SPMV_TRY(sums.alloc(P.nseg * sizeof(long long), s));
			SPMV_TRY(offs.alloc((P.nseg + 1) * sizeof(int64_t), s));
			SPMV_TRY(mx.alloc(sizeof(int), s));
			SPMV_TRY(err.alloc(sizeof(int), s));
			SPMV_CUDA_TRY(cudaMemsetAsync(mx.p, 0, sizeof(int), s));
			SPMV_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(int), s));
			const unsigned gs = (unsigned) spmv::ceil_div(P.nseg, 64);
			spmv::gen_degrees_kernel<<<gs, 64, 0, s>>>(P, deg.as<int32_t>(), sums.as<long long>());
			SPMV_CUDA_TRY(cudaGetLastError());
			SPMV_TRY(spmv::scan_exclusive(sums.as<int64_t>(), offs.as<int64_t>(), P.nseg, s));
			spmv::gen_max_kernel<<<(unsigned) spmv::ceil_div(rows, 256), 256, 0, s>>>(deg.as<int32_t>(), rows, mx.as<int>());
			SPMV_CUDA_TRY(cudaGetLastError());
			int64_t nnz = 0;
			int maxdeg = 0;
			SPMV_CUDA_TRY(cudaMemcpyAsync(&nnz, offs.as<int64_t>() + P.nseg, 8, cudaMemcpyDeviceToHost, s));
			SPMV_CUDA_TRY(cudaMemcpyAsync(&maxdeg, mx.p, 4, cudaMemcpyDeviceToHost, s));
			SPMV_CUDA_TRY(cudaStreamSynchronize(s));
			if (nnz > 0x7FFFFFFF - 64) {
				spmv::set_error(SPMV_ERR_OVERFLOW, "generator: %lld entries beyond the 32-bit range", (long long) nnz);
				return SPMV_ERR_OVERFLOW;
			}
			const double expected_cluster = 1 / (1 - P.p_right);
			P.bw_corrected = spmv::corrected_bandwidth((bw > 1 ? 1 : bw) * (double) cols,
					((double) nnz) / rows / expected_cluster);
			G->m = rows;
			G->n = cols;
			G->nnz = nnz;
			SPMV_TRY(G->rp.alloc((rows + 1) * sizeof(int32_t), s));
			SPMV_TRY(G->ci.alloc((nnz > 0 ? nnz : 1) * sizeof(int32_t), s));
			SPMV_TRY(G->v.alloc((nnz > 0 ? nnz : 1) * sizeof(double), s));
			const long long cap = maxdeg > 0 ? maxdeg : 1;
			if ((double) P.nseg * (double) cap * 4.0 > 8.0e9) {
				// one ordered set of the longest row per segment
				spmv::set_error(SPMV_ERR_ARG, "generator: %lld segments x rows of %lld entries need too much scratch",
						(long long) P.nseg, cap);
				return SPMV_ERR_ARG;
			}
			SPMV_TRY(sets.alloc((size_t) P.nseg * cap * sizeof(int32_t), s));
			spmv::gen_place_kernel<<<gs, 64, 0, s>>>(P, deg.as<int32_t>(), offs.as<long long>(), sets.as<int32_t>(), cap,
					G->rp.as<int32_t>(), G->ci.as<int32_t>(), G->v.as<double>(), err.as<int>());
			SPMV_CUDA_TRY(cudaGetLastError());
			const int32_t last = (int32_t) nnz;
			SPMV_CUDA_TRY(cudaMemcpyAsync(G->rp.as<int32_t>() + rows, &last, 4, cudaMemcpyHostToDevice, s));
			int bad = 0;
			SPMV_CUDA_TRY(cudaMemcpyAsync(&bad, err.p, 4, cudaMemcpyDeviceToHost, s));
			SPMV_CUDA_TRY(cudaStreamSynchronize(s));
			if (bad) {
				spmv::set_error(SPMV_ERR_ARG, "generator: a copied column was already in its row (the reference stops here)");
				return SPMV_ERR_ARG;
			}
			return SPMV_OK;
		};
		st = body();
		if (st != SPMV_OK) {
			delete G;
			G = nullptr;
		}
	}
	if (status)
		*status = st;
	return G;
}

int spmv_gen_info(const spmv_gen * G, int64_t * m, int64_t * n, int64_t * nnz)
{
	spmv::clear_error();
	if (!G) {
		spmv::set_error(SPMV_ERR_ARG, "null generator result");
		return SPMV_ERR_ARG;
	}
	if (m) *m = G->m;
	if (n) *n = G->n;
	if (nnz) *nnz = G->nnz;
	return SPMV_OK;
}

int spmv_gen_copy_device(const spmv_gen * G, int32_t * d_row_ptr, int32_t * d_col_ind, double * d_values, void * stream)
{
	spmv::clear_error();
	if (!G) {
		spmv::set_error(SPMV_ERR_ARG, "null generator result");
		return SPMV_ERR_ARG;
	}
	cudaStream_t s = (cudaStream_t) stream;
	if (d_row_ptr)
		SPMV_CUDA_TRY(cudaMemcpyAsync(d_row_ptr, G->rp.p, (G->m + 1) * 4, cudaMemcpyDeviceToDevice, s));
	if (d_col_ind && G->nnz)
		SPMV_CUDA_TRY(cudaMemcpyAsync(d_col_ind, G->ci.p, G->nnz * 4, cudaMemcpyDeviceToDevice, s));
	if (d_values && G->nnz)
		SPMV_CUDA_TRY(cudaMemcpyAsync(d_values, G->v.p, G->nnz * 8, cudaMemcpyDeviceToDevice, s));
	return SPMV_OK;
}

void spmv_gen_destroy(spmv_gen * G)
{
	delete G;
}

// Runs the generator's per-segment steps (the code the GPU kernels run) on the host, with
// the host's libm, into host arrays (row_ptr[rows+1], col/val of at most cap entries);
// returns nnz, or -1 on error.  A check of the GPU generator's code against the
// bit-exact host generator that needs no GPU.
int64_t spmv_gen_host_check(int64_t rows, int64_t cols, double avg, double std, const char * distribution,
		const char * placement, double bw, double skew, double neigh, double cross, uint32_t seed, int32_t * row_ptr,
		int32_t * col_ind, double * values, int64_t cap)
{
	spmv::clear_error();
	spmv::GenParams P;
	if (spmv::gen_params(rows, cols, avg, std, distribution, placement, bw, skew, neigh, cross, seed, P) != SPMV_OK)
		return -1;
	std::vector<int32_t> deg((size_t) rows);
	std::vector<long long> off((size_t) P.nseg + 1, 0);
	int maxdeg = 0;
	for (long long sg = 0; sg < P.nseg; sg++)
		off[(size_t) sg + 1] = off[(size_t) sg] + spmv::seg_degrees(P, sg, deg.data());
	for (int32_t d : deg)
		maxdeg = d > maxdeg ? d : maxdeg;
	const long long nnz = off[(size_t) P.nseg];
	if (nnz > cap) {
		spmv::set_error(SPMV_ERR_ARG, "generator check: %lld entries exceed the %lld given", nnz, (long long) cap);
		return -1;
	}
	P.bw_corrected = spmv::corrected_bandwidth((bw > 1 ? 1 : bw) * (double) cols,
			((double) nnz) / rows / (1 / (1 - P.p_right)));
	std::vector<int32_t> set((size_t) (maxdeg > 0 ? maxdeg : 1));
	for (long long sg = 0; sg < P.nseg; sg++)
		if (!spmv::seg_place(P, sg, deg.data(), off[(size_t) sg], set.data(), row_ptr, col_ind, values)) {
			spmv::set_error(SPMV_ERR_ARG, "generator: a copied column was already in its row");
			return -1;
		}
	row_ptr[rows] = (int32_t) nnz;
	return nnz;
}

}  // extern "C"
