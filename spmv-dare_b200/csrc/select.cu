// Learned format / tuning selector: GPU structural features of a CSR matrix and a small
// FP32 MLP (input -> h1 -> h2 -> classes, ReLU hidden layers) with hand-written forward,
// backward, softmax cross-entropy and Adam kernels.
//
// Features (after the generator's own statistics, artificial-matrix-generator/
// artificial_matrix_generation.c:529-570 and matrix_util.h:206-300, window 1):
//   0 log2(m + 1)                 1 log2(nnz + 1)
//   2 avg_nnz_per_row             3 std_nnz_per_row / avg (0 when avg = 0)
//   4 skew = (max - avg) / avg    5 avg_bw_scaled: mean over rows of (last - first + 1) / n
//                                   (0 for empty rows, as bandwidths[i] = 0 there)
//   6 avg scatter: mean over rows of degree / bandwidth
//   7 avg_num_neighbours: per entry, 2 x the entries of its row within +1 column after it
//     (csr_num_neighbours), averaged over nnz
//   8 cross-row similarity: per non-empty row, the share of its entries with an entry of
//     the next non-empty row within +-1 column, averaged over non-empty rows
//     (csr_cross_row_similarity)
//   9 avg clustering: mean over rows of groups of consecutive columns / degree
// All sums run in FP64 with atomics (order-independent up to FP64 rounding).
#include <mutex>

#include "internal.h"
#include "primitives.cuh"

namespace spmv {

namespace {

constexpr int FEAT_THREADS = 256;
enum { F_DEG = 0, F_DEG2, F_BW, F_SC, F_NEIGH, F_CRS, F_NONEMPTY, F_CLUST, F_NSUMS };

__device__ __forceinline__ double block_sum(double v, double * red)
{
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		v += __shfl_down_sync(0xffffffffu, v, o);
	__syncthreads();
	if ((threadIdx.x & 31) == 0)
		red[threadIdx.x >> 5] = v;
	__syncthreads();
	double t = 0.0;
	if (threadIdx.x == 0)
		for (int w = 0; w < (int) (blockDim.x >> 5); w++)
			t += red[w];
	return t;
}

// Last non-empty row before row i (-1 if none), found by the whole warp 32 rows at a time.
__device__ __forceinline__ int64_t prev_nonempty(const int32_t * rp, int64_t i, int lane)
{
	for (int64_t base = i - 1; base >= 0; base -= 32) {
		const int64_t r = base - lane;
		const bool ne = r >= 0 && rp[r + 1] > rp[r];
		const unsigned mask = __ballot_sync(0xffffffffu, ne);
		if (mask)
			return base - (__ffs(mask) - 1);       // the lowest lane is the nearest row
	}
	return -1;
}

// Per-row statistics, one warp per row (lanes split a row's entries, so long rows do not
// serialise).
__global__ void __launch_bounds__(FEAT_THREADS) features_kernel(const int32_t * rp, const int32_t * ci, int64_t m, int64_t n,
		double * sums, unsigned long long * maxdeg)
{
	__shared__ double red[FEAT_THREADS / 32];
	const int lane = threadIdx.x & 31;
	double acc[F_NSUMS];
	#pragma unroll
	for (int k = 0; k < F_NSUMS; k++)
		acc[k] = 0.0;
	long long mx = 0;
	const int64_t warps = (int64_t) gridDim.x * (blockDim.x >> 5);
	for (int64_t i = (int64_t) blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < m; i += warps) {
		const int64_t js = rp[i], je = rp[i + 1];
		const int64_t deg = je - js;
		if (deg <= 0)
			continue;
		// consecutive pairs (a neighbour within +1 column) and group starts of this row
		int64_t consecutive = 0, newgroups = 0;
		for (int64_t j = js + 1 + lane; j < je; j += 32) {
			const int32_t d = ci[j] - ci[j - 1];
			consecutive += d <= 1 ? 1 : 0;
			newgroups += d > 1 ? 1 : 0;
		}
		// this row is the next non-empty row of row p: entries of p with an entry here within +-1
		const int64_t p = prev_nonempty(rp, i, lane);
		int64_t sim = 0, ps = 0, pe = 0;
		if (p >= 0) {
			ps = rp[p];
			pe = rp[p + 1];
			for (int64_t j = ps + lane; j < pe; j += 32) {
				const int64_t c = ci[j];
				int64_t lo = js, hi = je;          // first entry of row i with column >= c - 1
				while (lo < hi) {
					const int64_t mid = (lo + hi) >> 1;
					if ((int64_t) ci[mid] < c - 1)
						lo = mid + 1;
					else
						hi = mid;
				}
				sim += (lo < je && (int64_t) ci[lo] <= c + 1) ? 1 : 0;
			}
		}
		#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			consecutive += __shfl_down_sync(0xffffffffu, consecutive, o);
			newgroups += __shfl_down_sync(0xffffffffu, newgroups, o);
			sim += __shfl_down_sync(0xffffffffu, sim, o);
		}
		if (lane == 0) {
			acc[F_DEG] += (double) deg;
			acc[F_DEG2] += (double) deg * (double) deg;
			mx = deg > mx ? deg : mx;
			acc[F_NONEMPTY] += 1.0;
			const double bw = (double) ci[je - 1] - (double) ci[js] + 1.0;
			acc[F_BW] += bw / (double) n;
			acc[F_SC] += (double) deg / bw;
			acc[F_NEIGH] += 2.0 * (double) consecutive;
			acc[F_CLUST] += (double) (1 + newgroups) / (double) deg;
			if (p >= 0)
				acc[F_CRS] += (double) sim / (double) (pe - ps);
		}
	}
	for (int k = 0; k < F_NSUMS; k++) {
		const double t = block_sum(acc[k], red);
		if (threadIdx.x == 0 && t != 0.0)
			atomicAdd(&sums[k], t);
	}
	atomicMax(maxdeg, (unsigned long long) mx);
}

// ------------------------------------------------------------------ MLP kernels
// Layer: Z[b, o] = sum_i W[o, i] X[b, i] + bias[o]; A = relu(Z) (hidden) or Z (output).
__global__ void dense_forward_kernel(const float * W, const float * bias, const float * X, int B, int in, int out,
		int relu, float * Z, float * A)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= B * out)
		return;
	const int b = idx / out, o = idx % out;
	const float * w = W + (size_t) o * in;
	const float * x = X + (size_t) b * in;
	float z = bias[o];
	for (int i = 0; i < in; i++)
		z = fmaf(w[i], x[i], z);
	if (Z)
		Z[idx] = z;
	A[idx] = relu ? fmaxf(z, 0.0f) : z;
}

// Softmax cross-entropy of logits [B, C] against integer labels: per-sample loss and
// dlogits = (softmax - onehot) / B.
__global__ void softmax_ce_kernel(const float * logits, const int32_t * labels, int B, int C, float * loss, float * dlogits)
{
	const int b = blockIdx.x * blockDim.x + threadIdx.x;
	if (b >= B)
		return;
	const float * z = logits + (size_t) b * C;
	float mx = z[0];
	for (int c = 1; c < C; c++)
		mx = fmaxf(mx, z[c]);
	float se = 0.0f;
	for (int c = 0; c < C; c++)
		se += expf(z[c] - mx);
	const float lse = mx + logf(se);
	const int y = labels[b];
	loss[b] = lse - z[y];
	for (int c = 0; c < C; c++)
		dlogits[(size_t) b * C + c] = (expf(z[c] - lse) - (c == y ? 1.0f : 0.0f)) / (float) B;
}

// dZ = dA * relu'(Z), in place on dA.
__global__ void relu_backward_kernel(float * dA, const float * Z, int count)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < count && Z[i] <= 0.0f)
		dA[i] = 0.0f;
}

// dW[o, i] = sum_b dZ[b, o] X[b, i]; db[o] = sum_b dZ[b, o] (fixed order over b).
__global__ void dense_wgrad_kernel(const float * dZ, const float * X, int B, int in, int out, float * dW, float * db)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx < out * in) {
		const int o = idx / in, i = idx % in;
		float g = 0.0f;
		for (int b = 0; b < B; b++)
			g = fmaf(dZ[(size_t) b * out + o], X[(size_t) b * in + i], g);
		dW[idx] = g;
	}
	if (idx < out) {
		float g = 0.0f;
		for (int b = 0; b < B; b++)
			g += dZ[(size_t) b * out + idx];
		db[idx] = g;
	}
}

// dX[b, i] = sum_o W[o, i] dZ[b, o].
__global__ void dense_xgrad_kernel(const float * W, const float * dZ, int B, int in, int out, float * dX)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= B * in)
		return;
	const int b = idx / in, i = idx % in;
	float g = 0.0f;
	for (int o = 0; o < out; o++)
		g = fmaf(W[(size_t) o * in + i], dZ[(size_t) b * out + o], g);
	dX[idx] = g;
}

// Mean of per-sample losses, one block of 256 threads, fixed order.
__global__ void mean_kernel(const float * v, int n, float * out)
{
	__shared__ float red[256];
	float s = 0.0f;
	for (int i = threadIdx.x; i < n; i += blockDim.x)
		s += v[i];
	red[threadIdx.x] = s;
	__syncthreads();
	for (int w = blockDim.x / 2; w > 0; w >>= 1) {
		if ((int) threadIdx.x < w)
			red[threadIdx.x] += red[threadIdx.x + w];
		__syncthreads();
	}
	if (threadIdx.x == 0)
		*out = red[0] / (float) (n > 0 ? n : 1);
}

// Adam (Kingma & Ba 2015) with bias correction and decoupled weight decay (AdamW).
__global__ void adam_kernel(float * p, const float * g, float * m1, float * m2, int count, float lr, float b1, float b2,
		float eps, float wd, float c1, float c2)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= count)
		return;
	const float gi = g[i];
	const float a = b1 * m1[i] + (1.0f - b1) * gi;
	const float v = b2 * m2[i] + (1.0f - b2) * gi * gi;
	m1[i] = a;
	m2[i] = v;
	const float mh = a / c1, vh = v / c2;
	p[i] -= lr * (mh / (sqrtf(vh) + eps) + wd * p[i]);
}

inline unsigned blocks_for(int64_t n, int t)
{
	return (unsigned) ((n + t - 1) / t);
}

}  // namespace

int features_device(const int32_t * d_rp, const int32_t * d_ci, int64_t m, int64_t n, int64_t nnz, double * out,
		cudaStream_t s)
{
	// one persistent scratch per device (the sums, then the maximum degree), so a query makes
	// no allocation: an allocation per call costs more than the whole computation
	static std::mutex mtx;
	static void * scratch[64] = {};
	constexpr size_t SCRATCH = F_NSUMS * sizeof(double) + sizeof(unsigned long long);
	int dev = 0;
	SPMV_CUDA_TRY(cudaGetDevice(&dev));
	if (dev < 0 || dev >= 64) {
		set_error(SPMV_ERR_ARG, "device index %d out of range", dev);
		return SPMV_ERR_ARG;
	}
	std::lock_guard<std::mutex> lock(mtx);
	if (!scratch[dev])
		SPMV_CUDA_TRY(cudaMalloc(&scratch[dev], SCRATCH));
	double * sums = static_cast<double *>(scratch[dev]);
	unsigned long long * mx = reinterpret_cast<unsigned long long *>(sums + F_NSUMS);
	SPMV_CUDA_TRY(cudaMemsetAsync(scratch[dev], 0, SCRATCH, s));
	if (m > 0) {
		int64_t grid = blocks_for(m, FEAT_THREADS / 32);     // a warp per row
		if (grid > 2048)
			grid = 2048;
		features_kernel<<<(unsigned) grid, FEAT_THREADS, 0, s>>>(d_rp, d_ci, m, n, sums, mx);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	struct {
		double h[F_NSUMS];
		unsigned long long hmx;
	} r;
	static_assert(sizeof(r) == SCRATCH, "scratch layout");
	SPMV_CUDA_TRY(cudaMemcpyAsync(&r, scratch[dev], SCRATCH, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	const double * h = r.h;
	const unsigned long long hmx = r.hmx;
	const double md = m > 0 ? (double) m : 1.0;
	const double avg = h[F_DEG] / md;
	const double var = h[F_DEG2] / md - avg * avg;
	out[0] = log2((double) m + 1.0);
	out[1] = log2((double) nnz + 1.0);
	out[2] = avg;
	out[3] = avg > 0 ? sqrt(var > 0 ? var : 0.0) / avg : 0.0;
	out[4] = avg > 0 ? ((double) hmx - avg) / avg : 0.0;
	out[5] = h[F_BW] / md;
	out[6] = h[F_SC] / md;
	out[7] = nnz > 0 ? h[F_NEIGH] / (double) nnz : 0.0;
	out[8] = h[F_NONEMPTY] > 0 ? h[F_CRS] / h[F_NONEMPTY] : 0.0;
	out[9] = h[F_CLUST] / md;
	return SPMV_OK;
}

// ------------------------------------------------------------------ MLP state
struct Mlp {
	int dims[4];                  // in, h1, h2, out
	int nparam = 0;
	float * p = nullptr;          // W1 b1 W2 b2 W3 b3, contiguous
	float * g = nullptr;
	float * m1 = nullptr;
	float * m2 = nullptr;
	int64_t step = 0;
	// activations of the last forward (batch capacity `cap`)
	int cap = 0;
	float *z1 = nullptr, *a1 = nullptr, *d1 = nullptr, *z2 = nullptr, *a2 = nullptr, *d2 = nullptr, *z3 = nullptr,
	      *d3 = nullptr, *loss = nullptr;
	float * lmean = nullptr;

	int off(int layer, bool bias) const
	{
		int o = 0;
		for (int l = 0; l < layer; l++)
			o += dims[l + 1] * dims[l] + dims[l + 1];
		return o + (bias ? dims[layer + 1] * dims[layer] : 0);
	}
	void free_acts()
	{
		for (float * q : {z1, a1, d1, z2, a2, d2, z3, d3, loss})
			if (q)
				cudaFree(q);
		z1 = a1 = d1 = z2 = a2 = d2 = z3 = d3 = loss = nullptr;
		cap = 0;
	}
	~Mlp()
	{
		free_acts();
		for (float * q : {p, g, m1, m2, lmean})
			if (q)
				cudaFree(q);
	}
	int ensure(int B)
	{
		if (B <= cap)
			return SPMV_OK;
		free_acts();
		const size_t h1 = (size_t) B * dims[1], h2 = (size_t) B * dims[2], o = (size_t) B * dims[3];
		float ** bufs[] = {&z1, &a1, &d1, &z2, &a2, &d2, &z3, &d3, &loss};
		const size_t sizes[] = {h1, h1, h1, h2, h2, h2, o, o, (size_t) B};
		for (int k = 0; k < 9; k++) {
			cudaError_t e = cudaMalloc((void **) bufs[k], sizes[k] * sizeof(float));
			if (e != cudaSuccess) {
				set_error(SPMV_ERR_NOMEM, "MLP activations: %s", cudaGetErrorString(e));
				return SPMV_ERR_NOMEM;
			}
		}
		cap = B;
		return SPMV_OK;
	}
	// keep: store the logits in z3 for a following backward (and copy them to `logits`
	// when given); otherwise write them to `logits` directly.
	int forward(const float * X, int B, float * logits, cudaStream_t s, bool keep)
	{
		SPMV_TRY(ensure(B));
		const int t = 128;
		dense_forward_kernel<<<blocks_for((int64_t) B * dims[1], t), t, 0, s>>>(p + off(0, false), p + off(0, true), X, B,
				dims[0], dims[1], 1, z1, a1);
		dense_forward_kernel<<<blocks_for((int64_t) B * dims[2], t), t, 0, s>>>(p + off(1, false), p + off(1, true), a1, B,
				dims[1], dims[2], 1, z2, a2);
		dense_forward_kernel<<<blocks_for((int64_t) B * dims[3], t), t, 0, s>>>(p + off(2, false), p + off(2, true), a2, B,
				dims[2], dims[3], 0, nullptr, keep ? z3 : logits);
		SPMV_CUDA_TRY(cudaGetLastError());
		if (keep && logits)
			SPMV_CUDA_TRY(cudaMemcpyAsync(logits, z3, (size_t) B * dims[3] * sizeof(float), cudaMemcpyDeviceToDevice, s));
		return SPMV_OK;
	}
	int backward(const float * X, const int32_t * labels, int B, cudaStream_t s)
	{
		const int t = 128;
		softmax_ce_kernel<<<blocks_for(B, t), t, 0, s>>>(z3, labels, B, dims[3], loss, d3);
		mean_kernel<<<1, 256, 0, s>>>(loss, B, lmean);
		dense_wgrad_kernel<<<blocks_for((int64_t) dims[3] * dims[2], t), t, 0, s>>>(d3, a2, B, dims[2], dims[3],
				g + off(2, false), g + off(2, true));
		dense_xgrad_kernel<<<blocks_for((int64_t) B * dims[2], t), t, 0, s>>>(p + off(2, false), d3, B, dims[2], dims[3], d2);
		relu_backward_kernel<<<blocks_for((int64_t) B * dims[2], t), t, 0, s>>>(d2, z2, B * dims[2]);
		dense_wgrad_kernel<<<blocks_for((int64_t) dims[2] * dims[1], t), t, 0, s>>>(d2, a1, B, dims[1], dims[2],
				g + off(1, false), g + off(1, true));
		dense_xgrad_kernel<<<blocks_for((int64_t) B * dims[1], t), t, 0, s>>>(p + off(1, false), d2, B, dims[1], dims[2], d1);
		relu_backward_kernel<<<blocks_for((int64_t) B * dims[1], t), t, 0, s>>>(d1, z1, B * dims[1]);
		dense_wgrad_kernel<<<blocks_for((int64_t) dims[1] * dims[0], t), t, 0, s>>>(d1, X, B, dims[0], dims[1],
				g + off(0, false), g + off(0, true));
		SPMV_CUDA_TRY(cudaGetLastError());
		return SPMV_OK;
	}
};

}  // namespace spmv

struct spmv_mlp {
	spmv::Mlp m;
};

using spmv::set_error;

extern "C" {

int spmv_features(const int32_t * row_ptr, const int32_t * col_ind, int64_t m, int64_t n, int64_t nnz, double * out10)
{
	spmv::clear_error();
	if (!out10 || m < 0 || n < 0 || nnz < 0 || !row_ptr || (nnz > 0 && !col_ind)) {
		set_error(SPMV_ERR_ARG, "spmv_features: bad arguments");
		return SPMV_ERR_ARG;
	}
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) {
		set_error(SPMV_ERR_NO_DEVICE, "no CUDA device");
		return SPMV_ERR_NO_DEVICE;
	}
	cudaStream_t s = cudaStreamLegacy;
	spmv::DevBuf rp, ci;
	SPMV_TRY(rp.alloc((m + 1) * sizeof(int32_t), s));
	SPMV_TRY(ci.alloc((nnz > 0 ? nnz : 1) * sizeof(int32_t), s));
	SPMV_CUDA_TRY(cudaMemcpyAsync(rp.p, row_ptr, (m + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, s));
	if (nnz > 0)
		SPMV_CUDA_TRY(cudaMemcpyAsync(ci.p, col_ind, nnz * sizeof(int32_t), cudaMemcpyHostToDevice, s));
	return spmv::features_device(rp.as<int32_t>(), ci.as<int32_t>(), m, n, nnz, out10, s);
}

int spmv_features_device(const int32_t * d_row_ptr, const int32_t * d_col_ind, int64_t m, int64_t n, int64_t nnz,
		double * out10, void * stream)
{
	spmv::clear_error();
	if (!out10 || m < 0 || n < 0 || nnz < 0 || !d_row_ptr || (nnz > 0 && !d_col_ind)) {
		set_error(SPMV_ERR_ARG, "spmv_features_device: bad arguments");
		return SPMV_ERR_ARG;
	}
	return spmv::features_device(d_row_ptr, d_col_ind, m, n, nnz, out10,
			stream ? (cudaStream_t) stream : cudaStreamLegacy);
}

spmv_mlp * spmv_mlp_create(int32_t in, int32_t h1, int32_t h2, int32_t out, const float * init_params, int * status)
{
	spmv::clear_error();
	int st = SPMV_OK;
	spmv_mlp * H = nullptr;
	if (in < 1 || h1 < 1 || h2 < 1 || out < 2 || in > 4096 || h1 > 4096 || h2 > 4096 || out > 4096 || !init_params) {
		set_error(SPMV_ERR_ARG, "spmv_mlp_create: bad dimensions or missing initial parameters");
		st = SPMV_ERR_ARG;
	} else {
		H = new spmv_mlp();
		spmv::Mlp & m = H->m;
		m.dims[0] = in;
		m.dims[1] = h1;
		m.dims[2] = h2;
		m.dims[3] = out;
		m.nparam = m.off(3, false);
		for (float ** q : {&m.p, &m.g, &m.m1, &m.m2})
			if (cudaMalloc((void **) q, (size_t) m.nparam * sizeof(float)) != cudaSuccess)
				st = SPMV_ERR_NOMEM;
		if (cudaMalloc((void **) &m.lmean, sizeof(float)) != cudaSuccess)
			st = SPMV_ERR_NOMEM;
		if (st == SPMV_OK) {
			cudaMemcpy(m.p, init_params, (size_t) m.nparam * sizeof(float), cudaMemcpyHostToDevice);
			cudaMemset(m.g, 0, (size_t) m.nparam * sizeof(float));
			cudaMemset(m.m1, 0, (size_t) m.nparam * sizeof(float));
			cudaMemset(m.m2, 0, (size_t) m.nparam * sizeof(float));
			if (cudaDeviceSynchronize() != cudaSuccess)
				st = SPMV_ERR_CUDA;
		}
		if (st != SPMV_OK) {
			set_error(st, "spmv_mlp_create: device allocation or copy failed");
			delete H;
			H = nullptr;
		}
	}
	if (status)
		*status = st;
	return H;
}

int32_t spmv_mlp_num_params(const spmv_mlp * H)
{
	return H ? H->m.nparam : 0;
}

int spmv_mlp_get(const spmv_mlp * H, int32_t which, float * host_out)
{
	spmv::clear_error();
	if (!H || !host_out || which < 0 || which > 3) {
		set_error(SPMV_ERR_ARG, "spmv_mlp_get: bad arguments");
		return SPMV_ERR_ARG;
	}
	const float * src = which == 0 ? H->m.p : which == 1 ? H->m.g : which == 2 ? H->m.m1 : H->m.m2;
	SPMV_CUDA_TRY(cudaMemcpy(host_out, src, (size_t) H->m.nparam * sizeof(float), cudaMemcpyDeviceToHost));
	return SPMV_OK;
}

int spmv_mlp_set(spmv_mlp * H, const float * host_params)
{
	spmv::clear_error();
	if (!H || !host_params) {
		set_error(SPMV_ERR_ARG, "spmv_mlp_set: bad arguments");
		return SPMV_ERR_ARG;
	}
	SPMV_CUDA_TRY(cudaMemcpy(H->m.p, host_params, (size_t) H->m.nparam * sizeof(float), cudaMemcpyHostToDevice));
	return SPMV_OK;
}

int spmv_mlp_forward(spmv_mlp * H, const float * d_x, int32_t batch, float * d_logits, void * stream)
{
	spmv::clear_error();
	if (!H || !d_x || !d_logits || batch < 1) {
		set_error(SPMV_ERR_ARG, "spmv_mlp_forward: bad arguments");
		return SPMV_ERR_ARG;
	}
	return H->m.forward(d_x, batch, d_logits, stream ? (cudaStream_t) stream : cudaStreamLegacy, false);
}

int spmv_mlp_forward_host(spmv_mlp * H, const float * x_host, int32_t batch, float * logits_host)
{
	spmv::clear_error();
	if (!H || !x_host || !logits_host || batch < 1) {
		set_error(SPMV_ERR_ARG, "spmv_mlp_forward_host: bad arguments");
		return SPMV_ERR_ARG;
	}
	spmv::Mlp & m = H->m;
	cudaStream_t s = cudaStreamLegacy;
	SPMV_TRY(m.ensure(batch));
	if (batch * m.dims[0] > m.cap * m.dims[1]) {
		set_error(SPMV_ERR_ARG, "spmv_mlp_forward_host: input wider than the first hidden layer");
		return SPMV_ERR_ARG;
	}
	float * xin = m.d1;                           // staging for the inputs (d1 holds B x h1 floats)
	SPMV_CUDA_TRY(cudaMemcpyAsync(xin, x_host, (size_t) batch * m.dims[0] * sizeof(float), cudaMemcpyHostToDevice, s));
	SPMV_TRY(m.forward(xin, batch, m.d3, s, false));
	SPMV_CUDA_TRY(cudaMemcpyAsync(logits_host, m.d3, (size_t) batch * m.dims[3] * sizeof(float), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	return SPMV_OK;
}

int spmv_mlp_loss_grad(spmv_mlp * H, const float * d_x, const int32_t * d_labels, int32_t batch, float * loss_out,
		void * stream)
{
	spmv::clear_error();
	if (!H || !d_x || !d_labels || batch < 1) {
		set_error(SPMV_ERR_ARG, "spmv_mlp_loss_grad: bad arguments");
		return SPMV_ERR_ARG;
	}
	cudaStream_t s = stream ? (cudaStream_t) stream : cudaStreamLegacy;
	SPMV_TRY(H->m.forward(d_x, batch, nullptr, s, true));
	SPMV_TRY(H->m.backward(d_x, d_labels, batch, s));
	if (loss_out) {
		SPMV_CUDA_TRY(cudaMemcpyAsync(loss_out, H->m.lmean, sizeof(float), cudaMemcpyDeviceToHost, s));
		SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	}
	return SPMV_OK;
}

int spmv_mlp_adam_step(spmv_mlp * H, float lr, float beta1, float beta2, float eps, float weight_decay, void * stream)
{
	spmv::clear_error();
	if (!H || !(lr >= 0) || !(beta1 >= 0 && beta1 < 1) || !(beta2 >= 0 && beta2 < 1) || !(eps > 0) || !(weight_decay >= 0)) {
		set_error(SPMV_ERR_ARG, "spmv_mlp_adam_step: bad arguments");
		return SPMV_ERR_ARG;
	}
	spmv::Mlp & m = H->m;
	m.step++;
	const float c1 = 1.0f - powf(beta1, (float) m.step), c2 = 1.0f - powf(beta2, (float) m.step);
	cudaStream_t s = stream ? (cudaStream_t) stream : cudaStreamLegacy;
	spmv::adam_kernel<<<spmv::blocks_for(m.nparam, 256), 256, 0, s>>>(m.p, m.g, m.m1, m.m2, m.nparam, lr, beta1, beta2,
			eps, weight_decay, c1, c2);
	SPMV_CUDA_TRY(cudaGetLastError());
	return SPMV_OK;
}

void spmv_mlp_destroy(spmv_mlp * H)
{
	delete H;
}

}  // extern "C"
