// DIV-RF on the GPU: the packetiser (csr_to_format of src/spmv_kernels/DIV/div.cpp with
// DIV_TYPE_RF) and the decoder + SpMV.  The byte streams are bit-identical to the
// reference's for the same thread count T, lane count L and packet size.
//
// Packet format (div_kernels_rf.h:65-79, :538-919):
//   header {u32 num_vals, num_vals_unique, num_rows, row_min, col_min; u8 row_bits,
//           col_bits; 2 zero bytes; u32 num_rfs; u32 lane_bytes[L]}
//   u32 rfs[num_rfs]; u32 unique_per_rf[num_rfs]
//   coordinates: (row - row_min) | (col - col_min) << row_bits, in coords_bytes LE bytes
//   one code byte per unique value: low nibble = payload bytes (0-8), high nibble = shift/4
//   L lane byte streams: per lane the shifted u64 differences of consecutive values.
// Entries are ordered by (value bits, row, col); rf = multiplicity of a value; groups of
// equal rf in ascending rf; per group the unique values are cut into L contiguous lane
// runs, interleaved value-wise, and the coordinates unit-wise (permutation_interleave,
// lib/macros/permutation.h:47-115).
//
// GPU mapping of the reference's sequential per-thread loop:
//   1. packet boundaries: one thread per reference thread range walks the chain of
//      select_num_vals_complete_last_row (div_kernels_rf.h:437-464) with binary searches;
//   2. per packet: coordinate bit widths from a warp min/max over its entries;
//   3. the per-packet 128-bit sort becomes LSD radix sorts over all entries:
//      (row, col) [only if a row's columns are not ascending], value bits, packet id;
//   4. rf = run lengths of equal (packet, value); a stable radix sort by (packet, rf);
//   5. unique values: lane, position and the delta code of each; byte offsets by scans;
//   6. scatter of headers, coordinates, codes and payload bytes.
//
// Decoder: one CTA per packet.  Threads are (lane, chunk of that lane's positions); a
// lane-wise scan of payload lengths gives byte offsets, a lane-wise scan of differences
// gives values, then each value's rf coordinates are decoded and y[row] accumulated in
// shared memory.  The summation order inside a row differs from the reference's
// value-sorted serial order, so DIV-RF y agrees with the reference within the stated
// tolerance, not bit for bit.
#include <algorithm>
#include <vector>

#include "internal.h"
#include "primitives.cuh"

namespace spmv {

namespace {

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ int bits_required_u64(uint64_t v)
{
	return v ? 64 - __clzll((long long) v) : 0;
}

// first index in [lo, hi] with A[idx] >= v (A ascending, A[hi] >= v)
__device__ __forceinline__ int64_t lb_i32(const int32_t * A, int64_t lo, int64_t hi, int64_t v)
{
	while (lo < hi) {
		int64_t mid = (lo + hi) >> 1;
		if ((int64_t) A[mid] < v)
			lo = mid + 1;
		else
			hi = mid;
	}
	return lo;
}

// select_num_vals_complete_last_row (div_kernels_rf.h:437-464), rows capped at 255
__device__ __forceinline__ int64_t div_select(const int32_t * rp, int64_t m, int64_t i_s, int64_t j_s, int64_t nv)
{
	int64_t j_e = j_s + nv;
	int64_t i_e = lb_i32(rp, i_s, m, j_e);
	if (j_e != (int64_t) rp[i_e] && i_e - 1 > i_s) {
		i_e--;
		j_e = rp[i_e];
	}
	if (i_e - i_s > 255)
		i_e = i_s + 255;
	int64_t r = (int64_t) rp[i_e] - j_s;
	return r > nv ? nv : r;
}

// Packet chain of one reference thread range (div.cpp:285-425).
template <bool WRITE>
__global__ void div_chain_kernel(const int32_t * rp, int64_t m, const int64_t * ranges, int T, int64_t P,
		int64_t * counts, const int64_t * offs, int32_t * pk_j, int32_t * pk_row, int32_t * pk_nv, uint8_t * pk_grp,
		int32_t * pk_thread)
{
	int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= T)
		return;
	const int64_t i_s = ranges[2 * t], i_e = ranges[2 * t + 1];
	int64_t j = rp[i_s];
	const int64_t j_e = rp[i_e];
	int64_t i = i_s;
	int64_t n = 0;
	const int64_t o = WRITE ? offs[t] : 0;
	while (j < j_e) {
		i = lb_i32(rp, i, i_e, j);
		if ((int64_t) rp[i] != j)
			i--;
		while (rp[i] == rp[i + 1])
			i++;
		const int64_t nv_max = (j + P <= j_e) ? P : j_e - j;
		const int64_t nv = div_select(rp, m, i, j, nv_max);
		if (WRITE) {
			pk_j[o + n] = (int32_t) j;
			pk_row[o + n] = (int32_t) i;
			pk_nv[o + n] = (int32_t) nv;
			pk_grp[o + n] = (j == (int64_t) rp[i]) ? 1 : 0;
			pk_thread[o + n] = t;
		}
		n++;
		j += nv;
	}
	if (!WRITE)
		counts[t] = n;
}

// reduce_precision (div_kernels_rf.h:467-510) with the host-computed number of dropped bits
__device__ __forceinline__ uint64_t div_round(uint64_t u, int drop)
{
	if (drop < 0 || u == 0)
		return u;
	if (__ffsll((long long) u) - 1 >= 53)
		return u;
	const uint64_t mask = (1ULL << drop) - 1;
	const uint64_t lo = u & ~mask;
	const uint64_t hi = (u + mask) & ~mask;
	const int tzl = lo ? __ffsll((long long) lo) - 1 : 64;
	const int tzh = hi ? __ffsll((long long) hi) - 1 : 64;
	return (tzl > tzh) ? lo : hi;
}

__global__ void div_entry_kernel(const int32_t * rp, const int32_t * ci, const double * v, int64_t m, int64_t nnz,
		const int32_t * pk_j, int64_t NP, int drop, int32_t * pkt_of, int32_t * row_of, uint64_t * val_of)
{
	int64_t j = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= nnz)
		return;
	// packet: last packet start <= j
	int64_t lo = 0, hi = NP - 1;
	while (lo < hi) {
		int64_t mid = (lo + hi + 1) >> 1;
		if ((int64_t) pk_j[mid] <= j)
			lo = mid;
		else
			hi = mid - 1;
	}
	pkt_of[j] = (int32_t) lo;
	// row: last row start <= j with a non-empty row
	int64_t r = lb_i32(rp, 0, m, j + 1) - 1;
	row_of[j] = (int32_t) r;
	val_of[j] = div_round(__double_as_longlong(v[j]), drop);
}

__global__ void cols_unsorted_kernel(const int32_t * rp, const int32_t * ci, const int32_t * row_of, int64_t nnz,
		int * flag)
{
	int64_t j = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (j + 1 < nnz && row_of[j] == row_of[j + 1] && ci[j] >= ci[j + 1])
		atomicOr(flag, 1);
}

__global__ void keys_from_kernel(const uint32_t * idx, int64_t n, int what, const int32_t * a32, const uint64_t * a64,
		uint64_t * keys)
{
	int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n)
		return;
	const uint32_t j = idx[s];
	keys[s] = (what == 0) ? (uint64_t) (uint32_t) a32[j] : a64[j];
}

__global__ void iota_kernel(uint32_t * a, int64_t n)
{
	int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s < n)
		a[s] = (uint32_t) s;
}

// run flags of equal (packet, value) in the value-sorted order
__global__ void run_flag_kernel(const uint32_t * idx, int64_t n, const int32_t * pkt_of, const uint64_t * val_of,
		int32_t * flag)
{
	int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n)
		return;
	const uint32_t j = idx[s];
	int f = 1;
	if (s > 0) {
		const uint32_t jp = idx[s - 1];
		f = (pkt_of[j] != pkt_of[jp] || val_of[j] != val_of[jp]) ? 1 : 0;
	}
	flag[s] = f;
}

__global__ void run_start_kernel(const int32_t * flag, const int64_t * ex, int64_t n, int64_t * run_pos)
{
	int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s < n && flag[s])
		run_pos[ex[s]] = s;
}

__global__ void rf_kernel(const uint32_t * idx, const int32_t * flag, const int64_t * ex, const int64_t * run_pos,
		int64_t nruns, int64_t n, const int32_t * pkt_of, int rf_bits, int32_t * rf_of, uint64_t * keys)
{
	int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n)
		return;
	const int64_t rid = ex[s] + flag[s] - 1;
	const int64_t end = (rid + 1 < nruns) ? run_pos[rid + 1] : n;
	const int32_t rf = (int32_t) (end - run_pos[rid]);
	const uint32_t j = idx[s];
	rf_of[j] = rf;
	keys[s] = ((uint64_t) (uint32_t) pkt_of[j] << rf_bits) | (uint64_t) rf;
}

__global__ void group_flag_kernel(const uint32_t * idx, int64_t n, const int32_t * pkt_of, const int32_t * rf_of,
		int32_t * flag)
{
	int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n)
		return;
	const uint32_t j = idx[s];
	int f = 1;
	if (s > 0) {
		const uint32_t jp = idx[s - 1];
		f = (pkt_of[j] != pkt_of[jp] || rf_of[j] != rf_of[jp]) ? 1 : 0;
	}
	flag[s] = f;
}

// per group: start position, packet, rf, unique count
__global__ void group_info_kernel(const uint32_t * idx, const int32_t * flag, const int64_t * ex, int64_t n,
		const int32_t * pkt_of, const int32_t * rf_of, int64_t G, int64_t * g_start, int32_t * g_pkt, int32_t * g_rf)
{
	int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s < n && flag[s]) {
		const int64_t g = ex[s];
		const uint32_t j = idx[s];
		g_start[g] = s;
		g_pkt[g] = pkt_of[j];
		g_rf[g] = rf_of[j];
	}
	if (s == 0)
		g_start[G] = n;
}

__global__ void group_unique_kernel(const int64_t * g_start, const int32_t * g_rf, int64_t G, int64_t * g_u,
		const int32_t * g_pkt, int32_t * pk_g0)
{
	int64_t g = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (g >= G)
		return;
	g_u[g] = (g_start[g + 1] - g_start[g]) / g_rf[g];
	if (g == 0 || g_pkt[g] != g_pkt[g - 1])
		pk_g0[g_pkt[g]] = (int32_t) g;
}

// per packet: coordinate geometry (div_kernels_rf.h:603-662), one warp per packet
__global__ void packet_meta_kernel(const int32_t * rp, const int32_t * ci, int64_t m, const int32_t * pk_j,
		const int32_t * pk_row, const int32_t * pk_nv, int64_t NP, int32_t * pk_rowmax, int32_t * pk_colmin,
		uint8_t * pk_rb, uint8_t * pk_cb_bits, uint8_t * pk_cbytes, int * err)
{
	const int64_t p = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (p >= NP)
		return;
	const int64_t j0 = pk_j[p], nv = pk_nv[p];
	int32_t cmin = INT32_MAX, cmax = INT32_MIN;
	for (int64_t e = lane; e < nv; e += 32) {
		const int32_t c = ci[j0 + e];
		cmin = min(cmin, c);
		cmax = max(cmax, c);
	}
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
		cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
	}
	if (lane != 0)
		return;
	const int64_t jl = j0 + nv - 1;
	const int64_t row_min = pk_row[p];
	const int64_t row_max = lb_i32(rp, row_min, m, jl + 1) - 1;
	int row_bits = bits_required_u64((uint64_t) (row_max - row_min));
	int col_bits = bits_required_u64((uint64_t) ((int64_t) cmax - cmin));
	const int cbytes = (row_bits + col_bits + 7) >> 3;
	if (row_bits % 8) {
		const int cmpl = 8 - row_bits % 8;
		if (((row_bits + cmpl + col_bits + 7) >> 3) == cbytes)
			row_bits += cmpl;
	}
	col_bits = cbytes * 8 - row_bits;
	if (row_bits > 8 || col_bits > 32)
		dev_flag_error(err, DEV_ERR_FORMAT);
	pk_rowmax[p] = (int32_t) row_max;
	pk_colmin[p] = cmin;
	pk_rb[p] = (uint8_t) row_bits;
	pk_cb_bits[p] = (uint8_t) col_bits;
	pk_cbytes[p] = (uint8_t) cbytes;
}

// lane of unique value q in a group of u values cut into L contiguous runs
__device__ __forceinline__ int lane_of(int64_t q, int64_t dv, int64_t md)
{
	if (q < (dv + 1) * md)
		return (int) (q / (dv + 1));
	return (int) (md + (q - (dv + 1) * md) / (dv > 0 ? dv : 1));
}

__device__ __forceinline__ int64_t seg_start(int i, int64_t dv, int64_t md)
{
	return (int64_t) i * dv + (i < md ? i : md);
}

// Delta code of one difference (div_kernels_rf.h:824-892).
__device__ __forceinline__ void encode_diff(uint64_t diff, uint8_t * code, uint64_t * payload, int * nbytes)
{
	if (diff == 0) {
		*code = 0;
		*payload = 0;
		*nbytes = 0;
		return;
	}
	uint64_t lz = __clzll((long long) diff), tz = __ffsll((long long) diff) - 1;
	const uint64_t rem_tz = tz & 3;
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
	const uint64_t tz4 = tz >> 2;
	tz = tz4 << 2;
	len_bits = 64 - lz - tz;
	len = (len_bits + 7) >> 3;
	*payload = diff >> tz;
	*nbytes = (int) len;
	*code = (uint8_t) (len | (tz4 << 4));
}

// one thread per unique value (global unique index ug)
__global__ void unique_kernel(const uint32_t * idx2, const uint64_t * val_of, const int64_t * g_start,
		const int32_t * g_rf, const int64_t * g_u, const int64_t * g_ustart, int64_t G, int64_t U, int L,
		uint8_t * u_code, int32_t * u_nbytes, uint64_t * u_payload)
{
	const int64_t ug = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (ug >= U)
		return;
	int64_t lo = 0, hi = G - 1;
	while (lo < hi) {
		int64_t mid = (lo + hi + 1) >> 1;
		if (g_ustart[mid] <= ug)
			lo = mid;
		else
			hi = mid - 1;
	}
	const int64_t g = lo;
	const int64_t q = ug - g_ustart[g];
	const int64_t u = g_u[g], rf = g_rf[g];
	const int64_t dv = u / L, md = u % L;
	const int i = lane_of(q, dv, md);
	const int64_t pos = q - seg_start(i, dv, md);
	const int64_t s = g_start[g] + q * rf;
	const uint64_t val = val_of[idx2[s]];
	const uint64_t prev = (pos > 0) ? val_of[idx2[s - rf]] : 0;
	uint8_t code;
	uint64_t pay;
	int nb;
	encode_diff(val - prev, &code, &pay, &nb);
	u_code[ug] = code;
	u_nbytes[ug] = nb;
	u_payload[ug] = pay;
}

// per packet: lane sizes and per-(group, lane) byte bases, lane-major (one thread per packet)
__global__ void lane_layout_kernel(const int32_t * pk_g0, int64_t NP, const int64_t * g_u, const int64_t * g_ustart,
		const int64_t * S, int L, int64_t * gl_base, int64_t * pk_lanes_total, uint32_t * pk_lane_bytes)
{
	const int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= NP)
		return;
	const int64_t g0 = pk_g0[p], g1 = pk_g0[p + 1];
	int64_t run = 0;
	for (int i = 0; i < L; i++) {
		int64_t lane_start = run;
		for (int64_t g = g0; g < g1; g++) {
			const int64_t u = g_u[g], dv = u / L, md = u % L;
			const int64_t q0 = seg_start(i, dv, md), q1 = seg_start(i + 1, dv, md);
			const int64_t b = S[g_ustart[g] + q1] - S[g_ustart[g] + q0];
			gl_base[g * L + i] = run;
			run += b;
		}
		pk_lane_bytes[p * L + i] = (uint32_t) (run - lane_start);
	}
	pk_lanes_total[p] = run;
}

__global__ void packet_size_kernel(const int32_t * pk_g0, const int32_t * pk_nv, const uint8_t * pk_cbytes,
		const int64_t * g_ustart, const int64_t * pk_lanes_total, int64_t NP, int L, int64_t * pk_size)
{
	const int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= NP)
		return;
	const int64_t nrf = pk_g0[p + 1] - pk_g0[p];
	const int64_t nu = g_ustart[pk_g0[p + 1]] - g_ustart[pk_g0[p]];
	pk_size[p] = (28 + 4 * (int64_t) L) + 8 * nrf + (int64_t) pk_cbytes[p] * pk_nv[p] + nu + pk_lanes_total[p];
}

__device__ __forceinline__ void put_u32(uint8_t * p, uint32_t v)
{
	p[0] = (uint8_t) v;
	p[1] = (uint8_t) (v >> 8);
	p[2] = (uint8_t) (v >> 16);
	p[3] = (uint8_t) (v >> 24);
}

__global__ void header_kernel(const int64_t * pk_off, const int32_t * pk_g0, const int32_t * pk_nv,
		const int32_t * pk_row, const int32_t * pk_rowmax, const int32_t * pk_colmin, const uint8_t * pk_rb,
		const uint8_t * pk_cb_bits, const int64_t * g_ustart, const int64_t * g_u, const int32_t * g_rf,
		const uint32_t * pk_lane_bytes, int64_t NP, int L, uint8_t * out)
{
	const int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= NP)
		return;
	uint8_t * h = out + pk_off[p];
	const int64_t g0 = pk_g0[p], g1 = pk_g0[p + 1];
	put_u32(h + 0, (uint32_t) pk_nv[p]);
	put_u32(h + 4, (uint32_t) (g_ustart[g1] - g_ustart[g0]));
	put_u32(h + 8, (uint32_t) (pk_rowmax[p] - pk_row[p] + 1));
	put_u32(h + 12, (uint32_t) pk_row[p]);
	put_u32(h + 16, (uint32_t) pk_colmin[p]);
	h[20] = pk_rb[p];
	h[21] = pk_cb_bits[p];
	h[22] = 0;
	h[23] = 0;
	put_u32(h + 24, (uint32_t) (g1 - g0));
	for (int i = 0; i < L; i++)
		put_u32(h + 28 + 4 * i, pk_lane_bytes[p * L + i]);
	uint8_t * r = h + 28 + 4 * L;
	const int64_t nrf = g1 - g0;
	for (int64_t g = g0; g < g1; g++) {
		put_u32(r + 4 * (g - g0), (uint32_t) g_rf[g]);
		put_u32(r + 4 * nrf + 4 * (g - g0), (uint32_t) g_u[g]);
	}
}

// one thread per entry position s of the (packet, rf, value, row, col) order
__global__ void coords_kernel(const uint32_t * idx2, int64_t n, const int32_t * pkt_of, const int32_t * row_of,
		const int32_t * ci, const int32_t * gid_flag, const int64_t * gid_ex, const int64_t * g_start,
		const int32_t * g_rf, const int64_t * g_u, const int32_t * pk_j, const int32_t * pk_row,
		const int32_t * pk_colmin, const uint8_t * pk_rb, const uint8_t * pk_cbytes, const int32_t * pk_g0,
		const int64_t * pk_off, int L, uint8_t * out)
{
	const int64_t s = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n)
		return;
	const uint32_t j = idx2[s];
	const int64_t p = pkt_of[j];
	const int64_t g = gid_ex[s] + gid_flag[s] - 1;
	const int64_t rf = g_rf[g], u = g_u[g];
	const int64_t dv = u / L, md = u % L;
	const int64_t e = s - g_start[g];
	const int64_t q = e / rf;
	const int i = lane_of(q, dv, md);
	const int64_t o = e - rf * seg_start(i, dv, md);
	const int64_t jj = (o < rf * dv) ? o * L + i : rf * dv * L + (int64_t) i * rf + (o - rf * dv);
	const int64_t slot = (g_start[g] - (int64_t) pk_j[p]) + jj;
	const int cb = pk_cbytes[p];
	const int64_t nrf = pk_g0[p + 1] - pk_g0[p];
	const uint64_t c = (uint64_t) (row_of[j] - pk_row[p]) | ((uint64_t) (ci[j] - pk_colmin[p]) << pk_rb[p]);
	uint8_t * dst = out + pk_off[p] + 28 + 4 * L + 8 * nrf + slot * cb;
	for (int b = 0; b < cb; b++)
		dst[b] = (uint8_t) (c >> (8 * b));
}

// one thread per unique value: its code byte and payload bytes
__global__ void values_kernel(const int64_t * g_start, const int32_t * g_pkt, const int64_t * g_u,
		const int64_t * g_ustart, int64_t G, int64_t U, const int32_t * pk_g0, const int32_t * pk_nv,
		const uint8_t * pk_cbytes, const int64_t * pk_off, const int64_t * gl_base, const int64_t * S,
		const uint8_t * u_code, const int32_t * u_nbytes, const uint64_t * u_payload, int L, uint8_t * out)
{
	const int64_t ug = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (ug >= U)
		return;
	int64_t lo = 0, hi = G - 1;
	while (lo < hi) {
		int64_t mid = (lo + hi + 1) >> 1;
		if (g_ustart[mid] <= ug)
			lo = mid;
		else
			hi = mid - 1;
	}
	const int64_t g = lo;
	const int64_t p = g_pkt[g];
	const int64_t q = ug - g_ustart[g];
	const int64_t u = g_u[g], dv = u / L, md = u % L;
	const int i = lane_of(q, dv, md);
	const int64_t q0 = seg_start(i, dv, md);
	const int64_t pos = q - q0;
	const int64_t g0 = pk_g0[p];
	const int64_t nrf = pk_g0[p + 1] - g0;
	const int64_t nu = g_ustart[pk_g0[p + 1]] - g_ustart[g0];
	const int64_t code_base = pk_off[p] + 28 + 4 * L + 8 * nrf + (int64_t) pk_cbytes[p] * pk_nv[p];
	const int64_t kslot = (g_ustart[g] - g_ustart[g0]) + pos * L + i;
	out[code_base + kslot] = u_code[ug];
	const int nb = u_nbytes[ug];
	if (nb > 0) {
		const int64_t dst = code_base + nu + gl_base[g * L + i] + (S[ug] - S[g_ustart[g] + q0]);
		const uint64_t pay = u_payload[ug];
		for (int b = 0; b < nb; b++)
			out[dst + b] = (uint8_t) (pay >> (8 * b));
	}
}

// packet groups per thread range: byte offsets relative to the thread's stream
__global__ void groups_kernel(const int64_t * pk_off, const uint8_t * pk_grp, const int32_t * pk_thread,
		const int64_t * th_first, int64_t NP, int T, const int64_t * grp_ex, const int64_t * grp_base_t,
		int64_t * groups, int64_t * th_bytes, int64_t * th_groups, int64_t total_bytes)
{
	const int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (p < NP && pk_grp[p]) {
		const int t = pk_thread[p];
		const int64_t gidx = grp_ex[p] - grp_ex[th_first[t]];   // group index inside the thread
		groups[grp_base_t[t] + t + gidx] = pk_off[p] - pk_off[th_first[t]];
	}
	if (p < T) {
		const int t = (int) p;
		const int64_t f = th_first[t], l = th_first[t + 1];
		const int64_t start = (f < NP) ? pk_off[f] : total_bytes;
		const int64_t end = (l < NP) ? pk_off[l] : total_bytes;
		th_bytes[t] = end - start;
		const int64_t ng = grp_base_t[t + 1] - grp_base_t[t];
		th_groups[t] = ng;
		groups[grp_base_t[t] + t + ng] = end - start;
	}
}

__global__ void thread_first_kernel(const int64_t * pk_count_ex, int T, int64_t * th_first)
{
	int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t <= T)
		th_first[t] = pk_count_ex[t];
}

__global__ void grp_i32_kernel(const uint8_t * g, int64_t n, int32_t * o)
{
	int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (p < n)
		o[p] = g[p];
}

// groups per thread: prefix of the group flags at the thread's first packet
__global__ void grp_base_kernel(const int64_t * grp_ex, const int64_t * th_first, int T, int64_t * base)
{
	int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t <= T)
		base[t] = grp_ex[th_first[t]];
}

// SpMV metadata per packet: byte offset, y rows to store / zero, shared first/last rows
__global__ void spmv_meta_kernel(const int32_t * rp, int64_t m, const int32_t * pk_j, const int32_t * pk_nv,
		const int32_t * pk_row, const int32_t * pk_rowmax, int64_t NP, int4 * meta, int32_t * split_flag)
{
	const int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= NP)
		return;
	const int64_t rmin = pk_row[p], rmax = pk_rowmax[p];
	const bool first_shared = (int64_t) pk_j[p] != (int64_t) rp[rmin];
	const bool last_shared = (int64_t) pk_j[p] + pk_nv[p] != (int64_t) rp[rmax + 1];
	// rows before this packet not covered by the previous packet (empty rows) are zeroed by it
	const int64_t zero_from = (p == 0) ? 0 : (int64_t) pk_rowmax[p - 1] + 1;
	int4 mt;
	mt.x = (int32_t) (zero_from < rmin ? zero_from : rmin);
	mt.y = (p == NP - 1) ? (int32_t) m : (int32_t) (rmax + 1);   // the last packet zeroes the tail rows
	mt.z = (first_shared ? 1 : 0) | (last_shared ? 2 : 0);
	mt.w = 0;
	meta[p] = mt;
	split_flag[p] = last_shared ? 1 : 0;
}

__global__ void split_rows_kernel(const int32_t * split_flag, const int64_t * ex, const int32_t * pk_rowmax, int64_t NP,
		int32_t * rows)
{
	const int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (p < NP && split_flag[p])
		rows[ex[p]] = pk_rowmax[p];
}

// ------------------------------------------------------------------ decoder + SpMV
constexpr int DEC_THREADS = 256;
constexpr int DEC_MAX_ROWS = 256;

// n <= 8 little-endian bytes at an unaligned address: two aligned 8-byte loads and a funnel
// shift.  The reads reach at most 15 bytes past p; the stream is padded by 16 bytes.
__device__ __forceinline__ uint64_t ld_bytes(const uint8_t * p, int n)
{
	const uintptr_t a = reinterpret_cast<uintptr_t>(p);
	const uint64_t * w = reinterpret_cast<const uint64_t *>(a & ~(uintptr_t) 7);
	const int sh = (int) (a & 7) * 8;
	const uint64_t lo = w[0];
	const uint64_t v = sh ? ((lo >> sh) | (w[1] << (64 - sh))) : lo;
	return n >= 8 ? v : (v & ((1ULL << (8 * n)) - 1));
}

__device__ __forceinline__ uint32_t ld_u32(const uint8_t * p)
{
	return (uint32_t) ld_bytes(p, 4);
}

struct DivArgs {
	const uint8_t * data;
	const int64_t * pkt_off;
	const int4 * meta;
	int64_t npackets;
	int L;
	const double * x;
	double * y;
	int pf;                  // warp decoder: prefetch distance in positions
};

// Exclusive scan over the threads of each lane (thread t: lane t % L, position t / L in its
// lane), in position order: the sum of v over the lane's earlier threads.  L is a power of two
// and DEC_THREADS threads take part.  Below 32 lanes a warp holds 32 / L threads of each lane,
// scanned with shuffles (strides L, 2L, ...), then the 8 warp totals of the lane are added from
// shared memory; from 32 lanes up a lane has at most 8 threads, one per warp, added directly.
// vals and wsum are DEC_THREADS-entry shared arrays; one barrier inside.
template <typename T>
__device__ __forceinline__ T lane_exclusive_scan(T v, int L, T * vals, T * wsum)
{
	const int t = threadIdx.x, lane = t % L, w = t >> 5, wl = t & 31;
	vals[t] = v;
	T inc = v;
	if (L < 32) {
		for (int d = L; d < 32; d <<= 1) {
			const T o = __shfl_up_sync(0xffffffffu, inc, d);
			if (wl >= d)
				inc += o;
		}
		if (wl >= 32 - L)
			wsum[w * L + (wl - (32 - L))] = inc;     // the warp's total of this lane
	}
	__syncthreads();
	T pre = inc - v;
	if (L < 32) {
		for (int q = 0; q < w; q++)
			pre += wsum[q * L + lane];
	} else {
		for (int c = 0; c < t / L; c++)
			pre += vals[c * L + lane];
	}
	return pre;
}

// One CTA per packet, at most 85 registers a thread so that 3 CTAs share an SM.  (Copying the
// packet into shared memory first was measured slower: the copy's shared memory leaves 2 CTAs
// an SM, and the byte reads conflict on the banks.)
__global__ void __launch_bounds__(DEC_THREADS, 3) div_spmv_kernel(DivArgs a)
{
	__shared__ double ys[DEC_MAX_ROWS];
	__shared__ int64_t scan_i[DEC_THREADS];
	__shared__ uint64_t scan_u[DEC_THREADS];
	__shared__ int64_t lane_cursor[DEC_THREADS];
	__shared__ int64_t wsum_i[DEC_THREADS];
	__shared__ uint64_t wsum_u[DEC_THREADS];
	const int64_t p = blockIdx.x;
	const uint8_t * h = a.data + a.pkt_off[p];
	const int L = a.L;
	const int64_t nv = ld_u32(h + 0), nu = ld_u32(h + 4), nrows = ld_u32(h + 8);
	const int64_t row_min = ld_u32(h + 12), col_min = ld_u32(h + 16);
	const int row_bits = h[20], col_bits = h[21];
	const int64_t nrf = ld_u32(h + 24);
	const int cb = (row_bits + col_bits + 7) >> 3;
	const uint8_t * rfs = h + 28 + 4 * L;
	const uint8_t * nus = rfs + 4 * nrf;
	const uint8_t * coords = nus + 4 * nrf;
	const uint8_t * codes = coords + cb * nv;
	const uint8_t * lanes = codes + nu;
	const uint64_t rmask = row_bits ? ((1ULL << row_bits) - 1) : 0;
	const uint64_t cmask = (col_bits >= 64) ? ~0ULL : ((1ULL << col_bits) - 1);
	for (int r = threadIdx.x; r < nrows && r < DEC_MAX_ROWS; r += blockDim.x)
		ys[r] = 0.0;
	// lane byte cursors: lane i starts after the streams of lanes < i
	if (threadIdx.x == 0) {
		int64_t run = 0;
		for (int i = 0; i < L; i++) {
			lane_cursor[i] = run;
			run += ld_u32(h + 28 + 4 * i);
		}
	}
	__syncthreads();
	const int tpl = blockDim.x / L;              // threads per lane
	const int lane = threadIdx.x % L;
	const int cidx = threadIdx.x / L;
	const bool active = cidx < tpl;
	// packet-local counts and offsets fit in 32 bits (a packet holds at most 2^31 values and bytes)
	int kstart = 0, cstart = 0;
	for (int g = 0; g < (int) nrf; g++) {
		const int rf = (int) ld_u32(rfs + 4 * g), u = (int) ld_u32(nus + 4 * g);
		const int dv = u / L, md = u % L;
		const int n_i = dv + (lane < md ? 1 : 0);          // positions of this lane
		const int per = (n_i + tpl - 1) / tpl;
		const int p0 = active ? cidx * per : 0;
		const int p1 = active ? min(n_i, p0 + per) : 0;
		// the chunk's coordinates, read only in pass 3, asked of L1 now: rf = 1 groups hold
		// them for positions [p0, p1) of all L lanes in one range, each of its L threads
		// prefetches every L-th line of it
		if (a.pf && rf == 1 && p1 > p0) {
			const uint8_t * c0 = coords + ((int64_t) cstart + (int64_t) p0 * L) * cb;
			const int64_t len = (int64_t) (p1 - p0) * L * cb;
			for (int64_t o = (int64_t) lane * 128; o < len; o += (int64_t) L * 128)
				asm volatile("prefetch.global.L1 [%0];" ::"l"(c0 + o));
		}
		// 1) payload bytes of this chunk
		int nbytes = 0;
		for (int pos = p0; pos < p1; pos++)
			nbytes += codes[kstart + pos * L + lane] & 15;
		const int bstart = (int) (lane_cursor[lane] + lane_exclusive_scan<int64_t>(nbytes, L, scan_i, wsum_i));
		__syncthreads();                 // every thread has read its lane's cursor
		if (active && cidx == tpl - 1)
			lane_cursor[lane] = bstart + nbytes;     // next group continues the lane stream
		// 2) value difference sum of this chunk
		uint64_t dsum = 0;
		{
			int b = bstart;
			for (int pos = p0; pos < p1; pos++) {
				const uint8_t code = codes[kstart + pos * L + lane];
				const int len = code & 15, tz = (code >> 2) & ~3;
				dsum += ld_bytes(lanes + b, len) << tz;
				b += len;
			}
		}
		const uint64_t dstart = lane_exclusive_scan<uint64_t>(dsum, L, scan_u, wsum_u);   // lanes restart at 0
		// 3) values, coordinates, products
		if (rf == 1) {
			// one coordinate per value (k = pos * L + lane): decode 4 positions, issue their x
			// loads together, then add the products in the same order
			uint64_t val = dstart;
			int b = bstart;
			for (int pos0 = p0; pos0 < p1; pos0 += 4) {
				double vv[4], xv[4];
				int rr[4];
				#pragma unroll
				for (int q = 0; q < 4; q++) {
					const int pos = pos0 + q;
					if (pos < p1) {
						const uint8_t code = codes[kstart + pos * L + lane];
						const int len = code & 15, tz = (code >> 2) & ~3;
						val += ld_bytes(lanes + b, len) << tz;
						b += len;
						vv[q] = __longlong_as_double((long long) val);
						const uint64_t c = ld_bytes(coords + (cstart + pos * L + lane) * cb, cb);
						rr[q] = (int) (c & rmask);
						xv[q] = __ldg(a.x + col_min + (int64_t) ((c >> row_bits) & cmask));
					}
				}
				#pragma unroll
				for (int q = 0; q < 4; q++)
					if (pos0 + q < p1)
						atomicAdd(&ys[rr[q]], vv[q] * xv[q]);
			}
		} else {
			uint64_t val = dstart;
			int b = bstart;
			for (int pos = p0; pos < p1; pos++) {
				const uint8_t code = codes[kstart + pos * L + lane];
				const int len = code & 15, tz = (code >> 2) & ~3;
				val += ld_bytes(lanes + b, len) << tz;
				b += len;
				const double vd = __longlong_as_double((long long) val);
				for (int j = 0; j < rf; j++) {
					const int k = (pos < dv) ? (pos * L) * rf + L * j + lane : (dv * L + lane) * rf + j;
					const uint64_t c = ld_bytes(coords + (cstart + k) * cb, cb);
					const int64_t rr = (int64_t) (c & rmask);
					const int64_t cc = (int64_t) ((c >> row_bits) & cmask);
					atomicAdd(&ys[rr], vd * __ldg(a.x + col_min + cc));
				}
			}
		}
		__syncthreads();
		kstart += u;
		cstart += rf * u;
	}
	__syncthreads();
	const int4 mt = a.meta[p];
	for (int64_t r = (int64_t) mt.x + threadIdx.x; r < (int64_t) mt.y; r += blockDim.x) {
		const int64_t rel = r - row_min;
		if (rel < 0 || rel >= nrows) {
			a.y[r] = 0.0;                                // empty rows between packets
		} else if ((rel == 0 && (mt.z & 1)) || (rel == nrows - 1 && (mt.z & 2))) {
			atomicAdd(&a.y[r], ys[rel]);                 // a row split across packets
		} else {
			a.y[r] = ys[rel];
		}
	}
}

// ------------------------------------------------------------------ warp decoder (32 lanes)
// With L = 32 every lane stream of a packet belongs to one lane of a warp, and the lane walks
// it once, in order: no scans over threads, every entry decoded once.  One warp per packet;
// per position the code byte (the 32 lanes read 32 neighbouring bytes), the lane's payload
// bytes through a streaming reader (two words in registers, one aligned 8-byte load per 8
// bytes consumed), the coordinates (neighbouring for rf = 1) and x; products go to the
// warp's row sums in shared memory, then the packet's rows are stored as in the CTA decoder.
constexpr int DIVW_WARPS = 8;

struct LaneReader {
	const uint64_t * w;      // next aligned word to load
	uint64_t cur, nxt;       // the words holding the read position and the one after it
	int sh;                  // read position within cur, in bytes
	__device__ __forceinline__ void init(const uint8_t * p)
	{
		const uintptr_t a = reinterpret_cast<uintptr_t>(p);
		w = reinterpret_cast<const uint64_t *>(a & ~(uintptr_t) 7);
		sh = (int) (a & 7);
		cur = w[0];
		nxt = w[1];
		w += 2;
	}
	// n <= 8 little-endian bytes; reads reach at most 15 bytes past the read position
	__device__ __forceinline__ uint64_t read(int n)
	{
		const uint64_t v = sh ? ((cur >> (8 * sh)) | (nxt << (64 - 8 * sh))) : cur;
		sh += n;
		if (sh >= 8) {
			sh -= 8;
			cur = nxt;
			nxt = *w++;
		}
		return n >= 8 ? v : (v & ((1ULL << (8 * n)) - 1));
	}
};

// PF 1 / 2: in groups of one coordinate per value, the lines of the code bytes and
// coordinates a.pf positions ahead (a multiple of 4, 8 by default) are prefetched into L1 /
// L2 (lane 0: the 128 code bytes of 4 positions; lanes 1..: the 128 * cb coordinate bytes),
// inside the group's full rows (L1: 0.744 against 0.830 ms on the 4M-row matrix, 4,096-value
// packets).

// MINB: CTAs an SM the registers are held to (3: 79 registers; 4: 64, a few spilled)
template <int PF, int MINB>
__global__ void __launch_bounds__(DIVW_WARPS * 32, MINB) div_warp_kernel(DivArgs a)
{
	__shared__ double ys_all[DIVW_WARPS][DEC_MAX_ROWS];
	const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
	const int64_t p = (int64_t) blockIdx.x * DIVW_WARPS + wib;
	if (p >= a.npackets)
		return;
	double * ys = ys_all[wib];
	const uint8_t * h = a.data + a.pkt_off[p];
	const int64_t nrows = ld_u32(h + 8);
	const int64_t row_min = ld_u32(h + 12), col_min = ld_u32(h + 16);
	const int row_bits = h[20], col_bits = h[21];
	const int nrf = (int) ld_u32(h + 24);
	const int cb = (row_bits + col_bits + 7) >> 3;
	const int64_t nv = ld_u32(h + 0), nu = ld_u32(h + 4);
	const uint8_t * rfs = h + 28 + 4 * 32;
	const uint8_t * nus = rfs + 4 * nrf;
	const uint8_t * coords = nus + 4 * nrf;
	const uint8_t * codes = coords + cb * nv;
	const uint8_t * lanes = codes + nu;
	const uint64_t rmask = row_bits ? ((1ULL << row_bits) - 1) : 0;
	const uint64_t cmask = (col_bits >= 64) ? ~0ULL : ((1ULL << col_bits) - 1);
	for (int r = lane; r < nrows && r < DEC_MAX_ROWS; r += 32)
		ys[r] = 0.0;
	// lane i's stream starts after the streams of lanes < i
	const uint32_t my_bytes = ld_u32(h + 28 + 4 * lane);
	uint32_t start = my_bytes;
	#pragma unroll
	for (int d = 1; d < 32; d <<= 1) {
		const uint32_t o = __shfl_up_sync(0xffffffffu, start, d);
		if (lane >= d)
			start += o;
	}
	start -= my_bytes;
	LaneReader rd;
	rd.init(lanes + start);
	__syncwarp();
	int kstart = 0, cstart = 0;
	for (int g = 0; g < nrf; g++) {
		const int rf = (int) ld_u32(rfs + 4 * g), u = (int) ld_u32(nus + 4 * g);
		const int dv = u >> 5, md = u & 31;
		const int n_i = dv + (lane < md ? 1 : 0);
		uint64_t val = 0;                                   // differences restart in every group
		if (rf == 1) {
			for (int pos0 = 0; pos0 < n_i; pos0 += 4) {
				if (PF && pos0 + a.pf + 4 <= dv) {
					const int64_t k0 = (int64_t) (pos0 + a.pf) * 32;
					const int cl = (128 * cb + 127) >> 7;      // coordinate lines of 4 positions
					const uint8_t * pa = lane == 0 ? codes + kstart + k0
							: lane <= cl ? coords + (cstart + k0) * cb + (int64_t) (lane - 1) * 128 : nullptr;
					if (pa && PF == 2)
						asm volatile("prefetch.global.L2 [%0];" ::"l"(pa));
					else if (pa)
						asm volatile("prefetch.global.L1 [%0];" ::"l"(pa));
				}
				double vv[4], xv[4];
				int rr[4];
				#pragma unroll
				for (int q = 0; q < 4; q++) {
					const int pos = pos0 + q;
					if (pos < n_i) {
						const int k = pos * 32 + lane;
						const uint8_t code = codes[kstart + k];
						val += rd.read(code & 15) << ((code >> 4) << 2);
						vv[q] = __longlong_as_double((long long) val);
						const uint64_t c = ld_bytes(coords + (int64_t) (cstart + k) * cb, cb);
						rr[q] = (int) (c & rmask);
						xv[q] = __ldg(a.x + col_min + (int64_t) ((c >> row_bits) & cmask));
					}
				}
				#pragma unroll
				for (int q = 0; q < 4; q++)
					if (pos0 + q < n_i)
						atomicAdd(&ys[rr[q]], vv[q] * xv[q]);
			}
		} else {
			for (int pos = 0; pos < n_i; pos++) {
				const uint8_t code = codes[kstart + pos * 32 + lane];
				val += rd.read(code & 15) << ((code >> 4) << 2);
				const double vd = __longlong_as_double((long long) val);
				for (int j = 0; j < rf; j++) {
					const int k = (pos < dv) ? (pos * 32) * rf + 32 * j + lane : (dv * 32 + lane) * rf + j;
					const uint64_t c = ld_bytes(coords + (int64_t) (cstart + k) * cb, cb);
					atomicAdd(&ys[(int) (c & rmask)], vd * __ldg(a.x + col_min + (int64_t) ((c >> row_bits) & cmask)));
				}
			}
		}
		kstart += u;
		cstart += rf * u;
	}
	__syncwarp();
	const int4 mt = a.meta[p];
	for (int64_t r = (int64_t) mt.x + lane; r < (int64_t) mt.y; r += 32) {
		const int64_t rel = r - row_min;
		if (rel < 0 || rel >= nrows) {
			a.y[r] = 0.0;                                // empty rows between packets
		} else if ((rel == 0 && (mt.z & 1)) || (rel == nrows - 1 && (mt.z & 2))) {
			atomicAdd(&a.y[r], ys[rel]);                 // a row split across packets
		} else {
			a.y[r] = ys[rel];
		}
	}
}

// ------------------------------------------------------------------ packet reordering
// DIV_PACKET_REORDERING (div.cpp:377-395, :455-498): every thread's packet groups are
// stored in ascending order of a median column.  The reference records, per packet, the
// median of its column indices (array_quantile_serial(ja, nv, 0.5), lib/array_metrics.c:
// 952-1088, method "median_unbiased": with N values, N <= 2 gives the largest, even N the
// order statistic N/2, odd N the mean of order statistics (N-1)/2 and (N+1)/2; truncated to
// an integer) and then sorts the thread's groups g by the median of its g-th PACKET with its
// quicksort.  Medians come from a GPU sort of (packet, column); the group permutation is
// computed on the host with the reference's quicksort restated (ref_quicksort below: equal
// keys end up where its partitioning puts them, so the same bytes result); the group byte
// ranges are then moved on the GPU.
__global__ void pkt_col_keys_kernel(const int32_t * pkt_of, const int32_t * ci, int64_t nnz, uint64_t * keys,
		uint32_t * vals)
{
	const int64_t j = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= nnz)
		return;
	keys[j] = ((uint64_t) (uint32_t) pkt_of[j] << 32) | (uint64_t) (uint32_t) ci[j];
	vals[j] = 0;
}

__global__ void pkt_median_kernel(const uint64_t * sorted, const int32_t * pk_j, const int32_t * pk_nv, int64_t NP,
		int64_t * med)
{
	const int64_t p = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= NP)
		return;
	const int64_t b = pk_j[p], N = pk_nv[p];
	const uint64_t * c = sorted + b;
	if (N <= 2) {
		med[p] = N > 0 ? (int64_t) (uint32_t) c[N - 1] : 0;
	} else if ((N & 1) == 0) {
		med[p] = (int64_t) (uint32_t) c[N / 2];
	} else {
		const double l = (double) (uint32_t) c[(N - 1) / 2], r = (double) (uint32_t) c[(N + 1) / 2];
		med[p] = (int64_t) (__dadd_rn(__dmul_rn(0.5, l), __dmul_rn(0.5, r)));
	}
}

__global__ void move_groups_kernel(const uint8_t * src, uint8_t * dst, const int64_t * plan, int64_t ngroups)
{
	// plan[3 g .. 3 g + 2]: source offset, destination offset, length of group g
	const int64_t g = blockIdx.x;
	if (g >= ngroups)
		return;
	const int64_t so = plan[3 * g], d = plan[3 * g + 1], len = plan[3 * g + 2];
	for (int64_t i = threadIdx.x; i < len; i += blockDim.x)
		dst[d + i] = src[so + i];
}

__global__ void zero_rows_kernel(const int32_t * rows, int64_t n, double * y)
{
	int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		y[rows[i]] = 0.0;
}

// The reference's quicksort of an index array A[0..N) by key[A[i]] ascending
// (lib/sort/quicksort/quicksort_gen.c:96-146 with partition_auto_serial /
// partition_serial_base, lib/sort/partition/partition_gen.c:100-195), restated: a
// median-of-three pivot, a two-cursor partition that swaps elements equal to the pivot, and
// the reference's loop that keeps the left bounds on a stack and shrinks the right end by
// one element per pop.  Equal keys end up where that procedure puts them.
static int ref_cmp(int a, int b, const int * key)
{
	return key[a] > key[b] ? 1 : key[a] < key[b] ? -1 : 0;
}

static long ref_partition_base(int pivot, int * A, long lo, long hi, const int * key)
{
	long s = lo, e = hi;
	for (;;) {
		while (s < e && ref_cmp(A[s], pivot, key) < 0)
			s++;
		while (s < e && ref_cmp(A[e], pivot, key) > 0)
			e--;
		if (s >= e)
			break;
		std::swap(A[s], A[e]);
		s++;
		e--;
	}
	if (ref_cmp(A[s], pivot, key) < 0)
		s++;
	return s;
}

static long ref_partition_auto(int * A, long lo, long end, const int * key)
{
	const long N = end - lo;
	if (N == 1)
		return lo;
	const long hi = end - 1, pv = (lo + hi) / 2;
	if (ref_cmp(A[lo], A[hi], key) > 0)
		std::swap(A[lo], A[hi]);
	if (N == 2)
		return hi;
	if (ref_cmp(A[lo], A[pv], key) > 0)
		std::swap(A[lo], A[pv]);
	if (ref_cmp(A[pv], A[hi], key) > 0)
		std::swap(A[pv], A[hi]);
	if (N == 3)
		return pv;
	return ref_partition_base(A[pv], A, lo + 1, hi - 1, key);
}

static void ref_quicksort(int * A, long N, const int * key)
{
	if (N < 2)
		return;
	std::vector<long> stack((size_t) N);
	long s = 0, e = N - 1, i = 0;
	for (;;) {
		while (s >= e) {
			if (s == 0)
				return;
			i--;
			e--;
			s = stack[(size_t) i];
		}
		const long m = ref_partition_auto(A, s, e + 1, key);
		stack[(size_t) i++] = s;
		s = m;
	}
}

int bits_for64(int64_t v)
{
	int b = 0;
	while (v) {
		b++;
		v >>= 1;
	}
	return b;
}

}  // namespace

int convert_div(Handle & h)
{
	cudaStream_t s = h.stream;
	const int T = h.desc.num_threads;
	const int L = h.desc.vec_len;
	const int64_t P = h.desc.div_packet_vals;
	const int64_t m = h.m, nnz = h.nnz;
	if (L > DEC_THREADS) {
		set_error(SPMV_ERR_ARG, "DIV-RF: vec_len %d above %d", L, DEC_THREADS);
		return SPMV_ERR_ARG;
	}
	// decoder: 2 = one warp per packet, one lane per lane stream (32 lanes only; the default
	// there); 0 = one CTA per packet, lanes shared by several threads (any lane count)
	h.exec_kernel = h.desc.kernel < 0 ? (L == 32 ? 2 : 0) : h.desc.kernel;
	if (h.exec_kernel != 0 && !(h.exec_kernel == 2 && L == 32)) {
		set_error(SPMV_ERR_ARG, "DIV-RF: kernel %d unavailable (0, or 2 with vec_len 32)", h.desc.kernel);
		return SPMV_ERR_ARG;
	}
	// dropped mantissa bits of the lossy mode (reduce_precision, div_kernels_rf.h:467-510)
	int drop = -1;
	if (h.desc.div_tolerance > 0) {
		const uint64_t prec = (uint64_t) ceil(fabs(log2(h.desc.div_tolerance)));
		if (prec < 52)
			drop = (int) (52 - prec);
	}
	SPMV_TRY(h.alloc(&h.d_ranges, 2 * T));
	SPMV_TRY(h.alloc(&h.d_thread_bytes, T));
	SPMV_TRY(h.alloc(&h.d_thread_groups, T));
	if (m > 0) {
		SPMV_TRY(partition_prefix_sums(h.d_rp, m, nnz, T, h.d_ranges, s));
	} else {
		SPMV_CUDA_TRY(cudaMemsetAsync(h.d_ranges, 0, 2 * T * sizeof(int64_t), s));
	}
	// 1) packet chains
	DevBuf cnt, cnt_ex;
	SPMV_TRY(cnt.alloc(T * sizeof(int64_t), s));
	SPMV_TRY(cnt_ex.alloc((T + 1) * sizeof(int64_t), s));
	const unsigned tg = (unsigned) ceil_div(T, 64);
	if (m > 0) {
		div_chain_kernel<false><<<tg, 64, 0, s>>>(h.d_rp, m, h.d_ranges, T, P, cnt.as<int64_t>(), nullptr, nullptr,
				nullptr, nullptr, nullptr, nullptr);
		SPMV_CUDA_TRY(cudaGetLastError());
	} else {
		SPMV_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, T * sizeof(int64_t), s));
	}
	SPMV_TRY(scan_exclusive(cnt.as<int64_t>(), cnt_ex.as<int64_t>(), T, s));
	int64_t NP = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&NP, cnt_ex.as<int64_t>() + T, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	h.num_packets = NP;
	SPMV_TRY(h.alloc(&h.d_pkt, NP + 1));
	SPMV_TRY(h.alloc(&h.d_pkt_meta, NP));
	if (NP == 0) {
		SPMV_CUDA_TRY(cudaMemsetAsync(h.d_pkt, 0, sizeof(int64_t), s));
		SPMV_CUDA_TRY(cudaMemsetAsync(h.d_thread_bytes, 0, T * sizeof(int64_t), s));
		SPMV_CUDA_TRY(cudaMemsetAsync(h.d_thread_groups, 0, T * sizeof(int64_t), s));
		h.num_group_entries = T;
		SPMV_TRY(h.alloc(&h.d_groups, T));
		SPMV_CUDA_TRY(cudaMemsetAsync(h.d_groups, 0, T * sizeof(int64_t), s));
		SPMV_TRY(h.alloc(&h.d_div, 1));
		h.div_bytes = 0;
		h.kernels_per_run = 0;
		return SPMV_OK;
	}
	DevBuf pk_j, pk_row, pk_nv, pk_grp, pk_thread;
	SPMV_TRY(pk_j.alloc(NP * 4, s));
	SPMV_TRY(pk_row.alloc(NP * 4, s));
	SPMV_TRY(pk_nv.alloc(NP * 4, s));
	SPMV_TRY(pk_grp.alloc(NP, s));
	SPMV_TRY(pk_thread.alloc(NP * 4, s));
	div_chain_kernel<true><<<tg, 64, 0, s>>>(h.d_rp, m, h.d_ranges, T, P, nullptr, cnt_ex.as<int64_t>(),
			pk_j.as<int32_t>(), pk_row.as<int32_t>(), pk_nv.as<int32_t>(), pk_grp.as<uint8_t>(),
			pk_thread.as<int32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());

	// 2) per-entry packet, row, value bits
	DevBuf pkt_of, row_of, val_of, flag;
	SPMV_TRY(pkt_of.alloc(nnz * 4, s));
	SPMV_TRY(row_of.alloc(nnz * 4, s));
	SPMV_TRY(val_of.alloc(nnz * 8, s));
	SPMV_TRY(flag.alloc(sizeof(int), s));
	const unsigned eg = (unsigned) ceil_div(nnz, 256);
	div_entry_kernel<<<eg, 256, 0, s>>>(h.d_rp, h.d_ci, h.d_v, m, nnz, pk_j.as<int32_t>(), NP, drop,
			pkt_of.as<int32_t>(), row_of.as<int32_t>(), val_of.as<uint64_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_CUDA_TRY(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
	cols_unsorted_kernel<<<eg, 256, 0, s>>>(h.d_rp, h.d_ci, row_of.as<int32_t>(), nnz, flag.as<int>());
	SPMV_CUDA_TRY(cudaGetLastError());
	int unsorted = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&unsorted, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));

	// 3) order by (packet, value, row, col): LSD passes
	DevBuf keys, idx;
	SPMV_TRY(keys.alloc(nnz * 8, s));
	SPMV_TRY(idx.alloc(nnz * 4, s));
	iota_kernel<<<eg, 256, 0, s>>>(idx.as<uint32_t>(), nnz);
	SPMV_CUDA_TRY(cudaGetLastError());
	if (unsorted) {
		keys_from_kernel<<<eg, 256, 0, s>>>(idx.as<uint32_t>(), nnz, 0, h.d_ci, nullptr, keys.as<uint64_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
		SPMV_TRY(radix_sort_pairs(keys.as<uint64_t>(), idx.as<uint32_t>(), nnz, 32, s));
		keys_from_kernel<<<eg, 256, 0, s>>>(idx.as<uint32_t>(), nnz, 0, row_of.as<int32_t>(), nullptr,
				keys.as<uint64_t>());
		SPMV_CUDA_TRY(cudaGetLastError());
		SPMV_TRY(radix_sort_pairs(keys.as<uint64_t>(), idx.as<uint32_t>(), nnz, bits_for64(m), s));
	}
	keys_from_kernel<<<eg, 256, 0, s>>>(idx.as<uint32_t>(), nnz, 1, nullptr, val_of.as<uint64_t>(), keys.as<uint64_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(radix_sort_pairs(keys.as<uint64_t>(), idx.as<uint32_t>(), nnz, 64, s));
	keys_from_kernel<<<eg, 256, 0, s>>>(idx.as<uint32_t>(), nnz, 0, pkt_of.as<int32_t>(), nullptr, keys.as<uint64_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(radix_sort_pairs(keys.as<uint64_t>(), idx.as<uint32_t>(), nnz, bits_for64(NP), s));

	// 4) replication factors, then order by (packet, rf) keeping the value order
	DevBuf rflag, rex, run_pos, rf_of;
	SPMV_TRY(rflag.alloc(nnz * 4, s));
	SPMV_TRY(rex.alloc((nnz + 1) * 8, s));
	SPMV_TRY(rf_of.alloc(nnz * 4, s));
	run_flag_kernel<<<eg, 256, 0, s>>>(idx.as<uint32_t>(), nnz, pkt_of.as<int32_t>(), val_of.as<uint64_t>(),
			rflag.as<int32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(scan_exclusive(rflag.as<int32_t>(), rex.as<int64_t>(), nnz, s));
	int64_t nruns = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&nruns, rex.as<int64_t>() + nnz, 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	SPMV_TRY(run_pos.alloc((nruns + 1) * 8, s));
	run_start_kernel<<<eg, 256, 0, s>>>(rflag.as<int32_t>(), rex.as<int64_t>(), nnz, run_pos.as<int64_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	const int rf_bits = bits_for64(P) + 1;
	rf_kernel<<<eg, 256, 0, s>>>(idx.as<uint32_t>(), rflag.as<int32_t>(), rex.as<int64_t>(), run_pos.as<int64_t>(),
			nruns, nnz, pkt_of.as<int32_t>(), rf_bits, rf_of.as<int32_t>(), keys.as<uint64_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(radix_sort_pairs(keys.as<uint64_t>(), idx.as<uint32_t>(), nnz, rf_bits + bits_for64(NP), s));

	// 5) groups of equal (packet, rf)
	DevBuf gflag, gex;
	SPMV_TRY(gflag.alloc(nnz * 4, s));
	SPMV_TRY(gex.alloc((nnz + 1) * 8, s));
	group_flag_kernel<<<eg, 256, 0, s>>>(idx.as<uint32_t>(), nnz, pkt_of.as<int32_t>(), rf_of.as<int32_t>(),
			gflag.as<int32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(scan_exclusive(gflag.as<int32_t>(), gex.as<int64_t>(), nnz, s));
	int64_t G = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&G, gex.as<int64_t>() + nnz, 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	DevBuf g_start, g_pkt, g_rf, g_u, g_ustart, pk_g0;
	SPMV_TRY(g_start.alloc((G + 1) * 8, s));
	SPMV_TRY(g_pkt.alloc(G * 4, s));
	SPMV_TRY(g_rf.alloc(G * 4, s));
	SPMV_TRY(g_u.alloc(G * 8, s));
	SPMV_TRY(g_ustart.alloc((G + 1) * 8, s));
	SPMV_TRY(pk_g0.alloc((NP + 1) * 4, s));
	group_info_kernel<<<eg, 256, 0, s>>>(idx.as<uint32_t>(), gflag.as<int32_t>(), gex.as<int64_t>(), nnz,
			pkt_of.as<int32_t>(), rf_of.as<int32_t>(), G, g_start.as<int64_t>(), g_pkt.as<int32_t>(),
			g_rf.as<int32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	group_unique_kernel<<<(unsigned) ceil_div(G, 256), 256, 0, s>>>(g_start.as<int64_t>(), g_rf.as<int32_t>(), G,
			g_u.as<int64_t>(), g_pkt.as<int32_t>(), pk_g0.as<int32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	{
		int32_t g = (int32_t) G;
		SPMV_CUDA_TRY(cudaMemcpyAsync(pk_g0.as<int32_t>() + NP, &g, 4, cudaMemcpyHostToDevice, s));
	}
	SPMV_TRY(scan_exclusive(g_u.as<int64_t>(), g_ustart.as<int64_t>(), G, s));
	int64_t U = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&U, g_ustart.as<int64_t>() + G, 8, cudaMemcpyDeviceToHost, s));

	// 6) packet geometry
	DevBuf pk_rowmax, pk_colmin, pk_rb, pk_cbb, pk_cbytes, err;
	SPMV_TRY(pk_rowmax.alloc(NP * 4, s));
	SPMV_TRY(pk_colmin.alloc(NP * 4, s));
	SPMV_TRY(pk_rb.alloc(NP, s));
	SPMV_TRY(pk_cbb.alloc(NP, s));
	SPMV_TRY(pk_cbytes.alloc(NP, s));
	SPMV_TRY(err.alloc(sizeof(int), s));
	SPMV_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(int), s));
	packet_meta_kernel<<<(unsigned) ceil_div(NP * 32, 256), 256, 0, s>>>(h.d_rp, h.d_ci, m, pk_j.as<int32_t>(),
			pk_row.as<int32_t>(), pk_nv.as<int32_t>(), NP, pk_rowmax.as<int32_t>(), pk_colmin.as<int32_t>(),
			pk_rb.as<uint8_t>(), pk_cbb.as<uint8_t>(), pk_cbytes.as<uint8_t>(), err.as<int>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));

	// 7) unique values: delta codes, byte offsets
	DevBuf u_code, u_nb, u_pay, S, gl_base, pk_lt, pk_lanes, pk_size;
	SPMV_TRY(u_code.alloc(U + 1, s));
	SPMV_TRY(u_nb.alloc((U + 1) * 4, s));
	SPMV_TRY(u_pay.alloc((U + 1) * 8, s));
	SPMV_TRY(S.alloc((U + 1) * 8, s));
	SPMV_TRY(gl_base.alloc(G * L * 8, s));
	SPMV_TRY(pk_lt.alloc(NP * 8, s));
	SPMV_TRY(pk_lanes.alloc(NP * L * 4, s));
	SPMV_TRY(pk_size.alloc(NP * 8, s));
	unique_kernel<<<(unsigned) ceil_div(U, 256), 256, 0, s>>>(idx.as<uint32_t>(), val_of.as<uint64_t>(),
			g_start.as<int64_t>(), g_rf.as<int32_t>(), g_u.as<int64_t>(), g_ustart.as<int64_t>(), G, U, L,
			u_code.as<uint8_t>(), u_nb.as<int32_t>(), u_pay.as<uint64_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(scan_exclusive(u_nb.as<int32_t>(), S.as<int64_t>(), U, s));
	lane_layout_kernel<<<(unsigned) ceil_div(NP, 128), 128, 0, s>>>(pk_g0.as<int32_t>(), NP, g_u.as<int64_t>(),
			g_ustart.as<int64_t>(), S.as<int64_t>(), L, gl_base.as<int64_t>(), pk_lt.as<int64_t>(),
			pk_lanes.as<uint32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	packet_size_kernel<<<(unsigned) ceil_div(NP, 256), 256, 0, s>>>(pk_g0.as<int32_t>(), pk_nv.as<int32_t>(),
			pk_cbytes.as<uint8_t>(), g_ustart.as<int64_t>(), pk_lt.as<int64_t>(), NP, L, pk_size.as<int64_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(scan_exclusive(pk_size.as<int64_t>(), h.d_pkt, NP, s));
	int64_t total = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&total, h.d_pkt + NP, 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	h.div_bytes = total;
	SPMV_TRY(h.alloc(&h.d_div, total + 16));     // 16 bytes of pad: the decoder reads whole words

	// 8) scatter the bytes
	header_kernel<<<(unsigned) ceil_div(NP, 128), 128, 0, s>>>(h.d_pkt, pk_g0.as<int32_t>(), pk_nv.as<int32_t>(),
			pk_row.as<int32_t>(), pk_rowmax.as<int32_t>(), pk_colmin.as<int32_t>(), pk_rb.as<uint8_t>(),
			pk_cbb.as<uint8_t>(), g_ustart.as<int64_t>(), g_u.as<int64_t>(), g_rf.as<int32_t>(),
			pk_lanes.as<uint32_t>(), NP, L, h.d_div);
	SPMV_CUDA_TRY(cudaGetLastError());
	coords_kernel<<<eg, 256, 0, s>>>(idx.as<uint32_t>(), nnz, pkt_of.as<int32_t>(), row_of.as<int32_t>(), h.d_ci,
			gflag.as<int32_t>(), gex.as<int64_t>(), g_start.as<int64_t>(), g_rf.as<int32_t>(), g_u.as<int64_t>(),
			pk_j.as<int32_t>(), pk_row.as<int32_t>(), pk_colmin.as<int32_t>(), pk_rb.as<uint8_t>(),
			pk_cbytes.as<uint8_t>(), pk_g0.as<int32_t>(), h.d_pkt, L, h.d_div);
	SPMV_CUDA_TRY(cudaGetLastError());
	values_kernel<<<(unsigned) ceil_div(U, 256), 256, 0, s>>>(g_start.as<int64_t>(), g_pkt.as<int32_t>(),
			g_u.as<int64_t>(), g_ustart.as<int64_t>(), G, U, pk_g0.as<int32_t>(), pk_nv.as<int32_t>(),
			pk_cbytes.as<uint8_t>(), h.d_pkt, gl_base.as<int64_t>(), S.as<int64_t>(), u_code.as<uint8_t>(),
			u_nb.as<int32_t>(), u_pay.as<uint64_t>(), L, h.d_div);
	SPMV_CUDA_TRY(cudaGetLastError());

	// 9) packet groups per reference thread (export) and thread byte counts
	DevBuf th_first, g32, gex2, gbase;
	SPMV_TRY(th_first.alloc((T + 1) * 8, s));
	SPMV_TRY(g32.alloc(NP * 4, s));
	SPMV_TRY(gex2.alloc((NP + 1) * 8, s));
	SPMV_TRY(gbase.alloc((T + 1) * 8, s));
	thread_first_kernel<<<(unsigned) ceil_div(T + 1, 64), 64, 0, s>>>(cnt_ex.as<int64_t>(), T, th_first.as<int64_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	grp_i32_kernel<<<(unsigned) ceil_div(NP, 256), 256, 0, s>>>(pk_grp.as<uint8_t>(), NP, g32.as<int32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(scan_exclusive(g32.as<int32_t>(), gex2.as<int64_t>(), NP, s));
	grp_base_kernel<<<(unsigned) ceil_div(T + 1, 64), 64, 0, s>>>(gex2.as<int64_t>(), th_first.as<int64_t>(), T,
			gbase.as<int64_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	int64_t ngroups = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&ngroups, gex2.as<int64_t>() + NP, 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	h.num_group_entries = ngroups + T;
	SPMV_TRY(h.alloc(&h.d_groups, h.num_group_entries));
	groups_kernel<<<(unsigned) ceil_div(NP > T ? NP : T, 256), 256, 0, s>>>(h.d_pkt, pk_grp.as<uint8_t>(),
			pk_thread.as<int32_t>(), th_first.as<int64_t>(), NP, T, gex2.as<int64_t>(), gbase.as<int64_t>(),
			h.d_groups, h.d_thread_bytes, h.d_thread_groups, total);
	SPMV_CUDA_TRY(cudaGetLastError());

	// 10) SpMV metadata: rows to store / zero per packet, rows split across packets
	DevBuf split_flag, split_ex;
	SPMV_TRY(split_flag.alloc(NP * 4, s));
	SPMV_TRY(split_ex.alloc((NP + 1) * 8, s));
	spmv_meta_kernel<<<(unsigned) ceil_div(NP, 256), 256, 0, s>>>(h.d_rp, m, pk_j.as<int32_t>(), pk_nv.as<int32_t>(),
			pk_row.as<int32_t>(), pk_rowmax.as<int32_t>(), NP, h.d_pkt_meta, split_flag.as<int32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(scan_exclusive(split_flag.as<int32_t>(), split_ex.as<int64_t>(), NP, s));
	int64_t nsplit = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&nsplit, split_ex.as<int64_t>() + NP, 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	h.num_split = nsplit;
	SPMV_TRY(h.alloc(&h.d_split_rows, nsplit));
	if (nsplit > 0) {
		split_rows_kernel<<<(unsigned) ceil_div(NP, 256), 256, 0, s>>>(split_flag.as<int32_t>(), split_ex.as<int64_t>(),
				pk_rowmax.as<int32_t>(), NP, h.d_split_rows);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	int e = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	if (e) {
		set_error(SPMV_ERR_BOUNDS, "DIV-RF: a packet needs more than 8 row bits or 32 column bits");
		return SPMV_ERR_BOUNDS;
	}
	h.kernels_per_run = nsplit > 0 ? 2 : 1;
	if (!h.desc.div_packet_reordering)
		return SPMV_OK;

	// 11) packet reordering: medians on the GPU, group order on the host, bytes moved on the GPU
	DevBuf rk, rv, med;
	SPMV_TRY(rk.alloc(nnz * 8, s));
	SPMV_TRY(rv.alloc(nnz * 4, s));
	SPMV_TRY(med.alloc(NP * 8, s));
	pkt_col_keys_kernel<<<eg, 256, 0, s>>>(pkt_of.as<int32_t>(), h.d_ci, nnz, rk.as<uint64_t>(), rv.as<uint32_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(radix_sort_pairs(rk.as<uint64_t>(), rv.as<uint32_t>(), nnz, 32 + bits_for64(NP), s));
	pkt_median_kernel<<<(unsigned) ceil_div(NP, 256), 256, 0, s>>>(rk.as<uint64_t>(), pk_j.as<int32_t>(),
			pk_nv.as<int32_t>(), NP, med.as<int64_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	std::vector<int64_t> hmed((size_t) NP), hoff((size_t) NP + 1), hfirst((size_t) T + 1), hgroups((size_t) h.num_group_entries),
			hbytes((size_t) T), hng((size_t) T);
	std::vector<uint8_t> hgrp((size_t) NP);
	SPMV_CUDA_TRY(cudaMemcpyAsync(hmed.data(), med.p, NP * 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaMemcpyAsync(hoff.data(), h.d_pkt, (NP + 1) * 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaMemcpyAsync(hfirst.data(), th_first.p, (T + 1) * 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaMemcpyAsync(hgroups.data(), h.d_groups, h.num_group_entries * 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaMemcpyAsync(hbytes.data(), h.d_thread_bytes, T * 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaMemcpyAsync(hng.data(), h.d_thread_groups, T * 8, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaMemcpyAsync(hgrp.data(), pk_grp.p, NP, cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	std::vector<int64_t> plan, new_groups((size_t) h.num_group_entries);
	int64_t gbase_t = 0, tbase = 0;
	for (int t = 0; t < T; t++) {
		const int64_t G = hng[(size_t) t];
		const int64_t * go = &hgroups[(size_t) gbase_t];        // G + 1 offsets, relative to the thread's stream
		const int64_t p0 = hfirst[(size_t) t], p1 = hfirst[(size_t) t + 1];
		std::vector<int> key((size_t) (G > 0 ? G : 1)), rev((size_t) (G > 0 ? G : 1));
		for (int64_t k = 0; k < G; k++) {
			key[(size_t) k] = (int) hmed[(size_t) (p0 + k)];        // the median of the thread's k-th packet
			rev[(size_t) k] = (int) k;
		}
		ref_quicksort(rev.data(), (long) G, key.data());
		std::vector<int64_t> newpos((size_t) G + 1), dest_of((size_t) (G > 0 ? G : 1));
		int64_t run = 0;
		for (int64_t k = 0; k < G; k++) {
			const int64_t g = rev[(size_t) k];
			newpos[(size_t) k] = run;
			dest_of[(size_t) g] = run;
			plan.push_back(tbase + go[g]);
			plan.push_back(tbase + run);
			plan.push_back(go[g + 1] - go[g]);
			run += go[g + 1] - go[g];
		}
		newpos[(size_t) G] = run;
		for (int64_t k = 0; k <= G; k++)
			new_groups[(size_t) (gbase_t + k)] = newpos[(size_t) k];
		// every packet moves with its group
		int64_t g = -1;
		for (int64_t p = p0; p < p1; p++) {
			if (hgrp[(size_t) p] || g < 0)
				g++;
			hoff[(size_t) p] = tbase + dest_of[(size_t) g] + (hoff[(size_t) p] - tbase - go[g]);
		}
		gbase_t += G + 1;
		tbase += hbytes[(size_t) t];
	}
	const int64_t nplan = (int64_t) plan.size() / 3;
	if (nplan > 0) {
		DevBuf dplan, old;
		SPMV_TRY(dplan.alloc(plan.size() * 8, s));
		SPMV_TRY(old.alloc(total + 16, s));
		SPMV_CUDA_TRY(cudaMemcpyAsync(dplan.p, plan.data(), plan.size() * 8, cudaMemcpyHostToDevice, s));
		SPMV_CUDA_TRY(cudaMemcpyAsync(old.p, h.d_div, total + 16, cudaMemcpyDeviceToDevice, s));
		move_groups_kernel<<<(unsigned) nplan, 256, 0, s>>>(old.as<uint8_t>(), h.d_div, dplan.as<int64_t>(), nplan);
		SPMV_CUDA_TRY(cudaGetLastError());
		SPMV_CUDA_TRY(cudaMemcpyAsync(h.d_pkt, hoff.data(), (NP + 1) * 8, cudaMemcpyHostToDevice, s));
		SPMV_CUDA_TRY(cudaMemcpyAsync(h.d_groups, new_groups.data(), h.num_group_entries * 8, cudaMemcpyHostToDevice, s));
		SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	}
	return SPMV_OK;
}

int launch_div(Handle & h, const double * d_x, double * d_y, cudaStream_t s)
{
	if (h.num_packets == 0) {
		if (h.m > 0)
			SPMV_CUDA_TRY(cudaMemsetAsync(d_y, 0, h.m * sizeof(double), s));
		return SPMV_OK;
	}
	if (h.num_split > 0) {
		zero_rows_kernel<<<(unsigned) ceil_div(h.num_split, 256), 256, 0, s>>>(h.d_split_rows, h.num_split, d_y);
		SPMV_CUDA_TRY(cudaGetLastError());
	}
	DivArgs a;
	a.data = h.d_div;
	a.pkt_off = h.d_pkt;
	a.meta = h.d_pkt_meta;
	a.npackets = h.num_packets;
	a.L = h.desc.vec_len;
	// block_nnz: the warp decoder's prefetch distance in positions (rounded up to 4); stages 1:
	// neither decoder prefetches
	a.pf = h.desc.stages == 1 ? 0 : h.desc.block_nnz > 0 ? (int) ((h.desc.block_nnz + 3) & ~3) : 8;
	a.x = d_x;
	a.y = d_y;
	if (h.exec_kernel == 2) {
		// code bytes and coordinates prefetched into L1 a.pf positions ahead (stages 1: not);
		// ctas_per_sm 4: the form held to 64 registers
		const unsigned g = (unsigned) ceil_div(h.num_packets, DIVW_WARPS);
		if (h.desc.stages == 1)
			div_warp_kernel<0, 3><<<g, DIVW_WARPS * 32, 0, s>>>(a);
		else if (h.desc.stages == 4)            // into L2 instead of L1
			div_warp_kernel<2, 3><<<g, DIVW_WARPS * 32, 0, s>>>(a);
		else if (h.desc.ctas_per_sm == 4)
			div_warp_kernel<1, 4><<<g, DIVW_WARPS * 32, 0, s>>>(a);
		else
			div_warp_kernel<1, 3><<<g, DIVW_WARPS * 32, 0, s>>>(a);
	} else {
		div_spmv_kernel<<<(unsigned) h.num_packets, DEC_THREADS, 0, s>>>(a);
	}
	SPMV_CUDA_TRY(cudaGetLastError());
	return SPMV_OK;
}

}  // namespace spmv
