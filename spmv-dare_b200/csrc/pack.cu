// Packed column indices of the staged blocks (a device-side copy; the exported CSR keeps the
// reference's int32 columns).
//
// A staged block covers the consecutive CSR entries [elem0, elem0 + elems).  Its columns
// are stored as (column - base) in `bits` bits each, base = the block's smallest column and
// bits = the width of (largest - smallest), little-endian in 32-bit words: entry e's field
// starts at bit e * bits of the block's stream.  Each stream starts on a 16-byte boundary
// (the bulk-copy unit) and carries one spare word past its last field, so a field is always
// read as two whole words and a funnel shift.  On the 4M-row configuration a block of 1,536
// entries spans about 200k columns: 18 bits an entry instead of 32.
#include "internal.h"
#include "primitives.cuh"

namespace spmv {

namespace {

__device__ __forceinline__ int width_of(uint32_t v)
{
	return v ? 32 - __clz(v) : 0;
}

// one warp per block: smallest and largest column, field width, stream size in 16-byte units
__global__ void pack_size_kernel(const StagedBlock * blocks, int64_t nb, const int32_t * ci, int4 * info,
		int64_t * units16)
{
	const int64_t b = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (b >= nb)
		return;
	const StagedBlock d = blocks[b];
	int32_t lo = INT32_MAX, hi = INT32_MIN;
	for (int e = lane; e < d.elems; e += 32) {
		const int32_t c = ci[(int64_t) d.elem0 + e];
		lo = min(lo, c);
		hi = max(hi, c);
	}
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
		hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
	}
	if (lane == 0) {
		if (d.elems == 0) {
			lo = 0;
			hi = 0;
		}
		const int bits = width_of((uint32_t) (hi - lo));
		const int64_t words = ((int64_t) d.elems * bits + 31) / 32 + 1;     // one spare word
		const int64_t u16 = (words + 3) / 4;
		info[b] = make_int4(0, lo, bits, (int) (u16 * 16));
		units16[b] = u16;
	}
}

// one CTA per block: word w of its stream holds the fields of entries e with
// e * bits in [32 w - bits + 1, 32 w + 32)
__global__ void pack_words_kernel(const StagedBlock * blocks, int64_t nb, const int32_t * ci, int4 * info,
		const int64_t * off16, uint32_t * out)
{
	const int64_t b = blockIdx.x;
	if (b >= nb)
		return;
	const StagedBlock d = blocks[b];
	int4 pi = info[b];
	const int64_t o = off16[b];
	if (threadIdx.x == 0) {
		pi.x = (int) o;
		info[b] = pi;
	}
	const int bits = pi.z, words = pi.w / 4;
	uint32_t * w0 = out + o * 4;
	for (int w = threadIdx.x; w < words; w += blockDim.x) {
		uint32_t acc = 0;
		if (bits > 0) {
			const int64_t bit0 = (int64_t) w * 32;
			int64_t e = bit0 / bits;
			for (; e < d.elems && e * bits < bit0 + 32; e++) {
				const uint64_t f = (uint64_t) (uint32_t) (ci[(int64_t) d.elem0 + e] - pi.y);
				const int64_t sh = e * bits - bit0;          // > -bits, < 32
				acc |= sh >= 0 ? (uint32_t) (f << sh) : (uint32_t) (f >> -sh);
			}
		}
		w0[w] = acc;
	}
}

}  // namespace

int build_packed_cols(Handle & h)
{
	cudaStream_t s = h.stream;
	const int64_t nb = h.num_blocks;
	SPMV_TRY(h.alloc(&h.d_pinfo, nb > 0 ? nb : 1));
	if (nb == 0) {
		SPMV_TRY(h.alloc(&h.d_pcols, 4));
		return SPMV_OK;
	}
	DevBuf u16, off;
	SPMV_TRY(u16.alloc(nb * sizeof(int64_t), s));
	SPMV_TRY(off.alloc((nb + 1) * sizeof(int64_t), s));
	pack_size_kernel<<<(unsigned) ceil_div(nb * 32, 256), 256, 0, s>>>(h.d_blocks, nb, h.d_ci, h.d_pinfo,
			u16.as<int64_t>());
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_TRY(scan_exclusive(u16.as<int64_t>(), off.as<int64_t>(), nb, s));
	int64_t total16 = 0;
	SPMV_CUDA_TRY(cudaMemcpyAsync(&total16, off.as<int64_t>() + nb, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	if (total16 > INT32_MAX) {
		set_error(SPMV_ERR_OVERFLOW, "packed columns: %lld bytes beyond the 32-bit offset range", (long long) total16 * 16);
		return SPMV_ERR_OVERFLOW;
	}
	SPMV_TRY(h.alloc(&h.d_pcols, total16 * 4 + 4));
	h.packed_bytes = total16 * 16;
	pack_words_kernel<<<(unsigned) nb, 128, 0, s>>>(h.d_blocks, nb, h.d_ci, h.d_pinfo, off.as<int64_t>(), h.d_pcols);
	SPMV_CUDA_TRY(cudaGetLastError());
	SPMV_CUDA_TRY(cudaStreamSynchronize(s));
	return SPMV_OK;
}

}  // namespace spmv
