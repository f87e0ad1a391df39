// FP32 variant (filled in below).
#include "internal.h"

namespace spmv {

int launch_spmv_f32(Handle & h, const float * d_x, float * d_y, cudaStream_t s)
{
	(void) h; (void) d_x; (void) d_y; (void) s;
	set_error(SPMV_ERR_UNSUPPORTED, "FP32 variant is not built yet");
	return SPMV_ERR_UNSUPPORTED;
}

}  // namespace spmv
