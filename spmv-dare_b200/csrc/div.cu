// DIV-RF: GPU packetiser and decoder (filled in below).
#include "internal.h"

namespace spmv {

int convert_div(Handle & h)
{
	(void) h;
	set_error(SPMV_ERR_UNSUPPORTED, "DIV-RF is not built yet");
	return SPMV_ERR_UNSUPPORTED;
}

int launch_div(Handle & h, const double * d_x, double * d_y, cudaStream_t s)
{
	(void) h; (void) d_x; (void) d_y; (void) s;
	set_error(SPMV_ERR_UNSUPPORTED, "DIV-RF is not built yet");
	return SPMV_ERR_UNSUPPORTED;
}

}  // namespace spmv
