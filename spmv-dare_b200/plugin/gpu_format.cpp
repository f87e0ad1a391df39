/*
 * Drop-in plugin: one GPU format behind the reference's Matrix_Format API
 * (src/spmv_kernels/spmv_kernel.h:8-29), forwarding to libspmv_b200.so's C ABI.
 *
 * Built like any reference format translation unit (one executable per format,
 * src/Makefile_in:47-74), with -DGPU_FORMAT_ID=<SPMV_FMT_*>, against the reference's own
 * bench driver (src/bench.cpp, src/bench_spmv.cpp), which then runs unchanged:
 *   csr_to_format()            -> spmv_create()   (validation + conversion on the GPU)
 *   Matrix_Format::spmv(x, y)  -> spmv_run()      (x, y are the bench's host buffers)
 *   statistics_print_labels / statistics_print_data -> the GPU statistics columns.
 * Errors keep the reference's behaviour: print and exit (error(), e.g. csr.cpp:131-132).
 *
 * Environment (config.sh:67-159 contract, plus the GPU knobs):
 *   CSRCV_NUM_PACKET_VALS, DIV_VC_TOLERANCE, DIV_PACKET_REORDERING   DIV-RF packet size /
 *                                             lossy tolerance / packet-group order
 *   SPMV_GPU_VEC_LEN, SPMV_GPU_SELLCS_C, SPMV_GPU_SELLCS_SIGMA, SPMV_GPU_EXACT,
 *   SPMV_GPU_BLOCK_NNZ, SPMV_GPU_STAGES, SPMV_GPU_THREADS, SPMV_GPU_KERNEL
 * The thread count that defines the reference layouts is omp_get_max_threads(), as in
 * every reference format.
 */
#include <stdlib.h>
#include <stdio.h>
#include <string.h>
#include <omp.h>

#include "macros/cpp_defines.h"

#include "spmv_kernel.h"

#ifdef __cplusplus
extern "C" {
#endif
	#include "macros/macrolib.h"
#ifdef __cplusplus
}
#endif

#include "spmv_b200.h"

#ifndef GPU_FORMAT_ID
	#error "define GPU_FORMAT_ID (SPMV_FMT_CSR_NAIVE, SPMV_FMT_SELL_C_S, ...)"
#endif

static long env_long(const char * name, long dflt)
{
	const char * v = getenv(name);
	return (v && *v) ? atol(v) : dflt;
}

static double env_double(const char * name, double dflt)
{
	const char * v = getenv(name);
	return (v && *v) ? atof(v) : dflt;
}

struct GPU_Format : Matrix_Format
{
	spmv_handle * h;
	char name[64];

	GPU_Format(long m, long n, long nnz) : Matrix_Format(m, n, nnz), h(NULL)
	{
		name[0] = 0;
	}

	~GPU_Format()
	{
		spmv_destroy(h);
	}

	void spmv(ValueType * x, ValueType * y)
	{
		int st;
#if DOUBLE == 1
		st = spmv_run(h, x, y);
#else
		st = spmv_run_f32(h, x, y);
#endif
		if (st != SPMV_OK)
			error("spmv_b200: %s", spmv_last_error());
	}

	void statistics_start()
	{
	}

	int statistics_print_data(char * buf, long buf_n)
	{
		return spmv_statistics_print_data(h, buf, buf_n);
	}
};


struct Matrix_Format *
csr_to_format(INT_T * row_ptr, INT_T * col_ind, ValueTypeReference * values, long m, long n, long nnz, long symmetric, long symmetry_expanded)
{
	// this translation unit's structs must be the library's (a stale build of either side
	// would read or write past them)
	if (spmv_format_desc_size() != sizeof(spmv_format_desc) || spmv_info_size() != sizeof(spmv_info))
		error("spmv_b200: header and library differ (spmv_format_desc %zu / %zu bytes, spmv_info %zu / %zu): rebuild",
				sizeof(spmv_format_desc), spmv_format_desc_size(), sizeof(spmv_info), spmv_info_size());
	spmv_format_desc d;
	spmv_format_desc_init(&d, GPU_FORMAT_ID);
	d.num_threads = omp_get_max_threads();
	d.vec_len = (int32_t) env_long("SPMV_GPU_VEC_LEN", d.vec_len);
	d.sellcs_c = (int32_t) env_long("SPMV_GPU_SELLCS_C", d.sellcs_c);
	d.sellcs_sigma = (int32_t) env_long("SPMV_GPU_SELLCS_SIGMA", d.sellcs_sigma);
	d.div_packet_vals = (int32_t) env_long("CSRCV_NUM_PACKET_VALS", d.div_packet_vals);
	d.div_tolerance = env_double("DIV_VC_TOLERANCE", d.div_tolerance);
	d.div_packet_reordering = (int32_t) env_long("DIV_PACKET_REORDERING", 0);
	d.exact = (int32_t) env_long("SPMV_GPU_EXACT", d.exact);
	d.block_nnz = (int32_t) env_long("SPMV_GPU_BLOCK_NNZ", 0);
	d.stages = (int32_t) env_long("SPMV_GPU_STAGES", 0);
	d.threads = (int32_t) env_long("SPMV_GPU_THREADS", 0);
	d.kernel = (int32_t) env_long("SPMV_GPU_KERNEL", d.kernel);
#if DOUBLE == 0
	d.values = SPMV_VALUES_F32;
#endif
	int st = SPMV_OK;
	spmv_handle * h = spmv_create(row_ptr, col_ind, values, m, n, nnz, symmetric, symmetry_expanded, &d, &st);
	if (h == NULL)
		error("spmv_b200: %s", spmv_last_error());
	GPU_Format * f = new GPU_Format(m, n, nnz);
	f->h = h;
	spmv_info info;
	spmv_get_info(h, &info);
	snprintf(f->name, sizeof(f->name), "%s", info.format_name);
	f->format_name = f->name;
	f->mem_footprint = info.mem_footprint;
	return f;
}


int
statistics_print_labels(char * buf, long buf_n)
{
	return spmv_statistics_print_labels(buf, buf_n);
}
