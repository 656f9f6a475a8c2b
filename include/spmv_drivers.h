/*
 * spmv_drivers.h — the per-format benchmark drivers of clSpMV with their
 * reference signatures (include/spmv_csr_scalar.h, spmv_csr_vector.h,
 * spmv_coo.h, spmv_dia.h, spmv_bdia.h, spmv_ell.h, spmv_sell.h,
 * spmv_bell.h, spmv_sbell.h, spmv_bcsr.h, mem_bandwidth.h), one header for
 * all of them.
 *
 * Each driver converts `mat` to its format for every variant the reference
 * sweeps, checks one SpMV against the host COO product, times `ntimes`
 * SpMVs with CUDA events and prints the reference's report lines (best
 * time, GFLOP/s, best variant). `oclfilename` and `deviceType` are
 * accepted and ignored (the kernels are compiled into the library and run
 * on the current CUDA device); `dim2Size` is ignored as well (it set the
 * second NDRange dimension of the OpenCL launches). Errors are printed,
 * never exit(); clspmv_run_method_f32 in clspmv_b200.h returns them with
 * the timings instead.
 */
#ifndef CLSPMV_SPMV_DRIVERS_H
#define CLSPMV_SPMV_DRIVERS_H

#include "cl_compat.h"
#include "matrix_storage.h"

void spmv_csr_scalar(char* oclfilename, coo_matrix<int, float>* mat, int dim2Size, int ntimes, cl_device_type deviceType);
void spmv_csr_vector(char* oclfilename, coo_matrix<int, float>* mat, int dim2Size, int ntimes, cl_device_type deviceType);
void spmv_coo(char* oclfilename, coo_matrix<int, float>* mat, int dim2Size, int ntimes, cl_device_type deviceType);
void spmv_dia(char* oclfilename, coo_matrix<int, float>* mat, int dim2Size, int ntimes, cl_device_type deviceType);
void spmv_bdia(char* oclfilename, coo_matrix<int, float>* mat, int dim2Size, int ntimes, cl_device_type deviceType);
void spmv_ell(char* oclfilename, coo_matrix<int, float>* mat, int dim2Size, int ntimes, cl_device_type deviceType);
void spmv_sell(char* oclfilename, coo_matrix<int, float>* mat, int dim2Size, int ntimes, cl_device_type deviceType);
void spmv_bell(char* oclfilename, coo_matrix<int, float>* mat, int dim2Size, int ntimes, cl_device_type deviceType);
void spmv_sbell(char* oclfilename, coo_matrix<int, float>* mat, int dim2Size, int ntimes, cl_device_type deviceType);
void spmv_bcsr(char* oclfilename, coo_matrix<int, float>* mat, int dim2Size, int ntimes, cl_device_type deviceType);
/* method 0 of spmv_all: copy bandwidth and launch overhead */
void bandwidth_test(char* oclfilename, cl_device_type deviceType, int dim2Size);

#endif /* CLSPMV_SPMV_DRIVERS_H */
