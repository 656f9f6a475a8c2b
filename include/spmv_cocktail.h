/*
 * spmv_cocktail.h — the Cocktail runtime API of clSpMV
 * (include/spmv_cocktail.h, src/spmv_cocktail.cpp) with its reference
 * names and signatures, on top of the opaque clspmv_cocktail_handle of
 * clspmv_b200.h. Implemented in libclspmv_b200 (csrc/compat.cpp).
 *
 * What is kept: the call sequence of src/eval.cpp (init_mat_kernels, then
 * cpy_* and do_spmv any number of times, then free_mat_kernels), the
 * members callers touch (gpumat.vec, gpumat.res, kernels.context,
 * kernels.cmdQueue, the ifuse* flags) and the semantics: every do_spmv
 * computes res = A * vec + res and returns when the GPU is done (the
 * reference ends each call with clFinish).
 *
 * What differs: a cl_mem here is a CUDA device pointer to float and
 * kernels.cmdQueue is the CUDA stream the calls are ordered on (created by
 * init_mat_kernels). The per-part cl_mem and cl_kernel members of the
 * reference structs are gone (the parts live in the handle), and so are the
 * image copies of x that `use_tex` asked for (the kernels read x through
 * the read-only data cache instead). The void functions print a message on
 * an error instead of exit(1); cocktail_last_status() returns the status of
 * the last call.
 */
#ifndef CLSPMV_SPMV_COCKTAIL_H
#define CLSPMV_SPMV_COCKTAIL_H

#include "analyze.h"
#include "cl_compat.h"
#include "clspmv_b200.h"

struct cocktail_gpu {
    cl_mem vec;        /* device x, mat_width floats  */
    cl_mem res;        /* device y, mat_height floats */
    int vec_size;
    int res_size;
    clspmv_cocktail_handle* handle;
    bool ifusebdia, ifusedia, ifusesbell, ifusebell, ifusebcsr, ifusesell, ifuseell, ifusecsr, ifusecoo;
};

struct cocktail_kernels {
    cl_context context;          /* unused, NULL */
    cl_command_queue cmdQueue;   /* cudaStream_t of all calls */
    clspmv_cocktail_handle* handle;
    cl_mem vec;
    cl_mem res;
    long long nnz;
};

void init_cocktail_gpu(cocktail_gpu& mat);
void free_cocktail_gpu(cocktail_gpu& mat);
void init_cocktail_kernels(cocktail_kernels& cocktail);
void free_cocktail_kernels(cocktail_kernels& cocktail);

/* Uploads the parts of `cpumat`, x = vec and y = res (src/spmv_cocktail.cpp:1590-1611). */
void init_mat_kernels(cocktail<int, int, float>& cpumat, float* vec, float* res, cocktail_gpu& gpumat,
                      cocktail_kernels& kernels, bool use_tex);
/* Releases the device parts, x, y and the stream (:1613-1618). */
void free_mat_kernels(cocktail_gpu& gpumat, cocktail_kernels& kernels);
/* `ntimes` SpMVs res = A*vec + res, then waits for the GPU (:1088-1132). */
void do_spmv(cocktail_kernels& kernels, cl_context& context, cl_command_queue& cmdQueue, int ntimes);

/* x from host memory / from a device buffer; y from host / from device;
 * y to host / to a device buffer (:1459-1587). Each waits for the copy. */
void cpy_vector_from_cpu(cocktail_gpu& gpumat, cl_context& context, cl_command_queue& cmdQueue, float* vec, int vec_size);
void cpy_vector_from_gpu(cocktail_gpu& gpumat, cl_context& context, cl_command_queue& cmdQueue, cl_mem vec, int vec_size);
void cpy_result_from_cpu(cocktail_gpu& gpumat, cl_context& context, cl_command_queue& cmdQueue, float* res, int res_size);
void cpy_result_from_gpu(cocktail_gpu& gpumat, cl_context& context, cl_command_queue& cmdQueue, cl_mem res, int res_size);
void cpy_result_to_cpu(cocktail_gpu& gpumat, cl_context& context, cl_command_queue& cmdQueue, float* res, int res_size);
void cpy_result_to_gpu(cocktail_gpu& gpumat, cl_context& context, cl_command_queue& cmdQueue, cl_mem res, int res_size);

/* One SpMV from `result` checked against `coores`, then 1000 timed SpMVs
 * (:1134-1154). */
void check_and_time(cocktail_gpu& gpumat, cocktail_kernels& kernels, cl_context& context, cl_command_queue& cmdQueue,
                    float* result, float* coores, int res_size, int nnz);
/* Prints which parts the partitioner chose and their sizes (:1351-1429). */
void output_cocktail_info(cocktail<int, int, float>& cpumat);
/* output_cocktail_info, upload, check_and_time, release (:1431-1455). */
void evaluate(cocktail<int, int, float>& cpumat, float* vec, float* res, float* coores);

/* Status of the last call above (CLSPMV_OK or a clspmv_status). */
int cocktail_last_status(void);

#endif /* CLSPMV_SPMV_COCKTAIL_H */
