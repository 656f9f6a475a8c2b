/*
 * clspmv_b200.h — C ABI of the B200 SpMV library (libclspmv_b200.so).
 *
 * Plain C: no CUDA or torch types appear here. Device pointers are plain
 * pointers, streams are passed as `clspmv_stream_t` (a cudaStream_t cast to
 * void*; NULL means the legacy default stream).
 *
 * Semantics of every SpMV entry point: y <- alpha * A * x + beta * y, FP32
 * values, int32 indices. The reference clSpMV kernels all compute
 * y <- A*x + y (they read `result` before accumulating, e.g.
 * kernels/spmv_ell.cl:7, kernels/spmv_coo.cl:43), which is alpha = beta = 1.
 * beta == 0 never reads y (BLAS convention).
 *
 * The format structs below are layout-identical to the reference's C++
 * templates instantiated with dimType = offsetType = int, dataType = float
 * (include/matrix_storage.h:15-365 of clSpMV), so a `coo_matrix<int,float>*`
 * may be passed where a `clspmv_coo_f32*` is expected. The same struct type is
 * used for host copies (converter outputs) and device copies (upload outputs):
 * only where the pointers point differs.
 *
 * Every function returns a clspmv_status (0 = success) and never exits the
 * process; the reference instead calls exit(1) from CHECKERROR
 * (include/oclcommon.h:11).
 */
#ifndef CLSPMV_B200_H
#define CLSPMV_B200_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef void* clspmv_stream_t;

typedef enum {
    CLSPMV_OK = 0,
    CLSPMV_ERR_ARG = 1,         /* null pointer, negative size, bad shape     */
    CLSPMV_ERR_ALLOC = 2,       /* host or device allocation failed           */
    CLSPMV_ERR_UNSUPPORTED = 3, /* block shape / slice height not supported   */
    CLSPMV_ERR_CUDA = 4,        /* a CUDA runtime call failed                 */
    CLSPMV_ERR_REFUSED = 5,     /* the reference converter refuses this input */
    CLSPMV_ERR_ALIGN = 6,       /* pointer or aligned length not 16-byte able */
    CLSPMV_ERR_NOT_SORTED = 7,  /* COO input must be sorted by (row, col)     */
    CLSPMV_ERR_TIMEOUT = 8      /* a bounded device wait ran out              */
} clspmv_status;

/* Reference constants (include/constant.h:7-45 of clSpMV). */
#define CLSPMV_GPU_ALIGNMENT 32
#define CLSPMV_COO_ALIGNMENT 32
#define CLSPMV_MAX_MEM_OBJ 268435456
#define CLSPMV_MAX_DIA_NUM 128
#define CLSPMV_MAX_BAND_NUM 31
#define CLSPMV_MAX_BAND_WIDTH 128
#define CLSPMV_WARPSIZE 32
#define CLSPMV_SELL_GROUP_SIZE 128

/* matrixInfo<int>: include/matrix_storage.h:15-25 */
typedef struct { int width; int height; int nnz; } clspmv_matinfo;

/* coo_matrix<int,float>: include/matrix_storage.h:141-152 */
typedef struct {
    clspmv_matinfo matinfo;
    int* coo_row_id; int* coo_col_id; float* coo_data;
} clspmv_coo_f32;

/* csr_matrix<int,float>: include/matrix_storage.h:155-166 */
typedef struct {
    clspmv_matinfo matinfo;
    int* csr_row_ptr; int* csr_col_id; float* csr_data;
} clspmv_csr_f32;

/* dia_matrix<int,int,float>: include/matrix_storage.h:30-47.
 * dia_data[d * dia_length_aligned + row] holds A[row, row + dia_offsets[d]]. */
typedef struct {
    clspmv_matinfo matinfo;
    int dia_num; int dia_length; int dia_length_aligned;
    int* dia_offsets; float* dia_data;
} clspmv_dia_f32;

/* bdia_matrix<int,int,float>: include/matrix_storage.h:72-94 */
typedef struct {
    clspmv_matinfo matinfo;
    int bdia_band_num; int bdia_length; int bdia_length_aligned;
    int* bdia_offsets; int* bdia_bptr; float* bdia_data;
} clspmv_bdia_f32;

/* ell_matrix<int,float>: include/matrix_storage.h:96-111 (column major) */
typedef struct {
    clspmv_matinfo matinfo;
    int ell_num; int ell_height_aligned;
    int* ell_col_id; float* ell_data;
} clspmv_ell_f32;

/* sell_matrix<int,float>: include/matrix_storage.h:122-137 */
typedef struct {
    clspmv_matinfo matinfo;
    unsigned int sell_slice_height; int sell_slice_num;
    int* sell_slice_ptr; int* sell_col_id; float* sell_data;
} clspmv_sell_f32;

/* bcsr_matrix<int,float>: include/matrix_storage.h:178-199 (host only) */
typedef struct {
    clspmv_matinfo matinfo;
    unsigned int bcsr_bwidth; unsigned int bcsr_bheight;
    int bcsr_row_num; int bcsr_aligned_size; int bcsr_block_num;
    int* bcsr_row_ptr; int* bcsr_col_id; float* bcsr_data;
} clspmv_bcsr_f32;

/* bell_matrix<int,float>: include/matrix_storage.h:215-236 (host only) */
typedef struct {
    clspmv_matinfo matinfo;
    unsigned int bell_bwidth; unsigned int bell_bheight;
    int bell_row_num; int bell_block_num; int bell_height_aligned; int bell_float4_aligned;
    int* bell_col_id; float* bell_data;
} clspmv_bell_f32;

/* b4csr_matrix<int,float>: include/matrix_storage.h:266-287 ("BCSR" on the GPU).
 * Column ids in float4 units; data plane (w4, h) holds one float4 per block:
 * b4csr_data[w4*aligned*bh + h*aligned + 4*block + w]. */
typedef struct {
    clspmv_matinfo matinfo;
    unsigned int b4csr_bwidth; unsigned int b4csr_bheight;
    int b4csr_row_num; int b4csr_aligned_size; int b4csr_block_num;
    int* b4csr_row_ptr; int* b4csr_col_id; float* b4csr_data;
} clspmv_b4csr_f32;

/* b4ell_matrix<int,float>: include/matrix_storage.h:311-332 ("BELL" on the GPU) */
typedef struct {
    clspmv_matinfo matinfo;
    unsigned int b4ell_bwidth; unsigned int b4ell_bheight;
    int b4ell_row_num; int b4ell_block_num; int b4ell_height_aligned; int b4ell_float4_aligned;
    int* b4ell_col_id; float* b4ell_data;
} clspmv_b4ell_f32;

/* sbell_matrix<int,float>: include/matrix_storage.h:344-365 */
typedef struct {
    clspmv_matinfo matinfo;
    unsigned int sbell_bwidth; unsigned int sbell_bheight; unsigned int sbell_slice_height;
    int sbell_slice_num; int sbell_row_num;
    int* sbell_slice_ptr; int* sbell_col_id; float* sbell_data;
} clspmv_sbell_f32;

/* cocktail<int,int,float>: include/analyze.h:105-144 of clSpMV. The result
 * of the Cocktail partitioner: which of the nine formats are used, the
 * kernel variant / work-group count the tables chose for each, and the
 * parts themselves (host arrays after analysis, device arrays after
 * clspmv_cocktail_upload). */
typedef struct {
    bool ifusebdia, ifusedia, ifusesbell, ifusebell, ifusebcsr, ifusesell, ifuseell, ifusecsr, ifusecoo;
    int bdia_meth_num, dia_meth_num, sbell_meth_num, bell_meth_num, bcsr_meth_num, sell_meth_num, ell_meth_num,
        csr_meth_num, coo_meth_num;
    int csr_group_num, coo_group_num;
    int mat_width, mat_height, mat_nnz;
    clspmv_bdia_f32 bdia;
    clspmv_dia_f32 dia;
    clspmv_sbell_f32 sbell;
    clspmv_b4ell_f32 bell;
    clspmv_b4csr_f32 bcsr;
    clspmv_sell_f32 sell;
    clspmv_ell_f32 ell;
    clspmv_csr_f32 csr;
    clspmv_coo_f32 coo;
} clspmv_cocktail_f32;

/* ------------------------------------------------------------------------ */
/* Library                                                                   */
/* ------------------------------------------------------------------------ */

/* Version string, e.g. "clspmv_b200 0.1 sm_100a". */
const char* clspmv_version(void);
/* Human readable text for a status code. */
const char* clspmv_status_string(int status);
/* Last CUDA error text seen by the library on this thread ("" if none). */
const char* clspmv_last_cuda_error(void);

/* ------------------------------------------------------------------------ */
/* Host converters. Outputs are malloc'ed; release with clspmv_free_<fmt>.   */
/* Byte-identical to the reference converters on sorted COO input.          */
/* ------------------------------------------------------------------------ */

/* sort_coo: include/matrix_storage.h:744-815 (row-major (row, col) order). */
int clspmv_sort_coo_f32(clspmv_coo_f32* mat);
/* if_sorted_coo: include/matrix_storage.h:731-741. Returns 1 if sorted. */
int clspmv_is_sorted_coo_f32(const clspmv_coo_f32* mat);
/* coo2csr: include/matrix_storage.h:1268-1307 */
int clspmv_coo2csr_f32(const clspmv_coo_f32* src, clspmv_csr_f32* dst);
/* pad_csr: src/util.cpp:31-72 (rows padded to a multiple of `alignment`
 * with the last column id and 0.0f). */
int clspmv_pad_csr_f32(const clspmv_csr_f32* src, clspmv_csr_f32* dst, int alignment);
/* coo2dia: include/matrix_storage.h:936-1014. CLSPMV_ERR_REFUSED when the
 * reference refuses (padded size rule at :972). */
int clspmv_coo2dia_f32(const clspmv_coo_f32* src, clspmv_dia_f32* dst, int alignment);
/* coo2bdia: include/matrix_storage.h:1184-1236 */
int clspmv_coo2bdia_f32(const clspmv_coo_f32* src, clspmv_bdia_f32* dst, int alignment);
/* coo2ell: include/matrix_storage.h:1339-1394. ellnum == 0 -> max row length.
 * CLSPMV_ERR_ARG when a row is longer than a given ellnum (reference
 * assert at :1379); CLSPMV_ERR_REFUSED when aligned_height*ellnum exceeds
 * INT_MAX (the reference overflows int there). */
int clspmv_coo2ell_f32(const clspmv_coo_f32* src, clspmv_ell_f32* dst, int alignment, int ellnum);
/* coo2sell: include/matrix_storage.h:1397-1513 */
int clspmv_coo2sell_f32(const clspmv_coo_f32* src, clspmv_sell_f32* dst, unsigned int slice_height);
/* coo2bcsr: include/matrix_storage.h:1593-1737 */
int clspmv_coo2bcsr_f32(const clspmv_coo_f32* src, clspmv_bcsr_f32* dst,
                        unsigned int bwidth, unsigned int bheight, int alignment);
/* coo2b4csr: include/matrix_storage.h:1740-1897 (refusal cap at :1863) */
int clspmv_coo2b4csr_f32(const clspmv_coo_f32* src, clspmv_b4csr_f32* dst,
                         unsigned int bwidth, unsigned int bheight, int alignment);
/* coo2bell: include/matrix_storage.h:1940-2006 */
int clspmv_coo2bell_f32(const clspmv_coo_f32* src, clspmv_bell_f32* dst,
                        unsigned int bwidth, unsigned int bheight, int alignment, int ellnum);
/* coo2b4ell: include/matrix_storage.h:2008-2200 (refusal cap at :2141) */
int clspmv_coo2b4ell_f32(const clspmv_coo_f32* src, clspmv_b4ell_f32* dst,
                         unsigned int bwidth, unsigned int bheight, int alignment, int ellnum);
/* coo2sbell: include/matrix_storage.h:2202-2409 (refusal cap at :2350) */
int clspmv_coo2sbell_f32(const clspmv_coo_f32* src, clspmv_sbell_f32* dst,
                         unsigned int bwidth, unsigned int bheight, unsigned int slice_height);

/* Inverse converters (allocate dst arrays). csr2coo :1238-1266, dia2coo
 * :825-863, bdia2coo :1136-1181, ell2coo :1309-1337, bcsr2coo :1545-1589,
 * bell2coo :1900-1938. The sell/b4csr/b4ell/sbell inverses have no
 * reference counterpart; they exist for round-trip checks of the layouts. */
int clspmv_csr2coo_f32(const clspmv_csr_f32* src, clspmv_coo_f32* dst);
int clspmv_dia2coo_f32(const clspmv_dia_f32* src, clspmv_coo_f32* dst);
int clspmv_bdia2coo_f32(const clspmv_bdia_f32* src, clspmv_coo_f32* dst);
int clspmv_ell2coo_f32(const clspmv_ell_f32* src, clspmv_coo_f32* dst);
int clspmv_bcsr2coo_f32(const clspmv_bcsr_f32* src, clspmv_coo_f32* dst);
int clspmv_bell2coo_f32(const clspmv_bell_f32* src, clspmv_coo_f32* dst);
int clspmv_sell2coo_f32(const clspmv_sell_f32* src, clspmv_coo_f32* dst);
int clspmv_b4csr2coo_f32(const clspmv_b4csr_f32* src, clspmv_coo_f32* dst);
/* Deep copy of a COO matrix (malloc'ed arrays). */
int clspmv_coo2coo_f32(const clspmv_coo_f32* src, clspmv_coo_f32* dst);
int clspmv_b4ell2coo_f32(const clspmv_b4ell_f32* src, clspmv_coo_f32* dst);
int clspmv_sbell2coo_f32(const clspmv_sbell_f32* src, clspmv_coo_f32* dst);

/* free_*: include/matrix_storage.h:529-652. Frees the arrays and nulls them. */
void clspmv_free_coo_f32(clspmv_coo_f32* m);
void clspmv_free_csr_f32(clspmv_csr_f32* m);
void clspmv_free_dia_f32(clspmv_dia_f32* m);
void clspmv_free_bdia_f32(clspmv_bdia_f32* m);
void clspmv_free_ell_f32(clspmv_ell_f32* m);
void clspmv_free_sell_f32(clspmv_sell_f32* m);
void clspmv_free_bcsr_f32(clspmv_bcsr_f32* m);
void clspmv_free_bell_f32(clspmv_bell_f32* m);
void clspmv_free_b4csr_f32(clspmv_b4csr_f32* m);
void clspmv_free_b4ell_f32(clspmv_b4ell_f32* m);
void clspmv_free_sbell_f32(clspmv_sbell_f32* m);

/* ------------------------------------------------------------------------ */
/* Device residency. upload: cudaMalloc + copy of every array of `host`     */
/* into `dev` (scalars copied). device_free: cudaFree of those arrays.      */
/* Replaces the ALLOCATE_GPU_READ uploads of the per-format drivers         */
/* (include/oclcommon.h:13-38) and the cpy_<fmt>_mat helpers of             */
/* src/spmv_cocktail.cpp:304-1009.                                          */
/* ------------------------------------------------------------------------ */
int clspmv_upload_coo_f32(const clspmv_coo_f32* host, clspmv_coo_f32* dev);
int clspmv_upload_csr_f32(const clspmv_csr_f32* host, clspmv_csr_f32* dev);
int clspmv_upload_dia_f32(const clspmv_dia_f32* host, clspmv_dia_f32* dev);
int clspmv_upload_bdia_f32(const clspmv_bdia_f32* host, clspmv_bdia_f32* dev);
int clspmv_upload_ell_f32(const clspmv_ell_f32* host, clspmv_ell_f32* dev);
int clspmv_upload_sell_f32(const clspmv_sell_f32* host, clspmv_sell_f32* dev);
int clspmv_upload_b4csr_f32(const clspmv_b4csr_f32* host, clspmv_b4csr_f32* dev);
int clspmv_upload_bcsr_f32(const clspmv_bcsr_f32* host, clspmv_bcsr_f32* dev);
int clspmv_upload_bell_f32(const clspmv_bell_f32* host, clspmv_bell_f32* dev);
int clspmv_upload_b4ell_f32(const clspmv_b4ell_f32* host, clspmv_b4ell_f32* dev);
int clspmv_upload_sbell_f32(const clspmv_sbell_f32* host, clspmv_sbell_f32* dev);
int clspmv_device_free_coo_f32(clspmv_coo_f32* dev);
int clspmv_device_free_csr_f32(clspmv_csr_f32* dev);
int clspmv_device_free_dia_f32(clspmv_dia_f32* dev);
int clspmv_device_free_bdia_f32(clspmv_bdia_f32* dev);
int clspmv_device_free_ell_f32(clspmv_ell_f32* dev);
int clspmv_device_free_sell_f32(clspmv_sell_f32* dev);
int clspmv_device_free_b4csr_f32(clspmv_b4csr_f32* dev);
int clspmv_device_free_bcsr_f32(clspmv_bcsr_f32* dev);
int clspmv_device_free_bell_f32(clspmv_bell_f32* dev);
int clspmv_device_free_b4ell_f32(clspmv_b4ell_f32* dev);
int clspmv_device_free_sbell_f32(clspmv_sbell_f32* dev);

/* ------------------------------------------------------------------------ */
/* Converters on the device. `coo` holds device arrays; the output struct   */
/* gets cudaMalloc'ed device arrays (release with clspmv_device_free_<fmt>) */
/* equal byte for byte to what the host converter of the same name without  */
/* `device_` makes from the same COO, with the same statuses (argument      */
/* checks, CLSPMV_ERR_NOT_SORTED, refusals). The COO is not modified. Each  */
/* call synchronises `stream`. They replace the host-side conversion the    */
/* reference does before every upload (include/matrix_storage.h:936-2409);  */
/* the reference has no device converter.                                   */
/* ------------------------------------------------------------------------ */
/* Stable sort of a device COO by (row, col), in place (sort_coo,
 * include/matrix_storage.h:744-815). */
int clspmv_device_sort_coo_f32(clspmv_coo_f32* coo, clspmv_stream_t stream);
/* coo2csr (include/matrix_storage.h:1268-1307). */
int clspmv_device_coo2csr_f32(const clspmv_coo_f32* coo, clspmv_csr_f32* dev, clspmv_stream_t stream);
/* coo2dia (:936-1014); any COO order, the last of a repeated (row, col) wins. */
int clspmv_device_coo2dia_f32(const clspmv_coo_f32* coo, clspmv_dia_f32* dev, int alignment, clspmv_stream_t stream);
/* coo2bdia (:1184-1236). */
int clspmv_device_coo2bdia_f32(const clspmv_coo_f32* coo, clspmv_bdia_f32* dev, int alignment, clspmv_stream_t stream);
/* coo2ell (:1339-1394); ellnum 0 = longest row. */
int clspmv_device_coo2ell_f32(const clspmv_coo_f32* coo, clspmv_ell_f32* dev, int alignment, int ellnum,
                              clspmv_stream_t stream);
/* coo2sell (:1397-1513). */
int clspmv_device_coo2sell_f32(const clspmv_coo_f32* coo, clspmv_sell_f32* dev, unsigned int slice_height,
                               clspmv_stream_t stream);
/* coo2b4csr (:1740-1897). */
int clspmv_device_coo2b4csr_f32(const clspmv_coo_f32* coo, clspmv_b4csr_f32* dev, unsigned int bwidth,
                                unsigned int bheight, int alignment, clspmv_stream_t stream);
/* coo2bcsr (:1593-1737), any block shape: the generic block CSR that only
 * the serial bcsr_spmv reads (col_id = a block's first column, data[k * len
 * + block], k = inner row * bwidth + inner column). */
int clspmv_device_coo2bcsr_f32(const clspmv_coo_f32* coo, clspmv_bcsr_f32* dev, unsigned int bwidth,
                               unsigned int bheight, int alignment, clspmv_stream_t stream);
/* coo2bell (:1940-2006), any block shape; ellnum 0 = most blocks in a block
 * row, CLSPMV_ERR_ARG when a block row holds more than a given ellnum. */
int clspmv_device_coo2bell_f32(const clspmv_coo_f32* coo, clspmv_bell_f32* dev, unsigned int bwidth,
                               unsigned int bheight, int alignment, int ellnum, clspmv_stream_t stream);
/* coo2b4ell (:2008-2200); ellnum 0 = most blocks in a block row. */
int clspmv_device_coo2b4ell_f32(const clspmv_coo_f32* coo, clspmv_b4ell_f32* dev, unsigned int bwidth,
                                unsigned int bheight, int alignment, int ellnum, clspmv_stream_t stream);
/* coo2sbell (:2202-2409). */
int clspmv_device_coo2sbell_f32(const clspmv_coo_f32* coo, clspmv_sbell_f32* dev, unsigned int bwidth,
                                unsigned int bheight, unsigned int slice_height, clspmv_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Compute entry points (device structs, device x and y).                    */
/* x has matinfo.width entries, y has matinfo.height entries; both 16-byte  */
/* aligned. All launches are asynchronous on `stream`.                      */
/* ------------------------------------------------------------------------ */

/* CSR, thread per row. Replaces gpu_csr_sc_pm / _u4 / _float4_noif
 * (kernels/spmv_csr_scalar.cl:5-209), driver src/spmv_csr_scalar.cpp:670-713.
 * Rows padded by pad_csr(.., 4) take the 128-bit load path automatically. */
int clspmv_csr_scalar_spmv_f32(const clspmv_csr_f32* dev, const float* x, float* y,
                               float alpha, float beta, clspmv_stream_t stream);

/* CSR, `threads_per_row` lanes per row (1,2,4,8,16,32; 0 = chosen from the
 * mean row length) with a shuffle reduction. Replaces gpu_csr_ve_slm_pm_fs /
 * gpu_csr_ve_reduction_fs (kernels/spmv_csr_vector.cl:4-191), driver
 * src/spmv_csr_vector.cpp:619-664. */
int clspmv_csr_vector_spmv_f32(const clspmv_csr_f32* dev, const float* x, float* y,
                               float alpha, float beta, int threads_per_row,
                               clspmv_stream_t stream);

/* CSR, nnz-balanced merge-path tiles: every CTA gets the same number of
 * (rows + nonzeros), so power-law rows cost the same as regular ones.
 * `tile_coord` is a device array of 2*(ntiles+1) ints made by
 * clspmv_csr_merge_plan (rows finished, nonzeros consumed at each tile
 * start). This is the CSR kernel the autotuner and the Cocktail runtime use. */
int clspmv_csr_merge_tiles(int rows, int nnz);
int clspmv_csr_merge_plan(const clspmv_csr_f32* dev, int* tile_coord, clspmv_stream_t stream);
int clspmv_csr_merge_spmv_f32(const clspmv_csr_f32* dev, const int* tile_coord,
                              const float* x, float* y, float alpha, float beta,
                              clspmv_stream_t stream);

/* CSR SpMV by nonzero chunks (replaces the same kernels as the merge path,
 * kernels/spmv_csr_scalar.cl and spmv_csr_vector.cl): a warp per 256
 * consecutive nonzeros, 128-bit loads of col_id / data, the rows recovered
 * from row_ptr and reduced with a warp segmented scan, rows cut by a chunk
 * edge added atomically (summation order differs from the reference's
 * serial one within the 1e-5 bound). The plan holds the first row of every
 * chunk: clspmv_csr_chunk_plan_size(nnz) ints, filled once per matrix by
 * clspmv_csr_chunk_plan. col_id and data must be 16-byte aligned. */
int clspmv_csr_chunk_plan_size(int nnz);
int clspmv_csr_chunk_plan(const clspmv_csr_f32* dev, int* chunk_row, clspmv_stream_t stream);
int clspmv_csr_chunk_spmv_f32(const clspmv_csr_f32* dev, const int* chunk_row, const float* x, float* y, float alpha,
                              float beta, clspmv_stream_t stream);

/* The same merge-path SpMV for callers that cannot allocate device memory at
 * the call (a running loop that must not call cudaMalloc/cudaFree, which can
 * wait for the whole device; a binding with no device allocator; a service
 * with a fixed memory budget). No counterpart in the reference. The tile
 * plan is rebuilt on every call in a fixed array that is part of the
 * library's device image (512 KiB per device), so the call allocates
 * nothing. Limits and rules:
 *  - rows + nnz must be at most clspmv_csr_merge_noalloc_max_tiles() * 2048
 *    (134,215,680); larger matrices get CLSPMV_ERR_UNSUPPORTED and nothing
 *    is launched;
 *  - the first call on each device (with that device current) looks the
 *    array up; make it before starting any stream capture on that device;
 *  - the looked-up address is kept for the life of the process: after
 *    cudaDeviceReset on a device (which destroys its copy of the array),
 *    do not call this entry point on that device again;
 *  - nothing needs to start at zero: each call writes the whole plan it
 *    reads, in `stream`, before its SpMV kernel;
 *  - there is one array per device, so calls on one device must not
 *    overlap: two in flight at once (other streams or threads) overwrite
 *    each other's plan. Issue them on one stream or wait in between. */
int clspmv_csr_merge_noalloc_max_tiles(void);
int clspmv_csr_merge_spmv_noalloc_f32(const clspmv_csr_f32* dev, const float* x, float* y,
                                      float alpha, float beta, clspmv_stream_t stream);

/* COO, single-pass warp segmented reduction (row-sorted input). Replaces the
 * two-pass gpu_coo_s1/gpu_coo_s2 (kernels/spmv_coo.cl:4-217), driver
 * src/spmv_coo.cpp:17-353. */
int clspmv_coo_spmv_f32(const clspmv_coo_f32* dev, const float* x, float* y,
                        float alpha, float beta, clspmv_stream_t stream);

/* DIA. Replaces gpu_dia{,_v4,_tx,_v4_tx} (kernels/spmv_dia.cl:4-170),
 * driver src/spmv_dia.cpp:366-395. x is not padded: out-of-range columns
 * are predicated off instead of read from an extended vector. */
int clspmv_dia_spmv_f32(const clspmv_dia_f32* dev, const float* x, float* y,
                        float alpha, float beta, clspmv_stream_t stream);

/* DIA and BDIA with the diagonals staged in shared memory by bulk copies:
 * per CTA one producer warp streams tiles of 1024 rows, 9 diagonals at a
 * time, into a ring of three shared-memory stages (cp.async.bulk, mbarrier
 * handoff with bounded waits) and eight consumer warps compute four rows per
 * thread from shared memory, x gathered through L1; two CTAs per SM, each
 * over an equal range of rows. The bytes in flight no longer depend on
 * registers. Requires dia_length_aligned (bdia_length_aligned) a multiple
 * of 32 and a 16-byte aligned data array (CLSPMV_ERR_ALIGN otherwise). Same
 * y as clspmv_dia_spmv_f32 / clspmv_bdia_spmv_f32 up to summation order. A
 * wait that runs out (about 2 s; none expected) ends the kernel and is
 * counted for clspmv_pipeline_timeouts. No counterpart in the reference. */
int clspmv_dia_bulk_spmv_f32(const clspmv_dia_f32* dev, const float* x, float* y,
                             float alpha, float beta, clspmv_stream_t stream);
int clspmv_bdia_bulk_spmv_f32(const clspmv_bdia_f32* dev, const float* x, float* y,
                              float alpha, float beta, clspmv_stream_t stream);
/* Reads and resets the number of bounded waits of the bulk-copy pipelines
 * that ran out since the last call (0 in normal operation). */
int clspmv_pipeline_timeouts(unsigned int* count);

/* BDIA with a shared-memory x window per band. Replaces gpu_bdia* variants
 * (kernels/spmv_bdia.cl:4-283), driver src/spmv_bdia.cpp:413-441. */
int clspmv_bdia_spmv_f32(const clspmv_bdia_f32* dev, const float* x, float* y,
                         float alpha, float beta, clspmv_stream_t stream);

/* ELL (column major), 4 rows per thread with 128-bit loads. Replaces
 * gpu_ell{,_v4,_tx,_v4_tx} (kernels/spmv_ell.cl:4-104). */
int clspmv_ell_spmv_f32(const clspmv_ell_f32* dev, const float* x, float* y,
                        float alpha, float beta, clspmv_stream_t stream);

/* SELL, any slice height that is a multiple of 4 (32 and 128 in the
 * reference). Replaces gpu_sell_warp / gpu_sell_group (kernels/spmv_sell.cl). */
int clspmv_sell_spmv_f32(const clspmv_sell_f32* dev, const float* x, float* y,
                         float alpha, float beta, clspmv_stream_t stream);

/* SELL without reading its padding. The converter pads each row of a slice
 * to the slice's widest row with the row's previous column id and value 0
 * (include/matrix_storage.h:1466-1491), so a slot equal to its predecessor's
 * column with value 0 adds nothing and a row's trailing run of such slots is
 * padding. clspmv_sell_plan_create finds where every row's real entries end
 * (synchronous, once per matrix; it allocates device memory, released with
 * clspmv_sell_plan_free). For slice heights 4..128 (powers of two) with
 * 16-byte aligned arrays the planned SpMV walks the slot space like
 * clspmv_sell_spmv_f32 (equal runs of slice columns per warp, 4 rows per
 * lane) but each lane loads a column only while one of its 4 rows still has
 * real entries, and only up to the slice's second-longest row; the longest
 * row's entries past it go to a warp per 256 entries, which reads their
 * column ids from a compact copy the plan made (structure only: the values
 * stay in the matrix, so the plan holds while they change, not while the
 * column ids do) and their values in place, the heads and the tails in one
 * launch (about a fifth of its CTAs on the tails); other slice heights sum each row's first
 * 32 entries with a thread per row and longer rows' tails with a warp per
 * 256 entries. Same y as clspmv_sell_spmv_f32 up to summation order, except
 * where x holds Inf or NaN at a skipped padding column. No counterpart in
 * the reference. */
typedef struct clspmv_sell_plan clspmv_sell_plan;
int clspmv_sell_plan_create(const clspmv_sell_f32* dev, clspmv_sell_plan** out);
int clspmv_sell_plan_spmv_f32(const clspmv_sell_f32* dev, const clspmv_sell_plan* plan, const float* x, float* y,
                              float alpha, float beta, clspmv_stream_t stream);
/* The planned SpMV with 16-bit values (clspmv_pack_values of this matrix:
 * CLSPMV_VALUES_BF16 / _F16 and the per-row scales); slice heights other than
 * 4..128 (powers of two) take the padded 16-bit read. */
int clspmv_sell_plan_spmv_packed(const clspmv_sell_f32* dev, const clspmv_sell_plan* plan, int value_type,
                                 const void* values, const float* row_scale, const float* x, float* y, float alpha,
                                 float beta, clspmv_stream_t stream);
/* stored entries the plan reads (real entries and explicit zeros before them), and its tail items */
long long clspmv_sell_plan_entries(const clspmv_sell_plan* plan);
long long clspmv_sell_plan_items(const clspmv_sell_plan* plan);
/* bytes of col and data in the 32-byte sectors that hold real entries: what
 * the planned SpMV must move from the matrix arrays */
long long clspmv_sell_plan_sector_bytes(const clspmv_sell_plan* plan);
/* bytes the planned SpMV (slice heights 4..128) must read at the 128-byte
 * line granularity of B200's DRAM traffic: the col and data lines holding
 * the heads' entries, a data line per tail entry, the tails' compact column
 * ids and the plan's own arrays */
long long clspmv_sell_plan_line_bytes(const clspmv_sell_plan* plan);
int clspmv_sell_plan_free(clspmv_sell_plan* plan);

/* BELL = b4ell, block shapes {1,2,4,8} x {4,8}. Replaces the 32 kernels of
 * kernels/spmv_bell.cl, driver src/spmv_bell.cpp:345-399. */
int clspmv_b4ell_spmv_f32(const clspmv_b4ell_f32* dev, const float* x, float* y,
                          float alpha, float beta, clspmv_stream_t stream);

/* SBELL, slice of `sbell_slice_height` block rows (32 in the reference).
 * Replaces the 16 kernels of kernels/spmv_sbell.cl. */
int clspmv_sbell_spmv_f32(const clspmv_sbell_f32* dev, const float* x, float* y,
                          float alpha, float beta, clspmv_stream_t stream);

/* BCSR = b4csr, block shapes {1,2,4,8} x {4,8}. Replaces the 16 kernels of
 * kernels/spmv_bcsr.cl, driver src/spmv_bcsr.cpp:224-278. */
int clspmv_b4csr_spmv_f32(const clspmv_b4csr_f32* dev, const float* x, float* y,
                          float alpha, float beta, clspmv_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Several right-hand sides and 16-bit value storage (no counterpart in the  */
/* reference, whose kernels multiply one vector per call).                   */
/* ------------------------------------------------------------------------ */

typedef enum {
    CLSPMV_FORMAT_CSR = 0, CLSPMV_FORMAT_COO = 1, CLSPMV_FORMAT_DIA = 2, CLSPMV_FORMAT_BDIA = 3,
    CLSPMV_FORMAT_ELL = 4, CLSPMV_FORMAT_SELL = 5, CLSPMV_FORMAT_B4CSR = 6, CLSPMV_FORMAT_B4ELL = 7,
    CLSPMV_FORMAT_SBELL = 8
} clspmv_format;

typedef enum { CLSPMV_VALUES_F32 = 0, CLSPMV_VALUES_BF16 = 1, CLSPMV_VALUES_F16 = 2 } clspmv_values;

/* Y <- alpha * A * X + beta * Y for the device matrix `dev` (a pointer to the
 * format's struct, e.g. clspmv_csr_f32*, with device arrays). X is width x k,
 * Y is height x k, both row major with leading dimensions ldx, ldy >= k,
 * 1 <= k <= 128 (k > 32 needs k, ldx, ldy multiples of 4 and 16-byte aligned
 * X, Y: CLSPMV_ERR_ALIGN otherwise). FP32 accumulation.
 * value_type CLSPMV_VALUES_F32 uses the struct's own values (`values`,
 * `row_scale` ignored); BF16 / F16 use the 16-bit array and per-row scales
 * made by clspmv_pack_values. CSR and COO must be row sorted; their rows
 * cut between work chunks are added atomically, so the last bits of Y may
 * differ between runs (within the FP32 bound). Kernel by case: at k = 4
 * (16-byte rows) CSR / COO take a warp per 256 nonzeros with a segmented
 * reduction; CSR rows averaging >= 128 nonzeros at k = 4 * 2^j take a warp
 * per row; otherwise lane groups per nonzero chunk (CSR / COO) or per row
 * (the other formats). */
int clspmv_spmm(int format, const void* dev, int value_type, const void* values, const float* row_scale, int k,
                const float* X, int ldx, float* Y, int ldy, float alpha, float beta, clspmv_stream_t stream);

/* Per-format FP32 forms of clspmv_spmm. */
int clspmv_csr_spmm_f32(const clspmv_csr_f32* dev, int k, const float* X, int ldx, float* Y, int ldy, float alpha, float beta, clspmv_stream_t stream);
int clspmv_coo_spmm_f32(const clspmv_coo_f32* dev, int k, const float* X, int ldx, float* Y, int ldy, float alpha, float beta, clspmv_stream_t stream);
int clspmv_dia_spmm_f32(const clspmv_dia_f32* dev, int k, const float* X, int ldx, float* Y, int ldy, float alpha, float beta, clspmv_stream_t stream);
int clspmv_bdia_spmm_f32(const clspmv_bdia_f32* dev, int k, const float* X, int ldx, float* Y, int ldy, float alpha, float beta, clspmv_stream_t stream);
int clspmv_ell_spmm_f32(const clspmv_ell_f32* dev, int k, const float* X, int ldx, float* Y, int ldy, float alpha, float beta, clspmv_stream_t stream);
int clspmv_sell_spmm_f32(const clspmv_sell_f32* dev, int k, const float* X, int ldx, float* Y, int ldy, float alpha, float beta, clspmv_stream_t stream);
int clspmv_b4csr_spmm_f32(const clspmv_b4csr_f32* dev, int k, const float* X, int ldx, float* Y, int ldy, float alpha, float beta, clspmv_stream_t stream);
int clspmv_b4ell_spmm_f32(const clspmv_b4ell_f32* dev, int k, const float* X, int ldx, float* Y, int ldy, float alpha, float beta, clspmv_stream_t stream);
int clspmv_sbell_spmm_f32(const clspmv_sbell_f32* dev, int k, const float* X, int ldx, float* Y, int ldy, float alpha, float beta, clspmv_stream_t stream);

/* clspmv_b4csr_spmm_f32 on the tensor cores (tcgen05.mma kind::tf32,
 * accumulators in tensor memory), for 4 x 4 blocks and k a multiple of 16 up
 * to 128 (CLSPMV_ERR_UNSUPPORTED otherwise). Every value of A and X is split
 * into a TF32 head and its remainder, so the products keep FP32 accuracy
 * (about 2^-21 of sum |a x|). X 16-byte aligned with ldx a multiple of 4
 * (CLSPMV_ERR_ALIGN otherwise); Y has no alignment rule. Up to 64 right-hand
 * sides per launch. */
int clspmv_b4csr_spmm_tc_f32(const clspmv_b4csr_f32* dev, int k, const float* X, int ldx, float* Y, int ldy,
                             float alpha, float beta, clspmv_stream_t stream);
/* Number of bounded device waits in the tensor-core kernels that ran out
 * since the last call (each ends its kernel early with Y incomplete);
 * synchronous, resets the count. */
int clspmv_tensor_timeouts(unsigned int* count);

/* Number of stored values (padding included) of the device matrix, i.e. the
 * length of its value array; reads one int from the device for BDIA, SELL
 * and SBELL. */
int clspmv_stored_values(int format, const void* dev, size_t* count);

/* Makes the 16-bit copy of a device matrix's values: row_scale[r] =
 * 2^ceil(log2(max_j |a_rj|)) (1 for empty rows) and values[i] = a_i /
 * row_scale[row of i], rounded to nearest (value_type BF16 or F16).
 * `values` holds clspmv_stored_values entries of 2 bytes, `row_scale` height
 * floats; stored positions outside the matrix get 0. Asynchronous. */
int clspmv_pack_values(int format, const void* dev, int value_type, void* values, float* row_scale,
                       clspmv_stream_t stream);

/* y <- alpha * A * x + beta * y with the 16-bit values and row scales of
 * clspmv_pack_values, in the format's own single-vector kernel (half the
 * value bytes of the FP32 call). `tile_coord` is the merge-path plan of the
 * matrix (clspmv_csr_merge_plan), used and required for CSR only. */
int clspmv_spmv_packed(int format, const void* dev, int value_type, const void* values, const float* row_scale,
                       const int* tile_coord, const float* x, float* y, float alpha, float beta,
                       clspmv_stream_t stream);
/* The same for CSR in the nonzero-chunk kernel (`chunk_row` from
 * clspmv_csr_chunk_plan); col_id 16-byte and values 8-byte aligned. */
int clspmv_csr_chunk_spmv_packed(const clspmv_csr_f32* dev, int value_type, const void* values,
                                 const float* row_scale, const int* chunk_row, const float* x, float* y,
                                 float alpha, float beta, clspmv_stream_t stream);

/* One Y <- alpha * A * X + beta * Y of a batch (fields as in clspmv_spmm). */
typedef struct {
    int format;              /* clspmv_format; every format but COO */
    const void* dev;         /* device matrix struct (read when the batch is set) */
    int value_type;          /* clspmv_values */
    const void* values;      /* 16-bit values (BF16 / F16 only) */
    const float* row_scale;  /* their row scales (BF16 / F16 only) */
    int k;
    const float* X;
    int ldx;
    float* Y;
    int ldy;
    float alpha, beta;
} clspmv_spmm_job;

/* A batch runs many jobs (different matrices, formats, value types and k)
 * in one persistent kernel launch: the rows of all jobs are cut into warp
 * tasks that every warp of a device-filling grid strides through. Jobs on
 * 4x4 blocks (b4csr, b4ell, SBELL) with 16-byte X / Y rows run in a second
 * persistent launch, one lane group per block row, as clspmv_spmm runs them.
 * A CSR job with beta == 1 (Y += alpha * A * X) whose rows hold 256 entries
 * or more on average is cut by nonzeros instead of rows, so very long rows
 * do not serialise one warp; for such matrices prefer beta == 1 (zero Y
 * first for a plain product). */
typedef struct clspmv_batch clspmv_batch;

/* Allocates the device job table for up to max_jobs jobs (and a pinned
 * staging copy). */
int clspmv_batch_create(int max_jobs, clspmv_batch** out);
/* Validates the jobs and uploads the table on `stream` (asynchronous; the
 * structs pointed to by jobs[i].dev are copied, so they may be released
 * after the call). On an invalid job returns its status and, if bad_job is
 * not NULL, its index; the batch is then empty. Waits only for this batch's
 * previous upload to leave the staging buffer. */
int clspmv_batch_set(clspmv_batch* b, const clspmv_spmm_job* jobs, int njobs, clspmv_stream_t stream, int* bad_job);
/* Runs the jobs last set: one kernel launch on `stream` (two when 4x4-block
 * jobs are among them), no allocation and no host synchronisation, so it can
 * be captured in a CUDA graph. Jobs must not write overlapping Y. */
int clspmv_batch_run(clspmv_batch* b, clspmv_stream_t stream);
int clspmv_batch_free(clspmv_batch* b);

/* ------------------------------------------------------------------------ */
/* Cocktail partitioning (src/analyze.cpp of clSpMV).                        */
/* ------------------------------------------------------------------------ */

/* analyze_matrix (src/analyze.cpp:3714-3900) with the benchmark tables read
 * from <table_dir>/benchmark/<fmt>.ben (NULL: $CLSPMVPATH, as the reference).
 * `coo` must be sorted by (row, col). `out` is initialised here; release it
 * with clspmv_free_cocktail_f32. CLSPMV_ERR_ARG when a table is missing or
 * empty (the reference segfaults there). */
int clspmv_analyze_matrix_f32(const clspmv_coo_f32* coo, clspmv_cocktail_f32* out, const char* table_dir,
                              float dia_priority_multiplier, int estimate_flat_partial, int estimate_flat_full);
/* free_cocktail (include/analyze.h:183-205) */
void clspmv_free_cocktail_f32(clspmv_cocktail_f32* m);

/* ------------------------------------------------------------------------ */
/* Cocktail runtime (src/spmv_cocktail.cpp of clSpMV).                       */
/* ------------------------------------------------------------------------ */

/* Opaque device residency of a partitioned matrix. */
typedef struct clspmv_cocktail_handle clspmv_cocktail_handle;

/* Uploads every used part of `host` (replaces init_mat_kernels / cpy_<fmt>_mat,
 * src/spmv_cocktail.cpp:304-1009, 1590-1611). Synchronous. */
int clspmv_cocktail_upload_f32(const clspmv_cocktail_f32* host, clspmv_cocktail_handle** out);
/* y <- alpha*A*x + beta*y over all parts (replaces do_spmv,
 * src/spmv_cocktail.cpp:1088-1132, which runs one kernel per part in
 * sequence). Two schedules (clspmv_cocktail_set_schedule):
 *  - PER_PART (the default, AUTO): one launch per part on internal streams
 *    forked from and joined into `stream`;
 *  - FUSED: ONE persistent launch. Every part is cut into tiles, the tiles of
 *    all parts are interleaved into one work list in proportion to each
 *    part's estimated time, and the CTAs take list entries from a device
 *    counter, so all parts run side by side on every SM (a small kernel
 *    before it applies beta and resets the counter). Measured on B200 it
 *    ties the per-part launches on the Cocktail benchmark matrix (4M rows,
 *    SBELL 4x4 + COO parts: 0.165 against 0.166 ms): the HBM-streaming and
 *    the x-gathering part share the L2, so overlapping them gains nothing
 *    there, and AUTO keeps the per-part launches. An x that is not 16-byte
 *    aligned takes the per-part launches.
 * Either way it is stream ordered and safe to capture in a CUDA graph; calls
 * on one handle must not overlap on the GPU (the work counter and the
 * streams belong to the handle). The parts' additions to y are atomic, so
 * the summation order (and the last bits of y) may differ from run to run
 * within the 1e-5 bound. */
int clspmv_cocktail_spmv_f32(clspmv_cocktail_handle* h, const float* x, float* y, float alpha, float beta,
                             clspmv_stream_t stream);
/* Schedule of a handle's SpMV: AUTO (the per-part launches), FUSED (one
 * persistent launch; refused with CLSPMV_ERR_UNSUPPORTED when the handle has
 * fewer than two parts or a part layout the fused kernel does not cover:
 * block shapes taller than 4, or 8 wide and taller than 2) or PER_PART. No
 * counterpart in the reference. */
#define CLSPMV_SCHEDULE_AUTO 0
#define CLSPMV_SCHEDULE_FUSED 1
#define CLSPMV_SCHEDULE_PER_PART 2
int clspmv_cocktail_set_schedule(clspmv_cocktail_handle* h, int schedule);
/* Work-list entries of the fused schedule, 0 when the handle has none (one
 * part, or a part the fused kernel does not cover). */
int clspmv_cocktail_fused_items(const clspmv_cocktail_handle* h);
/* 1 when the SELL part runs through a length plan (made at upload when the
 * plan's line bytes come to under 3/4 of the part's stored slots: slices
 * padded to a few long rows; clspmv_sell_plan_create), 0 when it takes the
 * padded read, -1 for a NULL handle. */
int clspmv_cocktail_sell_planned(const clspmv_cocktail_handle* h);
/* Kernel of the CSR part under the per-part schedule: 0 (default) nonzero
 * chunks, or CSR-vector with `lanes` (1, 2, 4, 8, 16 or 32) lanes per row,
 * the reference's threads-per-row knob (its CSR-vector driver sweeps the
 * work-group count, src/spmv_csr_vector.cpp:106; the Cocktail tables carry
 * it per part, src/spmv_cocktail.cpp:918-962). The partition tuner measures
 * the choices. */
int clspmv_cocktail_set_csr_lanes(clspmv_cocktail_handle* h, int lanes);
/* The reference's A^k x loop (src/eval.cpp:19-72) kept on the device:
 * `iterations` times y <- alpha*A*x + beta*y, then the first mat_height
 * entries of x <- y (cpy_vector_from_gpu, src/spmv_cocktail.cpp:1510-1556).
 * Stream ordered with no host synchronisation (the reference waits after
 * every step): whole groups of 16 steps replay one CUDA graph captured once
 * per (x, y, alpha, beta) and cached in the handle, the rest launch directly.
 * Requires mat_width >= mat_height and x != y. alpha = beta = 1 is the
 * reference's loop. */
int clspmv_cocktail_iterate_f32(clspmv_cocktail_handle* h, float* x, float* y, float alpha, float beta, int iterations,
                                clspmv_stream_t stream);
/* The device-side part structs (device pointers), e.g. to launch one part. */
int clspmv_cocktail_device_view(const clspmv_cocktail_handle* h, clspmv_cocktail_f32* out);
/* Releases the device parts (replaces free_mat_kernels, :1613-1618). */
int clspmv_cocktail_free(clspmv_cocktail_handle* h);

/* ------------------------------------------------------------------------ */
/* Benchmark drivers (src/spmv_all.cpp, src/spmv_<fmt>.cpp, src/eval.cpp).   */
/* ------------------------------------------------------------------------ */

/* Method numbers of the reference's spmv_all command line
 * (src/spmv_all.cpp:156-167); CSR_MERGE is this library's addition. */
enum {
    CLSPMV_METHOD_BANDWIDTH = 0,
    CLSPMV_METHOD_CSR_SCALAR = 1,
    CLSPMV_METHOD_CSR_VECTOR = 2,
    CLSPMV_METHOD_BDIA = 3,
    CLSPMV_METHOD_DIA = 4,
    CLSPMV_METHOD_ELL = 5,
    CLSPMV_METHOD_COO = 6,
    CLSPMV_METHOD_BELL = 7,
    CLSPMV_METHOD_BCSR = 8,
    CLSPMV_METHOD_SELL = 9,
    CLSPMV_METHOD_SBELL = 10,
    CLSPMV_METHOD_CSR_MERGE = 11
};

#define CLSPMV_BENCH_MAX_VARIANTS 16

/* One timed variant: a block shape (BELL, SBELL, BCSR), a slice height
 * (SELL), a lane count (CSR vector) or a row padding (CSR scalar). */
typedef struct {
    int status;            /* CLSPMV_OK, or why this variant did not run (converter refusal) */
    int param0, param1;    /* block height / block width, slice height, lanes, padding */
    double ms;             /* per SpMV, mean over the timed launches */
    double gflops;         /* 2 * nnz / time */
    double distance;       /* ||y_gpu - y_host||_2 after one SpMV from y = 0 */
    double max_diff;       /* max_i | |y_host[i]| - |y_gpu[i]| | (two_vec_compare, src/util.cpp:93-131) */
    double max_diff_ratio; /* the same difference over max(|y_host[i]|, |y_gpu[i]|) */
} clspmv_bench_variant;

typedef struct {
    int method;
    int nvariants;
    int best;              /* index of the fastest variant that ran, -1 if none */
    double best_ms, best_gflops;
    clspmv_bench_variant v[CLSPMV_BENCH_MAX_VARIANTS];
} clspmv_bench_result;

/* The per-format benchmark drivers spmv_<fmt>(oclfilename, mat, dim2Size,
 * ntimes, deviceType) of the reference (include/spmv_<fmt>.h;
 * src/spmv_csr_scalar.cpp:670-713, spmv_csr_vector.cpp:619-664,
 * spmv_bdia.cpp:413-441, spmv_dia.cpp:366-395, spmv_ell.cpp:330-359,
 * spmv_coo.cpp:17-353, spmv_bell.cpp:345-399, spmv_bcsr.cpp:224-278,
 * spmv_sell.cpp:331-412, spmv_sbell.cpp:225-305): convert the sorted COO
 * `coo` to the method's format for every variant the reference sweeps, run
 * one SpMV from y = 0 and compare it with the host coo_spmv answer, then
 * time `ntimes` SpMVs (after 3 untimed ones) with CUDA events. x is all
 * ones (i mod 1024 for SBELL, as the reference). With `verbose` the
 * reference's report lines are printed to stdout. `out` may be NULL.
 * Returns CLSPMV_ERR_REFUSED when no variant could be converted.
 * Allocates and frees its own device buffers; synchronous. */
int clspmv_run_method_f32(const clspmv_coo_f32* coo, int method, int ntimes, int verbose, clspmv_bench_result* out);

/* Method 0 of spmv_all (src/mem_bandwidth.cpp): device copy bandwidth over
 * `bytes` bytes and the launch overhead of an empty kernel, each the mean
 * of `ntimes` runs. */
int clspmv_bandwidth_test(size_t bytes, int ntimes, int verbose, double* copy_gbs, double* launch_us);

/* Random-gather throughput: `count` loads x[idx[i]] with uniformly random
 * idx over an x of x_len floats, in the load forms the SpMV kernels use
 * (indices streamed, x through L1 with an L2 keep policy); mean of ntimes
 * launches. This is the ceiling of the irregular formats (CSR, COO, ELL on
 * scattered columns), whose time is set by x gathers rather than bytes. No
 * counterpart in the reference. */
int clspmv_gather_test(int x_len, long long count, int ntimes, int verbose, double* gathers_per_s);

/* evaluate (src/spmv_cocktail.cpp:1431-1455): upload the partitioned
 * matrix, check one SpMV y = A*vec + res against `coores` (NULL: skip), then
 * time `ntimes` SpMVs (the reference uses 1000). Prints the reference's
 * report lines with `verbose`. Any of the out pointers may be NULL. */
int clspmv_cocktail_evaluate_f32(const clspmv_cocktail_f32* host, const float* vec, const float* res,
                                 const float* coores, int ntimes, int verbose, double* ms, double* gflops,
                                 double* max_diff);

/* ReadMMF (src/fileio.cpp:10-109): a Matrix Market coordinate file into a
 * row-sorted COO (1-based indices made 0-based; pattern entries read as
 * 1.0; a "symmetric" matrix gets its mirrored off-diagonal entries).
 * CLSPMV_ERR_ARG when the file cannot be opened or parsed,
 * CLSPMV_ERR_UNSUPPORTED for complex values. Release with
 * clspmv_free_coo_f32. */
int clspmv_read_mmf_f32(const char* filename, clspmv_coo_f32* out);

/* Number of kernels this library launched since load (all entry points). */
long long clspmv_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* CLSPMV_B200_H */
