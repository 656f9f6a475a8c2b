/*
 * constant.h — compile-time limits shared with clSpMV (include/constant.h:1-55
 * of the reference). The names and values are the reference's because the
 * storage layouts (alignment, refusal caps) and the Cocktail tables depend on
 * them; CONTEXTTYPE and the OpenCL texture constants have no meaning here.
 */
#ifndef CLSPMV_CONSTANT_H
#define CLSPMV_CONSTANT_H

/* matrix_storage.h */
#define DIAINCSIZE 200
#define MAX_LEVELS 1000
#define MAX_MEM_OBJ 268435456

/* image2d x layout of the reference's _tx kernels (kept for table parsing) */
#define WIDTH_MASK 1023
#define LOG_WIDTH 10
#define VEC2DWIDTH 1024

/* alignment of padded lengths */
#define GPU_ALIGNMENT 32
#define COO_ALIGNMENT 32

/* warp geometry */
#define WARPSIZE 32
#define MAX_WARP_NUM 480
#define MAX_WARP_PER_PROC 48
#define WAVEFRONTSIZE 64
#define MIN_WAVE_PER_GROUP 4
#define WORK_GROUP_SIZE 256

/* format limits */
#define MAX_BAND_NUM 31
#define MAX_BAND_WIDTH 128
#define MAX_DIA_NUM 128
#define CSR_VEC_GROUP_SIZE 64
#define BCSR_VEC_GROUP_SIZE 128
#define CSR_VEC_MIN_TH_NUM 5760
#define BELL_GROUP_SIZE 256
#define SELL_GROUP_SIZE 128
#define COO_GROUP_SIZE 64

/* number of kernel variants per format in the Cocktail benchmark tables */
#define BDIA_IMP_NUM 5
#define DIA_IMP_NUM 4
#define SBELL_IMP_NUM 1
#define BELL_IMP_NUM 2
#define BCSR_IMP_NUM 1
#define SELL_IMP_NUM 2
#define ELL_IMP_NUM 2
#define CSR_IMP_NUM 2
#define COO_IMP_NUM 1

#endif
