/*
 * util.h — host helpers, source-compatible with include/util.h of clSpMV
 * (src/util.cpp). Implemented in libclspmv_b200 (clspmv_mic_b200/csrc/compat.cpp).
 */
#ifndef CLSPMV_UTIL_H
#define CLSPMV_UTIL_H

#include "matrix_storage.h"

/* wall-clock seconds (src/util.cpp:10-15) */
double timestamp();
/* realSize rounded up to a multiple of alignment (:17-22) */
int findPaddedSize(int realSize, int alignment);
/* pad_csr (:31-72): rows padded to a multiple of `alignment` entries with
 * the row's last column and value 0. */
void pad_csr(csr_matrix<int, float>* source, csr_matrix<int, float>* dest, int alignment);
/* Euclidean distance of two vectors (:74-83) */
double distance(float* vec1, float* vec2, int size);
/* Checks res against a host COO product of mat and vec and prints the
 * comparison (:134-172). */
void correctness_check(coo_matrix<int, float>* mat, float* vec, float* res);
/* Prints size, diagonal-offset histogram and 16-column cache lines per row
 * (:174-245); sorts the matrix first if it is not sorted, as the reference. */
void printMatInfo(coo_matrix<int, float>* mat);
/* coores = A * vec from zero with the host COO product (:85-91) */
void spmv_only(coo_matrix<int, float>* mat, float* vec, float* coores);
/* Prints distance and largest differences of two result vectors (:93-131) */
void two_vec_compare(float* coovec, float* newvec, int size);
/* Re-lays a bell_matrix into float4 strips with float4 column ids
 * (:273-318): the b4ell data order on bell_matrix members. */
void rearrange_bell_4col(bell_matrix<int, float>* mat, int alignment);

#endif /* CLSPMV_UTIL_H */
