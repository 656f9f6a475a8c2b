/*
 * spmv_serial.h — host serial SpMV templates, source-compatible with
 * include/spmv_serial.h of clSpMV (same names, arguments and results).
 *
 * Every routine computes result += A * vec in the matrix's own storage
 * order, one FP32 accumulator per row where the reference keeps one, so a
 * caller that compared against the reference's serial results gets the same
 * numbers. These are host utilities (reference answers for the benchmark
 * drivers' correctness lines and for callers' own checks); the GPU entry
 * points of libclspmv_b200 never call them.
 */
#ifndef CLSPMV_SPMV_SERIAL_H
#define CLSPMV_SPMV_SERIAL_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "matrix_storage.h"

/* dia_spmv (reference :11-34): rows up to the aligned length, columns
 * outside [0, vec_size) read as 0; `result` holds dia_length_aligned rows. */
template <class dimType, class offsetType, class dataType>
void dia_spmv(dia_matrix<dimType, offsetType, dataType>* mat, dataType* vec, dataType* result, dimType vec_size)
{
    const dimType len = mat->dia_length_aligned;
    for (dimType row = 0; row < len; row++) {
        dataType acc = (dataType)0;
        for (dimType d = 0; d < mat->dia_num; d++) {
            const offsetType col = row + mat->dia_offsets[d];
            const dataType v = (col >= (offsetType)0 && col < (offsetType)vec_size) ? vec[col] : (dataType)0;
            acc += v * mat->dia_data[(size_t)row + (size_t)d * len];
        }
        result[row] += acc;
    }
}

/* dia_ext_spmv (reference :36-57): `vec` is already extended on both sides,
 * so no column test. */
template <class dimType, class offsetType, class dataType>
void dia_ext_spmv(dia_ext_matrix<dimType, offsetType, dataType>* mat, dataType* vec, dataType* result, dimType vec_size)
{
    (void)vec_size;
    const dimType len = mat->dia_length_aligned;
    for (dimType row = 0; row < len; row++) {
        dataType acc = (dataType)0;
        for (dimType d = 0; d < mat->dia_num; d++)
            acc += vec[row + mat->dia_offsets[d]] * mat->dia_data[(size_t)row + (size_t)d * len];
        result[row] += acc;
    }
}

/* bdia_spmv (reference :59-89): band b covers diagonals offsets[b] ..
 * offsets[b] + (bptr[b+1] - bptr[b]) - 1. */
template <class dimType, class offsetType, class dataType>
void bdia_spmv(bdia_matrix<dimType, offsetType, dataType>* mat, dataType* vec, dataType* result, dimType vec_size)
{
    const dimType len = mat->bdia_length_aligned;
    for (dimType row = 0; row < len; row++) {
        dataType acc = (dataType)0;
        for (dimType b = 0; b < mat->bdia_band_num; b++) {
            offsetType col = row + mat->bdia_offsets[b];
            for (dimType i = mat->bdia_bptr[b]; i < mat->bdia_bptr[b + 1]; i++, col++) {
                const dataType v = (col >= (offsetType)0 && col < (offsetType)vec_size) ? vec[col] : (dataType)0;
                acc += v * mat->bdia_data[(size_t)row + (size_t)i * len];
            }
        }
        result[row] += acc;
    }
}

/* ell_spmv (reference :92-110): slot-major, adding straight into result. */
template <class dimType, class dataType>
void ell_spmv(ell_matrix<dimType, dataType>* mat, dataType* vec, dataType* result, dimType vec_size)
{
    (void)vec_size;
    const size_t len = (size_t)mat->ell_height_aligned;
    for (dimType slot = 0; slot < mat->ell_num; slot++)
        for (dimType row = 0; row < mat->matinfo.height; row++) {
            const size_t k = (size_t)slot * len + (size_t)row;
            result[row] += mat->ell_data[k] * vec[mat->ell_col_id[k]];
        }
}

/* sell_spmv (reference :112-135): per slice, column by column. */
template <class dimType, class dataType>
void sell_spmv(sell_matrix<dimType, dataType>* mat, dataType* vec, dataType* result, dimType vec_size)
{
    (void)vec_size;
    const dimType sh = (dimType)mat->sell_slice_height;
    for (dimType s = 0; s < mat->sell_slice_num; s++) {
        const dimType start = mat->sell_slice_ptr[s];
        const dimType width = (mat->sell_slice_ptr[s + 1] - start) / sh;
        for (dimType c = 0; c < width; c++)
            for (dimType r = 0; r < sh && s * sh + r < mat->matinfo.height; r++) {
                const size_t k = (size_t)start + (size_t)r + (size_t)c * sh;
                result[s * sh + r] += mat->sell_data[k] * vec[mat->sell_col_id[k]];
            }
    }
}

/* sbell_spmv (reference :137-181): float4 strips of each block, x reads
 * stop at the matrix width. */
template <class dimType, class dataType>
void sbell_spmv(sbell_matrix<dimType, dataType>* mat, dataType* vec, dataType* result, dimType vec_size)
{
    (void)vec_size;
    const unsigned bw = mat->sbell_bwidth, bh = mat->sbell_bheight, sh = mat->sbell_slice_height;
    for (dimType sl = 0; sl < mat->sbell_slice_num; sl++) {
        const dimType start = mat->sbell_slice_ptr[sl];
        const dimType width = (mat->sbell_slice_ptr[sl + 1] - start) / (dimType)sh;
        for (unsigned s = 0; s < sh; s++) {
            size_t coloff = (size_t)start + s;
            size_t dataoff = (size_t)start * bw * bh + (size_t)s * 4;
            for (dimType j = 0; j < width; j++, coloff += sh) {
                dimType col = mat->sbell_col_id[coloff] * 4;
                for (unsigned w4 = 0; w4 < bw / 4; w4++, col += 4)
                    for (unsigned h = 0; h < bh; h++, dataoff += (size_t)sh * 4) {
                        const dimType row = (dimType)((sl * sh + s) * bh + h);
                        if (row >= mat->matinfo.height) continue;
                        for (unsigned w = 0; w < 4 && col + (dimType)w < mat->matinfo.width; w++)
                            result[row] += mat->sbell_data[dataoff + w] * vec[col + w];
                    }
            }
        }
    }
}

/* coo_spmv (reference :183-196): one addition per stored entry, in order. */
template <class dimType, class dataType>
void coo_spmv(coo_matrix<dimType, dataType>* mat, dataType* vec, dataType* result, dimType vec_size)
{
    (void)vec_size;
    for (dimType i = 0; i < mat->matinfo.nnz; i++)
        result[mat->coo_row_id[i]] += mat->coo_data[i] * vec[mat->coo_col_id[i]];
}

/* csr_spmv (reference :198-217): one accumulator per row. */
template <class dimType, class dataType>
void csr_spmv(csr_matrix<dimType, dataType>* mat, dataType* vec, dataType* result, dimType vec_size)
{
    (void)vec_size;
    for (dimType row = 0; row < mat->matinfo.height; row++) {
        dataType acc = (dataType)0;
        for (dimType j = mat->csr_row_ptr[row]; j < mat->csr_row_ptr[row + 1]; j++)
            acc += mat->csr_data[j] * vec[mat->csr_col_id[j]];
        result[row] += acc;
    }
}

/* bcsr_spmv (reference :219-249): element (ir, ic) of every block of a
 * block row, then the next element. */
template <class dimType, class dataType>
void bcsr_spmv(bcsr_matrix<dimType, dataType>* mat, dataType* vec, dataType* result, dimType vec_size)
{
    const unsigned bw = mat->bcsr_bwidth, bh = mat->bcsr_bheight;
    for (dimType br = 0; br < mat->bcsr_row_num; br++)
        for (unsigned k = 0; k < bw * bh; k++) {
            const dimType row = br * (dimType)bh + (dimType)(k / bw);
            for (dimType j = mat->bcsr_row_ptr[br]; j < mat->bcsr_row_ptr[br + 1]; j++) {
                const dimType col = mat->bcsr_col_id[j] + (dimType)(k % bw);
                if (col < vec_size && row < mat->matinfo.height)
                    result[row] += mat->bcsr_data[(size_t)j + (size_t)k * mat->bcsr_aligned_size] * vec[col];
            }
        }
}

/* bell_spmv (reference :251-279): block column by block column; `result`
 * must hold bell_row_num * bheight rows. */
template <class dimType, class dataType>
void bell_spmv(bell_matrix<dimType, dataType>* mat, dataType* vec, dataType* result, dimType vec_size)
{
    (void)vec_size;
    const unsigned bw = mat->bell_bwidth, bh = mat->bell_bheight;
    const size_t len = (size_t)mat->bell_height_aligned, plane = len * bw * bh;
    for (dimType i = 0; i < mat->bell_block_num; i++)
        for (dimType br = 0; br < mat->bell_row_num; br++)
            for (unsigned k = 0; k < bw * bh; k++) {
                const dimType col = mat->bell_col_id[(size_t)i * len + br] + (dimType)(k % bw);
                result[(size_t)br * bh + k / bw] += mat->bell_data[(size_t)br + k * len + (size_t)i * plane] * vec[col];
            }
}

/* compareVectors (reference :282-300): exact equality, first mismatch printed. */
template <class dimType, class dataType>
bool compareVectors(dataType* vec1, dataType* vec2, dimType vec_size)
{
    for (dimType i = 0; i < vec_size; i++)
        if (vec1[i] != vec2[i]) {
            dataType diff = vec1[i] - vec2[i];
            if (diff < 0) diff = -diff;
            printf("Diff: id %d vec1 %f vec2 %f diff %f\n", (int)i, (double)vec1[i], (double)vec2[i], (double)diff);
            return false;
        }
    return true;
}

template <class dimType, class dataType>
void initVectorZero(dataType* vec, dimType vec_size)
{
    for (dimType i = 0; i < vec_size; i++) vec[i] = (dataType)0;
}

template <class dimType, class dataType>
void initVectorOne(dataType* vec, dimType vec_size)
{
    for (dimType i = 0; i < vec_size; i++) vec[i] = (dataType)1;
}

/* initVectorArbitrary (reference :322-330): vec[i] = i mod 1024. */
template <class dimType, class dataType>
void initVectorArbitrary(dataType* vec, dimType vec_size)
{
    for (dimType i = 0; i < vec_size; i++) vec[i] = (dataType)(i % 1024);
}

/* The reference's do<FMT> self-checks (:332-565): convert `mat`, run the
 * format's serial SpMV and the CSR one on vec, and report whether the two
 * results are identical. Each returns that verdict (the reference prints
 * it only). */
namespace clspmv_serial_detail {
template <class dimType, class dataType>
dataType* csr_answer(coo_matrix<dimType, dataType>* mat, dataType* vec, dimType vec_size)
{
    csr_matrix<dimType, dataType> csr;
    coo2csr<dimType, dataType>(mat, &csr);
    dataType* res = (dataType*)calloc((size_t)mat->matinfo.height + 1, sizeof(dataType));
    csr_spmv<dimType, dataType>(&csr, vec, res, vec_size);
    free_csr_matrix(csr);
    return res;
}
template <class dimType, class dataType>
bool agree(dataType* ref, dataType* got, dimType n, const char* name)
{
    const bool ok = compareVectors<dimType, dataType>(ref, got, n);
    printf("%s serial check: %s\n", name, ok ? "identical" : "different");
    free(ref);
    free(got);
    return ok;
}
}  // namespace clspmv_serial_detail

template <class dimType, class offsetType, class dataType>
bool doDIA(coo_matrix<dimType, dataType>* mat, dataType* vec, dimType vec_size)
{
    dia_matrix<dimType, offsetType, dataType> dia;
    if (!coo2dia<dimType, offsetType, dataType>(mat, &dia, (dimType)1)) return false;
    dataType* got = (dataType*)calloc((size_t)dia.dia_length_aligned + 1, sizeof(dataType));
    dia_spmv<dimType, offsetType, dataType>(&dia, vec, got, vec_size);
    free_dia_matrix(dia);
    return clspmv_serial_detail::agree(clspmv_serial_detail::csr_answer(mat, vec, vec_size), got, mat->matinfo.height,
                                       "DIA");
}

template <class dimType, class offsetType, class dataType>
bool doBDIA(coo_matrix<dimType, dataType>* mat, dataType* vec, dimType vec_size)
{
    bdia_matrix<dimType, offsetType, dataType> bdia;
    if (!coo2bdia<dimType, offsetType, dataType>(mat, &bdia, (dimType)1)) return false;
    dataType* got = (dataType*)calloc((size_t)bdia.bdia_length_aligned + 1, sizeof(dataType));
    bdia_spmv<dimType, offsetType, dataType>(&bdia, vec, got, vec_size);
    free_bdia_matrix(bdia);
    return clspmv_serial_detail::agree(clspmv_serial_detail::csr_answer(mat, vec, vec_size), got, mat->matinfo.height,
                                       "BDIA");
}

template <class dimType, class dataType>
bool doELL(coo_matrix<dimType, dataType>* mat, dataType* vec, dimType vec_size)
{
    ell_matrix<dimType, dataType> ell;
    if (!coo2ell<dimType, dataType>(mat, &ell, (dimType)1, (dimType)0)) return false;
    dataType* got = (dataType*)calloc((size_t)mat->matinfo.height + 1, sizeof(dataType));
    ell_spmv<dimType, dataType>(&ell, vec, got, vec_size);
    free_ell_matrix(ell);
    return clspmv_serial_detail::agree(clspmv_serial_detail::csr_answer(mat, vec, vec_size), got, mat->matinfo.height,
                                       "ELL");
}

template <class dimType, class dataType>
bool doBCSR(coo_matrix<dimType, dataType>* mat, dataType* vec, dimType vec_size, unsigned bwidth = 4, unsigned bheight = 4)
{
    bcsr_matrix<dimType, dataType> bcsr;
    coo2bcsr<dimType, dataType>(mat, &bcsr, bwidth, bheight, (dimType)1);
    dataType* got = (dataType*)calloc((size_t)bcsr.bcsr_row_num * bheight + 1, sizeof(dataType));
    bcsr_spmv<dimType, dataType>(&bcsr, vec, got, vec_size);
    free_bcsr_matrix(bcsr);
    return clspmv_serial_detail::agree(clspmv_serial_detail::csr_answer(mat, vec, vec_size), got, mat->matinfo.height,
                                       "BCSR");
}

template <class dimType, class dataType>
bool doBELL(coo_matrix<dimType, dataType>* mat, dataType* vec, dimType vec_size, unsigned bwidth = 4, unsigned bheight = 4)
{
    bell_matrix<dimType, dataType> bell;
    if (!coo2bell<dimType, dataType>(mat, &bell, bwidth, bheight, (dimType)1, (dimType)0)) return false;
    dataType* got = (dataType*)calloc((size_t)bell.bell_row_num * bheight + 1, sizeof(dataType));
    bell_spmv<dimType, dataType>(&bell, vec, got, vec_size);
    free_bell_matrix(bell);
    return clspmv_serial_detail::agree(clspmv_serial_detail::csr_answer(mat, vec, vec_size), got, mat->matinfo.height,
                                       "BELL");
}

#endif /* CLSPMV_SPMV_SERIAL_H */
