/*
 * clspmv_oracle.c — CPU ORACLE for the parity tests. TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of clSpMV's serial SpMV routines (include/spmv_serial.h
 * of the reference), each computing result += A * vec in FP32 with the
 * reference's loop order, plus an FP64 CSR oracle that also returns the
 * per-row tolerance scale sum_j |a_ij * x_j|.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker or the timed CPU baseline; the
 * product path (libclspmv_b200.so) never calls it.
 *
 * Pinning: tests/test_oracle.py checks every routine here bit for bit
 * against the reference's own templates compiled from its sources
 * (oracle/_ref, built by oracle/Makefile) and against the committed golden
 * fixtures under tests/golden/, which were produced by that compiled
 * reference.
 *
 * Compile with -ffp-contract=off so that a*b+c is rounded twice, as the
 * reference's g++ build does on x86-64 without -mfma.
 */
#include <stddef.h>
#include "clspmv_b200.h"

/* coo_spmv: include/spmv_serial.h:183-196 */
void orc_coo_spmv_f32(const clspmv_coo_f32* m, const float* vec, float* result)
{
    for (int i = 0; i < m->matinfo.nnz; i++) {
        int row = m->coo_row_id[i];
        int col = m->coo_col_id[i];
        float data = m->coo_data[i];
        result[row] += data * vec[col];
    }
}

/* csr_spmv: include/spmv_serial.h:198-217 */
void orc_csr_spmv_f32(const clspmv_csr_f32* m, const float* vec, float* result)
{
    for (int row = 0; row < m->matinfo.height; row++) {
        float acc = 0.0f;
        for (int j = m->csr_row_ptr[row]; j < m->csr_row_ptr[row + 1]; j++) acc += m->csr_data[j] * vec[m->csr_col_id[j]];
        result[row] += acc;
    }
}

/* FP64 restatement of csr_spmv (same loop, double accumulation). Writes
 * result64[row] = sum_j a_ij x_j and scale[row] = sum_j |a_ij x_j|. */
void orc_csr_spmv_f64(const clspmv_csr_f32* m, const float* vec, double* result64, double* scale)
{
    for (int row = 0; row < m->matinfo.height; row++) {
        double acc = 0.0, s = 0.0;
        for (int j = m->csr_row_ptr[row]; j < m->csr_row_ptr[row + 1]; j++) {
            double p = (double)m->csr_data[j] * (double)vec[m->csr_col_id[j]];
            acc += p;
            s += p < 0 ? -p : p;
        }
        result64[row] = acc;
        scale[row] = s;
    }
}

/* dia_spmv: include/spmv_serial.h:11-34. Loops over the aligned length, so
 * `result` must hold dia_length_aligned entries; x entries past vec_size
 * read as 0. */
void orc_dia_spmv_f32(const clspmv_dia_f32* m, const float* vec, float* result, int vec_size)
{
    const int len = m->dia_length_aligned;
    for (int row = 0; row < len; row++) {
        float acc = 0.0f;
        for (int j = 0; j < m->dia_num; j++) {
            int col = row + m->dia_offsets[j];
            float a = m->dia_data[(size_t)row + (size_t)j * len];
            float v = 0.0f;
            if (col >= 0 && col < vec_size) v = vec[col];
            acc += v * a;
        }
        result[row] += acc;
    }
}

/* bdia_spmv: include/spmv_serial.h:59-89 (result sized bdia_length_aligned) */
void orc_bdia_spmv_f32(const clspmv_bdia_f32* m, const float* vec, float* result, int vec_size)
{
    const int len = m->bdia_length_aligned;
    for (int row = 0; row < len; row++) {
        float acc = 0.0f;
        for (int b = 0; b < m->bdia_band_num; b++) {
            int off = m->bdia_offsets[b];
            for (int i = m->bdia_bptr[b]; i < m->bdia_bptr[b + 1]; i++, off++) {
                int col = row + off;
                float a = m->bdia_data[(size_t)row + (size_t)i * len];
                float v = 0.0f;
                if (col >= 0 && col < vec_size) v = vec[col];
                acc += v * a;
            }
        }
        result[row] += acc;
    }
}

/* ell_spmv: include/spmv_serial.h:92-110 (slot-major accumulation into y) */
void orc_ell_spmv_f32(const clspmv_ell_f32* m, const float* vec, float* result)
{
    const size_t len = (size_t)m->ell_height_aligned;
    for (int i = 0; i < m->ell_num; i++)
        for (int j = 0; j < m->matinfo.height; j++) {
            size_t k = (size_t)i * len + (size_t)j;
            result[j] += m->ell_data[k] * vec[m->ell_col_id[k]];
        }
}

/* sell_spmv: include/spmv_serial.h:112-135 */
void orc_sell_spmv_f32(const clspmv_sell_f32* m, const float* vec, float* result)
{
    const int sh = (int)m->sell_slice_height;
    for (int s = 0; s < m->sell_slice_num; s++) {
        int start = m->sell_slice_ptr[s];
        int width = (m->sell_slice_ptr[s + 1] - start) / sh;
        for (int j = 0; j < width; j++)
            for (int row = s * sh; row < (s + 1) * sh && row < m->matinfo.height; row++) {
                size_t k = (size_t)start + (size_t)(row - s * sh) + (size_t)j * sh;
                result[row] += m->sell_data[k] * vec[m->sell_col_id[k]];
            }
    }
}

/* sbell_spmv: include/spmv_serial.h:137-181 (x reads stop at the matrix
 * width, :169-170) */
void orc_sbell_spmv_f32(const clspmv_sbell_f32* m, const float* vec, float* result)
{
    const unsigned bw = m->sbell_bwidth, bh = m->sbell_bheight, sh = m->sbell_slice_height;
    const unsigned bs = bw * bh;
    for (int i = 0; i < m->sbell_slice_num; i++) {
        int start = m->sbell_slice_ptr[i];
        int width = (m->sbell_slice_ptr[i + 1] - start) / (int)sh;
        for (unsigned s = 0; s < sh; s++) {
            size_t coloff = (size_t)start + s;
            size_t dataoff = (size_t)start * bs + (size_t)s * 4;
            for (int j = 0; j < width; j++) {
                int col = m->sbell_col_id[coloff] * 4;
                for (unsigned w4 = 0; w4 < bw / 4; w4++) {
                    for (unsigned h = 0; h < bh; h++) {
                        int row = (int)((i * sh + s) * bh + h);
                        if (row < m->matinfo.height) {
                            for (unsigned w = 0; w < 4; w++) {
                                float a = m->sbell_data[dataoff + w];
                                if (col + (int)w >= m->matinfo.width) break;
                                result[row] += a * vec[col + w];
                            }
                        }
                        dataoff += (size_t)sh * 4;
                    }
                    col += 4;
                }
                coloff += sh;
            }
        }
    }
}

/* bcsr_spmv: include/spmv_serial.h:219-249 */
void orc_bcsr_spmv_f32(const clspmv_bcsr_f32* m, const float* vec, float* result, int vec_size)
{
    const unsigned bw = m->bcsr_bwidth, bh = m->bcsr_bheight;
    for (int i = 0; i < m->bcsr_row_num; i++) {
        int r0 = i * (int)bh;
        for (unsigned k = 0; k < bw * bh; k++) {
            unsigned ic = k % bw, ir = k / bw;
            for (int j = m->bcsr_row_ptr[i]; j < m->bcsr_row_ptr[i + 1]; j++) {
                int col = m->bcsr_col_id[j] + (int)ic, row = r0 + (int)ir;
                if (col < vec_size && row < m->matinfo.height)
                    result[row] += m->bcsr_data[(size_t)j + (size_t)k * m->bcsr_aligned_size] * vec[col];
            }
        }
    }
}

/* bell_spmv: include/spmv_serial.h:251-279 (writes rows up to
 * bell_row_num * bheight, so `result` must be that long) */
void orc_bell_spmv_f32(const clspmv_bell_f32* m, const float* vec, float* result)
{
    const unsigned bw = m->bell_bwidth, bh = m->bell_bheight;
    const size_t len = (size_t)m->bell_height_aligned, colsz = len * bw * bh;
    for (int i = 0; i < m->bell_block_num; i++)
        for (int j = 0; j < m->bell_row_num; j++)
            for (unsigned k = 0; k < bw * bh; k++) {
                float a = m->bell_data[(size_t)j + k * len + (size_t)i * colsz];
                int col = m->bell_col_id[(size_t)i * len + j] + (int)(k % bw);
                result[(size_t)j * bh + k / bw] += a * vec[col];
            }
}

/* b4csr SpMV. The reference has no serial routine for this layout; this
 * restates its GPU kernels (kernels/spmv_bcsr.cl:4-1683): per block row, per
 * block in order, per row of the block, a 4-wide dot product per float4
 * strip, accumulated into that row. Columns past the width read as 0. */
void orc_b4csr_spmv_f32(const clspmv_b4csr_f32* m, const float* vec, float* result)
{
    const unsigned bw4 = m->b4csr_bwidth / 4, bh = m->b4csr_bheight;
    const size_t len = (size_t)m->b4csr_aligned_size;
    for (int br = 0; br < m->b4csr_row_num; br++)
        for (unsigned h = 0; h < bh; h++) {
            int row = br * (int)bh + (int)h;
            if (row >= m->matinfo.height) continue;
            float acc = 0.0f;
            for (int i = m->b4csr_row_ptr[br]; i < m->b4csr_row_ptr[br + 1]; i++)
                for (unsigned w4 = 0; w4 < bw4; w4++)
                    for (unsigned w = 0; w < 4; w++) {
                        int col = (m->b4csr_col_id[i] + (int)w4) * 4 + (int)w;
                        float a = m->b4csr_data[w4 * len * bh + h * len + (size_t)i * 4 + w];
                        float v = col < m->matinfo.width ? vec[col] : 0.0f;
                        acc += a * v;
                    }
            result[row] += acc;
        }
}

/* b4ell SpMV, restating kernels/spmv_bell.cl:4-1469 the same way. */
void orc_b4ell_spmv_f32(const clspmv_b4ell_f32* m, const float* vec, float* result)
{
    const unsigned bw4 = m->b4ell_bwidth / 4, bh = m->b4ell_bheight;
    const size_t f4 = (size_t)m->b4ell_float4_aligned, len = (size_t)m->b4ell_height_aligned;
    for (int br = 0; br < m->b4ell_row_num; br++)
        for (unsigned h = 0; h < bh; h++) {
            int row = br * (int)bh + (int)h;
            if (row >= m->matinfo.height) continue;
            float acc = 0.0f;
            for (int j = 0; j < m->b4ell_block_num; j++)
                for (unsigned w4 = 0; w4 < bw4; w4++)
                    for (unsigned w = 0; w < 4; w++) {
                        int col = (m->b4ell_col_id[(size_t)j * len + br] + (int)w4) * 4 + (int)w;
                        float a = m->b4ell_data[(size_t)j * f4 * bw4 * bh + w4 * f4 * bh + h * f4 + (size_t)br * 4 + w];
                        float v = col < m->matinfo.width ? vec[col] : 0.0f;
                        acc += a * v;
                    }
            result[row] += acc;
        }
}
