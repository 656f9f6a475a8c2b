// device_mem.cu — upload / device_free entry points: cudaMalloc + copy of
// every array of a host format struct into a device copy of the struct.
// They replace the ALLOCATE_GPU_READ uploads of the reference drivers
// (include/oclcommon.h:13-38) and cpy_<fmt>_mat of src/spmv_cocktail.cpp.
#include <cstring>
#include "clspmv_b200.h"
#include "api_internal.h"

using clspmv::cuda_status;

namespace {

template <class T>
int upload_array(T** dst, const T* src, size_t n)
{
    *dst = nullptr;
    if (n == 0) return CLSPMV_OK;
    if (!src) return CLSPMV_ERR_ARG;
    void* p = nullptr;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return CLSPMV_ERR_ALLOC;
    }
    int rc = cuda_status(cudaMemcpy(p, src, n * sizeof(T), cudaMemcpyHostToDevice));
    if (rc) {
        cudaFree(p);
        return rc;
    }
    *dst = static_cast<T*>(p);
    return CLSPMV_OK;
}

template <class T>
void release(T*& p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

// Uploads the listed arrays in order; on failure frees what was uploaded.
struct Uploader {
    void* done[4] = {nullptr, nullptr, nullptr, nullptr};
    int n = 0;
    int rc = CLSPMV_OK;
    template <class T>
    void add(T** dst, const T* src, size_t count)
    {
        if (rc) { *dst = nullptr; return; }
        rc = upload_array(dst, src, count);
        if (!rc) done[n++] = *dst;
    }
    int finish()
    {
        if (rc)
            for (int i = 0; i < n; i++)
                if (done[i]) cudaFree(done[i]);
        return rc;
    }
};

}  // namespace

extern "C" {

int clspmv_upload_coo_f32(const clspmv_coo_f32* h, clspmv_coo_f32* d)
{
    if (!h || !d || h->matinfo.nnz < 0) return CLSPMV_ERR_ARG;
    *d = *h;
    const size_t n = (size_t)h->matinfo.nnz;
    Uploader u;
    u.add(&d->coo_row_id, h->coo_row_id, n);
    u.add(&d->coo_col_id, h->coo_col_id, n);
    u.add(&d->coo_data, h->coo_data, n);
    return u.finish();
}

int clspmv_upload_csr_f32(const clspmv_csr_f32* h, clspmv_csr_f32* d)
{
    if (!h || !d || h->matinfo.nnz < 0 || h->matinfo.height < 0) return CLSPMV_ERR_ARG;
    *d = *h;
    const size_t n = (size_t)h->matinfo.nnz;
    Uploader u;
    u.add(&d->csr_row_ptr, h->csr_row_ptr, (size_t)h->matinfo.height + 1);
    u.add(&d->csr_col_id, h->csr_col_id, n);
    u.add(&d->csr_data, h->csr_data, n);
    return u.finish();
}

int clspmv_upload_dia_f32(const clspmv_dia_f32* h, clspmv_dia_f32* d)
{
    if (!h || !d || h->dia_num < 0 || h->dia_length_aligned < 0) return CLSPMV_ERR_ARG;
    *d = *h;
    Uploader u;
    u.add(&d->dia_offsets, h->dia_offsets, (size_t)h->dia_num);
    u.add(&d->dia_data, h->dia_data, (size_t)h->dia_num * (size_t)h->dia_length_aligned);
    return u.finish();
}

int clspmv_upload_bdia_f32(const clspmv_bdia_f32* h, clspmv_bdia_f32* d)
{
    if (!h || !d || h->bdia_band_num < 0 || (h->bdia_band_num > 0 && !h->bdia_bptr)) return CLSPMV_ERR_ARG;
    *d = *h;
    const size_t ndiag = h->bdia_band_num > 0 ? (size_t)h->bdia_bptr[h->bdia_band_num] : 0;
    Uploader u;
    u.add(&d->bdia_offsets, h->bdia_offsets, (size_t)h->bdia_band_num);
    u.add(&d->bdia_bptr, h->bdia_bptr, (size_t)h->bdia_band_num + (h->bdia_band_num > 0 ? 1 : 0));
    u.add(&d->bdia_data, h->bdia_data, ndiag * (size_t)h->bdia_length_aligned);
    return u.finish();
}

int clspmv_upload_ell_f32(const clspmv_ell_f32* h, clspmv_ell_f32* d)
{
    if (!h || !d || h->ell_num < 0 || h->ell_height_aligned < 0) return CLSPMV_ERR_ARG;
    *d = *h;
    const size_t n = (size_t)h->ell_num * (size_t)h->ell_height_aligned;
    Uploader u;
    u.add(&d->ell_col_id, h->ell_col_id, n);
    u.add(&d->ell_data, h->ell_data, n);
    return u.finish();
}

int clspmv_upload_sell_f32(const clspmv_sell_f32* h, clspmv_sell_f32* d)
{
    if (!h || !d || h->sell_slice_num < 0 || !h->sell_slice_ptr) return CLSPMV_ERR_ARG;
    *d = *h;
    const size_t n = (size_t)h->sell_slice_ptr[h->sell_slice_num];
    Uploader u;
    u.add(&d->sell_slice_ptr, h->sell_slice_ptr, (size_t)h->sell_slice_num + 1);
    u.add(&d->sell_col_id, h->sell_col_id, n);
    u.add(&d->sell_data, h->sell_data, n);
    return u.finish();
}

int clspmv_upload_b4csr_f32(const clspmv_b4csr_f32* h, clspmv_b4csr_f32* d)
{
    if (!h || !d || h->b4csr_row_num < 0 || h->b4csr_block_num < 0) return CLSPMV_ERR_ARG;
    *d = *h;
    const size_t n = (size_t)h->b4csr_aligned_size * h->b4csr_bheight * (h->b4csr_bwidth / 4);
    Uploader u;
    u.add(&d->b4csr_row_ptr, h->b4csr_row_ptr, (size_t)h->b4csr_row_num + 1);
    u.add(&d->b4csr_col_id, h->b4csr_col_id, (size_t)h->b4csr_block_num);
    u.add(&d->b4csr_data, h->b4csr_data, n);
    return u.finish();
}

int clspmv_upload_bcsr_f32(const clspmv_bcsr_f32* h, clspmv_bcsr_f32* d)
{
    if (!h || !d || h->bcsr_row_num < 0 || h->bcsr_block_num < 0 || h->bcsr_aligned_size < 0) return CLSPMV_ERR_ARG;
    *d = *h;
    Uploader u;
    u.add(&d->bcsr_row_ptr, h->bcsr_row_ptr, (size_t)h->bcsr_row_num + 1);
    u.add(&d->bcsr_col_id, h->bcsr_col_id, (size_t)h->bcsr_block_num);
    u.add(&d->bcsr_data, h->bcsr_data, (size_t)h->bcsr_aligned_size * h->bcsr_bwidth * h->bcsr_bheight);
    return u.finish();
}

int clspmv_upload_bell_f32(const clspmv_bell_f32* h, clspmv_bell_f32* d)
{
    if (!h || !d || h->bell_block_num < 0 || h->bell_height_aligned < 0) return CLSPMV_ERR_ARG;
    *d = *h;
    const size_t ncol = (size_t)h->bell_height_aligned * h->bell_block_num;
    Uploader u;
    u.add(&d->bell_col_id, h->bell_col_id, ncol);
    u.add(&d->bell_data, h->bell_data, ncol * h->bell_bwidth * h->bell_bheight);
    return u.finish();
}

int clspmv_upload_b4ell_f32(const clspmv_b4ell_f32* h, clspmv_b4ell_f32* d)
{
    if (!h || !d || h->b4ell_block_num < 0 || h->b4ell_height_aligned < 0) return CLSPMV_ERR_ARG;
    *d = *h;
    const size_t ncol = (size_t)h->b4ell_height_aligned * h->b4ell_block_num;
    const size_t ndata = (size_t)h->b4ell_float4_aligned * h->b4ell_bheight * (h->b4ell_bwidth / 4) * h->b4ell_block_num;
    Uploader u;
    u.add(&d->b4ell_col_id, h->b4ell_col_id, ncol);
    u.add(&d->b4ell_data, h->b4ell_data, ndata);
    return u.finish();
}

int clspmv_upload_sbell_f32(const clspmv_sbell_f32* h, clspmv_sbell_f32* d)
{
    if (!h || !d || h->sbell_slice_num < 0 || !h->sbell_slice_ptr) return CLSPMV_ERR_ARG;
    *d = *h;
    const size_t n = (size_t)h->sbell_slice_ptr[h->sbell_slice_num];
    Uploader u;
    u.add(&d->sbell_slice_ptr, h->sbell_slice_ptr, (size_t)h->sbell_slice_num + 1);
    u.add(&d->sbell_col_id, h->sbell_col_id, n);
    u.add(&d->sbell_data, h->sbell_data, n * h->sbell_bwidth * h->sbell_bheight);
    return u.finish();
}

int clspmv_device_free_coo_f32(clspmv_coo_f32* d) { if (!d) return CLSPMV_ERR_ARG; release(d->coo_row_id); release(d->coo_col_id); release(d->coo_data); return CLSPMV_OK; }
int clspmv_device_free_csr_f32(clspmv_csr_f32* d) { if (!d) return CLSPMV_ERR_ARG; release(d->csr_row_ptr); release(d->csr_col_id); release(d->csr_data); return CLSPMV_OK; }
int clspmv_device_free_dia_f32(clspmv_dia_f32* d) { if (!d) return CLSPMV_ERR_ARG; release(d->dia_offsets); release(d->dia_data); return CLSPMV_OK; }
int clspmv_device_free_bdia_f32(clspmv_bdia_f32* d) { if (!d) return CLSPMV_ERR_ARG; release(d->bdia_offsets); release(d->bdia_bptr); release(d->bdia_data); return CLSPMV_OK; }
int clspmv_device_free_ell_f32(clspmv_ell_f32* d) { if (!d) return CLSPMV_ERR_ARG; release(d->ell_col_id); release(d->ell_data); return CLSPMV_OK; }
int clspmv_device_free_sell_f32(clspmv_sell_f32* d) { if (!d) return CLSPMV_ERR_ARG; release(d->sell_slice_ptr); release(d->sell_col_id); release(d->sell_data); return CLSPMV_OK; }
int clspmv_device_free_b4csr_f32(clspmv_b4csr_f32* d) { if (!d) return CLSPMV_ERR_ARG; release(d->b4csr_row_ptr); release(d->b4csr_col_id); release(d->b4csr_data); return CLSPMV_OK; }
int clspmv_device_free_bcsr_f32(clspmv_bcsr_f32* d) { if (!d) return CLSPMV_ERR_ARG; release(d->bcsr_row_ptr); release(d->bcsr_col_id); release(d->bcsr_data); return CLSPMV_OK; }
int clspmv_device_free_bell_f32(clspmv_bell_f32* d) { if (!d) return CLSPMV_ERR_ARG; release(d->bell_col_id); release(d->bell_data); return CLSPMV_OK; }
int clspmv_device_free_b4ell_f32(clspmv_b4ell_f32* d) { if (!d) return CLSPMV_ERR_ARG; release(d->b4ell_col_id); release(d->b4ell_data); return CLSPMV_OK; }
int clspmv_device_free_sbell_f32(clspmv_sbell_f32* d) { if (!d) return CLSPMV_ERR_ARG; release(d->sbell_slice_ptr); release(d->sbell_col_id); release(d->sbell_data); return CLSPMV_OK; }

}  // extern "C"
