// api_internal.h — helpers shared by the .cu files of libclspmv_b200.so.
#pragma once
#include <cuda_runtime.h>
#include "clspmv_b200.h"

namespace clspmv {
// Maps a CUDA error to a clspmv_status, remembering its text per thread.
int cuda_status(cudaError_t e);
// Counts `n` kernel launches and returns the status of the last launch.
int after_launch(int n);

// Format launchers (spmv_api.cu). With `atomic`, alpha*A*x is added into y
// with red.global.add and beta is ignored (apply it first with
// launch_prescale); several launches may then target one y concurrently.
int launch_prescale(float* y, int n, float beta, cudaStream_t st);
int launch_dia(const clspmv_dia_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic);
int launch_bdia(const clspmv_bdia_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic);
int launch_ell(const clspmv_ell_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic);
int launch_sell(const clspmv_sell_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic);
int launch_sell_plan(const clspmv_sell_f32* m, const clspmv_sell_plan* plan, const float* x, float* y, float alpha,
                     float beta, cudaStream_t st, bool atomic);
int launch_csr_scalar(const clspmv_csr_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic);
int launch_csr_vector(const clspmv_csr_f32* m, const float* x, float* y, float alpha, float beta, int tpr, cudaStream_t st, bool atomic);
int launch_csr_merge(const clspmv_csr_f32* m, const int* tc, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic);
int launch_csr_merge_plan(const clspmv_csr_f32* m, int* tc, cudaStream_t st);
int launch_csr_chunk(const clspmv_csr_f32* m, const int* chunk_row, const float* x, float* y, float alpha, float beta,
                     cudaStream_t st, bool atomic);
int launch_csr_chunk_plan(const clspmv_csr_f32* m, int* chunk_row, cudaStream_t st);
int launch_coo(const clspmv_coo_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic);
int launch_b4ell(const clspmv_b4ell_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic);
int launch_sbell(const clspmv_sbell_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic);
int launch_packed(int format, const void* dev, int value_type, const void* values, const float* scale, const int* tc,
                  const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic);
int launch_b4csr(const clspmv_b4csr_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic);

// DIA / BDIA with the diagonals staged in shared memory by bulk copies
// (diag_bulk.cu); BDIA passes its bptr (the diagonal count is read on the
// device), DIA bptr = nullptr and its ndiag.
bool diag_bulk_supported(int len, const void* data);
int launch_diag_bulk(int rows, int cols, int ndiag, int len, const int* offsets, const int* bptr, int nband,
                     const float* data, const float* x, float* y, float alpha, float beta, cudaStream_t st);

// Fused Cocktail SpMV (cocktail_fused.cu): the parts of a partitioned matrix
// (device struct) cut into tiles, interleaved into one work list and run by
// one persistent launch. fused_plan_create returns CLSPMV_ERR_UNSUPPORTED
// when a part's layout is outside what the fused kernel covers.
struct FusedPlan;
int fused_plan_create(const clspmv_cocktail_f32* dev, const int* chunk_plan, FusedPlan** out);
int fused_spmv(const FusedPlan* plan, const float* x, float* y, float alpha, float beta, cudaStream_t st);
void fused_plan_free(FusedPlan* plan);
int fused_plan_items(const FusedPlan* plan);
}  // namespace clspmv
