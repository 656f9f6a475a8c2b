// api_internal.h — helpers shared by the .cu files of libclspmv_b200.so.
#pragma once
#include <cuda_runtime.h>

namespace clspmv {
// Maps a CUDA error to a clspmv_status, remembering its text per thread.
int cuda_status(cudaError_t e);
// Counts `n` kernel launches and returns the status of the last launch.
int after_launch(int n);
}  // namespace clspmv
