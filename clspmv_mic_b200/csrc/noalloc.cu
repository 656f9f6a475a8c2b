// noalloc.cu — merge-path CSR SpMV whose tile plan lives in a fixed,
// statically sized device array, so a call allocates nothing.
//
// clspmv_csr_merge_spmv_f32 needs a caller-owned device buffer of tile
// coordinates (clspmv_csr_merge_plan). Some callers cannot provide one at
// the point of the call: a loop that must not allocate once it is running
// (cudaFree waits for the whole device, and cudaMalloc may too), a host
// language binding with no way to allocate device memory of its own, or a
// service that admits work against a fixed memory budget. For them this
// entry point keeps the plan in the array below, which is part of the
// library's device image: it exists as soon as the library's kernels are
// loaded on a device and is never freed.
//
// Limits and rules (also stated in clspmv_b200.h):
//  * the plan holds kNoallocMaxTiles + 1 tile starts, which covers
//    rows + nnz <= kNoallocMaxTiles * 2048 = 134,215,680; larger matrices
//    are rejected with CLSPMV_ERR_UNSUPPORTED before anything is launched;
//  * the first call on each device (with that device current) looks up the
//    array's device address with cudaGetSymbolAddress; make that first call
//    before starting any stream capture on that device;
//  * nothing has to start at zero: every call writes all tile starts it
//    reads, in the same stream, before the SpMV kernel runs;
//  * there is one array per device, so calls on the same device must not
//    overlap: two calls in flight at once (other streams or host threads)
//    overwrite each other's plan. Order them on one stream, or otherwise
//    wait for one before issuing the next.
#include <mutex>
#include "clspmv_b200.h"
#include "api_internal.h"

using namespace clspmv;

namespace {

constexpr int kNoallocMaxTiles = 65535;
constexpr int kNoallocMaxDevices = 64;

// 2 ints per tile start (rows done, nonzeros done): 512 KiB
static __device__ __align__(256) int g_noalloc_plan[2 * (kNoallocMaxTiles + 1)];

std::mutex g_noalloc_mu;
int* g_noalloc_ptr[kNoallocMaxDevices] = {};

// Device address of g_noalloc_plan on the current device, looked up once per
// device and kept for the life of the process; a cudaDeviceReset destroys
// the device's copy of the array, so the cached address is not valid after
// one (documented at the entry point's declaration).
int noalloc_plan(int** out)
{
    int dev = 0;
    int rc = cuda_status(cudaGetDevice(&dev));
    if (rc) return rc;
    if (dev < 0 || dev >= kNoallocMaxDevices) return CLSPMV_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        rc = cuda_status(cudaGetSymbolAddress(&p, g_noalloc_plan));
        if (rc) return rc;
        g_noalloc_ptr[dev] = static_cast<int*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return CLSPMV_OK;
}

}  // namespace

extern "C" {

int clspmv_csr_merge_noalloc_max_tiles(void) { return kNoallocMaxTiles; }

int clspmv_csr_merge_spmv_noalloc_f32(const clspmv_csr_f32* dev, const float* x, float* y, float alpha, float beta,
                                      clspmv_stream_t stream)
{
    if (!dev || !x || !y || !dev->csr_row_ptr) return CLSPMV_ERR_ARG;
    const int tiles = clspmv_csr_merge_tiles(dev->matinfo.height, dev->matinfo.nnz);
    if (tiles < 0) return CLSPMV_ERR_ARG;
    if (tiles > kNoallocMaxTiles) return CLSPMV_ERR_UNSUPPORTED;
    if (dev->matinfo.height <= 0) return CLSPMV_OK;
    int* plan = nullptr;
    int rc = noalloc_plan(&plan);
    if (rc) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    rc = launch_csr_merge_plan(dev, plan, st);
    if (rc) return rc;
    return launch_csr_merge(dev, plan, x, y, alpha, beta, st, false);
}

}  // extern "C"
