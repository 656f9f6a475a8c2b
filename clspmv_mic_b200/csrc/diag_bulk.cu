// diag_bulk.cu — DIA and BDIA SpMV with the diagonals staged in shared
// memory by bulk copies (sm_100a).
//
// The register kernels of kernels.cuh (dia_cta / bdia_cta) keep four 128-bit
// loads of diagonal data in flight per thread; on B200 that leaves the
// stencil SpMV latency bound (most warps stalled on long scoreboard, about a
// quarter of issue slots used) at about 0.72 of the HBM copy rate. Here the
// bytes in flight no longer depend on registers: per CTA one producer warp
// streams, for tile after tile of kBulkRows rows, the tile's slice of every
// diagonal (kBulkRows contiguous floats of dia_data each, one cp.async.bulk
// per diagonal, kBulkChunk diagonals per stage) into a ring of shared-memory
// stages, and eight consumer warps compute four consecutive rows per thread
// from shared memory (128-bit reads), gathering x through L1. Stage handoff is by mbarrier pairs: the producer arms `full` with the
// stage's byte count and the copies complete it; the consumers arrive on
// `empty` when they are done with the stage. Two CTAs per SM keep up to
// 2 x (stages - 1) tiles of diagonal data in flight per SM.
//
// The layout is the reference's (dia_data[d * dia_length_aligned + row],
// include/matrix_storage.h:30-47; BDIA keeps the same data array with its
// diagonals grouped in bands of consecutive offsets, :72-94), so the kernel
// serves both: each diagonal's column offset is taken from the DIA offsets
// or from its band's first offset plus its place in the band.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include "clspmv_b200.h"
#include "common.cuh"
#include "pipeline.cuh"
#include "api_internal.h"

using namespace clspmv;

namespace {

// waits of the bulk-copy pipelines that ran out (clspmv_pipeline_timeouts)
__device__ unsigned int g_pipeline_timeouts;

constexpr int kBulkRows = 1024;                   // rows per tile
constexpr int kBulkChunk = 9;                     // diagonals per stage (the 27-point stencil: 3 stages a tile)
constexpr int kBulkStages = 3;
constexpr int kBulkMaxDiags = 1024;               // offsets kept in shared memory
constexpr size_t kBulkStageFloats = (size_t)kBulkChunk * kBulkRows;
constexpr size_t kBulkSmem = kBulkStages * kBulkStageFloats * 4 + kBulkMaxDiags * 4 + kBulkStages * 16;   // 112 KB

struct DiagBulkArgs {
    int rows, cols, ndiag, len;       // len = dia_length_aligned (multiple of 32); BDIA: ndiag = -1 (read from bptr)
    const int* offsets;               // DIA: one per diagonal; BDIA: first offset of each band
    const int* bptr;                  // BDIA: nband + 1 diagonal starts; DIA: nullptr
    int nband;
    const float* data;
    const float* x;
    float* y;
    float alpha, beta;
    int cta_rows;                     // rows per CTA, a multiple of 32
};

__device__ __forceinline__ float x_at(const float* x, long long c, int cols, uint64_t pol)
{
    return (unsigned long long)c < (unsigned long long)cols ? ld_x(x + c, pol) : 0.f;
}

// column offset of diagonal d (DIA: its own; BDIA: its band's first offset
// plus its place in the band)
__device__ __forceinline__ int diag_offset(const DiagBulkArgs& a, int d)
{
    if (!a.bptr) return a.offsets[d];
    int b = 0;
    while (b + 1 < a.nband && a.bptr[b + 1] <= d) b++;
    return a.offsets[b] + (d - a.bptr[b]);
}

// acc[i] += sum over the chunk's diagonals of data * x for the thread's RPT
// consecutive rows (RPT = 2 or 4: one 64- or 128-bit shared read per diagonal)
template <int RPT>
__device__ __forceinline__ void bulk_rows(const float* sd, int nd, const int* so, long long r0, int cols, const float* x,
                                          uint64_t pol, float (&acc)[RPT])
{
#pragma unroll 3
    for (int d = 0; d < nd; d++) {
        float v[RPT];
        if constexpr (RPT == 4) {
            const float4 w = *reinterpret_cast<const float4*>(sd + (size_t)d * kBulkRows);
            v[0] = w.x; v[1] = w.y; v[2] = w.z; v[3] = w.w;
        } else {
            const float2 w = *reinterpret_cast<const float2*>(sd + (size_t)d * kBulkRows);
            v[0] = w.x; v[1] = w.y;
        }
        const long long c = r0 + so[d];
        float xv[RPT];
        if (c >= 0 && c + RPT - 1 < cols) {
#pragma unroll
            for (int i = 0; i < RPT; i++) xv[i] = ld_x(x + c + i, pol);
        } else {
#pragma unroll
            for (int i = 0; i < RPT; i++) xv[i] = x_at(x, c + i, cols, pol);
        }
#pragma unroll
        for (int i = 0; i < RPT; i++) acc[i] = fmaf(v[i], xv[i], acc[i]);
    }
}

// A CTA owns rows [cta * cta_rows, ...), walked in tiles of kBulkRows rows
// (the last one partial); each tile in chunks of up to kBulkChunk diagonals.
// Unit u = (tile u / nchunk, chunk u % nchunk) goes through stage u % kBulkStages.
template <int CONS, int RPT>
__global__ void __launch_bounds__(CONS + 32, 2) k_diag_bulk(DiagBulkArgs a)
{
    static_assert(CONS * RPT == kBulkRows, "a tile is one row group per consumer thread");
    constexpr int kConsumerWarps = CONS / 32;
    extern __shared__ __align__(128) char smem[];
    float* sdata = reinterpret_cast<float*>(smem);
    int* soff = reinterpret_cast<int*>(smem + kBulkStages * kBulkStageFloats * 4);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kBulkStages * kBulkStageFloats * 4 + kBulkMaxDiags * 4);
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kBulkStages);

    const long long rb = (long long)blockIdx.x * a.cta_rows;
    const long long re = min((long long)a.rows, rb + a.cta_rows);
    if (rb >= re) return;
    const int ndiag = a.bptr ? (a.nband > 0 ? a.bptr[a.nband] : 0) : a.ndiag;
    if (ndiag <= 0) {   // no stored diagonal: y <- beta * y
        for (long long r = rb + threadIdx.x; r < re; r += blockDim.x) a.y[r] = a.beta == 0.0f ? 0.0f : a.beta * a.y[r];
        return;
    }
    for (int d = threadIdx.x; d < min(ndiag, kBulkMaxDiags); d += blockDim.x) soff[d] = diag_offset(a, d);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kBulkStages; s++) {
            pl_mbar_init(full0 + 8 * s, 1);
            pl_mbar_init(empty0 + 8 * s, kConsumerWarps);
        }
        pl_fence_init();
    }
    __syncthreads();

    const long long ntile = (re - rb + kBulkRows - 1) / kBulkRows;
    const int nchunk = (ndiag + kBulkChunk - 1) / kBulkChunk;
    const long long nunits = ntile * nchunk;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == kConsumerWarps) {
        // producer: one warp, each lane copying one diagonal of the chunk
        const uint64_t pe = policy_evict_first();
        for (long long u = 0; u < nunits; u++) {
            const int s = (int)(u % kBulkStages);
            if (u >= kBulkStages && !pl_wait(empty0 + 8 * s, (uint32_t)((u / kBulkStages - 1) & 1), &g_pipeline_timeouts))
                return;
            const long long row0 = rb + (u / nchunk) * kBulkRows;
            const int d0 = (int)(u % nchunk) * kBulkChunk, nd = min(kBulkChunk, ndiag - d0);
            // whole 32-row runs: never past dia_length_aligned (a multiple of 32 that is >= rows)
            const long long nrows = min((long long)kBulkRows, re - row0);
            const uint32_t bytes = (uint32_t)((nrows + 31) / 32 * 32) * 4u;
            const uint32_t full = full0 + 8 * s;
            if (lane == 0) pl_arrive_expect_tx(full, bytes * (uint32_t)nd);
            __syncwarp();
            const uint32_t dst = smem_u32(sdata + (size_t)s * kBulkStageFloats);
            if (lane < nd)
                pl_bulk_g2s(dst + (uint32_t)lane * kBulkRows * 4u, a.data + (size_t)(d0 + lane) * a.len + row0, bytes, full, pe);
        }
        // every copy issued has completed on its `full` barrier before the
        // consumers passed it; nothing is left in flight here
        return;
    }

    // consumers: RPT consecutive rows per thread
    const uint64_t pl = policy_evict_last();
    float acc[RPT];
#pragma unroll
    for (int i = 0; i < RPT; i++) acc[i] = 0.f;
    for (long long u = 0; u < nunits; u++) {
        const int s = (int)(u % kBulkStages);
        if (!pl_wait(full0 + 8 * s, (uint32_t)((u / kBulkStages) & 1), &g_pipeline_timeouts)) {
            // these copies never landed: wait (bounded) for the ones issued
            // into the other stages, then leave
            for (long long k = 1; k < kBulkStages && u + k < nunits; k++)
                pl_wait(full0 + 8 * ((u + k) % kBulkStages), (uint32_t)(((u + k) / kBulkStages) & 1), &g_pipeline_timeouts);
            return;
        }
        const long long r0 = rb + (u / nchunk) * kBulkRows + (long long)threadIdx.x * RPT;
        const int c = (int)(u % nchunk), d0 = c * kBulkChunk, nd = min(kBulkChunk, ndiag - d0);
        if (r0 < re) {
            const float* sd = sdata + (size_t)s * kBulkStageFloats + (size_t)threadIdx.x * RPT;
            if (d0 + nd <= kBulkMaxDiags) {
                bulk_rows<RPT>(sd, nd, soff + d0, r0, a.cols, a.x, pl, acc);
            } else {   // diagonals past the shared offset table: offsets from global memory
                int so[kBulkChunk];
                for (int d = 0; d < nd; d++) so[d] = diag_offset(a, d0 + d);
                bulk_rows<RPT>(sd, nd, so, r0, a.cols, a.x, pl, acc);
            }
        }
        __syncwarp();
        if (lane == 0) pl_arrive(empty0 + 8 * s);
        if (c == nchunk - 1) {
#pragma unroll
            for (int i = 0; i < RPT; i++) {
                if (r0 + i < re) {
                    const float old = a.beta == 0.0f ? 0.0f : a.beta * a.y[r0 + i];
                    a.y[r0 + i] = old + a.alpha * acc[i];
                }
                acc[i] = 0.f;
            }
        }
    }
}

}  // namespace

namespace clspmv {

// DIA / BDIA data the bulk kernel can stage: rows in whole 128-byte runs and
// a 16-byte aligned data array (any number of diagonals; BDIA's count is read
// on the device).
bool diag_bulk_supported(int len, const void* data)
{
    return (len & 31) == 0 && (reinterpret_cast<uintptr_t>(data) & 15u) == 0;
}

// y <- alpha * A x + beta * y for DIA (bptr == nullptr) or BDIA data laid out
// as dia_data; plain stores into y (the rows belong to this launch alone).
int launch_diag_bulk(int rows, int cols, int ndiag, int len, const int* offsets, const int* bptr, int nband,
                     const float* data, const float* x, float* y, float alpha, float beta, cudaStream_t st)
{
    // consumer shape: 256 threads x 4 rows or 512 x 2 (CLSPMV_BULK_CONSUMERS=512, for measurements)
    static const int cons = [] {
        const char* e = getenv("CLSPMV_BULK_CONSUMERS");
        return e && atoi(e) == 512 ? 512 : 256;
    }();
    auto go = [&](auto kernel, int threads) {
        int dev = 0, nsm = 148, per = 1;
        cudaGetDevice(&dev);
        // the shared-memory opt-in is a per-device function attribute
        static std::atomic<bool> configured[64];
        if (dev < 0 || dev >= 64) return (int)CLSPMV_ERR_UNSUPPORTED;
        if (!configured[dev].load()) {
            int rc = cuda_status(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBulkSmem));
            if (rc) return rc;
            configured[dev] = true;
        }
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, kBulkSmem) != cudaSuccess || per < 1) {
            cudaGetLastError();
            per = 1;
        }
        // equal row ranges (multiples of 32 rows) for all resident CTAs
        const long long want = std::max(1LL, (long long)nsm * per);
        long long cta_rows = ((long long)rows + want - 1) / want;
        cta_rows = std::max(32LL, (cta_rows + 31) / 32 * 32);
        const unsigned grid = (unsigned)(((long long)rows + cta_rows - 1) / cta_rows);
        DiagBulkArgs a{rows, cols, bptr ? -1 : ndiag, len, offsets, bptr, nband, data, x, y, alpha, beta, (int)cta_rows};
        kernel<<<grid, threads, kBulkSmem, st>>>(a);
        return after_launch(1);
    };
    if (cons == 512) return go(k_diag_bulk<512, 2>, 512 + 32);
    return go(k_diag_bulk<256, 4>, 256 + 32);
}

}  // namespace clspmv

extern "C" int clspmv_pipeline_timeouts(unsigned int* count)
{
    if (!count) return CLSPMV_ERR_ARG;
    const unsigned int zero = 0;
    if (cudaMemcpyFromSymbol(count, g_pipeline_timeouts, sizeof(unsigned int)) != cudaSuccess) return CLSPMV_ERR_CUDA;
    if (cudaMemcpyToSymbol(g_pipeline_timeouts, &zero, sizeof(unsigned int)) != cudaSuccess) return CLSPMV_ERR_CUDA;
    return CLSPMV_OK;
}
