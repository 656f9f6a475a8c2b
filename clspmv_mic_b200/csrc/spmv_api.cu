// spmv_api.cu — extern "C" compute and residency entry points of
// libclspmv_b200.so: argument checks, template dispatch, launches.
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <algorithm>
#include <mutex>
#include <unordered_map>
#include <vector>
#include <new>
#include "clspmv_b200.h"
#include "kernels.cuh"
#include "api_internal.h"

using namespace clspmv;

namespace clspmv {

static thread_local std::string g_last_cuda_error;
static std::atomic<long long> g_launches{0};

int cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return CLSPMV_OK;
    g_last_cuda_error = cudaGetErrorString(e);
    return CLSPMV_ERR_CUDA;
}

int after_launch(int n)
{
    g_launches += n;
    return cuda_status(cudaGetLastError());
}

}  // namespace clspmv

namespace {

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
// value arrays are read 4 values at a time
template <class V> inline bool aligned_v4(const V* p) { return (reinterpret_cast<uintptr_t>(p) & (4 * sizeof(V) - 1)) == 0; }
inline cudaStream_t S(clspmv_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }
inline unsigned grid_for(long long units, long long per_cta) { return (unsigned)((units + per_cta - 1) / per_cta); }

// ---------------------------------------------------------------------------
// __global__ wrappers: one tile per CTA.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_scale(float* y, int n, float beta)
{
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i < n) y[i] = beta == 0.0f ? 0.0f : beta * y[i];
}

template <bool A, class V, int XF>
__global__ void __launch_bounds__(kBlock) k_dia(DiaArgsT<V> a)
{
    __shared__ __align__(16) char smem[kDiaSmemBytes];
    dia_cta<A, V, XF>(a, blockIdx.x, gridDim.x, smem);
}

template <bool A, class V, bool XA>
__global__ void __launch_bounds__(kBlock) k_bdia(BdiaArgsT<V> a) { bdia_cta<A, V, XA>(a, blockIdx.x, gridDim.x, nullptr); }

// the same, capped at the registers that keep 8 (DIA) / 5 (BDIA) CTAs of 256 threads per SM
template <bool A, class V, int XF>
__global__ void __launch_bounds__(kBlock, 8) k_dia_occ(DiaArgsT<V> a)
{
    __shared__ __align__(16) char smem[kDiaSmemBytes];
    dia_cta<A, V, XF>(a, blockIdx.x, gridDim.x, smem);
}
template <bool A, class V, bool XA>
__global__ void __launch_bounds__(kBlock, 5) k_bdia_occ(BdiaArgsT<V> a) { bdia_cta<A, V, XA>(a, blockIdx.x, gridDim.x, nullptr); }

// Kernel form of the diagonal formats: 0 scalar x loads, 1 aligned x
// windows, 2 aligned x windows with the register cap, 3 (DIA) one aligned
// window per lane completed by shuffles, 4 diagonals staged in shared memory
// by bulk copies (diag_bulk.cu; FP32 values, own rows only). Measured on B200 (stencil27 128^3):
// DIA is fastest with form 0 (74.6 % of peak vs 60 / 72 / 53), BDIA with
// form 1 (78 % vs 69 / 75). CLSPMV_DIA_FORM overrides both (for
// measurements).
constexpr int kDiaDefaultForm = 0, kBdiaDefaultForm = 1;
int dia_form(int dflt)
{
    static int forced = [] {
        const char* e = getenv("CLSPMV_DIA_FORM");
        return e ? atoi(e) : -1;
    }();
    return forced >= 0 ? forced : dflt;
}

template <bool A, class V, int GX = 0>
__global__ void __launch_bounds__(kBlock) k_ell(EllArgsT<V> a) { ell_cta<A, V, GX>(a, blockIdx.x, gridDim.x, nullptr); }

template <int Q, bool A, class V>
__global__ void __launch_bounds__(kBlock) k_sell(SellArgsT<V> a) { sell_cta<Q, A>(a, blockIdx.x, gridDim.x, nullptr); }

template <bool A, class V>
__global__ void __launch_bounds__(kBlock) k_sell_rows(SellArgsT<V> a) { sell_rows_cta<A>(a, blockIdx.x, gridDim.x, nullptr); }

template <bool A, class V>
__global__ void __launch_bounds__(kBlock) k_sell_rows4(SellArgsT<V> a) { sell_rows4_cta<A>(a, blockIdx.x, gridDim.x, nullptr); }

__global__ void __launch_bounds__(kBlock) k_sell_rlen(const int* __restrict__ slice_ptr, const int* __restrict__ col,
                                                      const float* __restrict__ data, int sh, long long rows, int* rlen)
{
    for (long long r = blockIdx.x * (long long)kBlock + threadIdx.x; r < rows; r += (long long)gridDim.x * kBlock)
        rlen[r] = sell_row_length(slice_ptr, col, data, sh, r);
}

// 8 CTAs per SM (32 registers, a few spilled): measured on B200 over the
// power-law SELL-32 heads, 0.273 ms for the planned SpMV against 0.292 at 6
// CTAs (40 registers) and 0.318 at 4 (62 registers): the walk is latency
// bound, so warps in flight count more than the spills
template <int Q, bool A, class V = float>
__global__ void __launch_bounds__(kBlock, 8) k_sell_masked(SellArgsT<V> a, const int* __restrict__ rlen,
                                                           const int* __restrict__ head)
{
    sell_masked_cta<Q, A, V>(a, rlen, blockIdx.x, gridDim.x, head);
}
template <bool A>
__global__ void __launch_bounds__(kBlock) k_sell_head(SellArgs a, const int* __restrict__ rlen)
{
    sell_head_cta<A>(a, rlen, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(kBlock) k_sell_tail(SellArgs a, const int* __restrict__ rlen, const int2* __restrict__ items,
                                                      long long nitems)
{
    sell_tail_cta(a, rlen, items, nitems, blockIdx.x, gridDim.x);
}

template <class V = float>
__global__ void __launch_bounds__(kBlock) k_sell_tail_compact(SellArgsT<V> a, const int* __restrict__ rlen,
                                                              const int2* __restrict__ items, const int* __restrict__ tail_off,
                                                              const int* __restrict__ tail_col, long long nitems)
{
    sell_tail_compact_cta<V>(a, rlen, items, tail_off, tail_col, nitems, blockIdx.x, gridDim.x);
}

// The planned SELL walk in one launch: CTAs [0, ntail) take the long rows'
// tails, the rest the slice heads (every head update atomic, since a tail
// CTA may add to the same row meanwhile), so the latency-bound head walk and
// the bandwidth-bound tails share the SMs instead of running one after the
// other.
template <int Q, class V>
__global__ void __launch_bounds__(kBlock, 8) k_sell_planned_one(SellArgsT<V> a, const int* __restrict__ rlen,
                                                                const int* __restrict__ head, const int2* __restrict__ items,
                                                                const int* __restrict__ tail_off,
                                                                const int* __restrict__ tail_col, long long nitems, int ntail)
{
    if ((int)blockIdx.x < ntail)
        sell_tail_compact_cta<V>(a, rlen, items, tail_off, tail_col, nitems, blockIdx.x, ntail);
    else
        sell_masked_cta<Q, true, V>(a, rlen, blockIdx.x - ntail, gridDim.x - ntail, head);
}

// Share of the one launch's CTAs on the tails, per mille: measured on B200
// over the power-law SELL-32 (0.271 ms in two launches), 0.240 ms at 180,
// 0.250 at 250-300, 0.268 at 400, 0.308 at 550 (the latency-bound heads
// want most of the warps). CLSPMV_SELL_ONE overrides it (0: two launches;
// measurements).
int sell_one_permille()
{
    static const int v = [] {
        const char* e = getenv("CLSPMV_SELL_ONE");
        return e ? atoi(e) : 180;
    }();
    return v;
}

// tail_col[tail_off[t] + j] = column id of entry item.y + j of split item t
__global__ void k_sell_tail_cols(const int2* __restrict__ items, const int* __restrict__ tail_off, long long nitems,
                                 const int* __restrict__ slice_ptr, const int* __restrict__ col, int sh, int* tail_col)
{
    for (long long t = blockIdx.x; t < nitems; t += gridDim.x) {
        const int2 item = items[t];
        const int s = item.x / sh, lr = item.x - s * sh;
        const size_t base = (size_t)slice_ptr[s] + lr;
        const int o = tail_off[t], n = tail_off[t + 1] - o;
        for (int j = threadIdx.x; j < n; j += blockDim.x) tail_col[o + j] = col[base + (size_t)(item.y + j) * sh];
    }
}

template <bool A>
__global__ void __launch_bounds__(kBlock) k_csr_scalar(CsrArgs a) { csr_scalar_cta<A>(a, blockIdx.x, gridDim.x, nullptr); }

template <int T, bool A>
__global__ void __launch_bounds__(kBlock) k_csr_vector(CsrArgs a) { csr_vector_cta<T, A>(a, blockIdx.x, gridDim.x, nullptr); }

template <class V>
__global__ void __launch_bounds__(kBlock) k_csr_merge(CsrArgsT<V> a, const int* __restrict__ tc)
{
    extern __shared__ __align__(16) char dsmem[];
    csr_merge_tile(a, tc, blockIdx.x, dsmem);
}

__global__ void __launch_bounds__(kBlock) k_csr_merge_plan(int rows, int nnz, const int* __restrict__ row_ptr, int* tc, int ntiles)
{
    const int t = blockIdx.x * kBlock + threadIdx.x;
    if (t > ntiles) return;
    csr_merge_search(rows, nnz, row_ptr, (long long)t * kMergeTile, tc + 2 * t);
}

template <class V, int GX = 0, int MINB = 5>
__global__ void __launch_bounds__(kBlock, MINB) k_coo(CooArgsT<V> a) { coo_cta<V, GX>(a, blockIdx.x, gridDim.x, nullptr); }

template <class V, int GX = 0, int MINB = 5>
__global__ void __launch_bounds__(kBlock, MINB) k_csr_chunk(CsrArgsT<V> a, const int* __restrict__ chunk_row)
{
    csr_chunk_cta<V, GX>(a, chunk_row, blockIdx.x, gridDim.x);
}

// Resident CTAs per SM the gather kernels are compiled for (register cap):
// 5 (48 registers), 6 (40), 8 (32). Measured on B200 (power-law 2^20): CSR
// by chunks fits 32 registers without spilling and gains 2 % at 8 CTAs
// (90.4 -> 88.4 us); COO spills below 48 and loses (84.9 -> 89.1 / 103 us).
// CLSPMV_GATHER_OCC overrides both (measurements).
constexpr int kCsrChunkDefaultOcc = 8, kCooDefaultOcc = 5;
int gather_occ(int dflt)
{
    static int f = [] {
        const char* e = getenv("CLSPMV_GATHER_OCC");
        const int v = e ? atoi(e) : 0;
        return v == 5 || v == 6 || v == 8 ? v : 0;
    }();
    return f ? f : dflt;
}

// Form of the scattered x gathers of COO and CSR by chunks (ld_gx): 0 through
// L1 with allocation, 1 without. CLSPMV_GATHER_FORM overrides (measurements).
constexpr int kGatherDefaultForm = 0;
int gather_form()
{
    static int f = [] {
        const char* e = getenv("CLSPMV_GATHER_FORM");
        return e ? atoi(e) : kGatherDefaultForm;
    }();
    return f;
}

__global__ void __launch_bounds__(kBlock) k_csr_chunk_plan(const int* __restrict__ row_ptr, int rows, long long nchunks,
                                                           int* chunk_row)
{
    for (long long c = blockIdx.x * (long long)kBlock + threadIdx.x; c <= nchunks; c += (long long)gridDim.x * kBlock)
        chunk_row[c] = c < nchunks ? csr_row_of(row_ptr, rows, c * kCooWarpNnz) : rows - 1;
}

template <int BW4, int BH, bool A, class V>
__global__ void __launch_bounds__(kBlock) k_b4ell(B4ellArgsT<V> a) { b4ell_cta<BW4, BH, A>(a, blockIdx.x, gridDim.x, nullptr); }

template <int BW4, int BH, bool A, class V>
__global__ void __launch_bounds__(kBlock) k_sbell(SbellArgsT<V> a) { sbell_cta<BW4, BH, A>(a, blockIdx.x, gridDim.x, nullptr); }

template <int BW4, int BH, int T, bool A, class V>
__global__ void __launch_bounds__(kBlock) k_b4csr(B4csrArgsT<V> a) { b4csr_cta<BW4, BH, T, A>(a, blockIdx.x, gridDim.x, nullptr); }

// The 4x4-block kernels (FP32 values, own rows) compiled for MINB resident
// CTAs per SM (a register cap); CLSPMV_BLOCK_OCC = 6 or 8 selects them
// (measurements; 1 = the uncapped kernels above, the default). Measured on
// B200 (500k x 8 4x4 blocks): all three spill under the cap and lose
// (BELL 55 -> 63 / 72 us, SBELL 57 -> 66 / 63 us, BCSR 59 -> 61 / 98 us).
template <int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_b4ell_occ(B4ellArgsT<float> a) { b4ell_cta<1, 4, false>(a, blockIdx.x, gridDim.x, nullptr); }
template <int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_sbell_occ(SbellArgsT<float> a) { sbell_cta<1, 4, false>(a, blockIdx.x, gridDim.x, nullptr); }
template <int T, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_b4csr_occ(B4csrArgsT<float> a) { b4csr_cta<1, 4, T, false>(a, blockIdx.x, gridDim.x, nullptr); }
constexpr int kBlockDefaultOcc = 1;
int block_occ()
{
    static int f = [] {
        const char* e = getenv("CLSPMV_BLOCK_OCC");
        const int v = e ? atoi(e) : kBlockDefaultOcc;
        return v == 6 || v == 8 ? v : 1;
    }();
    return f;
}

// CTAs that fit on the device at once for `kernel` (SM count x resident
// CTAs per SM), cached per kernel.
int resident_ctas(const void* kernel, int smem_bytes)
{
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(kernel);
    if (it != cache.end()) return it->second;
    int dev = 0, nsm = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kBlock, smem_bytes) != cudaSuccess || per < 1) {
        cudaGetLastError();
        per = 1;
    }
    const int n = nsm * per;
    cache[kernel] = n;
    return n;
}

// Grid for a persistent launch: all resident CTAs, but no more CTAs than
// passes of work. With `whole`, when the work takes more than one wave of
// resident CTAs, as many CTAs as give every CTA the same whole number of
// passes (the last pass of a share otherwise runs part-empty on every CTA):
// measured on B200 over the 27-point stencil 128^3, DIA 53.7 -> 49.6 us and
// BDIA 53.3 -> 51.2 us, and over the 4x4-block matrix SBELL 55.6 -> 53.5 us;
// the gather-bound kernels and BELL lose 1-4 % with it and keep the full
// grid. CLSPMV_WHOLE_PASSES=0|1 overrides it for every kernel (measurements).
int whole_passes_override()
{
    static const int v = [] {
        const char* e = getenv("CLSPMV_WHOLE_PASSES");
        return e ? atoi(e) : -1;
    }();
    return v;
}

template <class K>
unsigned persistent_grid(K kernel, long long units, long long units_per_pass, int smem_bytes = 0, bool whole = false)
{
    const long long passes = (units + units_per_pass - 1) / units_per_pass;
    const long long res = resident_ctas(reinterpret_cast<const void*>(kernel), smem_bytes);
    const int ov = whole_passes_override();
    if ((ov >= 0 ? ov != 0 : whole) && passes > res) {
        const long long k = (passes + res - 1) / res;
        return (unsigned)((passes + k - 1) / k);
    }
    return (unsigned)std::max(1LL, std::min(passes, res));
}

// ---------------------------------------------------------------------------
// Shape dispatch helpers.
// ---------------------------------------------------------------------------
template <int V> using ic = std::integral_constant<int, V>;

// Calls f(ic<bwidth/4>, ic<bheight>) for the 8 block shapes of the
// reference ({1,2,4,8} x {4,8}, include/matrix_storage.h:241).
template <class F>
int dispatch_block(unsigned bw, unsigned bh, F&& f)
{
    if (bw == 4) {
        switch (bh) {
            case 1: return f(ic<1>{}, ic<1>{});
            case 2: return f(ic<1>{}, ic<2>{});
            case 4: return f(ic<1>{}, ic<4>{});
            case 8: return f(ic<1>{}, ic<8>{});
        }
    } else if (bw == 8) {
        switch (bh) {
            case 1: return f(ic<2>{}, ic<1>{});
            case 2: return f(ic<2>{}, ic<2>{});
            case 4: return f(ic<2>{}, ic<4>{});
            case 8: return f(ic<2>{}, ic<8>{});
        }
    }
    return CLSPMV_ERR_UNSUPPORTED;
}

// Calls f(ic<T>) for T in {1, 2, 4, 8, 16, 32}.
template <class F>
int dispatch_lanes(int t, F&& f)
{
    switch (t) {
        case 1: return f(ic<1>{});
        case 2: return f(ic<2>{});
        case 4: return f(ic<4>{});
        case 8: return f(ic<8>{});
        case 16: return f(ic<16>{});
        case 32: return f(ic<32>{});
    }
    return CLSPMV_ERR_ARG;
}

int pow2_lanes(double mean, int lo, int hi)
{
    int t = lo;
    while (t < hi && t < mean) t <<= 1;
    return t;
}

int prescale(float* y, int n, float beta, cudaStream_t st)
{
    if (beta == 1.0f || n == 0) return CLSPMV_OK;
    k_scale<<<grid_for(n, kBlock), kBlock, 0, st>>>(y, n, beta);
    return after_launch(1);
}

}  // namespace

// ---------------------------------------------------------------------------
// Internal launchers. `atomic` = add alpha*A*x into y with red.global.add
// (beta must already be applied); used by the Cocktail runtime, whose parts
// run concurrently into one y.
// ---------------------------------------------------------------------------
namespace clspmv {

int launch_prescale(float* y, int n, float beta, cudaStream_t st) { return prescale(y, n, beta, st); }

template <class V>
int launch_dia_v(const clspmv_dia_f32* m, const V* data, const float* scale, const float* x, float* y, float alpha, float beta,
                 cudaStream_t st, bool atomic)
{
    if (!m || !x || !y) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    if (rows <= 0) return CLSPMV_OK;
    if (m->dia_num > 0 && (!m->dia_offsets || !data)) return CLSPMV_ERR_ARG;
    if ((m->dia_length_aligned & 3) || !aligned_v4(data) || rows > m->dia_length_aligned) return CLSPMV_ERR_ALIGN;
    DiaArgsT<V> a{rows, m->matinfo.width, m->dia_num, m->dia_length_aligned, m->dia_offsets, data, x, y, alpha, beta, scale};
    const int form = aligned16(x) ? dia_form(kDiaDefaultForm) : 0;
    if constexpr (std::is_same<V, float>::value) {
        if (form == 4 && !atomic && m->dia_num > 0 && diag_bulk_supported(m->dia_length_aligned, data))
            return launch_diag_bulk(rows, m->matinfo.width, m->dia_num, m->dia_length_aligned, m->dia_offsets, nullptr, 0,
                                    data, x, y, alpha, beta, st);
    }
    auto go = [&](auto kernel) { kernel<<<persistent_grid(kernel, rows, kDiaRowsPerPass, 0, true), kBlock, 0, st>>>(a); };
    if (atomic) {
        if (form == 3) go(k_dia<true, V, 3>);
        else if (form == 2) go(k_dia_occ<true, V, 1>);
        else if (form == 1) go(k_dia<true, V, 1>);
        else go(k_dia<true, V, 0>);
    } else {
        if (form == 3) go(k_dia<false, V, 3>);
        else if (form == 2) go(k_dia_occ<false, V, 1>);
        else if (form == 1) go(k_dia<false, V, 1>);
        else go(k_dia<false, V, 0>);
    }
    return after_launch(1);
}

int launch_dia(const clspmv_dia_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic)
{
    return launch_dia_v<float>(m, m ? m->dia_data : nullptr, nullptr, x, y, alpha, beta, st, atomic);
}

template <class V>
int launch_bdia_v(const clspmv_bdia_f32* m, const V* data, const float* scale, const float* x, float* y, float alpha, float beta,
                  cudaStream_t st, bool atomic)
{
    if (!m || !x || !y) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    if (rows <= 0) return CLSPMV_OK;
    if (m->bdia_band_num > 0 && (!m->bdia_offsets || !m->bdia_bptr || !data)) return CLSPMV_ERR_ARG;
    if ((m->bdia_length_aligned & 3) || !aligned_v4(data) || rows > m->bdia_length_aligned) return CLSPMV_ERR_ALIGN;
    BdiaArgsT<V> a{rows, m->matinfo.width, m->bdia_band_num, m->bdia_length_aligned, m->bdia_offsets, m->bdia_bptr, data, x, y, alpha, beta, scale};
    const int form = aligned16(x) ? dia_form(kBdiaDefaultForm) : 0;
    if constexpr (std::is_same<V, float>::value) {
        if (form == 4 && !atomic && m->bdia_band_num > 0 && diag_bulk_supported(m->bdia_length_aligned, data))
            return launch_diag_bulk(rows, m->matinfo.width, 0, m->bdia_length_aligned, m->bdia_offsets, m->bdia_bptr,
                                    m->bdia_band_num, data, x, y, alpha, beta, st);
    }
    auto go = [&](auto kernel) { kernel<<<persistent_grid(kernel, rows, kBdiaRowsPerPass, 0, true), kBlock, 0, st>>>(a); };
    if (atomic) {
        if (form == 2) go(k_bdia_occ<true, V, true>);
        else if (form == 1) go(k_bdia<true, V, true>);
        else go(k_bdia<true, V, false>);
    } else {
        if (form == 2) go(k_bdia_occ<false, V, true>);
        else if (form == 1) go(k_bdia<false, V, true>);
        else go(k_bdia<false, V, false>);
    }
    return after_launch(1);
}

int launch_bdia(const clspmv_bdia_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic)
{
    return launch_bdia_v<float>(m, m ? m->bdia_data : nullptr, nullptr, x, y, alpha, beta, st, atomic);
}

template <class V>
int launch_ell_v(const clspmv_ell_f32* m, const V* data, const float* scale, const float* x, float* y, float alpha, float beta,
                 cudaStream_t st, bool atomic)
{
    if (!m || !x || !y) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    if (rows <= 0) return CLSPMV_OK;
    if (m->ell_num > 0 && (!m->ell_col_id || !data)) return CLSPMV_ERR_ARG;
    if ((m->ell_height_aligned & 3) || !aligned16(m->ell_col_id) || !aligned_v4(data) || rows > m->ell_height_aligned)
        return CLSPMV_ERR_ALIGN;
    EllArgsT<V> a{rows, m->ell_num, m->ell_height_aligned, m->ell_col_id, data, x, y, alpha, beta, scale};
    auto go = [&](auto kernel) { kernel<<<persistent_grid(kernel, rows, kEllRowsPerPass), kBlock, 0, st>>>(a); };
    if (gather_form() == 1) {
        if (atomic) go(k_ell<true, V, 1>);
        else go(k_ell<false, V, 1>);
    } else {
        if (atomic) go(k_ell<true, V, 0>);
        else go(k_ell<false, V, 0>);
    }
    return after_launch(1);
}

int launch_ell(const clspmv_ell_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic)
{
    return launch_ell_v<float>(m, m ? m->ell_data : nullptr, nullptr, x, y, alpha, beta, st, atomic);
}

template <class V>
int launch_sell_v(const clspmv_sell_f32* m, const V* data, const float* scale, const float* x, float* y, float alpha, float beta,
                  cudaStream_t st, bool atomic)
{
    if (!m || !x || !y || !m->sell_slice_ptr) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    const int sh = (int)m->sell_slice_height;
    if (rows <= 0) return CLSPMV_OK;
    if (sh <= 0 || (long long)m->sell_slice_num * sh < rows) return CLSPMV_ERR_ARG;
    SellArgsT<V> a{rows, sh, m->sell_slice_num, m->sell_slice_ptr, m->sell_col_id, data, x, y, alpha, beta, scale};
    const bool vec = aligned16(m->sell_col_id) && aligned_v4(data);
    // Narrow slices (about kSellNarrow stored entries per row or fewer): 4 rows
    // per thread. Wide or uneven slices: the column-balanced kernel, which
    // spreads one wide slice over many warps.
    if (vec && sh % 4 == 0 && (long long)m->matinfo.nnz <= (long long)kSellNarrow * rows) {
        if (atomic) k_sell_rows4<true, V><<<persistent_grid(k_sell_rows4<true, V>, rows, kBlock * 4), kBlock, 0, st>>>(a);
        else k_sell_rows4<false, V><<<persistent_grid(k_sell_rows4<false, V>, rows, kBlock * 4), kBlock, 0, st>>>(a);
        return after_launch(1);
    }
    if (vec && (sh == 4 || sh == 8 || sh == 16 || sh == 32 || sh == 64 || sh == 128)) {
        if (!atomic) {
            int rc = prescale(y, rows, beta, st);
            if (rc) return rc;
        }
        a.beta = 1.0f;
        return dispatch_lanes(sh / 4, [&](auto q) {
            constexpr int Q = decltype(q)::value;
            if (atomic) k_sell<Q, true, V><<<persistent_grid(k_sell<Q, true, V>, 1LL << 40, 1), kBlock, 0, st>>>(a);
            else k_sell<Q, false, V><<<persistent_grid(k_sell<Q, false, V>, 1LL << 40, 1), kBlock, 0, st>>>(a);
            return after_launch(1);
        });
    }
    if (atomic) k_sell_rows<true, V><<<persistent_grid(k_sell_rows<true, V>, rows, kBlock), kBlock, 0, st>>>(a);
    else k_sell_rows<false, V><<<persistent_grid(k_sell_rows<false, V>, rows, kBlock), kBlock, 0, st>>>(a);
    return after_launch(1);
}

int launch_sell(const clspmv_sell_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic)
{
    return launch_sell_v<float>(m, m ? m->sell_data : nullptr, nullptr, x, y, alpha, beta, st, atomic);
}

// Launches the planned walk as one kernel (k_sell_planned_one): tail CTAs
// by sell_one_permille, but no more than the tail items keep busy (a CTA
// walks 8 items at a time).
template <class V>
int launch_sell_one(const SellArgsT<V>& a, int sh, const int* rlen, const int* head, const int2* split_items,
                    long long nsplit, const int* tail_off, const int* tail_col, cudaStream_t st)
{
    return dispatch_lanes(sh / 4, [&](auto q) {
        constexpr int Q = decltype(q)::value;
        auto k = k_sell_planned_one<Q, V>;
        const unsigned grid = persistent_grid(k, 1LL << 40, 1);
        long long ntail = (long long)grid * sell_one_permille() / 1000;
        ntail = std::min(ntail, (nsplit + kBlock / 32 - 1) / (kBlock / 32));
        ntail = std::max(1LL, std::min((long long)grid - 1, ntail));
        k<<<grid, kBlock, 0, st>>>(a, rlen, head, split_items, tail_off, tail_col, nsplit, (int)ntail);
        return after_launch(1);
    });
}

// Padding-free SELL. Power-of-two slice heights with 16-byte aligned arrays:
// the column-balanced walk with each lane's loads cut at its rows' real
// length, either over every column of every slice (head == nullptr), or over
// each slice's columns up to its second-longest row (head: prefix table of
// those widths) and the longest rows' tails, a warp per item of up to
// kSellTailCols entries (split_items); with the tails' compact column ids
// both run in one launch (launch_sell_one). Other slice heights: each row's
// first kSellHead entries with a thread per row, then the tails (items).
int launch_sell_planned(const clspmv_sell_f32* m, const int* rlen, const int2* items, long long nitems, const int* head,
                        const int2* split_items, long long nsplit, const int* tail_off, const int* tail_col,
                        const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic)
{
    if (!m || !x || !y || !m->sell_slice_ptr || !rlen || (nitems > 0 && !items)) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    if (rows <= 0) return CLSPMV_OK;
    if (m->sell_slice_height == 0) return CLSPMV_ERR_ARG;
    SellArgs a{rows, (int)m->sell_slice_height, m->sell_slice_num, m->sell_slice_ptr, m->sell_col_id, m->sell_data,
               x, y, alpha, beta, nullptr};
    const int sh = (int)m->sell_slice_height;
    if (aligned16(m->sell_col_id) && aligned16(m->sell_data) && aligned16(rlen) &&
        (sh == 4 || sh == 8 || sh == 16 || sh == 32 || sh == 64 || sh == 128)) {
        if (!atomic) {
            int rc = prescale(y, rows, beta, st);
            if (rc) return rc;
        }
        a.beta = 1.0f;
        if (head && tail_col && nsplit > 0 && sell_one_permille() > 0)
            return launch_sell_one<float>(a, sh, rlen, head, split_items, nsplit, tail_off, tail_col, st);
        int rc = dispatch_lanes(sh / 4, [&](auto q) {
            constexpr int Q = decltype(q)::value;
            if (atomic) k_sell_masked<Q, true><<<persistent_grid(k_sell_masked<Q, true>, 1LL << 40, 1), kBlock, 0, st>>>(a, rlen, head);
            else k_sell_masked<Q, false><<<persistent_grid(k_sell_masked<Q, false>, 1LL << 40, 1), kBlock, 0, st>>>(a, rlen, head);
            return after_launch(1);
        });
        if (rc || !head || nsplit == 0) return rc;
        if (tail_col)
            k_sell_tail_compact<float><<<persistent_grid(k_sell_tail_compact<float>, nsplit, kBlock / 32), kBlock, 0, st>>>(
                a, rlen, split_items, tail_off, tail_col, nsplit);
        else
            k_sell_tail<<<persistent_grid(k_sell_tail, nsplit, kBlock / 32), kBlock, 0, st>>>(a, rlen, split_items, nsplit);
        return after_launch(1);
    }
    if (atomic) k_sell_head<true><<<persistent_grid(k_sell_head<true>, rows, kBlock), kBlock, 0, st>>>(a, rlen);
    else k_sell_head<false><<<persistent_grid(k_sell_head<false>, rows, kBlock), kBlock, 0, st>>>(a, rlen);
    int rc = after_launch(1);
    if (rc || nitems == 0) return rc;
    k_sell_tail<<<persistent_grid(k_sell_tail, nitems, kBlock / 32), kBlock, 0, st>>>(a, rlen, items, nitems);
    return after_launch(1);
}

// The planned walk with 16-bit values (per-row scales): slice heights
// 4..128 with the heads / compact tails split; otherwise the padded read.
template <class V>
int launch_sell_planned_packed(const clspmv_sell_f32* m, const V* data, const float* scale, const int* rlen, const int* head,
                               const int2* split_items, long long nsplit, const int* tail_off, const int* tail_col,
                               const float* x, float* y, float alpha, float beta, cudaStream_t st)
{
    if (!m || !x || !y || !m->sell_slice_ptr || !rlen || !data || !scale) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    if (rows <= 0) return CLSPMV_OK;
    const int sh = (int)m->sell_slice_height;
    if (!(head && tail_col && aligned16(m->sell_col_id) && aligned_v4(data) && aligned16(rlen) &&
          (sh == 4 || sh == 8 || sh == 16 || sh == 32 || sh == 64 || sh == 128)))
        return launch_sell_v<V>(m, data, scale, x, y, alpha, beta, st, false);
    SellArgsT<V> a{rows, sh, m->sell_slice_num, m->sell_slice_ptr, m->sell_col_id, data, x, y, alpha, 1.0f, scale};
    int rc = prescale(y, rows, beta, st);
    if (rc) return rc;
    if (nsplit > 0 && sell_one_permille() > 0)
        return launch_sell_one<V>(a, sh, rlen, head, split_items, nsplit, tail_off, tail_col, st);
    rc = dispatch_lanes(sh / 4, [&](auto q) {
        constexpr int Q = decltype(q)::value;
        k_sell_masked<Q, false, V><<<persistent_grid(k_sell_masked<Q, false, V>, 1LL << 40, 1), kBlock, 0, st>>>(a, rlen, head);
        return after_launch(1);
    });
    if (rc || nsplit == 0) return rc;
    k_sell_tail_compact<V><<<persistent_grid(k_sell_tail_compact<V>, nsplit, kBlock / 32), kBlock, 0, st>>>(
        a, rlen, split_items, tail_off, tail_col, nsplit);
    return after_launch(1);
}

int launch_csr_scalar(const clspmv_csr_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic)
{
    if (!m || !x || !y || !m->csr_row_ptr) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    if (rows <= 0) return CLSPMV_OK;
    if (!aligned16(m->csr_col_id) || !aligned16(m->csr_data)) return CLSPMV_ERR_ALIGN;
    CsrArgs a{rows, m->matinfo.nnz, m->csr_row_ptr, m->csr_col_id, m->csr_data, x, y, alpha, beta};
    // one pass per CTA: thread-per-row work is uneven, so CTAs are scheduled dynamically
    if (atomic) k_csr_scalar<true><<<grid_for(rows, kBlock), kBlock, 0, st>>>(a);
    else k_csr_scalar<false><<<grid_for(rows, kBlock), kBlock, 0, st>>>(a);
    return after_launch(1);
}

int launch_csr_vector(const clspmv_csr_f32* m, const float* x, float* y, float alpha, float beta, int tpr, cudaStream_t st, bool atomic)
{
    if (!m || !x || !y || !m->csr_row_ptr) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    if (rows <= 0) return CLSPMV_OK;
    if (!aligned16(m->csr_col_id) || !aligned16(m->csr_data)) return CLSPMV_ERR_ALIGN;
    if (tpr == 0) tpr = pow2_lanes((double)m->matinfo.nnz / rows, 2, 32);
    CsrArgs a{rows, m->matinfo.nnz, m->csr_row_ptr, m->csr_col_id, m->csr_data, x, y, alpha, beta};
    return dispatch_lanes(tpr, [&](auto t) {
        constexpr int T = decltype(t)::value;
        const unsigned grid = grid_for(rows, kBlock / T);
        if (atomic) k_csr_vector<T, true><<<grid, kBlock, 0, st>>>(a);
        else k_csr_vector<T, false><<<grid, kBlock, 0, st>>>(a);
        return after_launch(1);
    });
}

template <class V>
int launch_csr_merge_v(const clspmv_csr_f32* m, const V* data, const float* scale, const int* tc, const float* x, float* y,
                       float alpha, float beta, cudaStream_t st, bool atomic)
{
    if (!m || !tc || !x || !y || !m->csr_row_ptr) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    if (rows <= 0) return CLSPMV_OK;
    if (!atomic) {
        int rc = prescale(y, rows, beta, st);
        if (rc) return rc;
    }
    const int ntiles = clspmv_csr_merge_tiles(rows, m->matinfo.nnz);
    CsrArgsT<V> a{rows, m->matinfo.nnz, m->csr_row_ptr, m->csr_col_id, data, x, y, alpha, 1.0f, scale};
    k_csr_merge<V><<<ntiles, kBlock, kMergeSmemBytes, st>>>(a, tc);
    return after_launch(1);
}

int launch_csr_merge(const clspmv_csr_f32* m, const int* tc, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic)
{
    return launch_csr_merge_v<float>(m, m ? m->csr_data : nullptr, nullptr, tc, x, y, alpha, beta, st, atomic);
}

template <class V>
int launch_csr_chunk_v(const clspmv_csr_f32* m, const V* data, const float* scale, const int* chunk_row, const float* x,
                       float* y, float alpha, float beta, cudaStream_t st, bool atomic)
{
    if (!m || !chunk_row || !x || !y || !m->csr_row_ptr) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    if (rows <= 0) return CLSPMV_OK;
    if (!atomic) {
        int rc = prescale(y, rows, beta, st);
        if (rc) return rc;
    }
    if (m->matinfo.nnz <= 0) return CLSPMV_OK;
    if (!m->csr_col_id || !data) return CLSPMV_ERR_ARG;
    if (!aligned16(m->csr_col_id) || !aligned_v4(data)) return CLSPMV_ERR_ALIGN;
    CsrArgsT<V> a{rows, m->matinfo.nnz, m->csr_row_ptr, m->csr_col_id, data, x, y, alpha, 1.0f, scale};
    const long long nchunks = ((long long)m->matinfo.nnz + kCooWarpNnz - 1) / kCooWarpNnz;
    auto go = [&](auto kernel) { kernel<<<persistent_grid(kernel, nchunks, kBlock / 32), kBlock, 0, st>>>(a, chunk_row); };
    const int occ = gather_occ(kCsrChunkDefaultOcc);
    if (gather_form() == 1) {
        if (occ == 8) go(k_csr_chunk<V, 1, 8>);
        else if (occ == 6) go(k_csr_chunk<V, 1, 6>);
        else go(k_csr_chunk<V, 1, 5>);
    } else {
        if (occ == 8) go(k_csr_chunk<V, 0, 8>);
        else if (occ == 6) go(k_csr_chunk<V, 0, 6>);
        else go(k_csr_chunk<V, 0, 5>);
    }
    return after_launch(1);
}

int launch_csr_chunk(const clspmv_csr_f32* m, const int* chunk_row, const float* x, float* y, float alpha, float beta,
                     cudaStream_t st, bool atomic)
{
    return launch_csr_chunk_v<float>(m, m ? m->csr_data : nullptr, nullptr, chunk_row, x, y, alpha, beta, st, atomic);
}

int launch_csr_chunk_plan(const clspmv_csr_f32* m, int* chunk_row, cudaStream_t st)
{
    if (!m || !chunk_row || !m->csr_row_ptr || m->matinfo.height <= 0 || m->matinfo.nnz < 0) return CLSPMV_ERR_ARG;
    const long long nchunks = ((long long)m->matinfo.nnz + kCooWarpNnz - 1) / kCooWarpNnz;
    k_csr_chunk_plan<<<grid_for(nchunks + 1, kBlock), kBlock, 0, st>>>(m->csr_row_ptr, m->matinfo.height, nchunks, chunk_row);
    return after_launch(1);
}

template <class V>
int launch_coo_v(const clspmv_coo_f32* m, const V* data, const float* scale, const float* x, float* y, float alpha, float beta,
                 cudaStream_t st, bool atomic)
{
    if (!m || !x || !y) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    if (rows <= 0) return CLSPMV_OK;
    if (!atomic) {
        int rc = prescale(y, rows, beta, st);
        if (rc) return rc;
    }
    if (m->matinfo.nnz <= 0) return CLSPMV_OK;
    if (!m->coo_row_id || !m->coo_col_id || !data) return CLSPMV_ERR_ARG;
    if (!aligned16(m->coo_row_id) || !aligned16(m->coo_col_id) || !aligned_v4(data)) return CLSPMV_ERR_ALIGN;
    CooArgsT<V> a{m->matinfo.nnz, m->coo_row_id, m->coo_col_id, data, x, y, alpha, scale};
    const long long nchunks = ((long long)m->matinfo.nnz + kCooWarpNnz - 1) / kCooWarpNnz;
    auto go = [&](auto kernel) { kernel<<<persistent_grid(kernel, nchunks, kBlock / 32), kBlock, 0, st>>>(a); };
    const int occ = gather_occ(kCooDefaultOcc);
    if (gather_form() == 1) {
        if (occ == 8) go(k_coo<V, 1, 8>);
        else if (occ == 6) go(k_coo<V, 1, 6>);
        else go(k_coo<V, 1, 5>);
    } else {
        if (occ == 8) go(k_coo<V, 0, 8>);
        else if (occ == 6) go(k_coo<V, 0, 6>);
        else go(k_coo<V, 0, 5>);
    }
    return after_launch(1);
}

int launch_coo(const clspmv_coo_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic)
{
    return launch_coo_v<float>(m, m ? m->coo_data : nullptr, nullptr, x, y, alpha, beta, st, atomic);
}

template <class V>
int launch_b4ell_v(const clspmv_b4ell_f32* m, const V* data, const float* scale, const float* x, float* y, float alpha, float beta,
                   cudaStream_t st, bool atomic)
{
    if (!m || !x || !y) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    if (rows <= 0 || m->b4ell_row_num <= 0) return CLSPMV_OK;
    if (!m->b4ell_col_id || !data) return CLSPMV_ERR_ARG;
    if ((m->b4ell_float4_aligned & 3) || !aligned_v4(data) || !aligned16(x)) return CLSPMV_ERR_ALIGN;
    if ((long long)m->b4ell_row_num * m->b4ell_bheight < rows || m->b4ell_float4_aligned < 4 * m->b4ell_row_num) return CLSPMV_ERR_ARG;
    const B4ellArgsT<V> a{rows, m->matinfo.width, m->b4ell_row_num, m->b4ell_block_num, m->b4ell_height_aligned,
                          m->b4ell_float4_aligned, m->b4ell_col_id, data, x, y, alpha, beta, scale};
    if constexpr (std::is_same<V, float>::value) {
        if (!atomic && block_occ() != 1 && m->b4ell_bwidth == 4 && m->b4ell_bheight == 4) {
            auto go = [&](auto kernel) { kernel<<<persistent_grid(kernel, a.nbrow, kBlock), kBlock, 0, st>>>(a); };
            if (block_occ() == 8) go(k_b4ell_occ<8>);
            else go(k_b4ell_occ<6>);
            return after_launch(1);
        }
    }
    return dispatch_block(m->b4ell_bwidth, m->b4ell_bheight, [&](auto bw4, auto bh) {
        constexpr int BW4 = decltype(bw4)::value, BH = decltype(bh)::value;
        if (atomic) k_b4ell<BW4, BH, true, V><<<persistent_grid(k_b4ell<BW4, BH, true, V>, a.nbrow, kBlock), kBlock, 0, st>>>(a);
        else k_b4ell<BW4, BH, false, V><<<persistent_grid(k_b4ell<BW4, BH, false, V>, a.nbrow, kBlock), kBlock, 0, st>>>(a);
        return after_launch(1);
    });
}

int launch_b4ell(const clspmv_b4ell_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic)
{
    return launch_b4ell_v<float>(m, m ? m->b4ell_data : nullptr, nullptr, x, y, alpha, beta, st, atomic);
}

template <class V>
int launch_sbell_v(const clspmv_sbell_f32* m, const V* data, const float* scale, const float* x, float* y, float alpha, float beta,
                   cudaStream_t st, bool atomic)
{
    if (!m || !x || !y) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    if (rows <= 0 || m->sbell_row_num <= 0) return CLSPMV_OK;
    if (!m->sbell_slice_ptr || !m->sbell_col_id || !data || m->sbell_slice_height == 0) return CLSPMV_ERR_ARG;
    if (!aligned_v4(data) || !aligned16(x)) return CLSPMV_ERR_ALIGN;
    if ((long long)m->sbell_row_num * m->sbell_bheight < rows) return CLSPMV_ERR_ARG;
    const SbellArgsT<V> a{rows, m->matinfo.width, m->sbell_row_num, m->sbell_slice_num, (int)m->sbell_slice_height,
                          m->sbell_slice_ptr, m->sbell_col_id, data, x, y, alpha, beta, scale};
    if constexpr (std::is_same<V, float>::value) {
        if (!atomic && block_occ() != 1 && m->sbell_bwidth == 4 && m->sbell_bheight == 4) {
            auto go = [&](auto kernel) { kernel<<<persistent_grid(kernel, a.nbrow, kBlock), kBlock, 0, st>>>(a); };
            if (block_occ() == 8) go(k_sbell_occ<8>);
            else go(k_sbell_occ<6>);
            return after_launch(1);
        }
    }
    return dispatch_block(m->sbell_bwidth, m->sbell_bheight, [&](auto bw4, auto bh) {
        constexpr int BW4 = decltype(bw4)::value, BH = decltype(bh)::value;
        if (atomic) k_sbell<BW4, BH, true, V><<<persistent_grid(k_sbell<BW4, BH, true, V>, a.nbrow, kBlock), kBlock, 0, st>>>(a);
        else k_sbell<BW4, BH, false, V><<<persistent_grid(k_sbell<BW4, BH, false, V>, a.nbrow, kBlock, 0, true), kBlock, 0, st>>>(a);
        return after_launch(1);
    });
}

int launch_sbell(const clspmv_sbell_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic)
{
    return launch_sbell_v<float>(m, m ? m->sbell_data : nullptr, nullptr, x, y, alpha, beta, st, atomic);
}

template <class V>
int launch_b4csr_v(const clspmv_b4csr_f32* m, const V* data, const float* scale, const float* x, float* y, float alpha, float beta,
                   cudaStream_t st, bool atomic)
{
    if (!m || !x || !y) return CLSPMV_ERR_ARG;
    const int rows = m->matinfo.height;
    if (rows <= 0 || m->b4csr_row_num <= 0) return CLSPMV_OK;
    if (!m->b4csr_row_ptr || !m->b4csr_col_id || !data) return CLSPMV_ERR_ARG;
    if ((m->b4csr_aligned_size & 3) || !aligned_v4(data) || !aligned16(x)) return CLSPMV_ERR_ALIGN;
    if ((long long)m->b4csr_row_num * m->b4csr_bheight < rows) return CLSPMV_ERR_ARG;
    const B4csrArgsT<V> a{rows, m->matinfo.width, m->b4csr_row_num, m->b4csr_aligned_size,
                          m->b4csr_row_ptr, m->b4csr_col_id, data, x, y, alpha, beta, scale};
    // lanes per block row: about one block per lane (measured best on B200 against 2 and 4;
    // CLSPMV_BCSR_BPL overrides, for measurements)
    static const int bpl = [] {
        const char* e = getenv("CLSPMV_BCSR_BPL");
        return e ? std::max(1, atoi(e)) : 1;
    }();
    const int lanes = pow2_lanes((double)m->b4csr_block_num / m->b4csr_row_num / bpl, 1, 32);
    if constexpr (std::is_same<V, float>::value) {
        if (!atomic && block_occ() != 1 && m->b4csr_bwidth == 4 && m->b4csr_bheight == 4 && (lanes == 4 || lanes == 8)) {
            auto go = [&](auto kernel, int t) { kernel<<<persistent_grid(kernel, a.nbrow, kBlock / t), kBlock, 0, st>>>(a); };
            if (block_occ() == 8) {
                if (lanes == 8) go(k_b4csr_occ<8, 8>, 8);
                else go(k_b4csr_occ<4, 8>, 4);
            } else {
                if (lanes == 8) go(k_b4csr_occ<8, 6>, 8);
                else go(k_b4csr_occ<4, 6>, 4);
            }
            return after_launch(1);
        }
    }
    return dispatch_block(m->b4csr_bwidth, m->b4csr_bheight, [&](auto bw4, auto bh) {
        return dispatch_lanes(lanes, [&](auto t) {
            constexpr int T = decltype(t)::value;
            constexpr int BW4 = decltype(bw4)::value, BH = decltype(bh)::value;
            if (atomic)
                k_b4csr<BW4, BH, T, true, V><<<persistent_grid(k_b4csr<BW4, BH, T, true, V>, a.nbrow, kBlock / T), kBlock, 0, st>>>(a);
            else
                k_b4csr<BW4, BH, T, false, V><<<persistent_grid(k_b4csr<BW4, BH, T, false, V>, a.nbrow, kBlock / T), kBlock, 0, st>>>(a);
            return after_launch(1);
        });
    });
}

int launch_b4csr(const clspmv_b4csr_f32* m, const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic)
{
    return launch_b4csr_v<float>(m, m ? m->b4csr_data : nullptr, nullptr, x, y, alpha, beta, st, atomic);
}

// Single-vector SpMV with 16-bit values (clspmv_pack_values) in the format's
// dedicated kernel.
template <class V>
int launch_packed_t(int format, const void* dev, const V* vals, const float* scale, const int* tc, const float* x, float* y,
                    float alpha, float beta, cudaStream_t st, bool atomic)
{
    switch (format) {
        case CLSPMV_FORMAT_CSR: return launch_csr_merge_v(static_cast<const clspmv_csr_f32*>(dev), vals, scale, tc, x, y, alpha, beta, st, atomic);
        case CLSPMV_FORMAT_COO: return launch_coo_v(static_cast<const clspmv_coo_f32*>(dev), vals, scale, x, y, alpha, beta, st, atomic);
        case CLSPMV_FORMAT_DIA: return launch_dia_v(static_cast<const clspmv_dia_f32*>(dev), vals, scale, x, y, alpha, beta, st, atomic);
        case CLSPMV_FORMAT_BDIA: return launch_bdia_v(static_cast<const clspmv_bdia_f32*>(dev), vals, scale, x, y, alpha, beta, st, atomic);
        case CLSPMV_FORMAT_ELL: return launch_ell_v(static_cast<const clspmv_ell_f32*>(dev), vals, scale, x, y, alpha, beta, st, atomic);
        case CLSPMV_FORMAT_SELL: return launch_sell_v(static_cast<const clspmv_sell_f32*>(dev), vals, scale, x, y, alpha, beta, st, atomic);
        case CLSPMV_FORMAT_B4CSR: return launch_b4csr_v(static_cast<const clspmv_b4csr_f32*>(dev), vals, scale, x, y, alpha, beta, st, atomic);
        case CLSPMV_FORMAT_B4ELL: return launch_b4ell_v(static_cast<const clspmv_b4ell_f32*>(dev), vals, scale, x, y, alpha, beta, st, atomic);
        case CLSPMV_FORMAT_SBELL: return launch_sbell_v(static_cast<const clspmv_sbell_f32*>(dev), vals, scale, x, y, alpha, beta, st, atomic);
    }
    return CLSPMV_ERR_ARG;
}

int launch_packed(int format, const void* dev, int value_type, const void* values, const float* scale, const int* tc,
                  const float* x, float* y, float alpha, float beta, cudaStream_t st, bool atomic)
{
    if (!dev) return CLSPMV_ERR_ARG;
    if (format == CLSPMV_FORMAT_CSR && !tc) return CLSPMV_ERR_ARG;
    if (value_type == CLSPMV_VALUES_F32) {   // the struct's own FP32 values
        switch (format) {
            case CLSPMV_FORMAT_CSR: return launch_csr_merge(static_cast<const clspmv_csr_f32*>(dev), tc, x, y, alpha, beta, st, atomic);
            case CLSPMV_FORMAT_COO: return launch_coo(static_cast<const clspmv_coo_f32*>(dev), x, y, alpha, beta, st, atomic);
            case CLSPMV_FORMAT_DIA: return launch_dia(static_cast<const clspmv_dia_f32*>(dev), x, y, alpha, beta, st, atomic);
            case CLSPMV_FORMAT_BDIA: return launch_bdia(static_cast<const clspmv_bdia_f32*>(dev), x, y, alpha, beta, st, atomic);
            case CLSPMV_FORMAT_ELL: return launch_ell(static_cast<const clspmv_ell_f32*>(dev), x, y, alpha, beta, st, atomic);
            case CLSPMV_FORMAT_SELL: return launch_sell(static_cast<const clspmv_sell_f32*>(dev), x, y, alpha, beta, st, atomic);
            case CLSPMV_FORMAT_B4CSR: return launch_b4csr(static_cast<const clspmv_b4csr_f32*>(dev), x, y, alpha, beta, st, atomic);
            case CLSPMV_FORMAT_B4ELL: return launch_b4ell(static_cast<const clspmv_b4ell_f32*>(dev), x, y, alpha, beta, st, atomic);
            case CLSPMV_FORMAT_SBELL: return launch_sbell(static_cast<const clspmv_sbell_f32*>(dev), x, y, alpha, beta, st, atomic);
        }
        return CLSPMV_ERR_ARG;
    }
    if (!values || !scale) return CLSPMV_ERR_ARG;
    if (value_type == CLSPMV_VALUES_BF16)
        return launch_packed_t(format, dev, static_cast<const __nv_bfloat16*>(values), scale, tc, x, y, alpha, beta, st, atomic);
    if (value_type == CLSPMV_VALUES_F16)
        return launch_packed_t(format, dev, static_cast<const __half*>(values), scale, tc, x, y, alpha, beta, st, atomic);
    return CLSPMV_ERR_ARG;
}

int launch_csr_merge_plan(const clspmv_csr_f32* m, int* tc, cudaStream_t st)
{
    if (!m || !tc || !m->csr_row_ptr) return CLSPMV_ERR_ARG;
    const int ntiles = clspmv_csr_merge_tiles(m->matinfo.height, m->matinfo.nnz);
    if (ntiles < 0) return CLSPMV_ERR_ARG;
    k_csr_merge_plan<<<grid_for((long long)ntiles + 1, kBlock), kBlock, 0, st>>>(m->matinfo.height, m->matinfo.nnz, m->csr_row_ptr, tc, ntiles);
    return after_launch(1);
}

}  // namespace clspmv

// ---------------------------------------------------------------------------
// Compute entry points
// ---------------------------------------------------------------------------
extern "C" {

const char* clspmv_version(void) { return "clspmv_b200 0.1 sm_100a"; }

const char* clspmv_status_string(int s)
{
    switch (s) {
        case CLSPMV_OK: return "ok";
        case CLSPMV_ERR_ARG: return "invalid argument";
        case CLSPMV_ERR_ALLOC: return "allocation failed";
        case CLSPMV_ERR_UNSUPPORTED: return "unsupported shape";
        case CLSPMV_ERR_CUDA: return "CUDA error";
        case CLSPMV_ERR_REFUSED: return "refused by the format's size rule";
        case CLSPMV_ERR_ALIGN: return "misaligned pointer or length";
        case CLSPMV_ERR_NOT_SORTED: return "COO input is not sorted by (row, col)";
        case CLSPMV_ERR_TIMEOUT: return "bounded device wait timed out";
    }
    return "unknown status";
}

const char* clspmv_last_cuda_error(void) { return g_last_cuda_error.c_str(); }

long long clspmv_launch_count(void) { return g_launches.load(); }

int clspmv_csr_merge_tiles(int rows, int nnz)
{
    if (rows < 0 || nnz < 0) return -1;
    return (int)(((long long)rows + nnz + kMergeTile - 1) / kMergeTile);
}

int clspmv_csr_chunk_plan_size(int nnz)
{
    if (nnz < 0) return -1;
    return (int)(((long long)nnz + kCooWarpNnz - 1) / kCooWarpNnz + 1);
}

int clspmv_csr_chunk_plan(const clspmv_csr_f32* m, int* chunk_row, clspmv_stream_t s)
{
    return launch_csr_chunk_plan(m, chunk_row, S(s));
}

int clspmv_csr_chunk_spmv_f32(const clspmv_csr_f32* m, const int* chunk_row, const float* x, float* y, float alpha,
                              float beta, clspmv_stream_t s)
{
    return launch_csr_chunk(m, chunk_row, x, y, alpha, beta, S(s), false);
}

int clspmv_dia_spmv_f32(const clspmv_dia_f32* m, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{ return launch_dia(m, x, y, alpha, beta, S(s), false); }
int clspmv_dia_bulk_spmv_f32(const clspmv_dia_f32* m, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{
    if (!m || !x || !y) return CLSPMV_ERR_ARG;
    if (m->matinfo.height <= 0) return CLSPMV_OK;
    if (m->dia_num <= 0) return launch_dia(m, x, y, alpha, beta, S(s), false);
    if (!m->dia_offsets || !m->dia_data) return CLSPMV_ERR_ARG;
    if (m->matinfo.height > m->dia_length_aligned || !diag_bulk_supported(m->dia_length_aligned, m->dia_data))
        return CLSPMV_ERR_ALIGN;
    return launch_diag_bulk(m->matinfo.height, m->matinfo.width, m->dia_num, m->dia_length_aligned, m->dia_offsets, nullptr,
                            0, m->dia_data, x, y, alpha, beta, S(s));
}
int clspmv_bdia_bulk_spmv_f32(const clspmv_bdia_f32* m, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{
    if (!m || !x || !y) return CLSPMV_ERR_ARG;
    if (m->matinfo.height <= 0) return CLSPMV_OK;
    if (m->bdia_band_num <= 0) return launch_bdia(m, x, y, alpha, beta, S(s), false);
    if (!m->bdia_offsets || !m->bdia_bptr || !m->bdia_data) return CLSPMV_ERR_ARG;
    if (m->matinfo.height > m->bdia_length_aligned || !diag_bulk_supported(m->bdia_length_aligned, m->bdia_data))
        return CLSPMV_ERR_ALIGN;
    return launch_diag_bulk(m->matinfo.height, m->matinfo.width, 0, m->bdia_length_aligned, m->bdia_offsets, m->bdia_bptr,
                            m->bdia_band_num, m->bdia_data, x, y, alpha, beta, S(s));
}
int clspmv_bdia_spmv_f32(const clspmv_bdia_f32* m, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{ return launch_bdia(m, x, y, alpha, beta, S(s), false); }
int clspmv_ell_spmv_f32(const clspmv_ell_f32* m, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{ return launch_ell(m, x, y, alpha, beta, S(s), false); }
int clspmv_sell_spmv_f32(const clspmv_sell_f32* m, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{ return launch_sell(m, x, y, alpha, beta, S(s), false); }
struct clspmv_sell_plan {
    int* rlen = nullptr;       // device: stored length of every row (padding excluded)
    int2* items = nullptr;     // device: (row, first entry) of each tail item past the first kSellHead entries
    int* head = nullptr;       // device: prefix of per-slice widths up to the second-longest row
    int2* split_items = nullptr;   // device: (longest row, first entry) of each tail item past its slice's head
    int* tail_off = nullptr;   // device: prefix of the split items' entry counts (nsplit + 1)
    int* tail_col = nullptr;   // device: the split items' column ids, item after item (null: read in place)
    long long rows = 0, nitems = 0, nsplit = 0, entries = 0;
    long long sector_bytes = 0;   // col + data bytes of the 32-byte sectors holding real entries
    long long line_bytes = 0;     // bytes the split walk must read in 128-byte lines (see clspmv_sell_plan_line_bytes)
    bool split = true;         // walk the heads and the tails apart (power-of-two slice heights)
    bool compact = true;       // the tails' column ids from tail_col
};

int clspmv_sell_plan_create(const clspmv_sell_f32* m, clspmv_sell_plan** out)
{
    if (!m || !out || !m->sell_slice_ptr || m->sell_slice_height == 0) return CLSPMV_ERR_ARG;
    *out = nullptr;
    clspmv_sell_plan* p = new (std::nothrow) clspmv_sell_plan();
    if (!p) return CLSPMV_ERR_ALLOC;
    const long long rows = std::max(0, m->matinfo.height);
    p->rows = rows;
    std::vector<int> rlen((size_t)rows);
    std::vector<int2> items;
    int rc = cuda_status(cudaMalloc(&p->rlen, sizeof(int) * (size_t)std::max(1LL, rows)));
    if (!rc && rows) {
        k_sell_rlen<<<(unsigned)std::min<long long>((rows + kBlock - 1) / kBlock, 148LL * 32), kBlock>>>(
            m->sell_slice_ptr, m->sell_col_id, m->sell_data, (int)m->sell_slice_height, rows, p->rlen);
        rc = after_launch(1);
        if (!rc) rc = cuda_status(cudaMemcpy(rlen.data(), p->rlen, sizeof(int) * rows, cudaMemcpyDeviceToHost));
    }
    if (!rc) {
        for (long long r = 0; r < rows; r++) {
            p->entries += rlen[r];
            for (int k = kSellHead; k < rlen[r]; k += kSellTailCols) items.push_back(make_int2((int)r, k));
        }
        // heads and tails: per slice the width up to its second-longest row,
        // and the longest row's entries past it in items of kSellTailCols
        const long long shs = (long long)m->sell_slice_height, ns = m->sell_slice_num;
        std::vector<int> head((size_t)ns + 1, 0);
        std::vector<int2> split;
        for (long long sl = 0; sl < ns; sl++) {
            int l1 = 0, l2 = 0;
            long long arg = -1;
            for (long long r = sl * shs; r < std::min(rows, (sl + 1) * shs); r++) {
                const int l = rlen[(size_t)r];
                if (l > l1) { l2 = l1; l1 = l; arg = r; }
                else if (l > l2) l2 = l;
            }
            head[(size_t)sl + 1] = head[(size_t)sl] + l2;
            for (int k = l2; arg >= 0 && k < l1; k += kSellTailCols) split.push_back(make_int2((int)arg, k));
        }
        p->nsplit = (long long)split.size();
        rc = cuda_status(cudaMalloc(&p->head, sizeof(int) * head.size()));
        if (!rc) rc = cuda_status(cudaMemcpy(p->head, head.data(), sizeof(int) * head.size(), cudaMemcpyHostToDevice));
        if (!rc) rc = cuda_status(cudaMalloc(&p->split_items, sizeof(int2) * std::max<size_t>(1, split.size())));
        if (!rc && !split.empty())
            rc = cuda_status(cudaMemcpy(p->split_items, split.data(), sizeof(int2) * split.size(), cudaMemcpyHostToDevice));
        // the split items' column ids in one compact array (structure only: the
        // values stay in the matrix, so a plan stays valid while they change)
        std::vector<int> off(split.size() + 1, 0);
        for (size_t t = 0; t < split.size(); t++)
            off[t + 1] = off[t] + std::min(kSellTailCols, rlen[(size_t)split[t].x] - split[t].y);
        if (!rc) rc = cuda_status(cudaMalloc(&p->tail_off, sizeof(int) * off.size()));
        if (!rc) rc = cuda_status(cudaMemcpy(p->tail_off, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice));
        if (!rc) rc = cuda_status(cudaMalloc(&p->tail_col, sizeof(int) * std::max(1, off.back())));
        if (!rc && !split.empty()) {
            k_sell_tail_cols<<<(unsigned)std::min<size_t>(split.size(), 148 * 32), kBlock>>>(
                p->split_items, p->tail_off, (long long)split.size(), m->sell_slice_ptr, m->sell_col_id,
                (int)m->sell_slice_height, p->tail_col);
            rc = after_launch(1);
            if (!rc) rc = cuda_status(cudaDeviceSynchronize());
        }
        // The DRAM bytes of the split walk at 128-byte line granularity: the
        // lines of col and data holding a head entry, the data line of every
        // tail entry, the tails' compact column ids, and the plan's arrays
        // (row lengths, head table, items, item offsets).
        std::vector<int> sp((size_t)ns + 1);
        if (!rc) rc = cuda_status(cudaMemcpy(sp.data(), m->sell_slice_ptr, sizeof(int) * sp.size(), cudaMemcpyDeviceToHost));
        if (!rc) {
            const long long nlines = ((long long)sp[(size_t)ns] + 31) / 32 + 1;
            std::vector<uint64_t> dline((size_t)(nlines + 63) / 64, 0), cline((size_t)(nlines + 63) / 64, 0);
            auto mark = [](std::vector<uint64_t>& bm, long long l) { bm[(size_t)(l >> 6)] |= 1ull << (l & 63); };
            long long tail_entries = 0;
            for (long long sl = 0; sl < ns; sl++) {
                const int l2 = head[(size_t)sl + 1] - head[(size_t)sl];
                for (long long r = sl * shs; r < std::min(rows, (sl + 1) * shs); r++) {
                    const int len = rlen[(size_t)r];
                    for (int k = 0; k < len; k++) {
                        const long long pos = (long long)sp[(size_t)sl] + (long long)k * shs + (r - sl * shs);
                        mark(dline, pos >> 5);
                        if (k < l2) mark(cline, pos >> 5);
                        else tail_entries++;
                    }
                }
            }
            long long lines = 0;
            for (uint64_t w : dline) lines += __builtin_popcountll(w);
            for (uint64_t w : cline) lines += __builtin_popcountll(w);
            p->line_bytes = 128 * lines + 4 * tail_entries + 4 * rows + 4 * (ns + 1) + 12 * (long long)split.size() + 4;
        }
        // CLSPMV_SELL_SPLIT=0 walks every column instead, CLSPMV_SELL_TAIL_COMPACT=0
        // reads the tails' column ids in place (for measurements)
        const char* e = getenv("CLSPMV_SELL_SPLIT");
        p->split = !(e && atoi(e) == 0);
        const char* tcmp = getenv("CLSPMV_SELL_TAIL_COMPACT");
        p->compact = !(tcmp && atoi(tcmp) == 0);
    }
    if (!rc) {
        // a 32-byte sector of one slice column holds 8 consecutive rows (slice
        // starts are multiples of the slice height): per group of 8 rows, the
        // longest real length counts sectors in each of col and data
        const long long sh = (long long)m->sell_slice_height;
        for (long long r0 = 0; r0 < rows; r0 += 8) {
            int mx = 0;
            for (long long r = r0; r < std::min(rows, r0 + 8) && (r / sh) == (r0 / sh); r++) mx = std::max(mx, rlen[r]);
            p->sector_bytes += 2LL * 32 * mx;
        }
        p->nitems = (long long)items.size();
        rc = cuda_status(cudaMalloc(&p->items, sizeof(int2) * std::max<size_t>(1, items.size())));
        if (!rc && !items.empty())
            rc = cuda_status(cudaMemcpy(p->items, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice));
    }
    if (rc) {
        clspmv_sell_plan_free(p);
        return rc;
    }
    *out = p;
    return CLSPMV_OK;
}

}  // extern "C"

namespace clspmv {
// The planned walk for a caller that already applied beta and adds into y
// with the other parts of a Cocktail matrix (atomic = true).
int launch_sell_plan(const clspmv_sell_f32* m, const clspmv_sell_plan* p, const float* x, float* y, float alpha, float beta,
                     cudaStream_t st, bool atomic)
{
    if (!p) return CLSPMV_ERR_ARG;
    return launch_sell_planned(m, p->rlen, p->items, p->nitems, p->split ? p->head : nullptr, p->split_items, p->nsplit,
                               p->tail_off, p->compact ? p->tail_col : nullptr, x, y, alpha, beta, st, atomic);
}
}  // namespace clspmv

extern "C" {

int clspmv_sell_plan_spmv_f32(const clspmv_sell_f32* m, const clspmv_sell_plan* p, const float* x, float* y, float alpha,
                              float beta, clspmv_stream_t s)
{
    if (!p) return CLSPMV_ERR_ARG;
    return launch_sell_planned(m, p->rlen, p->items, p->nitems, p->split ? p->head : nullptr, p->split_items, p->nsplit,
                               p->tail_off, p->compact ? p->tail_col : nullptr, x, y, alpha, beta, S(s), false);
}

int clspmv_sell_plan_spmv_packed(const clspmv_sell_f32* m, const clspmv_sell_plan* p, int value_type, const void* values,
                                 const float* row_scale, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{
    if (!p) return CLSPMV_ERR_ARG;
    const int* head = p->split ? p->head : nullptr;
    const int* tc = p->compact ? p->tail_col : nullptr;
    if (value_type == CLSPMV_VALUES_BF16)
        return launch_sell_planned_packed(m, static_cast<const __nv_bfloat16*>(values), row_scale, p->rlen, head,
                                          p->split_items, p->nsplit, p->tail_off, tc, x, y, alpha, beta, S(s));
    if (value_type == CLSPMV_VALUES_F16)
        return launch_sell_planned_packed(m, static_cast<const __half*>(values), row_scale, p->rlen, head, p->split_items,
                                          p->nsplit, p->tail_off, tc, x, y, alpha, beta, S(s));
    return CLSPMV_ERR_ARG;
}

long long clspmv_sell_plan_entries(const clspmv_sell_plan* p) { return p ? p->entries : -1; }
long long clspmv_sell_plan_items(const clspmv_sell_plan* p) { return p ? p->nitems : -1; }
long long clspmv_sell_plan_sector_bytes(const clspmv_sell_plan* p) { return p ? p->sector_bytes : -1; }
long long clspmv_sell_plan_line_bytes(const clspmv_sell_plan* p) { return p ? p->line_bytes : -1; }

int clspmv_sell_plan_free(clspmv_sell_plan* p)
{
    if (!p) return CLSPMV_ERR_ARG;
    if (p->rlen) cudaFree(p->rlen);
    if (p->items) cudaFree(p->items);
    if (p->head) cudaFree(p->head);
    if (p->split_items) cudaFree(p->split_items);
    if (p->tail_off) cudaFree(p->tail_off);
    if (p->tail_col) cudaFree(p->tail_col);
    delete p;
    return CLSPMV_OK;
}

int clspmv_csr_scalar_spmv_f32(const clspmv_csr_f32* m, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{ return launch_csr_scalar(m, x, y, alpha, beta, S(s), false); }
int clspmv_csr_vector_spmv_f32(const clspmv_csr_f32* m, const float* x, float* y, float alpha, float beta, int tpr, clspmv_stream_t s)
{ return launch_csr_vector(m, x, y, alpha, beta, tpr, S(s), false); }
int clspmv_csr_merge_plan(const clspmv_csr_f32* m, int* tc, clspmv_stream_t s)
{ return launch_csr_merge_plan(m, tc, S(s)); }
int clspmv_csr_merge_spmv_f32(const clspmv_csr_f32* m, const int* tc, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{ return launch_csr_merge(m, tc, x, y, alpha, beta, S(s), false); }
int clspmv_coo_spmv_f32(const clspmv_coo_f32* m, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{ return launch_coo(m, x, y, alpha, beta, S(s), false); }
int clspmv_b4ell_spmv_f32(const clspmv_b4ell_f32* m, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{ return launch_b4ell(m, x, y, alpha, beta, S(s), false); }
int clspmv_sbell_spmv_f32(const clspmv_sbell_f32* m, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{ return launch_sbell(m, x, y, alpha, beta, S(s), false); }
int clspmv_b4csr_spmv_f32(const clspmv_b4csr_f32* m, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{ return launch_b4csr(m, x, y, alpha, beta, S(s), false); }
int clspmv_spmv_packed(int format, const void* dev, int value_type, const void* values, const float* row_scale,
                       const int* tile_coord, const float* x, float* y, float alpha, float beta, clspmv_stream_t s)
{ return launch_packed(format, dev, value_type, values, row_scale, tile_coord, x, y, alpha, beta, S(s), false); }
int clspmv_csr_chunk_spmv_packed(const clspmv_csr_f32* m, int value_type, const void* values, const float* row_scale,
                                 const int* chunk_row, const float* x, float* y, float alpha, float beta,
                                 clspmv_stream_t s)
{
    if (!values || !row_scale) return CLSPMV_ERR_ARG;
    if (value_type == CLSPMV_VALUES_BF16)
        return launch_csr_chunk_v(m, static_cast<const __nv_bfloat16*>(values), row_scale, chunk_row, x, y, alpha, beta,
                                  S(s), false);
    if (value_type == CLSPMV_VALUES_F16)
        return launch_csr_chunk_v(m, static_cast<const __half*>(values), row_scale, chunk_row, x, y, alpha, beta, S(s),
                                  false);
    return CLSPMV_ERR_ARG;
}

}  // extern "C"
