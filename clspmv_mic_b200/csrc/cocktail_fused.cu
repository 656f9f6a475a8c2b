// cocktail_fused.cu — one persistent launch for the SpMV of a partitioned
// (Cocktail) matrix.
//
// The reference enqueues one kernel per part and runs them one after another
// on an in-order queue (do_spmv, src/spmv_cocktail.cpp:1088-1132). Parts of a
// Cocktail partition are bound by different resources: the diagonal and block
// parts stream their arrays from HBM, the flat parts (COO, CSR, ELL, SELL of
// scattered columns) are bound by x gathers from L2. Run in sequence, the
// SpMV costs the sum of the parts. Here every part is cut into tiles (a tile
// is the share of CTA `t` of `ntiles` in the part's CTA-level function of
// kernels.cuh), the tiles of all parts are interleaved into one work list in
// proportion to each part's estimated time, and a persistent grid of CTAs
// takes list entries from a device counter. At any moment the SMs then hold
// a mix of streaming and gathering tiles, and all parts progress together.
// Every tile adds alpha * A_p x into y with red.global.add; beta is applied
// (and the counter reset) by a small kernel launched first, so the pair is
// stream ordered and can be captured in a CUDA graph.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>
#include "clspmv_b200.h"
#include "kernels.cuh"
#include "api_internal.h"

using namespace clspmv;

namespace clspmv {

enum FusedKind { FK_DIA, FK_BDIA, FK_SBELL, FK_BELL, FK_BCSR, FK_SELL_COLS, FK_SELL_ROWS4, FK_SELL_ROWS, FK_ELL, FK_CSR,
                 FK_COO };

// One part: its kind, the template variant (block shape BW4 * 16 + BH, SELL
// lanes per column, BCSR lanes per block row, BDIA aligned-x flag), its tile
// count and its argument block with device pointers (x, y and alpha are
// filled in per call from the kernel's parameters).
struct FusedPart {
    int kind, sub, lanes, ntiles;
    const int* aux;                   // CSR: chunk plan
    union Args {
        DiaArgs dia;
        BdiaArgs bdia;
        SbellArgs sbell;
        B4ellArgs bell;
        B4csrArgs bcsr;
        SellArgs sell;
        EllArgs ell;
        CsrArgs csr;
        CooArgs coo;
    } u;
};

struct FusedPlan {
    FusedPart* parts = nullptr;       // device, nparts
    int2* items = nullptr;            // device: (part, tile) in work order
    unsigned* counter = nullptr;      // device: next work item
    int nparts = 0, nitems = 0, rows = 0;
    int grid = 1;                     // resident CTAs of the fused kernel, at most nitems
    int min_ctas = 4;                 // register cap of the kernel variant (k_cocktail_fused<min_ctas>)
};

}  // namespace clspmv

namespace {

// Block shapes the fused kernel covers (sub = bwidth / 4 * 16 + bheight):
// the 4-wide shapes up to 4 high and the 8-wide shapes up to 2 high. The
// others keep as many accumulators as would cut the fused kernel's occupancy
// for every part, so a partition using them keeps the per-part launches.
constexpr bool fused_block_shape(int sub) { return sub == 17 || sub == 18 || sub == 20 || sub == 33 || sub == 34; }

template <class F>
__device__ __forceinline__ void block_shape(int sub, F&& f)
{
    switch (sub) {
        case 16 + 1: f(std::integral_constant<int, 1>{}, std::integral_constant<int, 1>{}); break;
        case 16 + 2: f(std::integral_constant<int, 1>{}, std::integral_constant<int, 2>{}); break;
        case 16 + 4: f(std::integral_constant<int, 1>{}, std::integral_constant<int, 4>{}); break;
        case 32 + 1: f(std::integral_constant<int, 2>{}, std::integral_constant<int, 1>{}); break;
        case 32 + 2: f(std::integral_constant<int, 2>{}, std::integral_constant<int, 2>{}); break;
    }
}

template <class F>
__device__ __forceinline__ void lanes_of(int t, F&& f)
{
    switch (t) {
        case 1: f(std::integral_constant<int, 1>{}); break;
        case 2: f(std::integral_constant<int, 2>{}); break;
        case 4: f(std::integral_constant<int, 4>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        case 16: f(std::integral_constant<int, 16>{}); break;
        case 32: f(std::integral_constant<int, 32>{}); break;
    }
}

template <class A>
__device__ __forceinline__ A with_call(A a, const float* x, float* y, float alpha)
{
    a.x = x;
    a.y = y;
    a.alpha = alpha;
    return a;
}

// One tile of one part; all threads of the CTA call it with the same item.
// Each kind is its own function, called (not inlined): inlined into one
// switch, the kinds' loops together spill heavily at any register cap;
// called, each is allocated on its own under the kernel's cap of 64
// registers (the single-format kernels use 32-53), and only the calls
// save and restore a few registers.
__device__ __noinline__ void tile_dia(const FusedPart* __restrict__ p, int tile, const float* x, float* y, float alpha, char* smem)
{
    DiaArgs a = with_call(p->u.dia, x, y, alpha);
    a.beta = 1.0f;
    dia_cta<true, float, 0>(a, tile, p->ntiles, smem);
}
__device__ __noinline__ void tile_bdia(const FusedPart* __restrict__ p, int tile, const float* x, float* y, float alpha)
{
    BdiaArgs a = with_call(p->u.bdia, x, y, alpha);
    a.beta = 1.0f;
    if (p->sub) bdia_cta<true, float, true>(a, tile, p->ntiles, nullptr);
    else bdia_cta<true, float, false>(a, tile, p->ntiles, nullptr);
}
template <int BW4, int BH>
__device__ __noinline__ void tile_sbell(const FusedPart* __restrict__ p, int tile, const float* x, float* y, float alpha)
{
    SbellArgs a = with_call(p->u.sbell, x, y, alpha);
    a.beta = 1.0f;
    sbell_cta<BW4, BH, true>(a, tile, p->ntiles, nullptr);
}
template <int BW4, int BH>
__device__ __noinline__ void tile_bell(const FusedPart* __restrict__ p, int tile, const float* x, float* y, float alpha)
{
    B4ellArgs a = with_call(p->u.bell, x, y, alpha);
    a.beta = 1.0f;
    b4ell_cta<BW4, BH, true>(a, tile, p->ntiles, nullptr);
}
template <int BW4, int BH, int T>
__device__ __noinline__ void tile_bcsr(const FusedPart* __restrict__ p, int tile, const float* x, float* y, float alpha)
{
    B4csrArgs a = with_call(p->u.bcsr, x, y, alpha);
    a.beta = 1.0f;
    b4csr_cta<BW4, BH, T, true>(a, tile, p->ntiles, nullptr);
}
template <int Q>
__device__ __noinline__ void tile_sell_cols(const FusedPart* __restrict__ p, int tile, const float* x, float* y, float alpha)
{
    const SellArgs a = with_call(p->u.sell, x, y, alpha);
    sell_cta<Q, true>(a, tile, p->ntiles, nullptr);
}
__device__ __noinline__ void tile_sell_rows4(const FusedPart* __restrict__ p, int tile, const float* x, float* y, float alpha)
{
    SellArgs a = with_call(p->u.sell, x, y, alpha);
    a.beta = 1.0f;
    sell_rows4_cta<true>(a, tile, p->ntiles, nullptr);
}
__device__ __noinline__ void tile_sell_rows(const FusedPart* __restrict__ p, int tile, const float* x, float* y, float alpha)
{
    SellArgs a = with_call(p->u.sell, x, y, alpha);
    a.beta = 1.0f;
    sell_rows_cta<true>(a, tile, p->ntiles, nullptr);
}
__device__ __noinline__ void tile_ell(const FusedPart* __restrict__ p, int tile, const float* x, float* y, float alpha)
{
    EllArgs a = with_call(p->u.ell, x, y, alpha);
    a.beta = 1.0f;
    ell_cta<true>(a, tile, p->ntiles, nullptr);
}
__device__ __noinline__ void tile_csr(const FusedPart* __restrict__ p, int tile, const float* x, float* y, float alpha)
{
    const CsrArgs a = with_call(p->u.csr, x, y, alpha);
    csr_chunk_cta(a, p->aux, tile, p->ntiles);
}
__device__ __noinline__ void tile_coo(const FusedPart* __restrict__ p, int tile, const float* x, float* y, float alpha)
{
    const CooArgs a = with_call(p->u.coo, x, y, alpha);
    coo_cta(a, tile, p->ntiles, nullptr);
}

__device__ __forceinline__ void run_tile(const FusedPart* __restrict__ p, int tile, const float* x, float* y, float alpha,
                                         char* smem)
{
    switch (p->kind) {
        case FK_DIA: tile_dia(p, tile, x, y, alpha, smem); break;
        case FK_BDIA: tile_bdia(p, tile, x, y, alpha); break;
        case FK_SBELL:
            block_shape(p->sub, [&](auto bw4, auto bh) { tile_sbell<decltype(bw4)::value, decltype(bh)::value>(p, tile, x, y, alpha); });
            break;
        case FK_BELL:
            block_shape(p->sub, [&](auto bw4, auto bh) { tile_bell<decltype(bw4)::value, decltype(bh)::value>(p, tile, x, y, alpha); });
            break;
        case FK_BCSR:
            block_shape(p->sub, [&](auto bw4, auto bh) {
                lanes_of(p->lanes, [&](auto t) {
                    tile_bcsr<decltype(bw4)::value, decltype(bh)::value, decltype(t)::value>(p, tile, x, y, alpha);
                });
            });
            break;
        case FK_SELL_COLS: lanes_of(p->sub, [&](auto q) { tile_sell_cols<decltype(q)::value>(p, tile, x, y, alpha); }); break;
        case FK_SELL_ROWS4: tile_sell_rows4(p, tile, x, y, alpha); break;
        case FK_SELL_ROWS: tile_sell_rows(p, tile, x, y, alpha); break;
        case FK_ELL: tile_ell(p, tile, x, y, alpha); break;
        case FK_CSR: tile_csr(p, tile, x, y, alpha); break;
        case FK_COO: tile_coo(p, tile, x, y, alpha); break;
    }
}

// The fused kernel, capped at the registers that keep MINCTAS CTAs of 256
// threads resident per SM (4: 64 registers, 5: 48).
template <int MINCTAS>
__global__ void __launch_bounds__(kBlock, MINCTAS) k_cocktail_fused(const FusedPart* __restrict__ parts,
                                                                    const int2* __restrict__ items, int nitems,
                                                                    unsigned* counter, const float* x, float* y, float alpha)
{
    __shared__ __align__(16) char smem[kDiaSmemBytes];
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int item = s_item;
        __syncthreads();              // every thread has read s_item before thread 0 takes the next one
        if (item >= nitems) return;
        const int2 it = __ldg(items + item);
        run_tile(parts + it.x, it.y, x, y, alpha, smem);
    }
}

// y <- beta * y and the work counter reset, ahead of the fused launch
__global__ void __launch_bounds__(kBlock) k_cocktail_fused_prepare(float* y, int n, float beta, unsigned* counter)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) *counter = 0u;
    if (beta == 1.0f) return;
    for (long long i = blockIdx.x * (long long)kBlock + threadIdx.x; i < n; i += (long long)gridDim.x * kBlock)
        y[i] = beta == 0.0f ? 0.0f : beta * y[i];
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int lanes_pow2(double mean, int lo, int hi)
{
    int t = lo;
    while (t < hi && t < mean) t <<= 1;
    return t;
}

// Estimated time of one part (seconds) for the interleave proportions:
// streaming of its stored arrays at about HBM speed, and for the flat formats
// one x gather per stored entry from L2 (the rates measured on B200 for the
// single-format kernels: ~6.5 TB/s copy, ~2.6e11 random 4-byte gathers/s).
double part_seconds(int format, const void* dev, int nnz, double index_bytes_per_value, bool gathers)
{
    size_t values = 0;
    if (clspmv_stored_values(format, dev, &values)) values = (size_t)std::max(0, nnz);
    const double bytes = (double)values * (4.0 + index_bytes_per_value);
    const double t_bytes = bytes / 6.5e12;
    const double t_gather = gathers ? (double)values / 2.6e11 : 0.0;
    return std::max(t_bytes, t_gather) + 1e-7;
}

long long cdiv(long long a, long long b) { return (a + b - 1) / b; }

int env_int(const char* name, int dflt, int lo, int hi)
{
    const char* e = getenv(name);
    if (!e) return dflt;
    return std::min(hi, std::max(lo, atoi(e)));
}

}  // namespace

namespace clspmv {

int fused_plan_create(const clspmv_cocktail_f32* d, const int* chunk_plan, FusedPlan** out)
{
    if (!d || !out) return CLSPMV_ERR_ARG;
    *out = nullptr;
    std::vector<FusedPart> parts;
    std::vector<double> secs;
    std::vector<long long> max_tiles;
    int rc = CLSPMV_OK;
    auto add = [&](FusedPart p, double s, long long mt) {
        parts.push_back(p);
        secs.push_back(s);
        max_tiles.push_back(std::max(1LL, mt));
    };
    const int rows = d->mat_height;
    if (d->ifusedia) {
        const clspmv_dia_f32& m = d->dia;
        if ((m.dia_length_aligned & 3) || m.matinfo.height > m.dia_length_aligned || !aligned16(m.dia_data))
            return CLSPMV_ERR_UNSUPPORTED;
        FusedPart p{};
        p.kind = FK_DIA;
        p.u.dia = DiaArgs{m.matinfo.height, m.matinfo.width, m.dia_num, m.dia_length_aligned, m.dia_offsets, m.dia_data,
                          nullptr, nullptr, 1.f, 1.f, nullptr};
        add(p, part_seconds(CLSPMV_FORMAT_DIA, &m, m.matinfo.nnz, 0.0, false), cdiv(m.matinfo.height, kDiaRowsPerPass));
    }
    if (d->ifusebdia) {
        const clspmv_bdia_f32& m = d->bdia;
        if ((m.bdia_length_aligned & 3) || m.matinfo.height > m.bdia_length_aligned || !aligned16(m.bdia_data))
            return CLSPMV_ERR_UNSUPPORTED;
        FusedPart p{};
        p.kind = FK_BDIA;
        p.sub = 1;
        p.u.bdia = BdiaArgs{m.matinfo.height, m.matinfo.width, m.bdia_band_num, m.bdia_length_aligned, m.bdia_offsets,
                            m.bdia_bptr, m.bdia_data, nullptr, nullptr, 1.f, 1.f, nullptr};
        add(p, part_seconds(CLSPMV_FORMAT_BDIA, &m, m.matinfo.nnz, 0.0, false), cdiv(m.matinfo.height, kBdiaRowsPerPass));
    }
    if (d->ifusesbell) {
        const clspmv_sbell_f32& m = d->sbell;
        if (!aligned16(m.sbell_data) || m.sbell_slice_height == 0 || (m.sbell_bwidth != 4 && m.sbell_bwidth != 8))
            return CLSPMV_ERR_UNSUPPORTED;
        FusedPart p{};
        p.kind = FK_SBELL;
        p.sub = (int)(m.sbell_bwidth / 4) * 16 + (int)m.sbell_bheight;
        if (!fused_block_shape(p.sub)) return CLSPMV_ERR_UNSUPPORTED;
        p.u.sbell = SbellArgs{m.matinfo.height, m.matinfo.width, m.sbell_row_num, m.sbell_slice_num, (int)m.sbell_slice_height,
                              m.sbell_slice_ptr, m.sbell_col_id, m.sbell_data, nullptr, nullptr, 1.f, 1.f, nullptr};
        add(p, part_seconds(CLSPMV_FORMAT_SBELL, &m, m.matinfo.nnz, 4.0 / (m.sbell_bwidth * m.sbell_bheight), false),
            cdiv(m.sbell_row_num, kBlock));
    }
    if (d->ifusebell) {
        const clspmv_b4ell_f32& m = d->bell;
        if (!aligned16(m.b4ell_data) || (m.b4ell_float4_aligned & 3) || (m.b4ell_bwidth != 4 && m.b4ell_bwidth != 8))
            return CLSPMV_ERR_UNSUPPORTED;
        FusedPart p{};
        p.kind = FK_BELL;
        p.sub = (int)(m.b4ell_bwidth / 4) * 16 + (int)m.b4ell_bheight;
        if (!fused_block_shape(p.sub)) return CLSPMV_ERR_UNSUPPORTED;
        p.u.bell = B4ellArgs{m.matinfo.height, m.matinfo.width, m.b4ell_row_num, m.b4ell_block_num, m.b4ell_height_aligned,
                             m.b4ell_float4_aligned, m.b4ell_col_id, m.b4ell_data, nullptr, nullptr, 1.f, 1.f, nullptr};
        add(p, part_seconds(CLSPMV_FORMAT_B4ELL, &m, m.matinfo.nnz, 4.0 / (m.b4ell_bwidth * m.b4ell_bheight), false),
            cdiv(m.b4ell_row_num, kBlock));
    }
    if (d->ifusebcsr) {
        const clspmv_b4csr_f32& m = d->bcsr;
        if (!aligned16(m.b4csr_data) || (m.b4csr_aligned_size & 3) || (m.b4csr_bwidth != 4 && m.b4csr_bwidth != 8) ||
            m.b4csr_row_num <= 0)
            return CLSPMV_ERR_UNSUPPORTED;
        FusedPart p{};
        p.kind = FK_BCSR;
        p.sub = (int)(m.b4csr_bwidth / 4) * 16 + (int)m.b4csr_bheight;
        if (!fused_block_shape(p.sub)) return CLSPMV_ERR_UNSUPPORTED;
        p.lanes = lanes_pow2((double)m.b4csr_block_num / m.b4csr_row_num, 1, 32);
        p.u.bcsr = B4csrArgs{m.matinfo.height, m.matinfo.width, m.b4csr_row_num, m.b4csr_aligned_size, m.b4csr_row_ptr,
                             m.b4csr_col_id, m.b4csr_data, nullptr, nullptr, 1.f, 1.f, nullptr};
        add(p, part_seconds(CLSPMV_FORMAT_B4CSR, &m, m.matinfo.nnz, 4.0 / (m.b4csr_bwidth * m.b4csr_bheight), false),
            cdiv(m.b4csr_row_num, kBlock / p.lanes));
    }
    if (d->ifusesell) {
        const clspmv_sell_f32& m = d->sell;
        const int sh = (int)m.sell_slice_height;
        if (sh <= 0 || (long long)m.sell_slice_num * sh < m.matinfo.height) return CLSPMV_ERR_UNSUPPORTED;
        FusedPart p{};
        p.u.sell = SellArgs{m.matinfo.height, sh, m.sell_slice_num, m.sell_slice_ptr, m.sell_col_id, m.sell_data, nullptr,
                            nullptr, 1.f, 1.f, nullptr};
        size_t slots = 0;
        if ((rc = clspmv_stored_values(CLSPMV_FORMAT_SELL, &m, &slots))) return rc;
        const bool vec = aligned16(m.sell_col_id) && aligned16(m.sell_data);
        long long mt;
        // the same kernel choice as the single-format SELL launcher
        if (vec && sh % 4 == 0 && (long long)m.matinfo.nnz <= (long long)kSellNarrow * m.matinfo.height) {
            p.kind = FK_SELL_ROWS4;
            mt = cdiv(m.matinfo.height, kBlock * 4);
        } else if (vec && (sh == 4 || sh == 8 || sh == 16 || sh == 32 || sh == 64 || sh == 128)) {
            p.kind = FK_SELL_COLS;
            p.sub = sh / 4;
            mt = cdiv((long long)slots / sh, (long long)kSellWarpCols * (kBlock / 32));
        } else {
            p.kind = FK_SELL_ROWS;
            mt = cdiv(m.matinfo.height, kBlock);
        }
        add(p, part_seconds(CLSPMV_FORMAT_SELL, &m, m.matinfo.nnz, 4.0, true), mt);
    }
    if (d->ifuseell) {
        const clspmv_ell_f32& m = d->ell;
        if ((m.ell_height_aligned & 3) || !aligned16(m.ell_col_id) || !aligned16(m.ell_data) ||
            m.matinfo.height > m.ell_height_aligned)
            return CLSPMV_ERR_UNSUPPORTED;
        FusedPart p{};
        p.kind = FK_ELL;
        p.u.ell = EllArgs{m.matinfo.height, m.ell_num, m.ell_height_aligned, m.ell_col_id, m.ell_data, nullptr, nullptr, 1.f,
                          1.f, nullptr};
        add(p, part_seconds(CLSPMV_FORMAT_ELL, &m, m.matinfo.nnz, 4.0, true), cdiv(m.matinfo.height, kEllRowsPerPass));
    }
    if (d->ifusecsr && d->csr.matinfo.nnz > 0) {
        const clspmv_csr_f32& m = d->csr;
        if (!chunk_plan || !aligned16(m.csr_col_id) || !aligned16(m.csr_data)) return CLSPMV_ERR_UNSUPPORTED;
        FusedPart p{};
        p.kind = FK_CSR;
        p.aux = chunk_plan;
        p.u.csr = CsrArgs{m.matinfo.height, m.matinfo.nnz, m.csr_row_ptr, m.csr_col_id, m.csr_data, nullptr, nullptr, 1.f,
                          1.f, nullptr};
        add(p, part_seconds(CLSPMV_FORMAT_CSR, &m, m.matinfo.nnz, 4.0, true),
            cdiv(cdiv(m.matinfo.nnz, kCooWarpNnz), kBlock / 32));
    }
    if (d->ifusecoo && d->coo.matinfo.nnz > 0) {
        const clspmv_coo_f32& m = d->coo;
        if (!aligned16(m.coo_row_id) || !aligned16(m.coo_col_id) || !aligned16(m.coo_data)) return CLSPMV_ERR_UNSUPPORTED;
        FusedPart p{};
        p.kind = FK_COO;
        p.u.coo = CooArgs{m.matinfo.nnz, m.coo_row_id, m.coo_col_id, m.coo_data, nullptr, nullptr, 1.f, nullptr};
        add(p, part_seconds(CLSPMV_FORMAT_COO, &m, m.matinfo.nnz, 8.0, true),
            cdiv(cdiv(m.matinfo.nnz, kCooWarpNnz), kBlock / 32));
    }
    if (parts.empty()) return CLSPMV_ERR_UNSUPPORTED;

    // tile counts: about items_per_cta list entries per resident CTA in all,
    // split in proportion to the parts' estimated times.
    // CLSPMV_FUSED_ITEMS / _ORDER / _CAP override the defaults (measurements)
    const int items_per_cta = env_int("CLSPMV_FUSED_ITEMS", 4, 1, 64);
    const int order = env_int("CLSPMV_FUSED_ORDER", 0, 0, 1);     // 0 interleaved, 1 part after part
    const int min_ctas = env_int("CLSPMV_FUSED_CAP", 4, 4, 5);
    int dev = 0, nsm = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const cudaError_t occ = min_ctas == 5
        ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cocktail_fused<5>, kBlock, 0)
        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cocktail_fused<4>, kBlock, 0);
    if (occ != cudaSuccess || per < 1) {
        cudaGetLastError();
        per = 1;
    }
    const long long resident = (long long)nsm * per;
    double total = 0.0;
    for (double s : secs) total += s;
    std::vector<int> tiles(parts.size());
    long long nitems = 0;
    for (size_t i = 0; i < parts.size(); i++) {
        const double want = (double)resident * items_per_cta * secs[i] / total;
        tiles[i] = (int)std::max(1LL, std::min(max_tiles[i], (long long)std::llround(want)));
        parts[i].ntiles = tiles[i];
        nitems += tiles[i];
    }
    // the work list: every part's tiles in order, merged by the fraction of
    // the part that precedes them, so the parts advance side by side
    std::vector<int2> items;
    items.reserve((size_t)nitems);
    std::vector<int> next(parts.size(), 0);
    for (long long k = 0; k < nitems; k++) {
        int best = -1;
        double best_f = 2.0;
        for (size_t i = 0; i < parts.size(); i++) {
            if (next[i] >= tiles[i]) continue;
            const double f = order == 1 ? (double)i : (next[i] + 0.5) / tiles[i];
            if (f < best_f) {
                best_f = f;
                best = (int)i;
            }
        }
        items.push_back(make_int2(best, next[best]++));
    }

    FusedPlan* plan = new (std::nothrow) FusedPlan();
    if (!plan) return CLSPMV_ERR_ALLOC;
    plan->nparts = (int)parts.size();
    plan->nitems = (int)nitems;
    plan->rows = rows;
    plan->grid = (int)std::max(1LL, std::min(resident, nitems));
    plan->min_ctas = min_ctas;
    rc = cuda_status(cudaMalloc(&plan->parts, sizeof(FusedPart) * parts.size()));
    if (!rc) rc = cuda_status(cudaMalloc(&plan->items, sizeof(int2) * items.size()));
    if (!rc) rc = cuda_status(cudaMalloc(&plan->counter, sizeof(unsigned)));
    if (!rc) rc = cuda_status(cudaMemcpy(plan->parts, parts.data(), sizeof(FusedPart) * parts.size(), cudaMemcpyHostToDevice));
    if (!rc) rc = cuda_status(cudaMemcpy(plan->items, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice));
    if (!rc) rc = cuda_status(cudaMemset(plan->counter, 0, sizeof(unsigned)));
    if (rc) {
        fused_plan_free(plan);
        return rc;
    }
    *out = plan;
    return CLSPMV_OK;
}

int fused_spmv(const FusedPlan* plan, const float* x, float* y, float alpha, float beta, cudaStream_t st)
{
    if (!plan || !x || !y) return CLSPMV_ERR_ARG;
    if (!aligned16(x)) return CLSPMV_ERR_ALIGN;
    const unsigned prep_grid = beta == 1.0f ? 1u : (unsigned)std::max(1LL, std::min(cdiv(plan->rows, kBlock), 148LL * 8));
    k_cocktail_fused_prepare<<<prep_grid, kBlock, 0, st>>>(y, plan->rows, beta, plan->counter);
    int rc = after_launch(1);
    if (rc) return rc;
    if (plan->min_ctas == 5)
        k_cocktail_fused<5><<<(unsigned)plan->grid, kBlock, 0, st>>>(plan->parts, plan->items, plan->nitems, plan->counter, x, y, alpha);
    else
        k_cocktail_fused<4><<<(unsigned)plan->grid, kBlock, 0, st>>>(plan->parts, plan->items, plan->nitems, plan->counter, x, y, alpha);
    return after_launch(1);
}

void fused_plan_free(FusedPlan* plan)
{
    if (!plan) return;
    if (plan->parts) cudaFree(plan->parts);
    if (plan->items) cudaFree(plan->items);
    if (plan->counter) cudaFree(plan->counter);
    delete plan;
}

int fused_plan_items(const FusedPlan* plan) { return plan ? plan->nitems : 0; }

}  // namespace clspmv
