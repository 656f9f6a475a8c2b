// kernels.cuh — CTA-level SpMV work functions of every storage format
// (sm_100a).
//
// All functions compute  y[r] <- alpha * (A x)[r] + beta * y[r]  for the rows
// they own. With ATOMIC = true they add alpha * (A x)[r] with red.global.add
// instead (beta must then have been applied beforehand); the Cocktail runtime
// uses that mode because several parts add into the same y, and the
// load-balanced kernels (CSR merge, COO, SELL) use it for rows that straddle
// two CTAs.
//
// Work distribution: a launch has `ncta` CTAs; CTA `cta` owns one contiguous,
// equal share of the format's units (rows, block rows, slice columns,
// nonzeros) and walks it in passes of one block of threads. Equal shares keep
// every CTA busy to the end of the launch (no partial last wave), and the
// functions take (cta, ncta) explicitly so that the fused Cocktail kernel can
// give each part its own range of CTAs.
//
// The reference's kernels (kernels/*.cl of clSpMV) run one work-item per row
// or block row and read x through the texture path. Here the matrix arrays
// are read with 128-bit, fully coalesced, L1-bypassing evict-first loads in
// each format's native layout; x is gathered through L1 with an evict-last
// L2 policy; BDIA stages its x window in shared memory; CSR-vector, COO and
// SELL reduce with warp shuffles.
#pragma once
#include <climits>
#include "common.cuh"

namespace clspmv {

constexpr unsigned kFull = 0xffffffffu;

// x as float4 at a float index c (c % 4 == 0), zero past `cols`.
__device__ __forceinline__ float4 load_x4_guarded(const float* x, int c, int cols, uint64_t pol)
{
    if (c + 3 < cols) return ld_x4(x + c, pol);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (c < cols) v.x = ld_x(x + c, pol);
    if (c + 1 < cols) v.y = ld_x(x + c + 1, pol);
    if (c + 2 < cols) v.z = ld_x(x + c + 2, pol);
    return v;
}

// x[b .. b+3] for b a multiple of 4 (x 16-byte aligned), zero outside [0, cols)
__device__ __forceinline__ float4 load_x4_window(const float* x, int b, int cols, uint64_t pol)
{
    if (b >= 0 && b + 3 < cols) return ld_x4(x + b, pol);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (b + 3 >= 0 && b < cols) {
        if ((unsigned)b < (unsigned)cols) v.x = ld_x(x + b, pol);
        if ((unsigned)(b + 1) < (unsigned)cols) v.y = ld_x(x + b + 1, pol);
        if ((unsigned)(b + 2) < (unsigned)cols) v.z = ld_x(x + b + 2, pol);
        if ((unsigned)(b + 3) < (unsigned)cols) v.w = ld_x(x + b + 3, pol);
    }
    return v;
}

__device__ __forceinline__ float x_or_zero(const float* x, int c, int cols, uint64_t pol)
{
    return (unsigned)c < (unsigned)cols ? ld_x(x + c, pol) : 0.f;
}

// Equal contiguous share [b, e) of `units` for CTA `cta` of `ncta`, with
// share boundaries on multiples of `quantum`.
__device__ __forceinline__ void cta_share(long long units, int quantum, int cta, int ncta, long long& b, long long& e)
{
    long long per = (units + ncta - 1) / ncta;
    per = (per + quantum - 1) / quantum * quantum;
    b = min(units, per * cta);
    e = min(units, b + per);
}

template <bool ATOMIC>
__device__ __forceinline__ void y_put4(const float* acc, long long row0, long long e, float* y, float alpha, float beta,
                                       const float* scale = nullptr)
{
#pragma unroll
    for (int i = 0; i < 4; i++)
        if (row0 + i < e) y_update<ATOMIC>(y, row0 + i, row_alpha(alpha, scale, row0 + i), beta, acc[i]);
}

// ---------------------------------------------------------------------------
// DIA (kernels/spmv_dia.cl:4-170): 4 consecutive rows per thread, one
// 128-bit load of dia_data per diagonal; offsets staged in shared memory 256
// at a time (the reference keeps <= MAX_DIA_NUM offsets in __local).
// ---------------------------------------------------------------------------
constexpr int kDiaRowsPerPass = kBlock * 4;
constexpr int kDiaSmemBytes = kBlock * sizeof(int);

// XF (x form), for a 16-byte aligned x: 0 four scalar x loads per diagonal;
// 1 one or two aligned 128-bit loads; 3 one aligned 128-bit load per thread,
// the next 4 values taken from the neighbouring lane by shuffles (the lanes
// of a warp own consecutive groups of 4 rows).
template <bool ATOMIC, class V, int XF = 0>
__device__ __forceinline__ void dia_cta(const DiaArgsT<V>& a, int cta, int ncta, char* smem)
{
    int* s_off = reinterpret_cast<int*>(smem);
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    long long b, e;
    cta_share(a.rows, 4, cta, ncta, b, e);
    const bool single_chunk = a.ndiag <= kBlock;
    if (single_chunk) {
        if (threadIdx.x < a.ndiag) s_off[threadIdx.x] = a.offsets[threadIdx.x];
        __syncthreads();
    }
    for (long long pass = b; pass < e; pass += kDiaRowsPerPass) {
        const long long row0 = pass + threadIdx.x * 4;
        const bool active = row0 < e;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        for (int d0 = 0; d0 < a.ndiag; d0 += kBlock) {
            const int nd = min(kBlock, a.ndiag - d0);
            if (!single_chunk) {
                __syncthreads();
                if (threadIdx.x < nd) s_off[threadIdx.x] = a.offsets[d0 + threadIdx.x];
                __syncthreads();
            }
            if (XF == 3) {
                // every lane runs the loop (the shuffles need the whole warp); inactive lanes load nothing
                const V* dp = a.data + (size_t)d0 * a.len + (active ? row0 : 0);
                const int lane = threadIdx.x & 31;
#pragma unroll 4
                for (int k = 0; k < nd; k++) {
                    const int c = (int)row0 + s_off[k];
                    const int sh = c & 3;           // the same for the whole CTA
                    const int base = c - sh;
                    const float4 v = active ? ldv4(dp + (size_t)k * a.len, pe) : make_float4(0.f, 0.f, 0.f, 0.f);
                    // inactive lanes still load their window: the lane below takes it by shuffle
                    const float4 xa = load_x4_window(a.x, base, a.cols, pl);
                    float x0 = xa.x, x1 = xa.y, x2 = xa.z, x3 = xa.w;
                    if (sh) {
                        float4 xb;
                        xb.x = __shfl_down_sync(kFull, xa.x, 1);
                        xb.y = __shfl_down_sync(kFull, xa.y, 1);
                        xb.z = __shfl_down_sync(kFull, xa.z, 1);
                        xb.w = __shfl_down_sync(kFull, xa.w, 1);
                        if (lane == 31) xb = load_x4_window(a.x, base + 4, a.cols, pl);
                        if (sh == 1) { x0 = xa.y; x1 = xa.z; x2 = xa.w; x3 = xb.x; }
                        else if (sh == 2) { x0 = xa.z; x1 = xa.w; x2 = xb.x; x3 = xb.y; }
                        else { x0 = xa.w; x1 = xb.x; x2 = xb.y; x3 = xb.z; }
                    }
                    acc[0] = fmaf(v.x, x0, acc[0]);
                    acc[1] = fmaf(v.y, x1, acc[1]);
                    acc[2] = fmaf(v.z, x2, acc[2]);
                    acc[3] = fmaf(v.w, x3, acc[3]);
                }
            } else if (active) {
                const V* dp = a.data + (size_t)d0 * a.len + row0;
#pragma unroll 4
                for (int k = 0; k < nd; k++) {
                    const int c = (int)row0 + s_off[k];
                    const float4 v = ldv4(dp + (size_t)k * a.len, pe);
                    float x0, x1, x2, x3;
                    const int base = c & ~3;   // rows start at multiples of 4: c & 3 is the same for the whole CTA
                    if (XF == 1 && base >= 0 && base + 7 < a.cols) {
                        // x[c .. c+3] from one or two aligned 128-bit loads
                        const float4 xa = ld_x4(a.x + base, pl);
                        switch (c & 3) {
                            case 0: x0 = xa.x; x1 = xa.y; x2 = xa.z; x3 = xa.w; break;
                            case 1: { const float4 xb = ld_x4(a.x + base + 4, pl); x0 = xa.y; x1 = xa.z; x2 = xa.w; x3 = xb.x; break; }
                            case 2: { const float4 xb = ld_x4(a.x + base + 4, pl); x0 = xa.z; x1 = xa.w; x2 = xb.x; x3 = xb.y; break; }
                            default: { const float4 xb = ld_x4(a.x + base + 4, pl); x0 = xa.w; x1 = xb.x; x2 = xb.y; x3 = xb.z; break; }
                        }
                    } else if (c >= 0 && c + 3 < a.cols) {
                        x0 = ld_x(a.x + c, pl);
                        x1 = ld_x(a.x + c + 1, pl);
                        x2 = ld_x(a.x + c + 2, pl);
                        x3 = ld_x(a.x + c + 3, pl);
                    } else {
                        x0 = x_or_zero(a.x, c, a.cols, pl);
                        x1 = x_or_zero(a.x, c + 1, a.cols, pl);
                        x2 = x_or_zero(a.x, c + 2, a.cols, pl);
                        x3 = x_or_zero(a.x, c + 3, a.cols, pl);
                    }
                    acc[0] = fmaf(v.x, x0, acc[0]);
                    acc[1] = fmaf(v.y, x1, acc[1]);
                    acc[2] = fmaf(v.z, x2, acc[2]);
                    acc[3] = fmaf(v.w, x3, acc[3]);
                }
            }
        }
        if (active) y_put4<ATOMIC>(acc, row0, e, a.y, a.alpha, a.beta, scl(a));
    }
}

// ---------------------------------------------------------------------------
// BDIA (kernels/spmv_bdia.cl:4-283): the reference stages, per band, an x
// window in __local memory and lets every diagonal of the band read it with
// a shifted index. Here the same reuse happens in registers: for each run of
// up to kBdiaRun diagonals of a band, a thread loads the kBdiaRun + 3 x
// values its 4 rows touch once (they stay L1-resident across neighbouring
// threads) and slides over them, so a band of w diagonals costs w + 3 x
// loads instead of 4 w, with no barrier. dia_data is read with one 128-bit
// evict-first load per diagonal.
// ---------------------------------------------------------------------------
constexpr int kBdiaRowsPerPass = kBlock * 4;
constexpr int kBdiaRun = 4;

template <bool ATOMIC, class V, bool XA = false>
__device__ __forceinline__ void bdia_cta(const BdiaArgsT<V>& a, int cta, int ncta, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    long long b, e;
    cta_share(a.rows, 4, cta, ncta, b, e);
    for (long long row0 = b + threadIdx.x * 4; row0 < e; row0 += kBdiaRowsPerPass) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        for (int bd = 0; bd < a.nband; bd++) {
            const int dbeg = a.bptr[bd], dend = a.bptr[bd + 1];
            const int boff = a.offsets[bd];
            for (int j0 = dbeg; j0 < dend; j0 += kBdiaRun) {
                const int n = min(kBdiaRun, dend - j0);
                const long long c0 = row0 + boff + (j0 - dbeg);
                float xw[kBdiaRun + 3];
                float4 v[kBdiaRun];
#pragma unroll
                for (int t = 0; t < kBdiaRun; t++)
                    if (t < n) v[t] = ldv4(a.data + (size_t)(j0 + t) * a.len + row0, pe);
                const long long base = c0 & ~3LL;   // c0 & 3 is the same for the whole CTA
                if (XA && base >= 0 && base + 11 < a.cols) {
                    // the window x[c0 .. c0+6] from three aligned 128-bit loads
                    const float4 w0 = ld_x4(a.x + base, pl), w1 = ld_x4(a.x + base + 4, pl), w2 = ld_x4(a.x + base + 8, pl);
                    const float win[12] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w, w2.x, w2.y, w2.z, w2.w};
                    switch (c0 & 3) {
                        case 0:
#pragma unroll
                            for (int t = 0; t < kBdiaRun + 3; t++) xw[t] = win[t];
                            break;
                        case 1:
#pragma unroll
                            for (int t = 0; t < kBdiaRun + 3; t++) xw[t] = win[t + 1];
                            break;
                        case 2:
#pragma unroll
                            for (int t = 0; t < kBdiaRun + 3; t++) xw[t] = win[t + 2];
                            break;
                        default:
#pragma unroll
                            for (int t = 0; t < kBdiaRun + 3; t++) xw[t] = win[t + 3];
                            break;
                    }
                } else {
#pragma unroll
                    for (int t = 0; t < kBdiaRun + 3; t++) {
                        const long long c = c0 + t;
                        xw[t] = (t < n + 3 && c >= 0 && c < a.cols) ? ld_x(a.x + c, pl) : 0.f;
                    }
                }
#pragma unroll
                for (int t = 0; t < kBdiaRun; t++) {
                    if (t < n) {
                        acc[0] = fmaf(v[t].x, xw[t], acc[0]);
                        acc[1] = fmaf(v[t].y, xw[t + 1], acc[1]);
                        acc[2] = fmaf(v[t].z, xw[t + 2], acc[2]);
                        acc[3] = fmaf(v[t].w, xw[t + 3], acc[3]);
                    }
                }
            }
        }
        y_put4<ATOMIC>(acc, row0, e, a.y, a.alpha, a.beta, scl(a));
    }
}

// ---------------------------------------------------------------------------
// ELL (kernels/spmv_ell.cl:4-104, the _v4 form): 4 rows per thread, int4 and
// float4 loads of each column-major slot.
// ---------------------------------------------------------------------------
constexpr int kEllRowsPerPass = kBlock * 4;

template <bool ATOMIC, class V, int GX = 0>
__device__ __forceinline__ void ell_cta(const EllArgsT<V>& a, int cta, int ncta, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    long long b, e;
    cta_share(a.rows, 4, cta, ncta, b, e);
    for (long long row0 = b + threadIdx.x * 4; row0 < e; row0 += kEllRowsPerPass) {
        const int* cp = a.col + row0;
        const V* dp = a.data + row0;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
        for (int k = 0; k < a.ell_num; k++) {
            const int4 c = ld_stream_i4(cp + (size_t)k * a.len, pe);
            const float4 v = ldv4(dp + (size_t)k * a.len, pe);
            acc[0] = fmaf(v.x, ld_gx<GX>(a.x + c.x, pl), acc[0]);
            acc[1] = fmaf(v.y, ld_gx<GX>(a.x + c.y, pl), acc[1]);
            acc[2] = fmaf(v.z, ld_gx<GX>(a.x + c.z, pl), acc[2]);
            acc[3] = fmaf(v.w, ld_gx<GX>(a.x + c.w, pl), acc[3]);
        }
        y_put4<ATOMIC>(acc, row0, e, a.y, a.alpha, a.beta, scl(a));
    }
}

// ---------------------------------------------------------------------------
// SELL (kernels/spmv_sell.cl:4-130), balanced by columns: the slot space of
// all slices is split into equal runs of slice columns (one column = the
// slice_height slots of one width step), so a slice 10,000 columns wide is
// shared by many warps instead of serialising one. Q = slice_height / 4
// lanes cover one column with 128-bit loads (4 rows per lane) and a warp
// steps 32 / Q columns at a time; partial row sums are combined with
// shuffles and added to y (directly when the warp saw the whole slice, with
// red.global.add when the slice is shared). Requires slice_height in
// {4, 8, 16, 32, 64, 128} and beta already applied.
// ---------------------------------------------------------------------------
constexpr int kSellWarpCols = 64;
constexpr int kSellNarrow = 12;   // mean nonzeros per row at or below which slices count as narrow

template <int Q, bool ATOMIC_ALL, class V>
__device__ __forceinline__ void sell_cta(const SellArgsT<V>& a, int cta, int ncta, char*)
{
    constexpr int G = 32 / Q;             // columns per warp step
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int sh = Q * 4;
    const long long total_cols = (long long)a.slice_ptr[a.nslice] / sh;
    const int lane = threadIdx.x & 31;
    const int g = lane / Q, q = lane % Q;
    const long long nwarps_total = (long long)ncta * (kBlock / 32);
    const long long wid = (long long)cta * (kBlock / 32) + (threadIdx.x >> 5);
    for (long long c0 = wid * kSellWarpCols; c0 < total_cols; c0 += nwarps_total * kSellWarpCols) {
        const long long c1 = min(c0 + kSellWarpCols, total_cols);
        // first slice whose column range ends after c0
        int lo = 0, hi = a.nslice - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((long long)a.slice_ptr[mid + 1] <= c0 * sh) lo = mid + 1;
            else hi = mid;
        }
        int s = lo;
        long long c = c0;
        while (c < c1) {
            const long long sb = a.slice_ptr[s] / sh, se = a.slice_ptr[s + 1] / sh;
            if (se <= c) {
                s++;
                continue;
            }
            const long long ce = min(c1, se);
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
            for (long long cc = c + g; cc < ce; cc += G) {
                const size_t base = (size_t)cc * sh + 4 * q;
                const int4 cv = ld_stream_i4(a.col + base, pe);
                const float4 v = ldv4(a.data + base, pe);
                acc[0] = fmaf(v.x, ld_x(a.x + cv.x, pl), acc[0]);
                acc[1] = fmaf(v.y, ld_x(a.x + cv.y, pl), acc[1]);
                acc[2] = fmaf(v.z, ld_x(a.x + cv.z, pl), acc[2]);
                acc[3] = fmaf(v.w, ld_x(a.x + cv.w, pl), acc[3]);
            }
#pragma unroll
            for (int off = Q; off < 32; off <<= 1) {
#pragma unroll
                for (int i = 0; i < 4; i++) acc[i] += __shfl_xor_sync(kFull, acc[i], off);
            }
            if (g == 0) {
                const bool whole = sb >= c0 && se <= c1;
                const long long row0 = (long long)s * sh + 4 * q;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (row0 + i < a.rows) {
                        const float al = row_alpha(a.alpha, scl(a), row0 + i);
                        if (whole && !ATOMIC_ALL) a.y[row0 + i] += al * acc[i];
                        else atomicAdd(a.y + row0 + i, al * acc[i]);
                    }
                }
            }
            c = ce;
            s++;
        }
    }
}

// Narrow slices (few columns each): 4 rows per thread inside one slice,
// int4 / float4 loads of each slice column, like ELL. Requires slice_height
// a multiple of 4 and 16-byte aligned arrays.
template <bool ATOMIC, class V>
__device__ __forceinline__ void sell_rows4_cta(const SellArgsT<V>& a, int cta, int ncta, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    long long b, e;
    cta_share(a.rows, 4, cta, ncta, b, e);
    const int sh = a.slice_height;
    for (long long row0 = b + threadIdx.x * 4; row0 < e; row0 += kBlock * 4) {
        const int s = (int)(row0 / sh), lr = (int)(row0 - (long long)s * sh);
        const int start = a.slice_ptr[s];
        const int width = (a.slice_ptr[s + 1] - start) / sh;
        const size_t base = (size_t)start + lr;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
        for (int k = 0; k < width; k++) {
            const int4 c = ld_stream_i4(a.col + base + (size_t)k * sh, pe);
            const float4 v = ldv4(a.data + base + (size_t)k * sh, pe);
            acc[0] = fmaf(v.x, ld_x(a.x + c.x, pl), acc[0]);
            acc[1] = fmaf(v.y, ld_x(a.x + c.y, pl), acc[1]);
            acc[2] = fmaf(v.z, ld_x(a.x + c.z, pl), acc[2]);
            acc[3] = fmaf(v.w, ld_x(a.x + c.w, pl), acc[3]);
        }
        y_put4<ATOMIC>(acc, row0, e, a.y, a.alpha, a.beta, scl(a));
    }
}

// ---------------------------------------------------------------------------
// SELL without its padding. The converter pads every row of a slice to the
// slice's widest row with the row's previous column id and value 0
// (include/matrix_storage.h:1466-1491): a slot whose column equals the slot
// before it and whose value is 0 adds nothing, and a row's trailing run of
// such slots is padding. sell_row_length finds where a row's real entries end
// (once per matrix). sell_head_cta then sums each row's first kSellHead
// entries with one thread per row (consecutive rows of a slice are adjacent,
// so a warp's loads are coalesced) and writes y; sell_tail_cta adds the rest
// of the long rows, a warp per item of up to kSellTailCols entries of one
// row, with red.global.add. A slice as wide as one power-law row then costs
// that row's entries instead of slice_height times them.
// ---------------------------------------------------------------------------
constexpr int kSellHead = 32;
constexpr int kSellTailCols = 256;

// Scans back from the slice's last column 16 slots at a time (the loads of a
// group are independent, so a row padded over thousands of columns costs
// hundreds of round trips, not thousands); the first slot always counts.
__device__ __forceinline__ int sell_row_length(const int* slice_ptr, const int* col, const float* data, int sh, long long row)
{
    constexpr int C = 16;
    const int s = (int)(row / sh), lr = (int)(row - (long long)s * sh);
    const int start = slice_ptr[s];
    int k = (slice_ptr[s + 1] - start) / sh;
    const size_t base = (size_t)start + lr;
    while (k > 1) {
        const int lo = max(1, k - C);   // slots lo .. k-1 are examined
        int c[C + 1];
        float d[C];
#pragma unroll
        for (int t = 0; t <= C; t++) {
            const int j = k - 1 - t;     // slot j, and j - 1 for the comparison
            c[t] = j >= lo - 1 ? col[base + (size_t)j * sh] : 0;
            if (t < C) d[t] = j >= lo ? data[base + (size_t)j * sh] : 0.0f;
        }
#pragma unroll
        for (int t = 0; t < C; t++) {
            const int j = k - 1 - t;
            if (j >= lo && (c[t] != c[t + 1] || d[t] != 0.0f)) return j + 1;
        }
        k = lo;
    }
    return k;
}

template <bool ATOMIC>
__device__ __forceinline__ void sell_head_cta(const SellArgs& a, const int* __restrict__ rlen, int cta, int ncta)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    long long b, e;
    cta_share(a.rows, 32, cta, ncta, b, e);
    const int sh = a.slice_height;
    for (long long row = b + threadIdx.x; row < e; row += kBlock) {
        const int s = (int)(row / sh), lr = (int)(row - (long long)s * sh);
        const size_t base = (size_t)__ldg(a.slice_ptr + s) + lr;
        const int n = min(__ldg(rlen + row), kSellHead);
        float acc = 0.f;
#pragma unroll 4
        for (int k = 0; k < n; k++) {
            const size_t i = base + (size_t)k * sh;
            acc = fmaf(ld_stream_f(a.data + i, pe), ld_x(a.x + ld_stream_i(a.col + i, pe), pl), acc);
        }
        y_update<ATOMIC>(a.y, row, a.alpha, a.beta, acc);
    }
}

// items: (row, first entry) pairs, first entry >= kSellHead; y already holds
// the row's head sum.
__device__ __forceinline__ void sell_tail_cta(const SellArgs& a, const int* __restrict__ rlen, const int2* __restrict__ items,
                                              long long nitems, int cta, int ncta)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int lane = threadIdx.x & 31;
    const long long nwarps = (long long)ncta * (kBlock / 32);
    const int sh = a.slice_height;
    for (long long it = (long long)cta * (kBlock / 32) + (threadIdx.x >> 5); it < nitems; it += nwarps) {
        const int2 item = __ldg(items + it);
        const int s = item.x / sh, lr = item.x - s * sh;
        const size_t base = (size_t)__ldg(a.slice_ptr + s) + lr;
        const int k1 = min(item.y + kSellTailCols, __ldg(rlen + item.x));
        float acc = 0.f;
#pragma unroll 4
        for (int k = item.y + lane; k < k1; k += 32) {
            const size_t i = base + (size_t)k * sh;
            acc = fmaf(ld_stream_f(a.data + i, pe), ld_x(a.x + ld_stream_i(a.col + i, pe), pl), acc);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(kFull, acc, off);
        if (lane == 0) atomicAdd(a.y + item.x, a.alpha * acc);
    }
}

// sell_tail_cta with the tail column ids copied by the plan into one
// compact array (tail_col[tail_off[it] + k - item.y]): the lanes of a warp
// read an item's column ids from consecutive words, and only its values
// from the slice's stride-sh column-major layout.
template <class V = float>
__device__ __forceinline__ void sell_tail_compact_cta(const SellArgsT<V>& a, const int* __restrict__ rlen,
                                                      const int2* __restrict__ items, const int* __restrict__ tail_off,
                                                      const int* __restrict__ tail_col, long long nitems, int cta, int ncta)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int lane = threadIdx.x & 31;
    const long long nwarps = (long long)ncta * (kBlock / 32);
    const int sh = a.slice_height;
    for (long long it = (long long)cta * (kBlock / 32) + (threadIdx.x >> 5); it < nitems; it += nwarps) {
        const int2 item = __ldg(items + it);
        const int s = item.x / sh, lr = item.x - s * sh;
        const size_t base = (size_t)__ldg(a.slice_ptr + s) + lr;
        const int n = __ldg(tail_off + it + 1) - __ldg(tail_off + it);
        const int* __restrict__ tc = tail_col + __ldg(tail_off + it) - item.y;
        float acc = 0.f;
#pragma unroll 4
        for (int k = item.y + lane; k < item.y + n; k += 32)
            acc = fmaf(ldv(a.data + base + (size_t)k * sh, pe), ld_x(a.x + ld_stream_i(tc + k, pe), pl), acc);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(kFull, acc, off);
        if (lane == 0) atomicAdd(a.y + item.x, row_alpha(a.alpha, scl(a), item.x) * acc);
    }
}

// SELL with the padding skipped, on the column-balanced mapping of sell_cta:
// the Q lanes of a column each own 4 rows of the slice, and a lane issues its
// 128-bit loads only for the columns before the longest real length of its 4
// rows (rlen, from the plan). A slice padded to the width of one long row then
// reads, in its tail columns, the 32-byte sectors of that row only (the
// padded read takes the whole 128-byte line of 32 rows per column and
// array), while the warp still walks the slot space in equal runs of columns.
// Requires slice_height = 4 Q, 16-byte aligned arrays and beta already
// applied.
//
// With `head` (a prefix table of per-slice head widths, nslice + 1 entries),
// only the first head[s+1] - head[s] columns of slice s are walked: the
// columns up to its second-longest row, the rest of its longest row being
// left to sell_tail_cta.
template <int Q, bool ATOMIC_ALL, class V = float>
__device__ __forceinline__ void sell_masked_cta(const SellArgsT<V>& a, const int* __restrict__ rlen, int cta, int ncta,
                                                const int* __restrict__ head = nullptr)
{
    constexpr int G = 32 / Q;             // columns per warp step
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int sh = Q * 4;
    const int* __restrict__ cptr = head ? head : a.slice_ptr;   // column-space prefix (slots / sh without head)
    const long long cdiv = head ? 1 : sh;
    const long long total_cols = (long long)cptr[a.nslice] / cdiv;
    const int lane = threadIdx.x & 31;
    const int g = lane / Q, q = lane % Q;
    const long long nwarps_total = (long long)ncta * (kBlock / 32);
    const long long wid = (long long)cta * (kBlock / 32) + (threadIdx.x >> 5);
    for (long long c0 = wid * kSellWarpCols; c0 < total_cols; c0 += nwarps_total * kSellWarpCols) {
        const long long c1 = min(c0 + kSellWarpCols, total_cols);
        int lo = 0, hi = a.nslice - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((long long)cptr[mid + 1] <= c0 * cdiv) lo = mid + 1;
            else hi = mid;
        }
        int s = lo;
        long long c = c0;
        while (c < c1) {
            const long long sb = cptr[s] / cdiv, se = cptr[s + 1] / cdiv;
            if (se <= c) {   // the next slice with a column at or past c (runs of empty slices are skipped at once)
                int l = s + 1, h = a.nslice - 1;
                while (l < h) {
                    const int mid = (l + h) >> 1;
                    if ((long long)cptr[mid + 1] <= c * cdiv) l = mid + 1;
                    else h = mid;
                }
                s = l;
                continue;
            }
            const long long ce = min(c1, se);
            // slot of column cc of this slice: (cc - sb) * sh + slice start
            const long long sbase = (long long)a.slice_ptr[s] - sb * sh;
            const long long row0 = (long long)s * sh + 4 * q;
            int live = 0;                 // columns sb .. sb + live - 1 hold real entries of this lane's rows
            if (row0 + 3 < a.rows) {
                const int4 l = __ldg(reinterpret_cast<const int4*>(rlen + row0));
                live = max(max(l.x, l.y), max(l.z, l.w));
            } else {
                for (int i = 0; i < 4; i++)
                    if (row0 + i < a.rows) live = max(live, __ldg(rlen + row0 + i));
            }
            const long long klim = sb + live;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
            for (long long cc = c + g; cc < ce; cc += G) {
                if (cc < klim) {
                    const size_t base = (size_t)(sbase + cc * sh) + 4 * q;
                    const int4 cv = ld_stream_i4(a.col + base, pe);
                    const float4 v = ldv4(a.data + base, pe);
                    acc[0] = fmaf(v.x, ld_x(a.x + cv.x, pl), acc[0]);
                    acc[1] = fmaf(v.y, ld_x(a.x + cv.y, pl), acc[1]);
                    acc[2] = fmaf(v.z, ld_x(a.x + cv.z, pl), acc[2]);
                    acc[3] = fmaf(v.w, ld_x(a.x + cv.w, pl), acc[3]);
                }
            }
#pragma unroll
            for (int off = Q; off < 32; off <<= 1) {
#pragma unroll
                for (int i = 0; i < 4; i++) acc[i] += __shfl_xor_sync(kFull, acc[i], off);
            }
            if (g == 0) {
                const bool whole = sb >= c0 && se <= c1;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (row0 + i < a.rows) {
                        const float al = row_alpha(a.alpha, scl(a), row0 + i);
                        if (whole && !ATOMIC_ALL) a.y[row0 + i] += al * acc[i];
                        else atomicAdd(a.y + row0 + i, al * acc[i]);
                    }
                }
            }
            c = ce;
            s++;
        }
    }
}

// Other slice heights: one row per thread, slice by slice.
template <bool ATOMIC, class V>
__device__ __forceinline__ void sell_rows_cta(const SellArgsT<V>& a, int cta, int ncta, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    long long b, e;
    cta_share(a.rows, 1, cta, ncta, b, e);
    const int sh = a.slice_height;
    for (long long row = b + threadIdx.x; row < e; row += kBlock) {
        const int s = (int)(row / sh), lr = (int)(row - (long long)s * sh);
        const int start = a.slice_ptr[s];
        const int width = (a.slice_ptr[s + 1] - start) / sh;
        float acc = 0.f;
#pragma unroll 4
        for (int k = 0; k < width; k++) {
            const size_t i = (size_t)start + (size_t)k * sh + lr;
            acc = fmaf(ldv(a.data + i, pe), ld_x(a.x + ld_stream_i(a.col + i, pe), pl), acc);
        }
        y_update<ATOMIC>(a.y, row, row_alpha(a.alpha, scl(a), row), a.beta, acc);
    }
}

// ---------------------------------------------------------------------------
// CSR scalar (kernels/spmv_csr_scalar.cl:5-209): one thread per row. Rows
// whose start and end are multiples of 4 (pad_csr(.., 4), the reference's
// _float4_noif input) use 128-bit loads.
// ---------------------------------------------------------------------------
template <bool ATOMIC>
__device__ __forceinline__ void csr_scalar_cta(const CsrArgs& a, int cta, int ncta, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    long long b, e;
    cta_share(a.rows, 1, cta, ncta, b, e);
    for (long long row = b + threadIdx.x; row < e; row += kBlock) {
        const int s = a.row_ptr[row], en = a.row_ptr[row + 1];
        float acc = 0.f;
        if (((s | en) & 3) == 0) {
            for (int j = s; j < en; j += 4) {
                const int4 c = ld_l1_i4(a.col + j, pe);
                const float4 v = ld_l1_f4(a.val + j, pe);
                acc = fmaf(v.x, ld_x(a.x + c.x, pl), acc);
                acc = fmaf(v.y, ld_x(a.x + c.y, pl), acc);
                acc = fmaf(v.z, ld_x(a.x + c.z, pl), acc);
                acc = fmaf(v.w, ld_x(a.x + c.w, pl), acc);
            }
        } else {
#pragma unroll 4
            for (int j = s; j < en; j++) acc = fmaf(ld_l1_f(a.val + j, pe), ld_x(a.x + ld_l1_i(a.col + j, pe), pl), acc);
        }
        y_update<ATOMIC>(a.y, row, a.alpha, a.beta, acc);
    }
}

// ---------------------------------------------------------------------------
// CSR vector (kernels/spmv_csr_vector.cl:4-191): T lanes per row with a
// shuffle reduction (the reference uses a volatile __local reduction that
// assumes lock-step warps). Rows padded to a multiple of 4 use 128-bit
// loads, 4 consecutive entries per lane.
// ---------------------------------------------------------------------------
template <int T, bool ATOMIC>
__device__ __forceinline__ void csr_vector_cta(const CsrArgs& a, int cta, int ncta, char*)
{
    constexpr int kRowsPerPass = kBlock / T;
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    long long b, e;
    cta_share(a.rows, 1, cta, ncta, b, e);
    const int l = threadIdx.x % T;
    for (long long pass = b; pass < e; pass += kRowsPerPass) {
        const long long g = pass + threadIdx.x / T;
        const bool active = g < e;
        float acc = 0.f;
        if (active) {
            const int s = a.row_ptr[g], en = a.row_ptr[g + 1];
            if (((s | en) & 3) == 0) {
                for (int j = s + 4 * l; j < en; j += 4 * T) {
                    const int4 c = ld_l1_i4(a.col + j, pe);
                    const float4 v = ld_l1_f4(a.val + j, pe);
                    acc = fmaf(v.x, ld_x(a.x + c.x, pl), acc);
                    acc = fmaf(v.y, ld_x(a.x + c.y, pl), acc);
                    acc = fmaf(v.z, ld_x(a.x + c.z, pl), acc);
                    acc = fmaf(v.w, ld_x(a.x + c.w, pl), acc);
                }
            } else {
#pragma unroll 4
                for (int j = s + l; j < en; j += T) acc = fmaf(ld_l1_f(a.val + j, pe), ld_x(a.x + ld_l1_i(a.col + j, pe), pl), acc);
            }
        }
#pragma unroll
        for (int off = T / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(kFull, acc, off, T);
        if (active && l == 0) y_update<ATOMIC>(a.y, g, a.alpha, a.beta, acc);
    }
}

// ---------------------------------------------------------------------------
// CSR merge path: tile t owns the kMergeTile consecutive items starting at
// diagonal t * kMergeTile of the merge of the row-end offsets row_ptr[1..m]
// with the nonzero indices 0..nnz-1, so every tile does the same work
// whatever the row-length distribution. The tile's row pointers and its
// nonzero products are staged in shared memory with fully unrolled loads;
// each thread walks kMergeIPT merge items and adds finished rows into a
// per-row shared sum with shared-memory atomics; the tile's rows are then
// added to y with red.global.add (rows that straddle tiles get one
// contribution per tile). beta must already be applied.
// ---------------------------------------------------------------------------
constexpr int kMergeIPT = 8;
constexpr int kMergeTile = kBlock * kMergeIPT;
constexpr int kMergeSmemBytes = (kMergeTile + 2) * sizeof(int) + kMergeTile * sizeof(float) + (kMergeTile + 1) * sizeof(float);

template <class V>
__device__ __forceinline__ void csr_merge_tile(const CsrArgsT<V>& a, const int* __restrict__ tc, int tile, char* smem)
{
    int* s_rp = reinterpret_cast<int*>(smem);
    float* s_prod = reinterpret_cast<float*>(s_rp + kMergeTile + 2);
    float* s_y = s_prod + kMergeTile;
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int x0 = tc[2 * tile], y0 = tc[2 * tile + 1];
    const int x1 = tc[2 * tile + 2], y1 = tc[2 * tile + 3];
    const int nfin = x1 - x0, nz = y1 - y0;
    {
        int cidx[kMergeIPT];
        float vv[kMergeIPT];
#pragma unroll
        for (int i = 0; i < kMergeIPT; i++) {
            const int k = threadIdx.x + i * kBlock;
            cidx[i] = k < nz ? ld_stream_i(a.col + y0 + k, pe) : 0;
        }
#pragma unroll
        for (int i = 0; i < kMergeIPT; i++) {
            const int k = threadIdx.x + i * kBlock;
            vv[i] = k < nz ? ldv(a.val + y0 + k, pe) : 0.f;
        }
#pragma unroll
        for (int i = 0; i <= kMergeIPT; i++) {
            const int k = threadIdx.x + i * kBlock;
            if (k <= nfin + 1) {
                const int r = x0 + k;
                s_rp[k] = r <= a.rows ? a.row_ptr[r] : INT_MAX;
            }
            if (k <= nfin) s_y[k] = 0.f;
        }
#pragma unroll
        for (int i = 0; i < kMergeIPT; i++) {
            const int k = threadIdx.x + i * kBlock;
            if (k < nz) s_prod[k] = vv[i] * ld_x(a.x + cidx[i], pl);
        }
    }
    __syncthreads();

    const int total = nfin + nz;
    const int d0 = min((int)threadIdx.x * kMergeIPT, total);
    const int d1 = min(d0 + kMergeIPT, total);
    int lo = max(d0 - nz, 0), hi = min(d0, nfin);
    while (lo < hi) {
        const int piv = (lo + hi) >> 1;
        if (s_rp[piv + 1] - y0 <= d0 - piv - 1) lo = piv + 1;
        else hi = piv;
    }
    int xi = lo, yj = d0 - lo;
    float acc = 0.f;
    for (int it = d0; it < d1; it++) {
        if (yj < nz && y0 + yj < s_rp[xi + 1]) {
            acc += s_prod[yj];
            yj++;
        } else {
            atomicAdd(s_y + xi, acc);
            acc = 0.f;
            xi++;
        }
    }
    if (acc != 0.f) atomicAdd(s_y + xi, acc);
    __syncthreads();

#pragma unroll
    for (int i = 0; i <= kMergeIPT; i++) {
        const int k = threadIdx.x + i * kBlock;
        if (k > nfin) break;
        const int r = x0 + k;
        if (r >= a.rows) break;
        const int rs = s_rp[k], re = s_rp[k + 1];
        const int from = max(rs, y0), to = k < nfin ? re : y1;
        if (to > from) atomicAdd(a.y + r, row_alpha(a.alpha, scl(a), r) * s_y[k]);
    }
}

// Tile start coordinates (rows finished, nonzeros consumed) of the merge
// path at diagonal `diag`.
__device__ __forceinline__ void csr_merge_search(int rows, int nnz, const int* row_ptr, long long diag, int* out)
{
    const long long total = (long long)rows + nnz;
    if (diag > total) diag = total;
    int lo = (int)max(diag - (long long)nnz, 0LL), hi = (int)min(diag, (long long)rows);
    while (lo < hi) {
        const int piv = (lo + hi) >> 1;
        if ((long long)row_ptr[piv + 1] <= diag - piv - 1) lo = piv + 1;
        else hi = piv;
    }
    out[0] = lo;
    out[1] = (int)(diag - lo);
}

// ---------------------------------------------------------------------------
// COO (kernels/spmv_coo.cl:4-217): single pass. A warp takes kCooWarpNnz
// consecutive nonzeros (row-sorted) in steps of 128: each lane loads 4
// consecutive (row, col, value) with 128-bit loads, reduces them in
// registers (rows that start and end inside the lane are added to y at
// once), and only each lane's leading and trailing row partials go through
// a warp segmented scan (segment starts from one ballot, 5 shuffles). The
// trailing row of a step is carried into the next step. Every finished row
// segment is added with red.global.add, so rows shared with the neighbouring
// chunk need no special case. The reference instead writes per-group carries
// to tmp_rowid/tmp_data and reduces them in a second kernel (gpu_coo_s2).
// beta must already be applied; arrays must be 16-byte aligned.
// ---------------------------------------------------------------------------
constexpr int kCooSteps = 2;
constexpr int kCooWarpNnz = 128 * kCooSteps;
constexpr int kCooCtaNnz = kCooWarpNnz * (kBlock / 32);
constexpr int kCooNoRow = INT_MAX;

// adds alpha * v (times the row's scale for 16-bit values) to y[row]
template <template <class> class ArgsT, class V>
__device__ __forceinline__ void coo_red(const ArgsT<V>& a, int row, float v)
{
    if (row != kCooNoRow) atomicAdd(a.y + row, row_alpha(a.alpha, scl(a), row) * v);
}

template <template <class> class ArgsT, class V>
__device__ __forceinline__ void warp_segments(const ArgsT<V>& a, const int (&r)[kCooSteps][4], const float (&p)[kCooSteps][4]);

template <class V, int GX = 0>
__device__ __forceinline__ void coo_warp_chunk(const CooArgsT<V>& a, long long base, uint64_t pe, uint64_t pl)
{
    const int lane = threadIdx.x & 31;
    int r[kCooSteps][4];
    float p[kCooSteps][4];
    {
        int c[kCooSteps][4];
#pragma unroll
        for (int s = 0; s < kCooSteps; s++) {
            const long long idx = base + s * 128 + lane * 4;
            if (idx + 3 < a.nnz) {
                const int4 rv = ld_stream_i4(a.row + idx, pe);
                const int4 cv = ld_stream_i4(a.col + idx, pe);
                const float4 vv = ldv4(a.val + idx, pe);
                r[s][0] = rv.x; r[s][1] = rv.y; r[s][2] = rv.z; r[s][3] = rv.w;
                c[s][0] = cv.x; c[s][1] = cv.y; c[s][2] = cv.z; c[s][3] = cv.w;
                p[s][0] = vv.x; p[s][1] = vv.y; p[s][2] = vv.z; p[s][3] = vv.w;
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const bool in = idx + j < a.nnz;
                    r[s][j] = in ? ld_stream_i(a.row + idx + j, pe) : kCooNoRow;
                    c[s][j] = in ? ld_stream_i(a.col + idx + j, pe) : 0;
                    p[s][j] = in ? ldv(a.val + idx + j, pe) : 0.f;
                }
            }
        }
#pragma unroll
        for (int s = 0; s < kCooSteps; s++)
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (r[s][j] != kCooNoRow) p[s][j] *= ld_gx<GX>(a.x + c[s][j], pl);
    }
    warp_segments(a, r, p);
}

// The reduction of a warp's kCooSteps x 128 (row, product) pairs in
// nonzero order (rows non-decreasing, kCooNoRow past the end): per-lane runs
// in registers, lane-boundary partials by a segmented scan, the trailing row
// carried across steps; every finished row segment is added to y with
// red.global.add.
template <template <class> class ArgsT, class V>
__device__ __forceinline__ void warp_segments(const ArgsT<V>& a, const int (&r)[kCooSteps][4], const float (&p)[kCooSteps][4])
{
    const int lane = threadIdx.x & 31;
    float carry = 0.f;
    int carry_row = -1;
#pragma unroll
    for (int s = 0; s < kCooSteps; s++) {
        const int head_row = r[s][0], tail_row = r[s][3];
        const bool single = head_row == tail_row;
        float head = 0.f, tail = 0.f;
        if (single) {
            tail = p[s][0] + p[s][1] + p[s][2] + p[s][3];
        } else {
            head = p[s][0];
            tail = p[s][3];
            int run_row = -1;
            float run = 0.f;
#pragma unroll
            for (int j = 1; j < 3; j++) {
                const int rj = r[s][j];
                if (rj == head_row) {
                    head += p[s][j];
                } else if (rj == tail_row) {
                    tail += p[s][j];
                } else if (rj == run_row) {
                    run += p[s][j];
                } else {
                    if (run_row >= 0) coo_red(a, run_row, run);
                    run_row = rj;
                    run = p[s][j];
                }
            }
            if (run_row >= 0) coo_red(a, run_row, run);
        }
        // the previous step's trailing row
        const int lead = __shfl_sync(kFull, head_row, 0);
        if (carry_row >= 0 && lead != carry_row) {
            if (lane == 0) coo_red(a, carry_row, carry);
            carry_row = -1;
            carry = 0.f;
        }
        if (lane == 0 && carry_row >= 0) {
            if (single) tail += carry;
            else head += carry;
        }
        // segmented inclusive scan of the lanes' trailing partials
        const int prev_tail_row = __shfl_up_sync(kFull, tail_row, 1);
        const bool start = lane == 0 || !single || prev_tail_row != tail_row;
        const unsigned smask = __ballot_sync(kFull, start);
        const int seg0 = 31 - __clz(smask & (0xffffffffu >> (31 - lane)));
        float v = tail;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const float t = __shfl_up_sync(kFull, v, off);
            if (lane - off >= seg0) v += t;
        }
        const float prev_v = __shfl_up_sync(kFull, v, 1);
        if (!single) {
            const float cin = (lane > 0 && prev_tail_row == head_row) ? prev_v : 0.f;
            coo_red(a, head_row, head + cin);
        }
        const int next_head = __shfl_down_sync(kFull, head_row, 1);
        if (lane < 31 && next_head != tail_row) coo_red(a, tail_row, v);
        carry = __shfl_sync(kFull, v, 31);
        carry_row = __shfl_sync(kFull, tail_row, 31);
        if (carry_row == kCooNoRow) carry_row = -1;
    }
    if (carry_row >= 0 && lane == 0) coo_red(a, carry_row, carry);
}

template <class V, int GX = 0>
__device__ __forceinline__ void coo_cta(const CooArgsT<V>& a, int cta, int ncta, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const long long nchunks = ((long long)a.nnz + kCooWarpNnz - 1) / kCooWarpNnz;
    long long b, e;
    cta_share(nchunks, 1, cta, ncta, b, e);
    for (long long ch = b + (threadIdx.x >> 5); ch < e; ch += kBlock / 32) coo_warp_chunk<V, GX>(a, ch * kCooWarpNnz, pe, pl);
}

// ---------------------------------------------------------------------------
// CSR by nonzero chunks: the COO kernel's mapping (a warp per kCooWarpNnz
// consecutive nonzeros, 4 per lane with 128-bit loads of col_id / data, the
// x gathers issued at once, the same segmented reduction) on CSR arrays,
// without a row id per nonzero: the rows come from row_ptr. A per-matrix
// plan holds, for every chunk, the row of its first nonzero (chunk_row); a
// lane finds the row of its first nonzero of a step by binary search of
// row_ptr between this chunk's and the next chunk's first rows (a few
// L1-resident loads), then steps over row ends for the other three.
// Matrix bytes are CSR's 8 nnz + 4 (m + 1) instead of COO's 12 nnz.
// beta must already be applied; col_id and data 16-byte aligned.
// ---------------------------------------------------------------------------
template <class V, int GX = 0>
__device__ __forceinline__ void csr_chunk_warp(const CsrArgsT<V>& a, const int* __restrict__ chunk_row, long long ch,
                                               uint64_t pe, uint64_t pl)
{
    const int lane = threadIdx.x & 31;
    const long long base = ch * kCooWarpNnz;
    int r[kCooSteps][4];
    float p[kCooSteps][4];
    {
        int c[kCooSteps][4];
#pragma unroll
        for (int s = 0; s < kCooSteps; s++) {
            const long long idx = base + s * 128 + lane * 4;
            if (idx + 3 < a.nnz) {
                const int4 cv = ld_stream_i4(a.col + idx, pe);
                const float4 vv = ldv4(a.val + idx, pe);
                c[s][0] = cv.x; c[s][1] = cv.y; c[s][2] = cv.z; c[s][3] = cv.w;
                p[s][0] = vv.x; p[s][1] = vv.y; p[s][2] = vv.z; p[s][3] = vv.w;
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const bool in = idx + j < a.nnz;
                    c[s][j] = in ? ld_stream_i(a.col + idx + j, pe) : 0;
                    p[s][j] = in ? ldv(a.val + idx + j, pe) : 0.f;
                }
            }
        }
#pragma unroll
        for (int s = 0; s < kCooSteps; s++)
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (base + s * 128 + lane * 4 + j < a.nnz) p[s][j] *= ld_gx<GX>(a.x + c[s][j], pl);
    }
    const int ra = __ldg(chunk_row + ch), rb = __ldg(chunk_row + ch + 1);
#pragma unroll
    for (int s = 0; s < kCooSteps; s++) {
        const long long q0 = base + s * 128 + lane * 4;
        if (q0 >= a.nnz) {
#pragma unroll
            for (int j = 0; j < 4; j++) r[s][j] = kCooNoRow;
            continue;
        }
        // largest row in [ra, rb] starting at or before q0
        int lo = ra, hi = rb;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(a.row_ptr + mid) <= q0) lo = mid;
            else hi = mid - 1;
        }
        int row = lo;
        r[s][0] = row;
#pragma unroll
        for (int j = 1; j < 4; j++) {
            const long long q = q0 + j;
            if (q < a.nnz) {
                while (__ldg(a.row_ptr + row + 1) <= q) row++;
                r[s][j] = row;
            } else {
                r[s][j] = kCooNoRow;
            }
        }
    }
    warp_segments(a, r, p);
}

template <class V, int GX = 0>
__device__ __forceinline__ void csr_chunk_cta(const CsrArgsT<V>& a, const int* __restrict__ chunk_row, int cta, int ncta)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const long long nchunks = ((long long)a.nnz + kCooWarpNnz - 1) / kCooWarpNnz;
    long long b, e;
    cta_share(nchunks, 1, cta, ncta, b, e);
    for (long long ch = b + (threadIdx.x >> 5); ch < e; ch += kBlock / 32) csr_chunk_warp<V, GX>(a, chunk_row, ch, pe, pl);
}

// chunk_row[c] = row of nonzero c * kCooWarpNnz (the largest row whose start
// is at or before it), for c < nchunks; chunk_row[nchunks] = rows - 1.
__device__ __forceinline__ int csr_row_of(const int* __restrict__ row_ptr, int rows, long long q)
{
    int lo = 0, hi = rows - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (row_ptr[mid] <= q) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// BELL = b4ell (kernels/spmv_bell.cl): one thread per block row; every
// (slot, w4, h) plane is a contiguous float4 array over block rows, so a warp
// reads 512 contiguous bytes per load. x blocks are 16-byte aligned float4.
// ---------------------------------------------------------------------------
template <int BW4, int BH, bool ATOMIC, class V>
__device__ __forceinline__ void b4ell_cta(const B4ellArgsT<V>& a, int cta, int ncta, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    long long b, e;
    cta_share(a.nbrow, 1, cta, ncta, b, e);
    const size_t colsz = (size_t)a.f4 * BW4 * BH;
    for (long long r = b + threadIdx.x; r < e; r += kBlock) {
        float acc[BH];
#pragma unroll
        for (int h = 0; h < BH; h++) acc[h] = 0.f;
        const V* base = a.data + (size_t)r * 4;
#pragma unroll 2
        for (int j = 0; j < a.ellnum; j++) {
            const int c4 = ld_stream_i(a.col + (size_t)j * a.len + r, pe);
            const V* bj = base + (size_t)j * colsz;
            float4 v[BW4][BH];
#pragma unroll
            for (int w4 = 0; w4 < BW4; w4++)
#pragma unroll
                for (int h = 0; h < BH; h++) v[w4][h] = ldv4(bj + (size_t)w4 * a.f4 * BH + (size_t)h * a.f4, pe);
#pragma unroll
            for (int w4 = 0; w4 < BW4; w4++) {
                const float4 xv = load_x4_guarded(a.x, (c4 + w4) * 4, a.cols, pl);
#pragma unroll
                for (int h = 0; h < BH; h++) acc[h] = dot4(v[w4][h], xv, acc[h]);
            }
        }
#pragma unroll
        for (int h = 0; h < BH; h++) {
            const long long row = r * BH + h;
            if (row < a.rows) y_update<ATOMIC>(a.y, row, row_alpha(a.alpha, scl(a), row), a.beta, acc[h]);
        }
    }
}

// ---------------------------------------------------------------------------
// SBELL (kernels/spmv_sbell.cl): slices of slice_height block rows; one
// thread per block row, so a 32-high slice is one warp and every plane load
// is 512 contiguous bytes.
// ---------------------------------------------------------------------------
template <int BW4, int BH, bool ATOMIC, class V>
__device__ __forceinline__ void sbell_cta(const SbellArgsT<V>& a, int cta, int ncta, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    long long b, e;
    cta_share(a.nbrow, 32, cta, ncta, b, e);
    const int sh = a.slice_height;
    const size_t bs = (size_t)BW4 * 4 * BH;
    const size_t colsz = (size_t)sh * BW4 * BH * 4, hsz = (size_t)sh * 4, w4sz = (size_t)sh * BH * 4;
    for (long long r = b + threadIdx.x; r < e; r += kBlock) {
        const int s = (int)(r / sh), lr = (int)(r - (long long)s * sh);
        const int cs = a.slice_ptr[s];
        const int width = (a.slice_ptr[s + 1] - cs) / sh;
        float acc[BH];
#pragma unroll
        for (int h = 0; h < BH; h++) acc[h] = 0.f;
        const V* base = a.data + (size_t)cs * bs + (size_t)lr * 4;
#pragma unroll 2
        for (int j = 0; j < width; j++) {
            const int c4 = ld_stream_i(a.col + (size_t)cs + lr + (size_t)j * sh, pe);
            const V* bj = base + (size_t)j * colsz;
            float4 v[BW4][BH];
#pragma unroll
            for (int w4 = 0; w4 < BW4; w4++)
#pragma unroll
                for (int h = 0; h < BH; h++) v[w4][h] = ldv4(bj + (size_t)w4 * w4sz + (size_t)h * hsz, pe);
#pragma unroll
            for (int w4 = 0; w4 < BW4; w4++) {
                const float4 xv = load_x4_guarded(a.x, (c4 + w4) * 4, a.cols, pl);
#pragma unroll
                for (int h = 0; h < BH; h++) acc[h] = dot4(v[w4][h], xv, acc[h]);
            }
        }
#pragma unroll
        for (int h = 0; h < BH; h++) {
            const long long row = r * BH + h;
            if (row < a.rows) y_update<ATOMIC>(a.y, row, row_alpha(a.alpha, scl(a), row), a.beta, acc[h]);
        }
    }
}

// ---------------------------------------------------------------------------
// BCSR = b4csr (kernels/spmv_bcsr.cl): T lanes per block row; lane l takes
// blocks start+l, start+l+T, ... Each (w4, h) plane holds one float4 per
// block, consecutive blocks adjacent, so the T lanes of a row and the rows of
// a warp read contiguous memory. Partial sums are combined with shuffles
// (the reference reduces in __local memory per 128-thread group).
// ---------------------------------------------------------------------------
template <int BW4, int BH, int T, bool ATOMIC, class V>
__device__ __forceinline__ void b4csr_cta(const B4csrArgsT<V>& a, int cta, int ncta, char*)
{
    constexpr int kRowsPerPass = kBlock / T;
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    long long b, e;
    cta_share(a.nbrow, 1, cta, ncta, b, e);
    const int l = threadIdx.x % T;
    const size_t plane_w4 = (size_t)a.len * BH;
    for (long long pass = b; pass < e; pass += kRowsPerPass) {
        const long long g = pass + threadIdx.x / T;
        const bool active = g < e;
        float acc[BH];
#pragma unroll
        for (int h = 0; h < BH; h++) acc[h] = 0.f;
        if (active) {
            const int s = a.row_ptr[g], en = a.row_ptr[g + 1];
#pragma unroll 2
            for (int i = s + l; i < en; i += T) {
                const int c4 = ld_stream_i(a.col + i, pe);
                const V* bi = a.data + (size_t)i * 4;
                float4 v[BW4][BH];
#pragma unroll
                for (int w4 = 0; w4 < BW4; w4++)
#pragma unroll
                    for (int h = 0; h < BH; h++) v[w4][h] = ldv4(bi + w4 * plane_w4 + (size_t)h * a.len, pe);
#pragma unroll
                for (int w4 = 0; w4 < BW4; w4++) {
                    const float4 xv = load_x4_guarded(a.x, (c4 + w4) * 4, a.cols, pl);
#pragma unroll
                    for (int h = 0; h < BH; h++) acc[h] = dot4(v[w4][h], xv, acc[h]);
                }
            }
        }
#pragma unroll
        for (int h = 0; h < BH; h++) {
#pragma unroll
            for (int off = T / 2; off > 0; off >>= 1) acc[h] += __shfl_xor_sync(kFull, acc[h], off, T);
        }
        if (active && l == 0) {
#pragma unroll
            for (int h = 0; h < BH; h++) {
                const long long row = g * BH + h;
                if (row < a.rows) y_update<ATOMIC>(a.y, row, row_alpha(a.alpha, scl(a), row), a.beta, acc[h]);
            }
        }
    }
}

}  // namespace clspmv
