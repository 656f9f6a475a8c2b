// kernels.cuh — CTA tile functions of every storage format (sm_100a).
//
// All tiles compute  y[r] <- alpha * (A x)[r] + beta * y[r]  for the rows they
// own. With ATOMIC = true they instead add alpha * (A x)[r] with atomicAdd
// (beta must then have been applied beforehand); the Cocktail runtime uses
// that mode because several parts add into the same y.
//
// The reference's kernels (kernels/*.cl of clSpMV) run one work-item per row
// or per block row and rely on the texture path for x. Here the matrix arrays
// are read with 128-bit, fully coalesced, L1-bypassing evict-first loads in
// each format's native layout; x is gathered through L1 with an evict-last
// L2 policy; banded formats stage their x window in shared memory; CSR-vector
// and COO reduce with warp shuffles.
#pragma once
#include <climits>
#include "common.cuh"

namespace clspmv {

constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------------------
// x as float4 at a float index c (c % 4 == 0), zero past `cols`.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float4 load_x4_guarded(const float* x, int c, int cols, uint64_t pol)
{
    if (c + 3 < cols) return ld_x4(x + c, pol);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (c < cols) v.x = ld_x(x + c, pol);
    if (c + 1 < cols) v.y = ld_x(x + c + 1, pol);
    if (c + 2 < cols) v.z = ld_x(x + c + 2, pol);
    return v;
}

__device__ __forceinline__ float x_or_zero(const float* x, int c, int cols, uint64_t pol)
{
    return (unsigned)c < (unsigned)cols ? ld_x(x + c, pol) : 0.f;
}

// ---------------------------------------------------------------------------
// DIA (kernels/spmv_dia.cl:4-170): 4 consecutive rows per thread, one
// 128-bit load of dia_data per diagonal; diagonal offsets staged in shared
// memory 256 at a time (the reference keeps <= MAX_DIA_NUM in __local).
// ---------------------------------------------------------------------------
constexpr int kDiaRowsPerTile = kBlock * 4;
constexpr int kDiaSmemBytes = kBlock * sizeof(int);

template <bool ATOMIC>
__device__ __forceinline__ void dia_tile(const DiaArgs& a, int tile, char* smem)
{
    int* s_off = reinterpret_cast<int*>(smem);
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int row0 = tile * kDiaRowsPerTile + threadIdx.x * 4;
    const bool active = row0 < a.rows;
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f, acc3 = 0.f;
    for (int d0 = 0; d0 < a.ndiag; d0 += kBlock) {
        const int nd = min(kBlock, a.ndiag - d0);
        __syncthreads();
        if (threadIdx.x < nd) s_off[threadIdx.x] = a.offsets[d0 + threadIdx.x];
        __syncthreads();
        if (active) {
            const float* dp = a.data + (size_t)d0 * a.len + row0;
#pragma unroll 4
            for (int k = 0; k < nd; k++) {
                const int c = row0 + s_off[k];
                const float4 v = ld_stream_f4(dp + (size_t)k * a.len, pe);
                float x0, x1, x2, x3;
                if (c >= 0 && c + 3 < a.cols) {
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
                acc0 = fmaf(v.x, x0, acc0);
                acc1 = fmaf(v.y, x1, acc1);
                acc2 = fmaf(v.z, x2, acc2);
                acc3 = fmaf(v.w, x3, acc3);
            }
        }
    }
    if (active) {
        y_update<ATOMIC>(a.y, row0, a.alpha, a.beta, acc0);
        if (row0 + 1 < a.rows) y_update<ATOMIC>(a.y, row0 + 1, a.alpha, a.beta, acc1);
        if (row0 + 2 < a.rows) y_update<ATOMIC>(a.y, row0 + 2, a.alpha, a.beta, acc2);
        if (row0 + 3 < a.rows) y_update<ATOMIC>(a.y, row0 + 3, a.alpha, a.beta, acc3);
    }
}

// ---------------------------------------------------------------------------
// BDIA (kernels/spmv_bdia.cl:4-283): per band, the x window
// [tile_row0 + offset, tile_row0 + offset + 1024 + width - 1) is staged in
// shared memory once and every diagonal of the band reads it with a shifted
// index, kept in a 4-register sliding window. Bands wider than kBdiaChunk
// diagonals are processed kBdiaChunk diagonals at a time.
// ---------------------------------------------------------------------------
constexpr int kBdiaRowsPerTile = kBlock * 4;
constexpr int kBdiaChunk = 128;
constexpr int kBdiaSmemBytes = (kBdiaRowsPerTile + kBdiaChunk) * sizeof(float);

template <bool ATOMIC>
__device__ __forceinline__ void bdia_tile(const BdiaArgs& a, int tile, char* smem)
{
    float* s_x = reinterpret_cast<float*>(smem);
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int rbase = tile * kBdiaRowsPerTile;
    const int l0 = threadIdx.x * 4;
    const int row0 = rbase + l0;
    const bool active = row0 < a.rows;
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f, acc3 = 0.f;
    for (int b = 0; b < a.nband; b++) {
        const int dbeg = a.bptr[b], dend = a.bptr[b + 1];
        const int boff = a.offsets[b];
        for (int j0 = 0; j0 < dend - dbeg; j0 += kBdiaChunk) {
            const int nj = min(kBdiaChunk, dend - dbeg - j0);
            const int wbase = rbase + boff + j0;
            const int wlen = kBdiaRowsPerTile + nj - 1;
            __syncthreads();
            for (int t = threadIdx.x; t < wlen; t += kBlock) s_x[t] = x_or_zero(a.x, wbase + t, a.cols, pl);
            __syncthreads();
            if (active) {
                const float* dp = a.data + (size_t)(dbeg + j0) * a.len + row0;
                float w0 = s_x[l0], w1 = s_x[l0 + 1], w2 = s_x[l0 + 2];
#pragma unroll 4
                for (int j = 0; j < nj; j++) {
                    const float w3 = s_x[l0 + j + 3];
                    const float4 v = ld_stream_f4(dp + (size_t)j * a.len, pe);
                    acc0 = fmaf(v.x, w0, acc0);
                    acc1 = fmaf(v.y, w1, acc1);
                    acc2 = fmaf(v.z, w2, acc2);
                    acc3 = fmaf(v.w, w3, acc3);
                    w0 = w1;
                    w1 = w2;
                    w2 = w3;
                }
            }
        }
    }
    if (active) {
        y_update<ATOMIC>(a.y, row0, a.alpha, a.beta, acc0);
        if (row0 + 1 < a.rows) y_update<ATOMIC>(a.y, row0 + 1, a.alpha, a.beta, acc1);
        if (row0 + 2 < a.rows) y_update<ATOMIC>(a.y, row0 + 2, a.alpha, a.beta, acc2);
        if (row0 + 3 < a.rows) y_update<ATOMIC>(a.y, row0 + 3, a.alpha, a.beta, acc3);
    }
}

// ---------------------------------------------------------------------------
// ELL (kernels/spmv_ell.cl:4-104, the _v4 form): 4 rows per thread, int4 and
// float4 loads of each column-major slot.
// ---------------------------------------------------------------------------
constexpr int kEllRowsPerTile = kBlock * 4;

template <bool ATOMIC>
__device__ __forceinline__ void ell_tile(const EllArgs& a, int tile, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int row0 = tile * kEllRowsPerTile + threadIdx.x * 4;
    if (row0 >= a.rows) return;
    const int* cp = a.col + row0;
    const float* dp = a.data + row0;
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f, acc3 = 0.f;
#pragma unroll 4
    for (int k = 0; k < a.ell_num; k++) {
        const int4 c = ld_stream_i4(cp + (size_t)k * a.len, pe);
        const float4 v = ld_stream_f4(dp + (size_t)k * a.len, pe);
        acc0 = fmaf(v.x, ld_x(a.x + c.x, pl), acc0);
        acc1 = fmaf(v.y, ld_x(a.x + c.y, pl), acc1);
        acc2 = fmaf(v.z, ld_x(a.x + c.z, pl), acc2);
        acc3 = fmaf(v.w, ld_x(a.x + c.w, pl), acc3);
    }
    y_update<ATOMIC>(a.y, row0, a.alpha, a.beta, acc0);
    if (row0 + 1 < a.rows) y_update<ATOMIC>(a.y, row0 + 1, a.alpha, a.beta, acc1);
    if (row0 + 2 < a.rows) y_update<ATOMIC>(a.y, row0 + 2, a.alpha, a.beta, acc2);
    if (row0 + 3 < a.rows) y_update<ATOMIC>(a.y, row0 + 3, a.alpha, a.beta, acc3);
}

// ---------------------------------------------------------------------------
// SELL (kernels/spmv_sell.cl:4-130): each thread owns 4 consecutive rows of a
// slice (slice height a multiple of 4), so slice height 128 is one warp per
// slice reading 512 contiguous bytes per slot, and slice height 32 is 8
// threads per slice. Slice starts are multiples of the slice height, hence
// 16-byte aligned.
// ---------------------------------------------------------------------------
template <bool ATOMIC>
__device__ __forceinline__ void sell_tile(const SellArgs& a, int tile, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int sh = a.slice_height;
    const int qps = sh >> 2;
    const int q = tile * kBlock + threadIdx.x;
    const int s = q / qps;
    if (s >= a.nslice) return;
    const int sub = q - s * qps;
    const int start = a.slice_ptr[s];
    const int width = (a.slice_ptr[s + 1] - start) / sh;
    const int* cp = a.col + start + sub * 4;
    const float* dp = a.data + start + sub * 4;
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f, acc3 = 0.f;
#pragma unroll 4
    for (int k = 0; k < width; k++) {
        const int4 c = ld_stream_i4(cp + (size_t)k * sh, pe);
        const float4 v = ld_stream_f4(dp + (size_t)k * sh, pe);
        acc0 = fmaf(v.x, ld_x(a.x + c.x, pl), acc0);
        acc1 = fmaf(v.y, ld_x(a.x + c.y, pl), acc1);
        acc2 = fmaf(v.z, ld_x(a.x + c.z, pl), acc2);
        acc3 = fmaf(v.w, ld_x(a.x + c.w, pl), acc3);
    }
    const int row0 = s * sh + sub * 4;
    if (row0 < a.rows) y_update<ATOMIC>(a.y, row0, a.alpha, a.beta, acc0);
    if (row0 + 1 < a.rows) y_update<ATOMIC>(a.y, row0 + 1, a.alpha, a.beta, acc1);
    if (row0 + 2 < a.rows) y_update<ATOMIC>(a.y, row0 + 2, a.alpha, a.beta, acc2);
    if (row0 + 3 < a.rows) y_update<ATOMIC>(a.y, row0 + 3, a.alpha, a.beta, acc3);
}

// Slice heights that are not a multiple of 4: one row per thread.
template <bool ATOMIC>
__device__ __forceinline__ void sell_tile_scalar(const SellArgs& a, int tile, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int row = tile * kBlock + threadIdx.x;
    if (row >= a.rows) return;
    const int sh = a.slice_height;
    const int s = row / sh, lr = row - s * sh;
    const int start = a.slice_ptr[s];
    const int width = (a.slice_ptr[s + 1] - start) / sh;
    float acc = 0.f;
#pragma unroll 4
    for (int k = 0; k < width; k++) {
        const size_t i = (size_t)start + (size_t)k * sh + lr;
        acc = fmaf(ld_stream_f(a.data + i, pe), ld_x(a.x + ld_stream_i(a.col + i, pe), pl), acc);
    }
    y_update<ATOMIC>(a.y, row, a.alpha, a.beta, acc);
}

// ---------------------------------------------------------------------------
// CSR scalar (kernels/spmv_csr_scalar.cl:5-209): one thread per row. Rows
// whose start and end are multiples of 4 (pad_csr(.., 4), the reference's
// _float4_noif input) use 128-bit loads.
// ---------------------------------------------------------------------------
template <bool ATOMIC>
__device__ __forceinline__ void csr_scalar_tile(const CsrArgs& a, int tile, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int row = tile * kBlock + threadIdx.x;
    if (row >= a.rows) return;
    const int s = a.row_ptr[row], e = a.row_ptr[row + 1];
    float acc = 0.f;
    if (((s | e) & 3) == 0) {
        for (int j = s; j < e; j += 4) {
            const int4 c = ld_l1_i4(a.col + j, pe);
            const float4 v = ld_l1_f4(a.val + j, pe);
            acc = fmaf(v.x, ld_x(a.x + c.x, pl), acc);
            acc = fmaf(v.y, ld_x(a.x + c.y, pl), acc);
            acc = fmaf(v.z, ld_x(a.x + c.z, pl), acc);
            acc = fmaf(v.w, ld_x(a.x + c.w, pl), acc);
        }
    } else {
#pragma unroll 4
        for (int j = s; j < e; j++) acc = fmaf(ld_l1_f(a.val + j, pe), ld_x(a.x + ld_l1_i(a.col + j, pe), pl), acc);
    }
    y_update<ATOMIC>(a.y, row, a.alpha, a.beta, acc);
}

// ---------------------------------------------------------------------------
// CSR vector (kernels/spmv_csr_vector.cl:4-191): T lanes per row with a
// shuffle reduction (the reference uses a volatile __local reduction that
// assumes lock-step warps). Rows padded to a multiple of 4 use 128-bit
// loads, 4 consecutive entries per lane.
// ---------------------------------------------------------------------------
template <int T, bool ATOMIC>
__device__ __forceinline__ void csr_vector_tile(const CsrArgs& a, int tile, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int g = (tile * kBlock + threadIdx.x) / T;
    const int l = threadIdx.x % T;
    const bool active = g < a.rows;
    float acc = 0.f;
    if (active) {
        const int s = a.row_ptr[g], e = a.row_ptr[g + 1];
        if (((s | e) & 3) == 0) {
            for (int j = s + 4 * l; j < e; j += 4 * T) {
                const int4 c = ld_l1_i4(a.col + j, pe);
                const float4 v = ld_l1_f4(a.val + j, pe);
                acc = fmaf(v.x, ld_x(a.x + c.x, pl), acc);
                acc = fmaf(v.y, ld_x(a.x + c.y, pl), acc);
                acc = fmaf(v.z, ld_x(a.x + c.z, pl), acc);
                acc = fmaf(v.w, ld_x(a.x + c.w, pl), acc);
            }
        } else {
#pragma unroll 4
            for (int j = s + l; j < e; j += T) acc = fmaf(ld_l1_f(a.val + j, pe), ld_x(a.x + ld_l1_i(a.col + j, pe), pl), acc);
        }
    }
#pragma unroll
    for (int off = T / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(kFull, acc, off, T);
    if (active && l == 0) y_update<ATOMIC>(a.y, g, a.alpha, a.beta, acc);
}

// ---------------------------------------------------------------------------
// CSR merge path: a tile owns kMergeTile consecutive items of the merge of
// the row-end offsets row_ptr[1..m] with the nonzero indices 0..nnz-1, so
// every CTA does the same work whatever the row-length distribution. The
// tile's row pointers and its nonzero products are staged in shared memory;
// each thread walks kMergeIPT merge items and accumulates finished rows into
// a shared per-row sum with shared-memory atomics. Rows that cross a tile
// boundary are added to y with global atomics; rows owned by the tile are
// written directly.
// ---------------------------------------------------------------------------
constexpr int kMergeIPT = 8;
constexpr int kMergeTile = kBlock * kMergeIPT;
constexpr int kMergeSmemBytes = (kMergeTile + 2) * sizeof(int) + kMergeTile * sizeof(float) + (kMergeTile + 1) * sizeof(float);

template <bool ATOMIC_ALL>
__device__ __forceinline__ void csr_merge_tile(const CsrArgs& a, const int* __restrict__ tc, int tile, char* smem)
{
    int* s_rp = reinterpret_cast<int*>(smem);
    float* s_prod = reinterpret_cast<float*>(s_rp + kMergeTile + 2);
    float* s_y = s_prod + kMergeTile;
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int x0 = tc[2 * tile], y0 = tc[2 * tile + 1];
    const int x1 = tc[2 * tile + 2], y1 = tc[2 * tile + 3];
    const int nfin = x1 - x0, nz = y1 - y0;
    for (int k = threadIdx.x; k <= nfin + 1; k += kBlock) {
        const int r = x0 + k;
        s_rp[k] = r <= a.rows ? a.row_ptr[r] : INT_MAX;
    }
    for (int k = threadIdx.x; k < nz; k += kBlock) {
        const int j = y0 + k;
        s_prod[k] = ld_stream_f(a.val + j, pe) * ld_x(a.x + ld_stream_i(a.col + j, pe), pl);
    }
    for (int k = threadIdx.x; k <= nfin; k += kBlock) s_y[k] = 0.f;
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

    for (int k = threadIdx.x; k <= nfin; k += kBlock) {
        const int r = x0 + k;
        if (r >= a.rows) continue;
        const int rs = s_rp[k], re = s_rp[k + 1];
        const float v = s_y[k];
        const bool ends_here = k < nfin;
        if (rs >= y0 && ends_here) {
            if (rs != re) {
                if (ATOMIC_ALL) atomicAdd(a.y + r, a.alpha * v);
                else a.y[r] = a.y[r] + a.alpha * v;
            }
        } else {
            const int from = max(rs, y0), to = ends_here ? re : y1;
            if (to > from) atomicAdd(a.y + r, a.alpha * v);
        }
    }
}

// Tile start coordinates (rows finished, nonzeros consumed) of the merge
// path at diagonals t * kMergeTile, t = 0..ntiles.
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
// COO (kernels/spmv_coo.cl:4-217): single pass. A warp takes 32*kCooK
// consecutive nonzeros (row-sorted), loads them lane-striped (coalesced),
// and runs a segmented inclusive scan per 32-wide step with shuffles, the
// row id acting as the segment key. The running tail is carried across
// steps; the first and last row of a warp chunk may be shared with the
// neighbouring chunk and are added with atomics, interior rows directly.
// The reference instead writes per-group carries to tmp_rowid/tmp_data and
// reduces them in a second kernel (gpu_coo_s2).
// ---------------------------------------------------------------------------
constexpr int kCooK = 8;
constexpr int kCooWarpNnz = 32 * kCooK;
constexpr int kCooTileNnz = kCooWarpNnz * (kBlock / 32);

template <bool ATOMIC_ALL>
__device__ __forceinline__ void coo_put(float* y, int row, float v, int first_row)
{
    if (ATOMIC_ALL || row == first_row) atomicAdd(y + row, v);
    else y[row] += v;
}

template <bool ATOMIC_ALL>
__device__ __forceinline__ void coo_tile(const CooArgs& a, int tile, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int lane = threadIdx.x & 31;
    const long long base = (long long)tile * kCooTileNnz + (long long)(threadIdx.x >> 5) * kCooWarpNnz;
    if (base >= a.nnz) return;
    int r[kCooK], c[kCooK];
    float p[kCooK];
#pragma unroll
    for (int k = 0; k < kCooK; k++) {
        const long long idx = base + k * 32 + lane;
        if (idx < a.nnz) {
            r[k] = ld_stream_i(a.row + idx, pe);
            c[k] = ld_stream_i(a.col + idx, pe);
            p[k] = ld_stream_f(a.val + idx, pe);
        } else {
            r[k] = -1;
            c[k] = 0;
            p[k] = 0.f;
        }
    }
#pragma unroll
    for (int k = 0; k < kCooK; k++)
        if (r[k] >= 0) p[k] *= ld_x(a.x + c[k], pl);
    const int first_row = __shfl_sync(kFull, r[0], 0);
    float carry = 0.f;
    int carry_row = -1;
#pragma unroll
    for (int k = 0; k < kCooK; k++) {
        const int rr = r[k];
        float v = p[k];
        const int lead = __shfl_sync(kFull, rr, 0);
        if (carry_row >= 0 && lead != carry_row) {
            if (lane == 0) coo_put<ATOMIC_ALL>(a.y, carry_row, a.alpha * carry, first_row);
            carry = 0.f;
            carry_row = -1;
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const float vu = __shfl_up_sync(kFull, v, off);
            const int ru = __shfl_up_sync(kFull, rr, off);
            if (lane >= off && ru == rr) v += vu;
        }
        if (rr == carry_row) v += carry;
        const int rn = __shfl_down_sync(kFull, rr, 1);
        const bool tail = lane == 31 || rn != rr;
        const float v31 = __shfl_sync(kFull, v, 31);
        const int r31 = __shfl_sync(kFull, rr, 31);
        if (tail && lane != 31 && rr >= 0) coo_put<ATOMIC_ALL>(a.y, rr, a.alpha * v, first_row);
        carry = v31;
        carry_row = r31;
    }
    if (carry_row >= 0 && lane == 0) atomicAdd(a.y + carry_row, a.alpha * carry);
}

// ---------------------------------------------------------------------------
// BELL = b4ell (kernels/spmv_bell.cl): one thread per block row; every
// (slot, w4, h) plane is a contiguous float4 array over block rows, so a warp
// reads 512 contiguous bytes per load. x blocks are 16-byte aligned float4.
// ---------------------------------------------------------------------------
template <int BW4, int BH, bool ATOMIC>
__device__ __forceinline__ void b4ell_tile(const B4ellArgs& a, int tile, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int r = tile * kBlock + threadIdx.x;
    if (r >= a.nbrow) return;
    float acc[BH];
#pragma unroll
    for (int h = 0; h < BH; h++) acc[h] = 0.f;
    const size_t colsz = (size_t)a.f4 * BW4 * BH;
    const float* base = a.data + (size_t)r * 4;
    for (int j = 0; j < a.ellnum; j++) {
        const int c4 = ld_stream_i(a.col + (size_t)j * a.len + r, pe);
        const float* bj = base + (size_t)j * colsz;
#pragma unroll
        for (int w4 = 0; w4 < BW4; w4++) {
            const float4 xv = load_x4_guarded(a.x, (c4 + w4) * 4, a.cols, pl);
#pragma unroll
            for (int h = 0; h < BH; h++) {
                const float4 v = ld_stream_f4(bj + (size_t)w4 * a.f4 * BH + (size_t)h * a.f4, pe);
                acc[h] = dot4(v, xv, acc[h]);
            }
        }
    }
#pragma unroll
    for (int h = 0; h < BH; h++) {
        const int row = r * BH + h;
        if (row < a.rows) y_update<ATOMIC>(a.y, row, a.alpha, a.beta, acc[h]);
    }
}

// ---------------------------------------------------------------------------
// SBELL (kernels/spmv_sbell.cl): slices of slice_height block rows; one
// thread per block row, so a 32-high slice is one warp and every plane load
// is 512 contiguous bytes.
// ---------------------------------------------------------------------------
template <int BW4, int BH, bool ATOMIC>
__device__ __forceinline__ void sbell_tile(const SbellArgs& a, int tile, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int r = tile * kBlock + threadIdx.x;
    if (r >= a.nbrow) return;
    const int sh = a.slice_height;
    const int s = r / sh, lr = r - s * sh;
    const int cs = a.slice_ptr[s];
    const int width = (a.slice_ptr[s + 1] - cs) / sh;
    float acc[BH];
#pragma unroll
    for (int h = 0; h < BH; h++) acc[h] = 0.f;
    const size_t bs = (size_t)BW4 * 4 * BH;
    const size_t colsz = (size_t)sh * BW4 * BH * 4, hsz = (size_t)sh * 4, w4sz = (size_t)sh * BH * 4;
    const float* base = a.data + (size_t)cs * bs + (size_t)lr * 4;
    for (int j = 0; j < width; j++) {
        const int c4 = ld_stream_i(a.col + (size_t)cs + lr + (size_t)j * sh, pe);
        const float* bj = base + (size_t)j * colsz;
#pragma unroll
        for (int w4 = 0; w4 < BW4; w4++) {
            const float4 xv = load_x4_guarded(a.x, (c4 + w4) * 4, a.cols, pl);
#pragma unroll
            for (int h = 0; h < BH; h++) {
                const float4 v = ld_stream_f4(bj + (size_t)w4 * w4sz + (size_t)h * hsz, pe);
                acc[h] = dot4(v, xv, acc[h]);
            }
        }
    }
#pragma unroll
    for (int h = 0; h < BH; h++) {
        const int row = r * BH + h;
        if (row < a.rows) y_update<ATOMIC>(a.y, row, a.alpha, a.beta, acc[h]);
    }
}

// ---------------------------------------------------------------------------
// BCSR = b4csr (kernels/spmv_bcsr.cl): T lanes per block row; lane l takes
// blocks start+l, start+l+T, ... Each (w4, h) plane holds one float4 per
// block, consecutive blocks adjacent, so the T lanes of a row and the rows of
// a warp read contiguous memory. Partial sums are combined with shuffles
// (the reference reduces in __local memory per 128-thread group).
// ---------------------------------------------------------------------------
template <int BW4, int BH, int T, bool ATOMIC>
__device__ __forceinline__ void b4csr_tile(const B4csrArgs& a, int tile, char*)
{
    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    const int g = (tile * kBlock + threadIdx.x) / T;
    const int l = threadIdx.x % T;
    const bool active = g < a.nbrow;
    float acc[BH];
#pragma unroll
    for (int h = 0; h < BH; h++) acc[h] = 0.f;
    if (active) {
        const int s = a.row_ptr[g], e = a.row_ptr[g + 1];
        const size_t plane_w4 = (size_t)a.len * BH;
        for (int i = s + l; i < e; i += T) {
            const int c4 = ld_stream_i(a.col + i, pe);
            const float* bi = a.data + (size_t)i * 4;
#pragma unroll
            for (int w4 = 0; w4 < BW4; w4++) {
                const float4 xv = load_x4_guarded(a.x, (c4 + w4) * 4, a.cols, pl);
#pragma unroll
                for (int h = 0; h < BH; h++) {
                    const float4 v = ld_stream_f4(bi + w4 * plane_w4 + (size_t)h * a.len, pe);
                    acc[h] = dot4(v, xv, acc[h]);
                }
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
            const int row = g * BH + h;
            if (row < a.rows) y_update<ATOMIC>(a.y, row, a.alpha, a.beta, acc[h]);
        }
    }
}

}  // namespace clspmv
