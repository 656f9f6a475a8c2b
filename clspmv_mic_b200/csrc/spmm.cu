// spmm.cu — several right-hand sides at once, Y <- alpha * A * X + beta * Y,
// for every device format, with FP32 values or values stored as BF16 / FP16
// (indices untouched, per-row power-of-two scale, FP32 accumulation).
//
// The reference multiplies one vector per call (its kernels read `vec` and
// `result`, e.g. kernels/spmv_ell.cl:4-30). Here X is n x k and Y is m x k,
// both row major with leading dimensions ldx / ldy, k <= 128. Each row of A
// is handled by a group of G lanes that split the k columns between them
// (VEC = 4 columns per lane with 128-bit loads when X / Y rows are 16-byte
// aligned, else 1), so every stored element of A is read once per group and
// multiplies one contiguous row of X. The regular formats (DIA, BDIA, ELL,
// SELL, b4csr, b4ell, SBELL) walk their own layout row by row; CSR and COO
// split the nonzeros into equal chunks per group (power-law rows cost the
// same as short ones) and add the partial sums of rows cut by a chunk edge
// with vector atomics.
//
// Reduced-precision storage: clspmv_pack_values converts a device matrix's
// FP32 values in place of a caller-supplied 16-bit array: every value of row
// r is divided by s_r = 2^ceil(log2(max_j |a_rj|)) (exact) before rounding,
// so FP16 keeps its full precision whatever the row's magnitude, and the
// kernels multiply the row sum by s_r.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <type_traits>
#include <new>
#include "clspmv_b200.h"
#include "api_internal.h"
#include "common.cuh"

using namespace clspmv;

namespace {

constexpr int kSpmmBlock = 256;
constexpr int kSpmmMaxK = 128;

template <class T> __device__ __forceinline__ float to_f(T v);
template <> __device__ __forceinline__ float to_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }

template <class T> __device__ __forceinline__ T from_f(float v);
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }

template <class T> __device__ __forceinline__ T ld_val(const T* p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// Row walks: for_row(m, r, f) calls f(col, idx) for every stored element of
// row r whose column lies inside the matrix, idx indexing the value array.
// ---------------------------------------------------------------------------
template <class F>
__device__ __forceinline__ void for_row(const clspmv_dia_f32& m, int r, F&& f)
{
    const size_t len = (size_t)m.dia_length_aligned;
    for (int d = 0; d < m.dia_num; d++) {
        const int col = r + __ldg(m.dia_offsets + d);
        if (col >= 0 && col < m.matinfo.width) f(col, (size_t)d * len + r);
    }
}

template <class F>
__device__ __forceinline__ void for_row(const clspmv_bdia_f32& m, int r, F&& f)
{
    const size_t len = (size_t)m.bdia_length_aligned;
    for (int b = 0; b < m.bdia_band_num; b++) {
        const int i0 = __ldg(m.bdia_bptr + b), i1 = __ldg(m.bdia_bptr + b + 1);
        int col = r + __ldg(m.bdia_offsets + b);
        for (int i = i0; i < i1; i++, col++)
            if (col >= 0 && col < m.matinfo.width) f(col, (size_t)i * len + r);
    }
}

template <class F>
__device__ __forceinline__ void for_row(const clspmv_ell_f32& m, int r, F&& f)
{
    const size_t len = (size_t)m.ell_height_aligned;
    for (int s = 0; s < m.ell_num; s++) {
        const size_t idx = (size_t)s * len + r;
        f(__ldg(m.ell_col_id + idx), idx);
    }
}

template <class F>
__device__ __forceinline__ void for_row(const clspmv_sell_f32& m, int r, F&& f)
{
    const int sh = (int)m.sell_slice_height;
    const int sl = r / sh;
    const int start = __ldg(m.sell_slice_ptr + sl);
    const int width = (__ldg(m.sell_slice_ptr + sl + 1) - start) / sh;
    for (int s = 0; s < width; s++) {
        const size_t idx = (size_t)start + (size_t)s * sh + (r - sl * sh);
        f(__ldg(m.sell_col_id + idx), idx);
    }
}

// CSR rows for the batched kernel (one group per row; the single-matrix
// path splits CSR by nonzeros instead).
template <class F>
__device__ __forceinline__ void for_row(const clspmv_csr_f32& m, int r, F&& f)
{
    const int j1 = __ldg(m.csr_row_ptr + r + 1);
    for (int j = __ldg(m.csr_row_ptr + r); j < j1; j++) f(__ldg(m.csr_col_id + j), (size_t)j);
}

// Four consecutive columns of one float4 strip of a block (col0 .. col0+3),
// stopping at the matrix width like the reference's serial sbell_spmv.
template <class F>
__device__ __forceinline__ void strip(int col0, size_t idx0, int width, F&& f)
{
#pragma unroll
    for (int w = 0; w < 4; w++)
        if (col0 + w < width) f(col0 + w, idx0 + w);
}

template <class F>
__device__ __forceinline__ void for_row(const clspmv_b4csr_f32& m, int r, F&& f)
{
    const int bh = (int)m.b4csr_bheight, bw4 = (int)m.b4csr_bwidth / 4;
    const int br = r / bh, h = r - br * bh;
    const size_t len = (size_t)m.b4csr_aligned_size;
    const int i0 = __ldg(m.b4csr_row_ptr + br), i1 = __ldg(m.b4csr_row_ptr + br + 1);
    for (int i = i0; i < i1; i++) {
        const int c4 = __ldg(m.b4csr_col_id + i);
        for (int w4 = 0; w4 < bw4; w4++)
            strip((c4 + w4) * 4, (size_t)w4 * len * bh + (size_t)h * len + (size_t)i * 4, m.matinfo.width, f);
    }
}

template <class F>
__device__ __forceinline__ void for_row(const clspmv_b4ell_f32& m, int r, F&& f)
{
    const int bh = (int)m.b4ell_bheight, bw4 = (int)m.b4ell_bwidth / 4;
    const int br = r / bh, h = r - br * bh;
    const size_t len = (size_t)m.b4ell_height_aligned, f4 = (size_t)m.b4ell_float4_aligned;
    for (int j = 0; j < m.b4ell_block_num; j++) {
        const int c4 = __ldg(m.b4ell_col_id + (size_t)j * len + br);
        for (int w4 = 0; w4 < bw4; w4++)
            strip((c4 + w4) * 4, (size_t)j * f4 * bw4 * bh + (size_t)w4 * f4 * bh + (size_t)h * f4 + (size_t)br * 4,
                  m.matinfo.width, f);
    }
}

template <class F>
__device__ __forceinline__ void for_row(const clspmv_sbell_f32& m, int r, F&& f)
{
    const int bh = (int)m.sbell_bheight, bw4 = (int)m.sbell_bwidth / 4, sh = (int)m.sbell_slice_height;
    const int br = r / bh, h = r - br * bh;
    const int sl = br / sh, s = br - sl * sh;
    const int start = __ldg(m.sbell_slice_ptr + sl);
    const int width = (__ldg(m.sbell_slice_ptr + sl + 1) - start) / sh;
    const size_t base = (size_t)start * bw4 * 4 * bh + (size_t)s * 4;
    for (int j = 0; j < width; j++) {
        const int c4 = __ldg(m.sbell_col_id + (size_t)start + s + (size_t)j * sh);
        for (int w4 = 0; w4 < bw4; w4++)
            strip((c4 + w4) * 4, base + ((size_t)(j * bw4 + w4) * bh + h) * sh * 4, m.matinfo.width, f);
    }
}

// ---------------------------------------------------------------------------
// Lane helpers: a lane owns VEC consecutive columns c0 .. c0+VEC-1 of X / Y.
// ---------------------------------------------------------------------------
template <int VEC> struct Acc;
template <> struct Acc<1> {
    using X = float;
    float v = 0.0f;
    __device__ static X load(const float* x) { return __ldg(x); }
    __device__ static X zero() { return 0.0f; }
    __device__ void fma_v(float a, X xv) { v = fmaf(a, xv, v); }
    __device__ void fma(float a, const float* x) { v = fmaf(a, __ldg(x), v); }
    __device__ void store(float* y, float alpha, float beta) const
    {
        *y = beta == 0.0f ? alpha * v : fmaf(beta, *y, alpha * v);
    }
    __device__ void add(float* y, float alpha) const { *y += alpha * v; }
    __device__ void atomic(float* y, float alpha) const { atomicAdd(y, alpha * v); }
};
template <> struct Acc<4> {
    using X = float4;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    __device__ static X load(const float* x) { return __ldg(reinterpret_cast<const float4*>(x)); }
    __device__ static X zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
    __device__ void fma_v(float a, X xv)
    {
        v.x = fmaf(a, xv.x, v.x);
        v.y = fmaf(a, xv.y, v.y);
        v.z = fmaf(a, xv.z, v.z);
        v.w = fmaf(a, xv.w, v.w);
    }
    __device__ void fma(float a, const float* x)
    {
        const float4 xv = __ldg(reinterpret_cast<const float4*>(x));
        v.x = fmaf(a, xv.x, v.x);
        v.y = fmaf(a, xv.y, v.y);
        v.z = fmaf(a, xv.z, v.z);
        v.w = fmaf(a, xv.w, v.w);
    }
    __device__ void store(float* y, float alpha, float beta) const
    {
        float4 o = make_float4(alpha * v.x, alpha * v.y, alpha * v.z, alpha * v.w);
        if (beta != 0.0f) {
            const float4 p = *reinterpret_cast<const float4*>(y);
            o.x = fmaf(beta, p.x, o.x);
            o.y = fmaf(beta, p.y, o.y);
            o.z = fmaf(beta, p.z, o.z);
            o.w = fmaf(beta, p.w, o.w);
        }
        *reinterpret_cast<float4*>(y) = o;
    }
    __device__ void add(float* y, float alpha) const
    {
        float4 p = *reinterpret_cast<float4*>(y);
        p.x += alpha * v.x;
        p.y += alpha * v.y;
        p.z += alpha * v.z;
        p.w += alpha * v.w;
        *reinterpret_cast<float4*>(y) = p;
    }
    __device__ void atomic(float* y, float alpha) const
    {
        atomicAdd(reinterpret_cast<float4*>(y), make_float4(alpha * v.x, alpha * v.y, alpha * v.z, alpha * v.w));
    }
};

struct Dense {
    int k;
    const float* X;
    int ldx;
    float* Y;
    int ldy;
    float alpha, beta;
    const float* scale;   // per-row scale of packed values, or nullptr
    int lshift;           // log2 of lanes per row group
    int x_form;           // block-row kernel: X rows through L1 (0), with an L2 evict-last hint (1), past L1 (2)
};

// Row-walk kernel: one group of 2^lshift lanes per row, grid-stride over rows.
template <int VEC, class T, class M>
__global__ void __launch_bounds__(kSpmmBlock) k_spmm_rows(M m, const T* __restrict__ vals, Dense d)
{
    const int G = 1 << d.lshift;
    const long long t = (long long)blockIdx.x * kSpmmBlock + threadIdx.x;
    const int lane = (int)(t & (G - 1));
    const int c0 = lane * VEC;
    if (c0 >= d.k) return;                      // lanes past k have no columns
    const long long groups = ((long long)gridDim.x * kSpmmBlock) >> d.lshift;
    for (long long r = t >> d.lshift; r < m.matinfo.height; r += groups) {
        Acc<VEC> acc;
        for_row(m, (int)r, [&](int col, size_t idx) { acc.fma(to_f(ld_val(vals + idx)), d.X + (size_t)col * d.ldx + c0); });
        const float a = d.scale ? d.alpha * d.scale[r] : d.alpha;
        acc.store(d.Y + (size_t)r * d.ldy + c0, a, d.beta);
    }
}

// ---------------------------------------------------------------------------
// Block walks: for_block(m, br, f) calls f(c4, base, s4, sh) for every stored
// block of block row br. The block's first column is 4 * c4; the value of its
// row h, column 4 * w4 + w sits at base + w4 * s4 + h * sh + w, so each
// (w4, h) strip is 4 consecutive values. Same addressing as for_row.
// ---------------------------------------------------------------------------
template <class F>
__device__ __forceinline__ void for_block(const clspmv_b4csr_f32& m, int br, F&& f)
{
    const size_t len = (size_t)m.b4csr_aligned_size, bh = m.b4csr_bheight;
    const int i1 = __ldg(m.b4csr_row_ptr + br + 1);
    for (int i = __ldg(m.b4csr_row_ptr + br); i < i1; i++) f(__ldg(m.b4csr_col_id + i), (size_t)i * 4, len * bh, len);
}

template <class F>
__device__ __forceinline__ void for_block(const clspmv_b4ell_f32& m, int br, F&& f)
{
    const size_t len = (size_t)m.b4ell_height_aligned, f4 = (size_t)m.b4ell_float4_aligned;
    const size_t bh = m.b4ell_bheight, bw4 = m.b4ell_bwidth / 4;
    for (int j = 0; j < m.b4ell_block_num; j++)
        f(__ldg(m.b4ell_col_id + (size_t)j * len + br), (size_t)j * f4 * bw4 * bh + (size_t)br * 4, f4 * bh, f4);
}

template <class F>
__device__ __forceinline__ void for_block(const clspmv_sbell_f32& m, int br, F&& f)
{
    const size_t bh = m.sbell_bheight, bw4 = m.sbell_bwidth / 4, sh = m.sbell_slice_height;
    const int sl = (int)(br / sh), s = br - sl * (int)sh;
    const int start = __ldg(m.sbell_slice_ptr + sl);
    const int width = (__ldg(m.sbell_slice_ptr + sl + 1) - start) / (int)sh;
    const size_t base = (size_t)start * bw4 * 4 * bh + (size_t)s * 4;
    for (int j = 0; j < width; j++)
        f(__ldg(m.sbell_col_id + (size_t)start + s + (size_t)j * sh), base + (size_t)j * bw4 * bh * sh * 4, bh * sh * 4,
          sh * 4);
}

// 4 consecutive values of a block strip. b4csr keeps a block row's blocks
// side by side (block i at 4 * i in each (w4, h) plane), so a group's next
// blocks share the line of this one: those loads allocate in L1 and carry no
// evict-first hint, so that the line is still in L2 when L1 has lost it. In
// b4ell and SBELL the neighbouring groups (block rows) read the rest of the
// line in the same instruction, and the loads stream past L1.
template <class M> struct StripsInL1 { static constexpr bool value = false; };
__device__ __forceinline__ float4 ld_x4_na(const float* p)
{
    float4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
    return v;
}
template <> struct StripsInL1<clspmv_b4csr_f32> { static constexpr bool value = true; };

__device__ __forceinline__ uint2 ld_l1_u2(const void* p) { return __ldg(reinterpret_cast<const uint2*>(p)); }
template <bool L1> __device__ __forceinline__ float4 strip4(const float* p, uint64_t pol)
{
    return L1 ? __ldg(reinterpret_cast<const float4*>(p)) : ld_stream_f4(p, pol);
}
template <bool L1> __device__ __forceinline__ float4 strip4(const __nv_bfloat16* p, uint64_t pol)
{
    const uint2 u = L1 ? ld_l1_u2(p) : ld_stream_u2(p, pol);
    return make_float4(bf16_lo(u.x), bf16_hi(u.x), bf16_lo(u.y), bf16_hi(u.y));
}
template <bool L1> __device__ __forceinline__ float4 strip4(const __half* p, uint64_t pol)
{
    const uint2 u = L1 ? ld_l1_u2(p) : ld_stream_u2(p, pol);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
    return make_float4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ float4 load_x(const float* p, int form, uint64_t pol)
{
    return form == 0 ? __ldg(reinterpret_cast<const float4*>(p)) : form == 1 ? ld_x4(p, pol) : ld_x4_na(p);
}

// One block row of the block-row kernel: the group's lane holds columns
// c0 .. c0+3 of all BH rows of Y. A block's 4 x 4 slice of X is loaded once
// (the 4 X rows in flight together) and multiplies its BH rows from registers
// (the row walk loads it once per row), and each (w4, h) strip of values is
// one 4-value load. Every row accumulates in the same order as the row walk
// (block, strip, column), so the two give the same bits.
template <int BH, int BW4, class T, class M>
__device__ __forceinline__ void block_row(const M& m, const T* __restrict__ vals, int br, int c0, const float* __restrict__ X,
                                          int ldx, float* __restrict__ Y, int ldy, float alpha, float beta,
                                          const float* __restrict__ scale, int x_form)
{
    const int height = m.matinfo.height, width = m.matinfo.width;
    const uint64_t pol = policy_evict_first(), xpol = policy_evict_last();
    Acc<4> acc[BH];
    for_block(m, br, [&](int c4, size_t base, size_t s4, size_t sh) {
#pragma unroll
        for (int w4 = 0; w4 < BW4; w4++) {
            float4 a[BH];
#pragma unroll
            for (int h = 0; h < BH; h++)
                a[h] = strip4<StripsInL1<M>::value>(vals + base + (size_t)w4 * s4 + (size_t)h * sh, pol);
            const int col0 = (c4 + w4) * 4;
            const int ncol = min(4, width - col0);   // the reference stops a block at the matrix width
            float4 xv[4];
            if (ncol == 4) {                         // the 4 X rows in flight together
#pragma unroll
                for (int w = 0; w < 4; w++) xv[w] = load_x(X + (size_t)(col0 + w) * ldx + c0, x_form, xpol);
            } else {
#pragma unroll
                for (int w = 0; w < 4; w++)
                    xv[w] = w < ncol ? load_x(X + (size_t)(col0 + w) * ldx + c0, x_form, xpol) : Acc<4>::zero();
            }
#pragma unroll
            for (int w = 0; w < 4; w++) {
                if (w >= ncol) break;
#pragma unroll
                for (int h = 0; h < BH; h++) {
                    const float av = w == 0 ? a[h].x : w == 1 ? a[h].y : w == 2 ? a[h].z : a[h].w;
                    acc[h].fma_v(av, xv[w]);
                }
            }
        }
    });
#pragma unroll
    for (int h = 0; h < BH; h++) {
        const long long r = (long long)br * BH + h;
        if (r >= height) break;
        const float al = scale ? alpha * scale[r] : alpha;
        acc[h].store(Y + (size_t)r * ldy + c0, al, beta);
    }
}

// Block-row kernel for the 4-wide block formats: one group of 2^lshift lanes
// per BH-high block row (block_row), grid-stride over block rows.
template <int BH, int BW4, class T, class M>
__global__ void __launch_bounds__(kSpmmBlock, BH >= 8 ? 1 : 4) k_spmm_blocks(M m, const T* __restrict__ vals, Dense d)
{
    const long long t = (long long)blockIdx.x * kSpmmBlock + threadIdx.x;
    const int c0 = (int)(t & ((1 << d.lshift) - 1)) * 4;
    if (c0 >= d.k) return;
    const long long groups = ((long long)gridDim.x * kSpmmBlock) >> d.lshift;
    const long long nbr = ((long long)m.matinfo.height + BH - 1) / BH;
    for (long long br = t >> d.lshift; br < nbr; br += groups)
        block_row<BH, BW4>(m, vals, (int)br, c0, d.X, d.ldx, d.Y, d.ldy, d.alpha, d.beta, d.scale, d.x_form);
}

// Nonzero-chunk kernel for CSR (row_ptr) and row-sorted COO (row_id). Y must
// already hold beta * Y. A row wholly inside a chunk is added with a plain
// read-modify-write; a row cut by a chunk edge is added atomically.
constexpr int kChunkPrefetch = 4;

template <int VEC, class T, bool IS_CSR>
__global__ void __launch_bounds__(kSpmmBlock) k_spmm_chunks(int rows, int nnz, const int* __restrict__ row_ptr,
                                                            const int* __restrict__ row_id, const int* __restrict__ col_id,
                                                            const T* __restrict__ vals, int chunk, Dense d)
{
    const int G = 1 << d.lshift;
    const long long t = (long long)blockIdx.x * kSpmmBlock + threadIdx.x;
    const int lane = (int)(t & (G - 1));
    const int c0 = lane * VEC;
    if (c0 >= d.k) return;
    const long long g = t >> d.lshift;
    const long long e0l = g * chunk;
    if (e0l >= nnz) return;
    const int e0 = (int)e0l;
    const int e1 = (int)min((long long)nnz, e0l + chunk);
    int row, row_end = 0;
    if (IS_CSR) {   // last row whose start is <= e0 (skips empty rows)
        int lo = 0, hi = rows;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(row_ptr + mid) <= e0) lo = mid;
            else hi = mid - 1;
        }
        row = lo;
        row_end = __ldg(row_ptr + row + 1);
    } else {
        row = __ldg(row_id + e0);
    }
    bool first = true;   // the current row may have started before e0
    Acc<VEC> acc;
    // A row is cut by the chunk if it started before e0 (only the first row
    // can) or continues past e1 (only the last row can).
    auto flush = [&](bool last) {
        const float a = d.scale ? d.alpha * d.scale[row] : d.alpha;
        float* y = d.Y + (size_t)row * d.ldy + c0;
        bool cut = false;
        if (first) cut = IS_CSR ? __ldg(row_ptr + row) < e0 : (e0 > 0 && __ldg(row_id + e0 - 1) == row);
        if (last) cut = cut || (IS_CSR ? row_end > e1 : (e1 < nnz && __ldg(row_id + e1) == row));
        if (cut) acc.atomic(y, a);
        else acc.add(y, a);
    };
    // kChunkPrefetch nonzeros at a time: their column ids, values and X
    // slices are all requested before the first is used, so a lane keeps
    // that many gathers in flight
    constexpr int U = kChunkPrefetch;
    for (int e = e0; e < e1; e += U) {
        int cc[U], rr[U];
        float vv[U];
        typename Acc<VEC>::X xv[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const bool in = e + u < e1;
            cc[u] = in ? __ldg(col_id + e + u) : 0;
            vv[u] = in ? to_f(ld_val(vals + e + u)) : 0.f;
            rr[u] = (!IS_CSR && in) ? __ldg(row_id + e + u) : 0;
        }
#pragma unroll
        for (int u = 0; u < U; u++) xv[u] = e + u < e1 ? Acc<VEC>::load(d.X + (size_t)cc[u] * d.ldx + c0) : Acc<VEC>::zero();
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int ee = e + u;
            if (ee >= e1) break;
            if (IS_CSR) {
                if (ee >= row_end) {
                    flush(false);
                    first = false;
                    acc = Acc<VEC>();
                    do {
                        row++;
                        row_end = __ldg(row_ptr + row + 1);
                    } while (ee >= row_end);
                }
            } else if (rr[u] != row) {
                flush(false);
                first = false;
                acc = Acc<VEC>();
                row = rr[u];
            }
            acc.fma_v(vv[u], xv[u]);
        }
    }
    flush(true);
}

// ---------------------------------------------------------------------------
// Warp-segmented CSR / COO product for k a multiple of 4 (used at k = 4)
// with 16-byte rows of X and Y: the mapping of the single-vector COO kernel (a warp per 256
// consecutive nonzeros, 4 per lane, all of a step's X gathers issued at
// once) applied to each group of 4 columns in turn, with float4 partial sums
// reduced by the same per-lane runs + warp segmented scan and added to Y with
// vector red.global.add. The nonzero-chunk kernel above walks a chunk's
// nonzeros one after another per lane group; this one keeps 8 gathers of 16
// bytes in flight per lane. CSR rows come from row_ptr: a warp-wide 32-way
// search finds the first and last row of the chunk, each lane then searches
// between them. Y must already hold beta * Y.
// ---------------------------------------------------------------------------
constexpr unsigned kWarpAll = 0xffffffffu;
constexpr int kSegNoRow = 0x7fffffff;
constexpr int kSegSteps = 2;
constexpr int kSegChunk = 128 * kSegSteps;

__device__ __forceinline__ float4 f4add(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 f4up(float4 v, int off)
{
    return make_float4(__shfl_up_sync(kWarpAll, v.x, off), __shfl_up_sync(kWarpAll, v.y, off),
                       __shfl_up_sync(kWarpAll, v.z, off), __shfl_up_sync(kWarpAll, v.w, off));
}
__device__ __forceinline__ float4 f4from(float4 v, int src)
{
    return make_float4(__shfl_sync(kWarpAll, v.x, src), __shfl_sync(kWarpAll, v.y, src), __shfl_sync(kWarpAll, v.z, src),
                       __shfl_sync(kWarpAll, v.w, src));
}

// Largest r in [0, rows) with row_ptr[r] <= q (q < nnz), by the whole warp:
// each round the 32 lanes probe 32 evenly spaced rows of the interval.
__device__ __forceinline__ int warp_row_of(const int* __restrict__ row_ptr, int rows, long long q, int lane)
{
    int lo = 0, hi = rows - 1;   // invariant: row_ptr[lo] <= q
    while (hi - lo >= 32) {
        const long long span = (long long)hi - lo;
        const int p = lo + (int)(span * lane / 32);
        const unsigned m = __ballot_sync(kWarpAll, __ldg(row_ptr + p) <= q);
        const int j = 31 - __clz(m);
        const int nlo = __shfl_sync(kWarpAll, p, j);
        const int next = __shfl_sync(kWarpAll, p, j < 31 ? j + 1 : 31);
        hi = j < 31 ? next - 1 : hi;
        lo = nlo;
    }
    const int p = lo + lane;
    const unsigned m = __ballot_sync(kWarpAll, p <= hi && __ldg(row_ptr + min(p, hi)) <= q);
    return lo + (31 - __clz(m));
}

__device__ __forceinline__ void seg_red(const Dense& d, int row, int c0, float4 v)
{
    if (row == kSegNoRow) return;
    const float a = d.scale ? d.alpha * d.scale[row] : d.alpha;
    atomicAdd(reinterpret_cast<float4*>(d.Y + (size_t)row * d.ldy + c0), make_float4(a * v.x, a * v.y, a * v.z, a * v.w));
}

// The segmented reduction of the COO kernel (per-lane runs, lane-boundary
// partials by a warp scan, the trailing row carried across steps) on float4
// sums of 4 columns.
__device__ __forceinline__ void seg_reduce4(const Dense& d, int c0, const int (&r)[kSegSteps][4],
                                            const float4 (&p)[kSegSteps][4], int lane)
{
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 carry = zero;
    int carry_row = -1;
#pragma unroll
    for (int s = 0; s < kSegSteps; s++) {
        const int head_row = r[s][0], tail_row = r[s][3];
        const bool single = head_row == tail_row;
        float4 head = zero, tail = zero;
        if (single) {
            tail = f4add(f4add(p[s][0], p[s][1]), f4add(p[s][2], p[s][3]));
        } else {
            head = p[s][0];
            tail = p[s][3];
            int run_row = -1;
            float4 run = zero;
#pragma unroll
            for (int j = 1; j < 3; j++) {
                const int rj = r[s][j];
                if (rj == head_row) {
                    head = f4add(head, p[s][j]);
                } else if (rj == tail_row) {
                    tail = f4add(tail, p[s][j]);
                } else if (rj == run_row) {
                    run = f4add(run, p[s][j]);
                } else {
                    if (run_row >= 0) seg_red(d, run_row, c0, run);
                    run_row = rj;
                    run = p[s][j];
                }
            }
            if (run_row >= 0) seg_red(d, run_row, c0, run);
        }
        const int lead = __shfl_sync(kWarpAll, head_row, 0);
        if (carry_row >= 0 && lead != carry_row) {
            if (lane == 0) seg_red(d, carry_row, c0, carry);
            carry_row = -1;
            carry = zero;
        }
        if (lane == 0 && carry_row >= 0) {
            if (single) tail = f4add(tail, carry);
            else head = f4add(head, carry);
        }
        const int prev_tail_row = __shfl_up_sync(kWarpAll, tail_row, 1);
        const bool start = lane == 0 || !single || prev_tail_row != tail_row;
        const unsigned smask = __ballot_sync(kWarpAll, start);
        const int seg0 = 31 - __clz(smask & (0xffffffffu >> (31 - lane)));
        float4 v = tail;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const float4 t = f4up(v, off);
            if (lane - off >= seg0) v = f4add(v, t);
        }
        const float4 prev_v = f4up(v, 1);
        if (!single) seg_red(d, head_row, c0, (lane > 0 && prev_tail_row == head_row) ? f4add(head, prev_v) : head);
        const int next_head = __shfl_down_sync(kWarpAll, head_row, 1);
        if (lane < 31 && next_head != tail_row) seg_red(d, tail_row, c0, v);
        carry = f4from(v, 31);
        carry_row = __shfl_sync(kWarpAll, tail_row, 31);
        if (carry_row == kSegNoRow) carry_row = -1;
    }
    if (carry_row >= 0 && lane == 0) seg_red(d, carry_row, c0, carry);
}

template <class T, bool IS_CSR>
__device__ __forceinline__ void seg_chunk(int rows, int nnz, const int* __restrict__ row_ptr, const int* __restrict__ row_id,
                                          const int* __restrict__ col_id, const T* __restrict__ vals, const Dense& d,
                                          long long ch, int lane)
{
    const long long base = ch * kSegChunk;
    int r[kSegSteps][4], c[kSegSteps][4];
    float v[kSegSteps][4];
#pragma unroll
    for (int s = 0; s < kSegSteps; s++) {
        const long long idx = base + s * 128 + lane * 4;
        if (idx + 3 < nnz) {
            const int4 cv = __ldg(reinterpret_cast<const int4*>(col_id + idx));
            c[s][0] = cv.x; c[s][1] = cv.y; c[s][2] = cv.z; c[s][3] = cv.w;
            if constexpr (std::is_same<T, float>::value) {
                const float4 vv = __ldg(reinterpret_cast<const float4*>(vals + idx));
                v[s][0] = vv.x; v[s][1] = vv.y; v[s][2] = vv.z; v[s][3] = vv.w;
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++) v[s][j] = to_f(ld_val(vals + idx + j));
            }
            if (!IS_CSR) {
                const int4 rv = __ldg(reinterpret_cast<const int4*>(row_id + idx));
                r[s][0] = rv.x; r[s][1] = rv.y; r[s][2] = rv.z; r[s][3] = rv.w;
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const bool in = idx + j < nnz;
                c[s][j] = in ? __ldg(col_id + idx + j) : 0;
                v[s][j] = in ? to_f(ld_val(vals + idx + j)) : 0.f;
                if (!IS_CSR) r[s][j] = in ? __ldg(row_id + idx + j) : kSegNoRow;
            }
        }
    }
    if (IS_CSR) {
        const int ra = warp_row_of(row_ptr, rows, base, lane);
        const int rb = warp_row_of(row_ptr, rows, min(base + kSegChunk - 1, (long long)nnz - 1), lane);
#pragma unroll
        for (int s = 0; s < kSegSteps; s++) {
            const long long q0 = base + s * 128 + lane * 4;
            if (q0 >= nnz) {
#pragma unroll
                for (int j = 0; j < 4; j++) r[s][j] = kSegNoRow;
                continue;
            }
            int lo = ra, hi = rb;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(row_ptr + mid) <= q0) lo = mid;
                else hi = mid - 1;
            }
            int row = lo;
            r[s][0] = row;
#pragma unroll
            for (int j = 1; j < 4; j++) {
                const long long q = q0 + j;
                if (q < nnz) {
                    while (__ldg(row_ptr + row + 1) <= q) row++;
                    r[s][j] = row;
                } else {
                    r[s][j] = kSegNoRow;
                }
            }
        }
    }
    for (int c0 = 0; c0 < d.k; c0 += 4) {
        float4 p[kSegSteps][4];
#pragma unroll
        for (int s = 0; s < kSegSteps; s++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (r[s][j] != kSegNoRow) {
                    const float4 xv = __ldg(reinterpret_cast<const float4*>(d.X + (size_t)c[s][j] * d.ldx + c0));
                    p[s][j] = make_float4(v[s][j] * xv.x, v[s][j] * xv.y, v[s][j] * xv.z, v[s][j] * xv.w);
                } else {
                    p[s][j] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
        seg_reduce4(d, c0, r, p, lane);
    }
}

template <class T, bool IS_CSR>
__global__ void __launch_bounds__(kSpmmBlock) k_spmm_seg(int rows, int nnz, const int* __restrict__ row_ptr,
                                                         const int* __restrict__ row_id, const int* __restrict__ col_id,
                                                         const T* __restrict__ vals, Dense d)
{
    const int lane = threadIdx.x & 31;
    const long long nchunks = ((long long)nnz + kSegChunk - 1) / kSegChunk;
    const long long nwarps = (long long)gridDim.x * (kSpmmBlock / 32);
    for (long long ch = (long long)blockIdx.x * (kSpmmBlock / 32) + (threadIdx.x >> 5); ch < nchunks; ch += nwarps)
        seg_chunk<T, IS_CSR>(rows, nnz, row_ptr, row_id, col_id, vals, d, ch, lane);
}

// ---------------------------------------------------------------------------
// Long CSR rows at k a multiple of 4: a warp per row. The warp's lanes form
// 32 / G nonzero slots of G = k / 4 lanes (4 columns each); a step covers
// 32 / G consecutive nonzeros of the row with coalesced col_id / value loads
// and one float4 X load per lane, and the slots' partial sums are combined
// once per row by shuffles. The row is owned by its warp, so Y is written
// directly (alpha, beta applied there). Used when rows average
// kWarpRowMin nonzeros or more: the nonzero-chunk kernel walks a long row's
// nonzeros one after another per lane group.
// ---------------------------------------------------------------------------
constexpr int kWarpRowMin = 128;

template <class T>
__global__ void __launch_bounds__(kSpmmBlock) k_spmm_warp_rows(int rows, const int* __restrict__ row_ptr,
                                                               const int* __restrict__ col_id, const T* __restrict__ vals,
                                                               Dense d)
{
    const int lane = threadIdx.x & 31;
    const int G = d.k >> 2;                     // lanes per nonzero slot, 1..32 (k <= 128)
    const int lg = 31 - __clz(G);               // G is a power of two (checked by the launcher)
    const int slots = 32 >> lg;
    const int slot = lane >> lg, c0 = (lane & (G - 1)) * 4;
    const long long nwarps = (long long)gridDim.x * (kSpmmBlock / 32);
    for (long long r = (long long)blockIdx.x * (kSpmmBlock / 32) + (threadIdx.x >> 5); r < rows; r += nwarps) {
        const int j0 = __ldg(row_ptr + r), j1 = __ldg(row_ptr + r + 1);
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        int j = j0 + slot;
        // two nonzeros per slot in flight
        for (; j + slots < j1; j += 2 * slots) {
            const int ca = __ldg(col_id + j), cb = __ldg(col_id + j + slots);
            const float va = to_f(ld_val(vals + j)), vb = to_f(ld_val(vals + j + slots));
            const float4 xa = __ldg(reinterpret_cast<const float4*>(d.X + (size_t)ca * d.ldx + c0));
            const float4 xb = __ldg(reinterpret_cast<const float4*>(d.X + (size_t)cb * d.ldx + c0));
            acc.x = fmaf(va, xa.x, acc.x); acc.y = fmaf(va, xa.y, acc.y);
            acc.z = fmaf(va, xa.z, acc.z); acc.w = fmaf(va, xa.w, acc.w);
            acc.x = fmaf(vb, xb.x, acc.x); acc.y = fmaf(vb, xb.y, acc.y);
            acc.z = fmaf(vb, xb.z, acc.z); acc.w = fmaf(vb, xb.w, acc.w);
        }
        if (j < j1) {
            const int ca = __ldg(col_id + j);
            const float va = to_f(ld_val(vals + j));
            const float4 xa = __ldg(reinterpret_cast<const float4*>(d.X + (size_t)ca * d.ldx + c0));
            acc.x = fmaf(va, xa.x, acc.x); acc.y = fmaf(va, xa.y, acc.y);
            acc.z = fmaf(va, xa.z, acc.z); acc.w = fmaf(va, xa.w, acc.w);
        }
        for (int off = 16; off >= G; off >>= 1) {
            acc.x += __shfl_xor_sync(kWarpAll, acc.x, off);
            acc.y += __shfl_xor_sync(kWarpAll, acc.y, off);
            acc.z += __shfl_xor_sync(kWarpAll, acc.z, off);
            acc.w += __shfl_xor_sync(kWarpAll, acc.w, off);
        }
        if (slot == 0) {
            const float a = d.scale ? d.alpha * d.scale[r] : d.alpha;
            float4* y = reinterpret_cast<float4*>(d.Y + (size_t)r * d.ldy + c0);
            float4 o = make_float4(a * acc.x, a * acc.y, a * acc.z, a * acc.w);
            if (d.beta != 0.0f) {
                const float4 p = *y;
                o.x = fmaf(d.beta, p.x, o.x); o.y = fmaf(d.beta, p.y, o.y);
                o.z = fmaf(d.beta, p.z, o.z); o.w = fmaf(d.beta, p.w, o.w);
            }
            *y = o;
        }
    }
}

__global__ void k_scale_rows(float* Y, int rows, int k, int ldy, float beta)
{
    const long long n = (long long)rows * k;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / k, c = i - r * k;
        float* p = Y + r * ldy + c;
        *p = beta == 0.0f ? 0.0f : beta * *p;
    }
}

// Packing: per-row scale (pass 1), then the scaled 16-bit values (pass 2).
__device__ __forceinline__ float pow2_at_least(float s)
{
    if (!(s > 0.0f) || isinf(s)) return 1.0f;
    int e;
    const float f = frexpf(s, &e);   // s = f * 2^e, f in [0.5, 1)
    (void)f;
    return ldexpf(1.0f, e);
}

template <class T, class M>
__global__ void k_pack_rows(M m, const float* __restrict__ src, T* __restrict__ dst, float* __restrict__ scale)
{
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < m.matinfo.height;
         r += (long long)gridDim.x * blockDim.x) {
        float mx = 0.0f;
        for_row(m, (int)r, [&](int, size_t idx) { mx = fmaxf(mx, fabsf(src[idx])); });
        const float s = pow2_at_least(mx), inv = 1.0f / s;   // exact: s is a power of two
        scale[r] = s;
        for_row(m, (int)r, [&](int, size_t idx) { dst[idx] = from_f<T>(src[idx] * inv); });
    }
}

template <class T>
__global__ void k_pack_csr(int rows, const int* __restrict__ row_ptr, const float* __restrict__ src, T* __restrict__ dst,
                           float* __restrict__ scale)
{
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (long long)gridDim.x * blockDim.x) {
        const int a = row_ptr[r], b = row_ptr[r + 1];
        float mx = 0.0f;
        for (int j = a; j < b; j++) mx = fmaxf(mx, fabsf(src[j]));
        const float s = pow2_at_least(mx), inv = 1.0f / s;
        scale[r] = s;
        for (int j = a; j < b; j++) dst[j] = from_f<T>(src[j] * inv);
    }
}

// COO rows are runs of equal row ids: the thread at the start of a run packs it.
template <class T>
__global__ void k_pack_coo(int nnz, const int* __restrict__ row_id, const float* __restrict__ src, T* __restrict__ dst,
                           float* __restrict__ scale)
{
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (long long)gridDim.x * blockDim.x) {
        const int r = row_id[e];
        if (e > 0 && row_id[e - 1] == r) continue;
        long long f = e;
        float mx = 0.0f;
        for (; f < nnz && row_id[f] == r; f++) mx = fmaxf(mx, fabsf(src[f]));
        const float s = pow2_at_least(mx), inv = 1.0f / s;
        scale[r] = s;
        for (long long j = e; j < f; j++) dst[j] = from_f<T>(src[j] * inv);
    }
}

__global__ void k_fill(float* p, int n, float v)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) p[i] = v;
}

int grid_of(long long threads, int block = kSpmmBlock)
{
    long long g = (threads + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 148LL * 64) g = 148LL * 64;
    return (int)g;
}

int log2_ceil(int v)
{
    int s = 0;
    while ((1 << s) < v) s++;
    return s;
}

// Lanes per row group and the vector width for k, X and Y.
int plan_lanes(int k, const float* X, int ldx, const float* Y, int ldy, int* vec, int* lshift)
{
    if (k < 1 || k > kSpmmMaxK || ldx < k || ldy < k) return CLSPMV_ERR_ARG;
    const bool v4 = k % 4 == 0 && ldx % 4 == 0 && ldy % 4 == 0 && ((uintptr_t)X & 15) == 0 && ((uintptr_t)Y & 15) == 0;
    if (!v4 && k > 32) return CLSPMV_ERR_ALIGN;   // more than 32 lanes per row otherwise
    *vec = v4 ? 4 : 1;
    *lshift = log2_ceil(v4 ? k / 4 : k);
    return CLSPMV_OK;
}

template <class M> const float* values_of(const M& m);
template <> const float* values_of(const clspmv_dia_f32& m) { return m.dia_data; }
template <> const float* values_of(const clspmv_bdia_f32& m) { return m.bdia_data; }
template <> const float* values_of(const clspmv_ell_f32& m) { return m.ell_data; }
template <> const float* values_of(const clspmv_sell_f32& m) { return m.sell_data; }
template <> const float* values_of(const clspmv_b4csr_f32& m) { return m.b4csr_data; }
template <> const float* values_of(const clspmv_b4ell_f32& m) { return m.b4ell_data; }
template <> const float* values_of(const clspmv_sbell_f32& m) { return m.sbell_data; }

template <class T, class M>
int launch_rows(const M& m, const void* vals, Dense d, int vec, cudaStream_t st)
{
    const long long threads = (long long)m.matinfo.height << d.lshift;
    const int grid = grid_of(threads);
    const T* v = static_cast<const T*>(vals);
    if (vec == 4) k_spmm_rows<4, T, M><<<grid, kSpmmBlock, 0, st>>>(m, v, d);
    else k_spmm_rows<1, T, M><<<grid, kSpmmBlock, 0, st>>>(m, v, d);
    return after_launch(1);
}

// CLSPMV_SPMM_BLOCK_ROWS=0 keeps the row walk for the block formats (measurements).
bool block_rows_enabled()
{
    static const bool on = [] {
        const char* e = getenv("CLSPMV_SPMM_BLOCK_ROWS");
        return !(e && atoi(e) == 0);
    }();
    return on;
}

inline int bheight_of(const clspmv_b4csr_f32& m) { return (int)m.b4csr_bheight; }
inline int bheight_of(const clspmv_b4ell_f32& m) { return (int)m.b4ell_bheight; }
inline int bheight_of(const clspmv_sbell_f32& m) { return (int)m.sbell_bheight; }
inline int bwidth_of(const clspmv_b4csr_f32& m) { return (int)m.b4csr_bwidth; }
inline int bwidth_of(const clspmv_b4ell_f32& m) { return (int)m.b4ell_bwidth; }
inline int bwidth_of(const clspmv_sbell_f32& m) { return (int)m.sbell_bwidth; }
// strides of for_block in values, which 4-value loads need to be multiples of 4
inline bool strips_aligned(const clspmv_b4csr_f32& m) { return m.b4csr_aligned_size % 4 == 0; }
inline bool strips_aligned(const clspmv_b4ell_f32& m) { return m.b4ell_float4_aligned % 4 == 0; }
inline bool strips_aligned(const clspmv_sbell_f32&) { return true; }

// CLSPMV_SPMM_X_FORM: how the block-row kernel reads X rows (Dense::x_form; measurements)
int x_form()
{
    static const int f = [] {
        const char* e = getenv("CLSPMV_SPMM_X_FORM");
        return e ? atoi(e) : 0;
    }();
    return f;
}

template <int BH, int BW4, class T, class M>
void launch_block_kernel(const M& m, const T* v, Dense d, cudaStream_t st)
{
    d.x_form = x_form();
    const long long nbr = ((long long)m.matinfo.height + BH - 1) / BH;
    k_spmm_blocks<BH, BW4, T, M><<<grid_of(nbr << d.lshift), kSpmmBlock, 0, st>>>(m, v, d);
}

// Block formats with 128-bit X rows: the block-row kernel; otherwise (X rows
// of single columns, or strips off a 4-value boundary) the row walk.
template <class T, class M>
int launch_blocks(const M& m, const void* vals, Dense d, int vec, cudaStream_t st)
{
    const T* v = static_cast<const T*>(vals);
    const int bh = bheight_of(m), bw4 = bwidth_of(m) / 4;
    if (vec != 4 || !block_rows_enabled() || !strips_aligned(m) || ((uintptr_t)v % (4 * sizeof(T))) != 0 ||
        (bw4 != 1 && bw4 != 2))
        return launch_rows<T>(m, vals, d, vec, st);
    if (m.matinfo.height <= 0) return CLSPMV_OK;
#define BLK(BH)                                                        \
    case BH:                                                           \
        if (bw4 == 1) launch_block_kernel<BH, 1, T>(m, v, d, st);      \
        else launch_block_kernel<BH, 2, T>(m, v, d, st);               \
        break;
    switch (bh) {
        BLK(1)
        BLK(2)
        BLK(4)
        BLK(8)
        default: return launch_rows<T>(m, vals, d, vec, st);
    }
#undef BLK
    return after_launch(1);
}

// CLSPMV_SPMM_WARP_ROWS=0 keeps the nonzero-chunk kernel for long CSR rows (measurements).
bool warp_rows_enabled()
{
    static const bool on = [] {
        const char* e = getenv("CLSPMV_SPMM_WARP_ROWS");
        return !(e && atoi(e) == 0);
    }();
    return on;
}

// CLSPMV_SPMM_SEG=0 keeps the nonzero-chunk kernel for CSR / COO (measurements).
bool seg_enabled()
{
    static const bool on = [] {
        const char* e = getenv("CLSPMV_SPMM_SEG");
        return !(e && atoi(e) == 0);
    }();
    return on;
}

template <class T, bool IS_CSR>
int launch_chunks(int rows, int nnz, const int* row_ptr, const int* row_id, const int* col_id, const void* vals, Dense d,
                  int vec, cudaStream_t st)
{
    if (d.beta != 1.0f) {
        k_scale_rows<<<grid_of((long long)rows * d.k), kSpmmBlock, 0, st>>>(d.Y, rows, d.k, d.ldy, d.beta);
        int rc = after_launch(1);
        if (rc) return rc;
    }
    if (nnz <= 0) return CLSPMV_OK;
    // k = 4: the warp-segmented kernel (measured on the power-law matrix: CSR 0.19 against 0.26 ms, COO 0.12
    // against 0.68 ms); from k = 8 on the per-column scans cost more than the lane-per-column walk saves
    if (vec == 4 && d.k == 4 && seg_enabled() && ((uintptr_t)col_id & 15) == 0 && (IS_CSR || ((uintptr_t)row_id & 15) == 0) &&
        (!std::is_same<T, float>::value || ((uintptr_t)vals & 15) == 0)) {
        const long long nchunks = ((long long)nnz + kSegChunk - 1) / kSegChunk;
        const int grid = (int)std::min<long long>((nchunks + kSpmmBlock / 32 - 1) / (kSpmmBlock / 32), 148LL * 8);
        k_spmm_seg<T, IS_CSR><<<grid, kSpmmBlock, 0, st>>>(rows, nnz, row_ptr, row_id, col_id,
                                                          static_cast<const T*>(vals), d);
        return after_launch(1);
    }
    // about 16 row-sum updates of X per lane: enough work to hide the search
    const int chunk = d.k <= 4 ? 32 : 16;
    const long long groups = ((long long)nnz + chunk - 1) / chunk;
    const long long threads = groups << d.lshift;
    const int grid = (int)((threads + kSpmmBlock - 1) / kSpmmBlock);
    const T* v = static_cast<const T*>(vals);
    if (vec == 4) k_spmm_chunks<4, T, IS_CSR><<<grid, kSpmmBlock, 0, st>>>(rows, nnz, row_ptr, row_id, col_id, v, chunk, d);
    else k_spmm_chunks<1, T, IS_CSR><<<grid, kSpmmBlock, 0, st>>>(rows, nnz, row_ptr, row_id, col_id, v, chunk, d);
    return after_launch(1);
}

template <class T>
int spmm_typed(int format, const void* dev, const void* vals, Dense d, int vec, cudaStream_t st)
{
    switch (format) {
        case CLSPMV_FORMAT_CSR: {
            const auto& m = *static_cast<const clspmv_csr_f32*>(dev);
            if (!m.csr_row_ptr) return CLSPMV_ERR_ARG;
            const int G = d.k / 4;
            if (vec == 4 && (G & (G - 1)) == 0 && m.matinfo.height > 0 &&
                (long long)m.matinfo.nnz >= (long long)kWarpRowMin * m.matinfo.height && warp_rows_enabled()) {
                const long long warps = m.matinfo.height;
                const int grid = (int)std::min<long long>((warps + kSpmmBlock / 32 - 1) / (kSpmmBlock / 32), 148LL * 16);
                k_spmm_warp_rows<T><<<grid, kSpmmBlock, 0, st>>>(m.matinfo.height, m.csr_row_ptr, m.csr_col_id,
                                                                 static_cast<const T*>(vals ? vals : m.csr_data), d);
                return after_launch(1);
            }
            return launch_chunks<T, true>(m.matinfo.height, m.matinfo.nnz, m.csr_row_ptr, nullptr, m.csr_col_id,
                                          vals ? vals : m.csr_data, d, vec, st);
        }
        case CLSPMV_FORMAT_COO: {
            const auto& m = *static_cast<const clspmv_coo_f32*>(dev);
            return launch_chunks<T, false>(m.matinfo.height, m.matinfo.nnz, nullptr, m.coo_row_id, m.coo_col_id,
                                           vals ? vals : m.coo_data, d, vec, st);
        }
#define ROWS(FMT, TYPE)                                                              \
    case FMT: {                                                                      \
        const auto& m = *static_cast<const TYPE*>(dev);                              \
        return launch_rows<T>(m, vals ? vals : values_of(m), d, vec, st);            \
    }
        ROWS(CLSPMV_FORMAT_DIA, clspmv_dia_f32)
        ROWS(CLSPMV_FORMAT_BDIA, clspmv_bdia_f32)
        ROWS(CLSPMV_FORMAT_ELL, clspmv_ell_f32)
        ROWS(CLSPMV_FORMAT_SELL, clspmv_sell_f32)
#undef ROWS
#define BLOCKS(FMT, TYPE)                                                            \
    case FMT: {                                                                      \
        const auto& m = *static_cast<const TYPE*>(dev);                              \
        return launch_blocks<T>(m, vals ? vals : values_of(m), d, vec, st);          \
    }
        BLOCKS(CLSPMV_FORMAT_B4CSR, clspmv_b4csr_f32)
        BLOCKS(CLSPMV_FORMAT_B4ELL, clspmv_b4ell_f32)
        BLOCKS(CLSPMV_FORMAT_SBELL, clspmv_sbell_f32)
#undef BLOCKS
    }
    return CLSPMV_ERR_ARG;
}

int read_int(const int* dev_ptr, int* out)
{
    return cuda_status(cudaMemcpy(out, dev_ptr, sizeof(int), cudaMemcpyDeviceToHost));
}

bool block_ok(unsigned bw, unsigned bh) { return (bw == 4 || bw == 8) && (bh == 1 || bh == 2 || bh == 4 || bh == 8); }

template <class T>
int pack_typed(int format, const void* dev, T* dst, float* scale, cudaStream_t st)
{
    switch (format) {
        case CLSPMV_FORMAT_CSR: {
            const auto& m = *static_cast<const clspmv_csr_f32*>(dev);
            k_pack_csr<T><<<grid_of(m.matinfo.height), kSpmmBlock, 0, st>>>(m.matinfo.height, m.csr_row_ptr, m.csr_data,
                                                                           dst, scale);
            return after_launch(1);
        }
        case CLSPMV_FORMAT_COO: {
            const auto& m = *static_cast<const clspmv_coo_f32*>(dev);
            k_fill<<<grid_of(m.matinfo.height), kSpmmBlock, 0, st>>>(scale, m.matinfo.height, 1.0f);
            int rc = after_launch(1);
            if (rc || m.matinfo.nnz <= 0) return rc;
            k_pack_coo<T><<<grid_of(m.matinfo.nnz), kSpmmBlock, 0, st>>>(m.matinfo.nnz, m.coo_row_id, m.coo_data, dst, scale);
            return after_launch(1);
        }
#define PACK(FMT, TYPE)                                                                       \
    case FMT: {                                                                               \
        const auto& m = *static_cast<const TYPE*>(dev);                                       \
        k_pack_rows<T, TYPE><<<grid_of(m.matinfo.height), kSpmmBlock, 0, st>>>(m, values_of(m), dst, scale); \
        return after_launch(1);                                                               \
    }
        PACK(CLSPMV_FORMAT_DIA, clspmv_dia_f32)
        PACK(CLSPMV_FORMAT_BDIA, clspmv_bdia_f32)
        PACK(CLSPMV_FORMAT_ELL, clspmv_ell_f32)
        PACK(CLSPMV_FORMAT_SELL, clspmv_sell_f32)
        PACK(CLSPMV_FORMAT_B4CSR, clspmv_b4csr_f32)
        PACK(CLSPMV_FORMAT_B4ELL, clspmv_b4ell_f32)
        PACK(CLSPMV_FORMAT_SBELL, clspmv_sbell_f32)
#undef PACK
    }
    return CLSPMV_ERR_ARG;
}

int check_struct(int format, const void* dev)
{
    if (!dev) return CLSPMV_ERR_ARG;
    switch (format) {
        case CLSPMV_FORMAT_B4CSR: {
            const auto& m = *static_cast<const clspmv_b4csr_f32*>(dev);
            return block_ok(m.b4csr_bwidth, m.b4csr_bheight) ? CLSPMV_OK : CLSPMV_ERR_UNSUPPORTED;
        }
        case CLSPMV_FORMAT_B4ELL: {
            const auto& m = *static_cast<const clspmv_b4ell_f32*>(dev);
            return block_ok(m.b4ell_bwidth, m.b4ell_bheight) ? CLSPMV_OK : CLSPMV_ERR_UNSUPPORTED;
        }
        case CLSPMV_FORMAT_SBELL: {
            const auto& m = *static_cast<const clspmv_sbell_f32*>(dev);
            return block_ok(m.sbell_bwidth, m.sbell_bheight) && m.sbell_slice_height > 0 ? CLSPMV_OK : CLSPMV_ERR_UNSUPPORTED;
        }
        case CLSPMV_FORMAT_SELL:
            return static_cast<const clspmv_sell_f32*>(dev)->sell_slice_height > 0 ? CLSPMV_OK : CLSPMV_ERR_UNSUPPORTED;
        case CLSPMV_FORMAT_CSR:
        case CLSPMV_FORMAT_COO:
        case CLSPMV_FORMAT_DIA:
        case CLSPMV_FORMAT_BDIA:
        case CLSPMV_FORMAT_ELL:
            return CLSPMV_OK;
    }
    return CLSPMV_ERR_ARG;
}

// every format struct starts with its matinfo
int matrix_rows(const void* dev) { return static_cast<const clspmv_matinfo*>(dev)->height; }


// ---------------------------------------------------------------------------
// Batches: many (matrix, X, Y) jobs in one persistent launch. Each job is cut
// into warp tasks of 32 / G rows (G lanes per row for its k) -- or, for a CSR
// job that adds into Y (beta 1), of 32 / G equal chunks of nonzeros, so that
// rows of thousands of entries are shared between groups; the tasks of all
// jobs form one index space that every warp strides through, finding its job
// by binary search over the jobs' first task numbers.
// ---------------------------------------------------------------------------
constexpr int kBatchLongRow = 256;

struct BatchJob {
    int format, value_type, k, lshift, vec, rows;
    int bh;                    // 4: a 4x4-block job, one lane group per block row (block_row); 0: rows
    int chunk, nnz;            // CSR accumulating into Y (beta 1): nonzeros per lane group, else 0 (row mode)
    long long task_begin;
    int ldx, ldy;
    float alpha, beta;
    const void* values;
    const float* scale;
    const float* X;
    float* Y;
    union {
        clspmv_csr_f32 csr;
        clspmv_dia_f32 dia;
        clspmv_bdia_f32 bdia;
        clspmv_ell_f32 ell;
        clspmv_sell_f32 sell;
        clspmv_b4csr_f32 b4csr;
        clspmv_b4ell_f32 b4ell;
        clspmv_sbell_f32 sbell;
    } m;
};

template <int VEC, class T, class M>
__device__ __forceinline__ void batch_row(const M& m, const BatchJob& J, int r, int c0)
{
    const T* vals = static_cast<const T*>(J.values);
    Acc<VEC> acc;
    for_row(m, r, [&](int col, size_t idx) { acc.fma(to_f(ld_val(vals + idx)), J.X + (size_t)col * J.ldx + c0); });
    const float a = J.scale ? J.alpha * J.scale[r] : J.alpha;
    acc.store(J.Y + (size_t)r * J.ldy + c0, a, J.beta);
}

template <int VEC, class T>
__device__ __forceinline__ void batch_dispatch(const BatchJob& J, int r, int c0)
{
    switch (J.format) {
        case CLSPMV_FORMAT_CSR: batch_row<VEC, T>(J.m.csr, J, r, c0); break;
        case CLSPMV_FORMAT_DIA: batch_row<VEC, T>(J.m.dia, J, r, c0); break;
        case CLSPMV_FORMAT_BDIA: batch_row<VEC, T>(J.m.bdia, J, r, c0); break;
        case CLSPMV_FORMAT_ELL: batch_row<VEC, T>(J.m.ell, J, r, c0); break;
        case CLSPMV_FORMAT_SELL: batch_row<VEC, T>(J.m.sell, J, r, c0); break;
        case CLSPMV_FORMAT_B4CSR: batch_row<VEC, T>(J.m.b4csr, J, r, c0); break;
        case CLSPMV_FORMAT_B4ELL: batch_row<VEC, T>(J.m.b4ell, J, r, c0); break;
        case CLSPMV_FORMAT_SBELL: batch_row<VEC, T>(J.m.sbell, J, r, c0); break;
    }
}

template <class T>
__device__ __forceinline__ void batch_blocks(const BatchJob& J, int br, int c0)
{
    const T* v = static_cast<const T*>(J.values);
    switch (J.format) {
        case CLSPMV_FORMAT_B4CSR: block_row<4, 1>(J.m.b4csr, v, br, c0, J.X, J.ldx, J.Y, J.ldy, J.alpha, J.beta, J.scale, 0); break;
        case CLSPMV_FORMAT_B4ELL: block_row<4, 1>(J.m.b4ell, v, br, c0, J.X, J.ldx, J.Y, J.ldy, J.alpha, J.beta, J.scale, 0); break;
        case CLSPMV_FORMAT_SBELL: block_row<4, 1>(J.m.sbell, v, br, c0, J.X, J.ldx, J.Y, J.ldy, J.alpha, J.beta, J.scale, 0); break;
    }
}

// CSR job accumulating into Y: the group owns nonzeros [e0, e0 + chunk); rows
// cut by the chunk's edges are added atomically, the others with a plain add
// (as k_spmm_chunks, with Y already holding beta * Y = Y).
template <int VEC, class T>
__device__ __forceinline__ void batch_chunk(const BatchJob& J, int e0, int c0)
{
    const clspmv_csr_f32& m = J.m.csr;
    const T* vals = static_cast<const T*>(J.values);
    const int e1 = min(J.nnz, e0 + J.chunk);
    int lo = 0, hi = J.rows;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(m.csr_row_ptr + mid) <= e0) lo = mid;
        else hi = mid - 1;
    }
    int row = lo, row_end = __ldg(m.csr_row_ptr + row + 1);
    bool first = true;
    Acc<VEC> acc;
    auto flush = [&](bool last) {
        const float a = J.scale ? J.alpha * J.scale[row] : J.alpha;
        float* y = J.Y + (size_t)row * J.ldy + c0;
        bool cut = first && __ldg(m.csr_row_ptr + row) < e0;
        if (last) cut = cut || row_end > e1;
        if (cut) acc.atomic(y, a);
        else acc.add(y, a);
    };
    for (int e = e0; e < e1; e++) {
        if (e >= row_end) {
            flush(false);
            first = false;
            acc = Acc<VEC>();
            do {
                row++;
                row_end = __ldg(m.csr_row_ptr + row + 1);
            } while (e >= row_end);
        }
        acc.fma(to_f(ld_val(vals + e)), J.X + (size_t)__ldg(m.csr_col_id + e) * J.ldx + c0);
    }
    flush(true);
}

__global__ void __launch_bounds__(kSpmmBlock) k_batch(const BatchJob* __restrict__ jobs, int njobs, long long tasks)
{
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * kSpmmBlock) >> 5;
    for (long long t = ((long long)blockIdx.x * kSpmmBlock + threadIdx.x) >> 5; t < tasks; t += nwarps) {
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].task_begin <= t) lo = mid;
            else hi = mid - 1;
        }
        const BatchJob& J = jobs[lo];
        const long long r = (t - J.task_begin) * (32 >> J.lshift) + (lane >> J.lshift);
        const int c0 = (lane & ((1 << J.lshift) - 1)) * J.vec;
        if (J.chunk > 0) {   // r counts chunks of nonzeros here
            const long long e0 = r * J.chunk;
            if (e0 >= J.nnz || c0 >= J.k) continue;
            if (J.vec == 4) {
                if (J.value_type == CLSPMV_VALUES_F32) batch_chunk<4, float>(J, (int)e0, c0);
                else if (J.value_type == CLSPMV_VALUES_BF16) batch_chunk<4, __nv_bfloat16>(J, (int)e0, c0);
                else batch_chunk<4, __half>(J, (int)e0, c0);
            } else {
                if (J.value_type == CLSPMV_VALUES_F32) batch_chunk<1, float>(J, (int)e0, c0);
                else if (J.value_type == CLSPMV_VALUES_BF16) batch_chunk<1, __nv_bfloat16>(J, (int)e0, c0);
                else batch_chunk<1, __half>(J, (int)e0, c0);
            }
            continue;
        }
        if (r >= J.rows || c0 >= J.k) continue;
        if (J.vec == 4) {
            if (J.value_type == CLSPMV_VALUES_F32) batch_dispatch<4, float>(J, (int)r, c0);
            else if (J.value_type == CLSPMV_VALUES_BF16) batch_dispatch<4, __nv_bfloat16>(J, (int)r, c0);
            else batch_dispatch<4, __half>(J, (int)r, c0);
        } else {
            if (J.value_type == CLSPMV_VALUES_F32) batch_dispatch<1, float>(J, (int)r, c0);
            else if (J.value_type == CLSPMV_VALUES_BF16) batch_dispatch<1, __nv_bfloat16>(J, (int)r, c0);
            else batch_dispatch<1, __half>(J, (int)r, c0);
        }
    }
}

// The 4x4-block jobs of a batch (bh = 4) in their own persistent launch: warp
// tasks of 32 / G block rows, one lane group per block row (block_row). Kept
// apart from k_batch, whose other jobs would otherwise run at this path's
// register count.
__global__ void __launch_bounds__(kSpmmBlock, 3) k_batch_blocks(const BatchJob* __restrict__ jobs, int njobs, long long tasks)
{
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * kSpmmBlock) >> 5;
    for (long long t = ((long long)blockIdx.x * kSpmmBlock + threadIdx.x) >> 5; t < tasks; t += nwarps) {
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].task_begin <= t) lo = mid;
            else hi = mid - 1;
        }
        const BatchJob& J = jobs[lo];
        const long long br = (t - J.task_begin) * (32 >> J.lshift) + (lane >> J.lshift);
        const int c0 = (lane & ((1 << J.lshift) - 1)) * 4;
        if (br >= (J.rows + 3) / 4 || c0 >= J.k) continue;
        if (J.value_type == CLSPMV_VALUES_F32) batch_blocks<float>(J, (int)br, c0);
        else if (J.value_type == CLSPMV_VALUES_BF16) batch_blocks<__nv_bfloat16>(J, (int)br, c0);
        else batch_blocks<__half>(J, (int)br, c0);
    }
}

int persistent_grid(const void* kernel, int* cache)
{
    if (!*cache) {
        int dev = 0, nsm = 148, per = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kSpmmBlock, 0) != cudaSuccess || per < 1) {
            cudaGetLastError();
            per = 1;
        }
        *cache = nsm * per;
    }
    return *cache;
}

int batch_blocks_grid()
{
    static int grid = 0;
    return persistent_grid((const void*)k_batch_blocks, &grid);
}

int batch_grid()
{
    static int grid = 0;
    return persistent_grid((const void*)k_batch, &grid);
}

// Fills one device job from a caller's job description.
int make_job(const clspmv_spmm_job& in, BatchJob& out)
{
    int rc = check_struct(in.format, in.dev);
    if (rc) return rc;
    if (in.format == CLSPMV_FORMAT_COO) return CLSPMV_ERR_UNSUPPORTED;   // no row starts to walk
    if (!in.X || !in.Y) return CLSPMV_ERR_ARG;
    if (in.value_type != CLSPMV_VALUES_F32 && in.value_type != CLSPMV_VALUES_BF16 && in.value_type != CLSPMV_VALUES_F16)
        return CLSPMV_ERR_ARG;
    if (in.value_type != CLSPMV_VALUES_F32 && (!in.values || !in.row_scale)) return CLSPMV_ERR_ARG;
    memset(&out, 0, sizeof(out));
    if ((rc = plan_lanes(in.k, in.X, in.ldx, in.Y, in.ldy, &out.vec, &out.lshift))) return rc;
    out.format = in.format;
    out.value_type = in.value_type;
    out.k = in.k;
    out.rows = matrix_rows(in.dev);
    out.ldx = in.ldx;
    out.ldy = in.ldy;
    out.alpha = in.alpha;
    out.beta = in.beta;
    out.scale = in.value_type == CLSPMV_VALUES_F32 ? nullptr : in.row_scale;
    out.X = in.X;
    out.Y = in.Y;
    switch (in.format) {
        case CLSPMV_FORMAT_CSR: out.m.csr = *static_cast<const clspmv_csr_f32*>(in.dev); out.values = out.m.csr.csr_data; break;
        case CLSPMV_FORMAT_DIA: out.m.dia = *static_cast<const clspmv_dia_f32*>(in.dev); out.values = out.m.dia.dia_data; break;
        case CLSPMV_FORMAT_BDIA: out.m.bdia = *static_cast<const clspmv_bdia_f32*>(in.dev); out.values = out.m.bdia.bdia_data; break;
        case CLSPMV_FORMAT_ELL: out.m.ell = *static_cast<const clspmv_ell_f32*>(in.dev); out.values = out.m.ell.ell_data; break;
        case CLSPMV_FORMAT_SELL: out.m.sell = *static_cast<const clspmv_sell_f32*>(in.dev); out.values = out.m.sell.sell_data; break;
        case CLSPMV_FORMAT_B4CSR: out.m.b4csr = *static_cast<const clspmv_b4csr_f32*>(in.dev); out.values = out.m.b4csr.b4csr_data; break;
        case CLSPMV_FORMAT_B4ELL: out.m.b4ell = *static_cast<const clspmv_b4ell_f32*>(in.dev); out.values = out.m.b4ell.b4ell_data; break;
        case CLSPMV_FORMAT_SBELL: out.m.sbell = *static_cast<const clspmv_sbell_f32*>(in.dev); out.values = out.m.sbell.sbell_data; break;
    }
    if (in.value_type != CLSPMV_VALUES_F32) out.values = in.values;
    if (out.format == CLSPMV_FORMAT_CSR && !out.m.csr.csr_row_ptr) return CLSPMV_ERR_ARG;
    // 4x4 blocks with 128-bit X rows: one lane group per block row, as clspmv_spmm does
    const size_t vsize = in.value_type == CLSPMV_VALUES_F32 ? 4 : 2;
    if (out.vec == 4 && block_rows_enabled() && ((uintptr_t)out.values % (4 * vsize)) == 0) {
        bool four = false;
        switch (out.format) {
            case CLSPMV_FORMAT_B4CSR: four = bheight_of(out.m.b4csr) == 4 && bwidth_of(out.m.b4csr) == 4 && strips_aligned(out.m.b4csr); break;
            case CLSPMV_FORMAT_B4ELL: four = bheight_of(out.m.b4ell) == 4 && bwidth_of(out.m.b4ell) == 4 && strips_aligned(out.m.b4ell); break;
            case CLSPMV_FORMAT_SBELL: four = bheight_of(out.m.sbell) == 4 && bwidth_of(out.m.sbell) == 4; break;
        }
        if (four) out.bh = 4;
    }
    // CSR adding into Y with long rows (mean >= kBatchLongRow entries): equal chunks of
    // nonzeros, so long rows are shared between groups (shorter rows: one group per row
    // is faster, measured on B200)
    if (out.format == CLSPMV_FORMAT_CSR && in.beta == 1.0f && out.m.csr.matinfo.nnz > 0 &&
        (long long)out.m.csr.matinfo.nnz >= (long long)kBatchLongRow * out.rows) {
        out.chunk = in.k <= 4 ? 64 : 32;
        out.nnz = out.m.csr.matinfo.nnz;
    }
    return CLSPMV_OK;
}

}  // namespace

struct clspmv_batch {
    int capacity = 0;
    int njobs = 0;
    int nrow_jobs = 0;            // jobs [0, nrow_jobs) run in k_batch, the rest (4x4 blocks) in k_batch_blocks
    long long tasks = 0;
    long long block_tasks = 0;
    BatchJob* host = nullptr;     // pinned staging of the job table
    BatchJob* dev = nullptr;
    cudaEvent_t copied = nullptr; // the last table upload has left `host`
};

namespace {
}  // namespace

extern "C" {

int clspmv_stored_values(int format, const void* dev, size_t* count)
{
    int rc = check_struct(format, dev);
    if (rc) return rc;
    if (!count) return CLSPMV_ERR_ARG;
    int last = 0;
    switch (format) {
        case CLSPMV_FORMAT_CSR: *count = (size_t)static_cast<const clspmv_csr_f32*>(dev)->matinfo.nnz; return CLSPMV_OK;
        case CLSPMV_FORMAT_COO: *count = (size_t)static_cast<const clspmv_coo_f32*>(dev)->matinfo.nnz; return CLSPMV_OK;
        case CLSPMV_FORMAT_DIA: {
            const auto& m = *static_cast<const clspmv_dia_f32*>(dev);
            *count = (size_t)m.dia_num * m.dia_length_aligned;
            return CLSPMV_OK;
        }
        case CLSPMV_FORMAT_BDIA: {
            const auto& m = *static_cast<const clspmv_bdia_f32*>(dev);
            if (m.bdia_band_num > 0 && (rc = read_int(m.bdia_bptr + m.bdia_band_num, &last))) return rc;
            *count = (size_t)last * m.bdia_length_aligned;
            return CLSPMV_OK;
        }
        case CLSPMV_FORMAT_ELL: {
            const auto& m = *static_cast<const clspmv_ell_f32*>(dev);
            *count = (size_t)m.ell_num * m.ell_height_aligned;
            return CLSPMV_OK;
        }
        case CLSPMV_FORMAT_SELL: {
            const auto& m = *static_cast<const clspmv_sell_f32*>(dev);
            if ((rc = read_int(m.sell_slice_ptr + m.sell_slice_num, &last))) return rc;
            *count = (size_t)last;
            return CLSPMV_OK;
        }
        case CLSPMV_FORMAT_B4CSR: {
            const auto& m = *static_cast<const clspmv_b4csr_f32*>(dev);
            *count = (size_t)m.b4csr_aligned_size * m.b4csr_bwidth * m.b4csr_bheight / 4;
            return CLSPMV_OK;
        }
        case CLSPMV_FORMAT_B4ELL: {
            const auto& m = *static_cast<const clspmv_b4ell_f32*>(dev);
            *count = (size_t)m.b4ell_block_num * m.b4ell_float4_aligned * (m.b4ell_bwidth / 4) * m.b4ell_bheight;
            return CLSPMV_OK;
        }
        case CLSPMV_FORMAT_SBELL: {
            const auto& m = *static_cast<const clspmv_sbell_f32*>(dev);
            if ((rc = read_int(m.sbell_slice_ptr + m.sbell_slice_num, &last))) return rc;
            *count = (size_t)last * m.sbell_bwidth * m.sbell_bheight;
            return CLSPMV_OK;
        }
    }
    return CLSPMV_ERR_ARG;
}

int clspmv_pack_values(int format, const void* dev, int value_type, void* values, float* row_scale,
                       clspmv_stream_t stream)
{
    int rc = check_struct(format, dev);
    if (rc) return rc;
    if (!values || !row_scale) return CLSPMV_ERR_ARG;
    size_t count = 0;
    if ((rc = clspmv_stored_values(format, dev, &count))) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    // entries no row walk reaches (padding rows, out-of-range diagonals) stay 0
    if ((rc = cuda_status(cudaMemsetAsync(values, 0, count * 2, st)))) return rc;
    if (matrix_rows(dev) <= 0) return CLSPMV_OK;
    if (value_type == CLSPMV_VALUES_BF16) return pack_typed(format, dev, static_cast<__nv_bfloat16*>(values), row_scale, st);
    if (value_type == CLSPMV_VALUES_F16) return pack_typed(format, dev, static_cast<__half*>(values), row_scale, st);
    return CLSPMV_ERR_ARG;
}

int clspmv_spmm(int format, const void* dev, int value_type, const void* values, const float* row_scale, int k,
                const float* X, int ldx, float* Y, int ldy, float alpha, float beta, clspmv_stream_t stream)
{
    int rc = check_struct(format, dev);
    if (rc) return rc;
    if (!X || !Y) return CLSPMV_ERR_ARG;
    if (value_type != CLSPMV_VALUES_F32 && (!values || !row_scale)) return CLSPMV_ERR_ARG;
    int vec = 1, lshift = 0;
    if ((rc = plan_lanes(k, X, ldx, Y, ldy, &vec, &lshift))) return rc;
    if (matrix_rows(dev) <= 0) return CLSPMV_OK;
    Dense d{k, X, ldx, Y, ldy, alpha, beta, value_type == CLSPMV_VALUES_F32 ? nullptr : row_scale, lshift};
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    // one contiguous vector: the format's own single-vector kernel (CSR's needs a merge plan)
    if (k == 1 && ldx == 1 && ldy == 1 && format != CLSPMV_FORMAT_CSR) {
        rc = launch_packed(format, dev, value_type, values, row_scale, nullptr, X, Y, alpha, beta, st, false);
        if (rc != CLSPMV_ERR_ALIGN) return rc;
    }
    switch (value_type) {
        case CLSPMV_VALUES_F32: return spmm_typed<float>(format, dev, nullptr, d, vec, st);
        case CLSPMV_VALUES_BF16: return spmm_typed<__nv_bfloat16>(format, dev, values, d, vec, st);
        case CLSPMV_VALUES_F16: return spmm_typed<__half>(format, dev, values, d, vec, st);
    }
    return CLSPMV_ERR_ARG;
}

int clspmv_batch_create(int max_jobs, clspmv_batch** out)
{
    if (!out || max_jobs < 1) return CLSPMV_ERR_ARG;
    *out = nullptr;
    clspmv_batch* b = new (std::nothrow) clspmv_batch();
    if (!b) return CLSPMV_ERR_ALLOC;
    b->capacity = max_jobs;
    int rc = cuda_status(cudaMallocHost(&b->host, sizeof(BatchJob) * max_jobs));
    if (!rc) rc = cuda_status(cudaMalloc(&b->dev, sizeof(BatchJob) * max_jobs));
    if (!rc) rc = cuda_status(cudaEventCreateWithFlags(&b->copied, cudaEventDisableTiming));
    if (rc) {
        clspmv_batch_free(b);
        return rc;
    }
    *out = b;
    return CLSPMV_OK;
}

int clspmv_batch_set(clspmv_batch* b, const clspmv_spmm_job* jobs, int njobs, clspmv_stream_t stream, int* bad_job)
{
    if (bad_job) *bad_job = -1;
    if (!b || (!jobs && njobs > 0) || njobs < 0) return CLSPMV_ERR_ARG;
    if (njobs > b->capacity) return CLSPMV_ERR_ARG;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int rc = cuda_status(cudaEventSynchronize(b->copied));   // staging free again
    if (rc) return rc;
    // row jobs first (k_batch), then the 4x4-block jobs (k_batch_blocks), each
    // with its own task numbering; a job's place in the table changes nothing
    // in its Y
    b->njobs = 0;
    b->tasks = b->block_tasks = 0;
    b->nrow_jobs = 0;
    int nblock = 0;
    for (int i = 0; i < njobs; i++) {
        BatchJob J;
        if ((rc = make_job(jobs[i], J))) {
            if (bad_job) *bad_job = i;
            return rc;
        }
        if (J.bh) b->host[njobs - 1 - nblock++] = J;   // filled from the end, reversed below
        else b->host[b->nrow_jobs++] = J;
    }
    std::reverse(b->host + b->nrow_jobs, b->host + njobs);
    long long tasks = 0, block_tasks = 0;
    for (int i = 0; i < njobs; i++) {
        BatchJob& J = b->host[i];
        long long& t = J.bh ? block_tasks : tasks;
        J.task_begin = t;
        const long long units = J.chunk > 0 ? ((long long)J.nnz + J.chunk - 1) / J.chunk
                                : J.bh ? ((long long)J.rows + J.bh - 1) / J.bh : J.rows;
        t += (units + (32 >> J.lshift) - 1) / (32 >> J.lshift);
    }
    b->njobs = njobs;
    b->tasks = tasks;
    b->block_tasks = block_tasks;
    if (njobs == 0) return CLSPMV_OK;
    rc = cuda_status(cudaMemcpyAsync(b->dev, b->host, sizeof(BatchJob) * njobs, cudaMemcpyHostToDevice, st));
    if (!rc) rc = cuda_status(cudaEventRecord(b->copied, st));
    return rc;
}

int clspmv_batch_run(clspmv_batch* b, clspmv_stream_t stream)
{
    if (!b) return CLSPMV_ERR_ARG;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int n = 0;
    if (b->tasks > 0) {
        const long long grid = std::min<long long>(batch_grid(), (b->tasks + 7) / 8);
        k_batch<<<(int)grid, kSpmmBlock, 0, st>>>(b->dev, b->nrow_jobs, b->tasks);
        n++;
    }
    if (b->block_tasks > 0) {
        const long long grid = std::min<long long>(batch_blocks_grid(), (b->block_tasks + 7) / 8);
        k_batch_blocks<<<(int)grid, kSpmmBlock, 0, st>>>(b->dev + b->nrow_jobs, b->njobs - b->nrow_jobs, b->block_tasks);
        n++;
    }
    return n ? after_launch(n) : CLSPMV_OK;
}

int clspmv_batch_free(clspmv_batch* b)
{
    if (!b) return CLSPMV_ERR_ARG;
    if (b->copied) {
        cudaEventSynchronize(b->copied);
        cudaEventDestroy(b->copied);
    }
    if (b->host) cudaFreeHost(b->host);
    if (b->dev) cudaFree(b->dev);
    delete b;
    return CLSPMV_OK;
}

#define SPMM_ENTRY(name, FMT, TYPE)                                                                        \
    int clspmv_##name##_spmm_f32(const TYPE* dev, int k, const float* X, int ldx, float* Y, int ldy, float alpha, \
                                 float beta, clspmv_stream_t stream)                                              \
    {                                                                                                             \
        return clspmv_spmm(FMT, dev, CLSPMV_VALUES_F32, nullptr, nullptr, k, X, ldx, Y, ldy, alpha, beta, stream); \
    }
SPMM_ENTRY(csr, CLSPMV_FORMAT_CSR, clspmv_csr_f32)
SPMM_ENTRY(coo, CLSPMV_FORMAT_COO, clspmv_coo_f32)
SPMM_ENTRY(dia, CLSPMV_FORMAT_DIA, clspmv_dia_f32)
SPMM_ENTRY(bdia, CLSPMV_FORMAT_BDIA, clspmv_bdia_f32)
SPMM_ENTRY(ell, CLSPMV_FORMAT_ELL, clspmv_ell_f32)
SPMM_ENTRY(sell, CLSPMV_FORMAT_SELL, clspmv_sell_f32)
SPMM_ENTRY(b4csr, CLSPMV_FORMAT_B4CSR, clspmv_b4csr_f32)
SPMM_ENTRY(b4ell, CLSPMV_FORMAT_B4ELL, clspmv_b4ell_f32)
SPMM_ENTRY(sbell, CLSPMV_FORMAT_SBELL, clspmv_sbell_f32)
#undef SPMM_ENTRY

}  // extern "C"
