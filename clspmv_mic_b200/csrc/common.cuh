// common.cuh — load/store helpers and argument blocks shared by the SpMV
// tile functions (sm_100a only).
//
// Every format is written as a CTA-level tile function
//     template <...> __device__ void <fmt>_tile(const <Fmt>Args&, int tile, char* smem)
// for a fixed block of kBlock threads. A per-format __global__ wrapper runs
// one tile per CTA; the fused Cocktail kernel maps CTA ranges to the tiles of
// several formats, so all tile functions share the block size and take their
// shared memory from the caller.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

namespace clspmv {

constexpr int kBlock = 256;      // threads per CTA for every SpMV tile
constexpr int kWarp = 32;

// ---------------------------------------------------------------------------
// Cache-policy loads. Matrix arrays are streamed once per SpMV: they are read
// through the non-coherent path without L1 allocation and marked evict-first
// in L2, so that x (reused by many rows) keeps its L2 lines. x is read with
// an evict-last policy for the same reason.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t policy_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t policy_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ float4 ld_stream_f4(const float* p, uint64_t pol)
{
    float4 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ int4 ld_stream_i4(const int* p, uint64_t pol)
{
    int4 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_stream_f(const float* p, uint64_t pol)
{
    float v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ int ld_stream_i(const int* p, uint64_t pol)
{
    int v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}
// Loads for thread-per-row walks (CSR scalar / vector): consecutive loads
// of one thread share sectors, so these keep the L1 allocation.
__device__ __forceinline__ float ld_l1_f(const float* p, uint64_t pol)
{
    float v;
    asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ int ld_l1_i(const int* p, uint64_t pol)
{
    int v;
    asm volatile("ld.global.nc.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float4 ld_l1_f4(const float* p, uint64_t pol)
{
    float4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ int4 ld_l1_i4(const int* p, uint64_t pol)
{
    int4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
// x gathers: read-only path, L1 allocation kept (neighbouring rows share
// lines), evict-last in L2.
__device__ __forceinline__ float ld_x(const float* p, uint64_t pol)
{
    float v;
    asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float4 ld_x4(const float* p, uint64_t pol)
{
    float4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}

// x gathers at scattered columns (COO, CSR by chunks): GX = 0 allocates the
// line in L1 like ld_x; GX = 1 does not (with uniformly scattered columns
// almost no gather hits L1, and the line fill costs L1 bandwidth).
__device__ __forceinline__ float ld_x_na(const float* p, uint64_t pol)
{
    float v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
template <int GX>
__device__ __forceinline__ float ld_gx(const float* p, uint64_t pol)
{
    if constexpr (GX == 1) return ld_x_na(p, pol);
    else return ld_x(p, pol);
}

// Matrix values stored as FP32, BF16 or FP16, read as float: ldv4 loads 4
// consecutive values (16 bytes, or 8 for 16-bit storage; 4-value aligned),
// ldv one. Streamed like the other matrix arrays.
__device__ __forceinline__ uint2 ld_stream_u2(const void* p, uint64_t pol)
{
    uint2 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0,%1}, [%2], %3;"
                 : "=r"(v.x), "=r"(v.y)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ unsigned short ld_stream_u16(const void* p, uint64_t pol)
{
    unsigned short v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(pol));
    return v;
}
// bf16 is the upper half of an FP32 word
__device__ __forceinline__ float bf16_lo(unsigned w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(unsigned w) { return __uint_as_float(w & 0xffff0000u); }

__device__ __forceinline__ float4 ldv4(const float* p, uint64_t pol) { return ld_stream_f4(p, pol); }
__device__ __forceinline__ float4 ldv4(const __nv_bfloat16* p, uint64_t pol)
{
    const uint2 u = ld_stream_u2(p, pol);
    return make_float4(bf16_lo(u.x), bf16_hi(u.x), bf16_lo(u.y), bf16_hi(u.y));
}
__device__ __forceinline__ float4 ldv4(const __half* p, uint64_t pol)
{
    const uint2 u = ld_stream_u2(p, pol);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
    return make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float ldv(const float* p, uint64_t pol) { return ld_stream_f(p, pol); }
__device__ __forceinline__ float ldv(const __nv_bfloat16* p, uint64_t pol) { return __uint_as_float((unsigned)ld_stream_u16(p, pol) << 16); }
__device__ __forceinline__ float ldv(const __half* p, uint64_t pol) { return __half2float(__ushort_as_half(ld_stream_u16(p, pol))); }

// alpha for one row: 16-bit values carry a per-row scale
__device__ __forceinline__ float row_alpha(float alpha, const float* scale, long long row)
{
    return scale ? alpha * __ldg(scale + row) : alpha;
}

// The row scales of an argument block: none for FP32 values, known at
// compile time so the FP32 kernels keep their registers.
template <template <class> class ArgsT, class V>
__device__ __forceinline__ const float* scl(const ArgsT<V>& a)
{
    if constexpr (std::is_same<V, float>::value) return nullptr;
    else return a.scale;
}

// y update. ATOMIC is used when another CTA (or another Cocktail part) may
// add to the same row; otherwise the row belongs to this thread alone.
template <bool ATOMIC>
__device__ __forceinline__ void y_update(float* y, long long row, float alpha, float beta, float acc)
{
    if (ATOMIC) {
        atomicAdd(y + row, alpha * acc);
    } else {
        float old = beta == 0.0f ? 0.0f : beta * y[row];
        y[row] = old + alpha * acc;
    }
}

__device__ __forceinline__ float dot4(float4 a, float4 b, float acc)
{
    acc = fmaf(a.x, b.x, acc);
    acc = fmaf(a.y, b.y, acc);
    acc = fmaf(a.z, b.z, acc);
    acc = fmaf(a.w, b.w, acc);
    return acc;
}

// ---------------------------------------------------------------------------
// Argument blocks (device pointers + sizes), one per format.
// ---------------------------------------------------------------------------
template <class V>
struct DiaArgsT {
    int rows, cols, ndiag, len;       // len = dia_length_aligned (multiple of 4)
    const int* offsets;
    const V* data;
    const float* x;
    float* y;
    float alpha, beta;
    const float* scale;               // per-row scale of 16-bit values, or nullptr
};
using DiaArgs = DiaArgsT<float>;

template <class V>
struct BdiaArgsT {
    int rows, cols, nband, len;
    const int* offsets;               // first offset of each band
    const int* bptr;                  // nband + 1
    const V* data;
    const float* x;
    float* y;
    float alpha, beta;
    const float* scale;               // per-row scale of 16-bit values, or nullptr
};
using BdiaArgs = BdiaArgsT<float>;

template <class V>
struct EllArgsT {
    int rows, ell_num, len;           // len = ell_height_aligned (multiple of 4)
    const int* col;
    const V* data;
    const float* x;
    float* y;
    float alpha, beta;
    const float* scale;               // per-row scale of 16-bit values, or nullptr
};
using EllArgs = EllArgsT<float>;

template <class V>
struct SellArgsT {
    int rows, slice_height, nslice;
    const int* slice_ptr;
    const int* col;
    const V* data;
    const float* x;
    float* y;
    float alpha, beta;
    const float* scale;               // per-row scale of 16-bit values, or nullptr
};
using SellArgs = SellArgsT<float>;

template <class V>
struct CsrArgsT {
    int rows, nnz;
    const int* row_ptr;
    const int* col;
    const V* val;
    const float* x;
    float* y;
    float alpha, beta;
    const float* scale;               // per-row scale of 16-bit values, or nullptr
};
using CsrArgs = CsrArgsT<float>;

template <class V>
struct CooArgsT {
    int nnz;
    const int* row;
    const int* col;
    const V* val;
    const float* x;
    float* y;
    float alpha;
    const float* scale;               // per-row scale of 16-bit values, or nullptr
};
using CooArgs = CooArgsT<float>;

template <class V>
struct B4ellArgsT {
    int rows, cols, nbrow, ellnum, len, f4;   // len = height_aligned, f4 = float4_aligned
    const int* col;                           // float4 units
    const V* data;
    const float* x;
    float* y;
    float alpha, beta;
    const float* scale;               // per-row scale of 16-bit values, or nullptr
};
using B4ellArgs = B4ellArgsT<float>;

template <class V>
struct SbellArgsT {
    int rows, cols, nbrow, nslice, slice_height;
    const int* slice_ptr;
    const int* col;
    const V* data;
    const float* x;
    float* y;
    float alpha, beta;
    const float* scale;               // per-row scale of 16-bit values, or nullptr
};
using SbellArgs = SbellArgsT<float>;

template <class V>
struct B4csrArgsT {
    int rows, cols, nbrow, len;               // len = aligned_size
    const int* row_ptr;
    const int* col;
    const V* data;
    const float* x;
    float* y;
    float alpha, beta;
    const float* scale;               // per-row scale of 16-bit values, or nullptr
};
using B4csrArgs = B4csrArgsT<float>;

}  // namespace clspmv
