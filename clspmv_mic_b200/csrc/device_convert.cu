// device_convert.cu — COO -> format converters that run on the device.
//
// clspmv_device_coo2<fmt>_f32 takes a COO whose arrays are in device memory
// and writes a device copy of the format struct holding, array for array and
// byte for byte, what the host converter clspmv_coo2<fmt>_f32 (the templates
// of matrix_storage.h, restating include/matrix_storage.h:936-2409 of
// clSpMV) makes from the same COO, with the same statuses: the same argument
// checks, the same refusals, and CLSPMV_ERR_NOT_SORTED where the host
// converter wants a (row, col)-sorted COO (every format but DIA / BDIA, which
// keep the last value of a repeated (row, col) in COO order).
// clspmv_device_sort_coo_f32 sorts a device COO in place, stably, as
// clspmv_sort_coo_f32 does on the host.
//
// Output arrays are cudaMalloc'ed and released with clspmv_device_free_<fmt>
// (an empty array still gets a 4-byte allocation, so no pointer is NULL after
// a success). Every call synchronises `stream`: sizes are read back to size
// the outputs.
//
// The work is integer index arithmetic over the COO: row pointers by binary
// search of the sorted row ids, slot-parallel fills of the padded layouts
// (every slot written once, coalesced), scatters for DIA and the block
// formats. Block grouping sorts the entries by (block row, block column) with
// a stable radix sort (CUB), which keeps COO order inside a block, so the
// last of a repeated (row, col) is the one written, as in the host loops.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

#include "api_internal.h"
#include "clspmv_b200.h"

using clspmv::cuda_status;

namespace {

constexpr int kT = 256;

int grid_for(long long n)
{
    const long long b = (n + kT - 1) / kT;
    return (int)std::max(1LL, std::min(b, 148LL * 32));
}

#define GRID_STRIDE(i, n) \
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

long long aligned_len(long long n, long long a) { return n % a == 0 ? n : n + (a - n % a); }

int bits_for(long long n)   // bits of the largest value in [0, n)
{
    int b = 0;
    while (b < 62 && (1LL << b) < n) b++;
    return b;
}

// cudaMalloc'ed arrays released at scope exit unless kept.
struct Allocs {
    std::vector<void*> ptrs;
    int rc = CLSPMV_OK;
    bool keep = false;
    template <class T>
    T* get(size_t n)
    {
        if (rc) return nullptr;
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            rc = CLSPMV_ERR_ALLOC;
            return nullptr;
        }
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    ~Allocs()
    {
        if (!keep)
            for (void* p : ptrs) cudaFree(p);
    }
};

template <class T>
int read_back(const T* dev, T* host, cudaStream_t st)
{
    int rc = cuda_status(cudaMemcpyAsync(host, dev, sizeof(T), cudaMemcpyDeviceToHost, st));
    if (!rc) rc = cuda_status(cudaStreamSynchronize(st));
    return rc;
}

int launched(cudaStream_t st, int n = 1)
{
    (void)st;
    return clspmv::after_launch(n);
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// flags bit 0: some neighbour pair is out of (row, col) order; bit 1: an id
// is outside the matrix.
__global__ void k_check_coo(const int* __restrict__ row, const int* __restrict__ col, long long n, int h, int w,
                            int* flags)
{
    int f = 0;
    GRID_STRIDE(i, n)
    {
        const int r = row[i], c = col[i];
        if (r < 0 || r >= h || c < 0 || c >= w) f |= 2;
        if (i > 0) {
            const int pr = row[i - 1], pc = col[i - 1];
            if (pr > r || (pr == r && pc > c)) f |= 1;
        }
    }
    f = __reduce_or_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && f) atomicOr(flags, f);
}

__global__ void k_coo_keys(const int* __restrict__ row, const int* __restrict__ col, long long n, int colbits,
                           unsigned long long* keys, int* idx)
{
    GRID_STRIDE(i, n)
    {
        keys[i] = ((unsigned long long)(unsigned)row[i] << colbits) | (unsigned)col[i];
        idx[i] = (int)i;
    }
}

__global__ void k_block_keys(const int* __restrict__ row, const int* __restrict__ col, long long n, int bw, int bh,
                             int colbits, unsigned long long* keys, int* idx)
{
    GRID_STRIDE(i, n)
    {
        keys[i] = ((unsigned long long)(unsigned)(row[i] / bh) << colbits) | (unsigned)(col[i] / bw);
        idx[i] = (int)i;
    }
}

template <class T>
__global__ void k_gather(const int* __restrict__ idx, const T* __restrict__ src, long long n, T* dst)
{
    GRID_STRIDE(i, n) dst[i] = src[idx[i]];
}

// rp[r] = first position whose sorted id is >= r, for r in [0, nrows].
__global__ void k_lower_bounds(const int* __restrict__ ids, long long n, int nrows, int* rp)
{
    GRID_STRIDE(r, (long long)nrows + 1)
    {
        long long lo = 0, hi = n;
        while (lo < hi) {
            const long long mid = (lo + hi) >> 1;
            if (ids[mid] < r) lo = mid + 1;
            else hi = mid;
        }
        rp[r] = (int)lo;
    }
}

__global__ void k_max_len(const int* __restrict__ rp, int nrows, int* out)
{
    int m = 0;
    GRID_STRIDE(r, nrows) m = max(m, rp[r + 1] - rp[r]);
    m = __reduce_max_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// wsh[s] = (longest row of slice s) * sh; wsh[ns] = 0.
__global__ void k_slice_slots(const int* __restrict__ rp, int nrows, int sh, int ns, long long* wsh)
{
    GRID_STRIDE(s, (long long)ns + 1)
    {
        int m = 0;
        if (s < ns) {
            const long long r1 = min((long long)nrows, (s + 1) * (long long)sh);
            for (long long r = s * (long long)sh; r < r1; r++) m = max(m, rp[r + 1] - rp[r]);
        }
        wsh[s] = (long long)m * sh;
    }
}

__global__ void k_to_int(const long long* __restrict__ a, long long n, int* b)
{
    GRID_STRIDE(i, n) b[i] = (int)a[i];
}

// Largest s in [0, ns) with ptr[s] <= t: the slice holding slot t (a
// zero-width slice shares its start with the next one and is never chosen).
__device__ __forceinline__ int slice_of(const int* __restrict__ ptr, int ns, long long t)
{
    int lo = 0, hi = ns - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((long long)ptr[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ELL slot (k, r) = t: entry k of row r, else the row's last column (0 for
// an empty row) with value 0; rows past the height are all zero
// (include/matrix_storage.h:1385-1389).
__global__ void k_ell_fill(const int* __restrict__ rp, const int* __restrict__ col, const float* __restrict__ val,
                           int h, long long len, long long total, int* ocol, float* oval)
{
    GRID_STRIDE(t, total)
    {
        const long long k = t / len, r = t - k * len;
        int c = 0;
        float v = 0.f;
        if (r < h) {
            const int a = rp[r], b = rp[r + 1];
            if (k < b - a) {
                c = col[a + k];
                v = val[a + k];
            } else if (b > a) {
                c = col[b - 1];
            }
        }
        ocol[t] = c;
        oval[t] = v;
    }
}

// SELL slot t: entry k of row r of its slice, else padding that copies the
// slot to its left (the row's last column), and for an empty row (or a row
// past the height) slot 0 of the slice, itself 0 when the slice's first row
// is empty (include/matrix_storage.h:1466-1496).
__global__ void k_sell_fill(const int* __restrict__ ptr, int ns, const int* __restrict__ rp,
                            const int* __restrict__ col, const float* __restrict__ val, int h, int sh, long long total,
                            int* ocol, float* oval)
{
    GRID_STRIDE(t, total)
    {
        const int s = slice_of(ptr, ns, t);
        const long long off = t - ptr[s];
        const long long k = off / sh;
        const long long r = (long long)s * sh + (off - k * sh);
        int c;
        float v = 0.f;
        const int a = r < h ? rp[r] : 0, b = r < h ? rp[r + 1] : 0;
        if (k < b - a) {
            c = col[a + k];
            v = val[a + k];
        } else if (b > a) {
            c = col[b - 1];
        } else {
            const long long r0 = (long long)s * sh;
            c = rp[r0 + 1] > rp[r0] ? col[rp[r0]] : 0;
        }
        ocol[t] = c;
        oval[t] = v;
    }
}

__global__ void k_dia_mark(const int* __restrict__ row, const int* __restrict__ col, long long n, int h, int* flag)
{
    GRID_STRIDE(i, n) flag[(long long)col[i] - row[i] + h - 1] = 1;
}

// flags[0] = 1 when some row id is >= len
__global__ void k_rows_at_least(const int* __restrict__ row, long long n, long long len, int* flags)
{
    int f = 0;
    GRID_STRIDE(i, n) if (row[i] >= len) f = 1;
    f = __reduce_or_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && f) atomicOr(flags, f);
}

__global__ void k_dia_offsets(const int* __restrict__ flag, const int* __restrict__ rank, long long nd, int h, int* off)
{
    GRID_STRIDE(p, nd)
    if (flag[p]) off[rank[p]] = (int)(p - (h - 1));
}

// Sorted input: the last of a run of equal (row, col) is the one written.
__global__ void k_dia_scatter_sorted(const int* __restrict__ row, const int* __restrict__ col,
                                     const float* __restrict__ val, long long n, int h, const int* __restrict__ rank,
                                     long long len, float* data)
{
    GRID_STRIDE(i, n)
    {
        const int r = row[i], c = col[i];
        if (i + 1 < n && row[i + 1] == r && col[i + 1] == c) continue;
        data[(long long)rank[(long long)c - r + h - 1] * len + r] = val[i];
    }
}

// Unsorted input: each slot keeps the value of its highest COO position.
__global__ void k_dia_claim(const int* __restrict__ row, const int* __restrict__ col, long long n, int h,
                            const int* __restrict__ rank, long long len, int* owner)
{
    GRID_STRIDE(i, n)
    {
        const int r = row[i], c = col[i];
        atomicMax(owner + (long long)rank[(long long)c - r + h - 1] * len + r, (int)i);
    }
}

__global__ void k_dia_scatter_owned(const int* __restrict__ row, const int* __restrict__ col,
                                    const float* __restrict__ val, long long n, int h, const int* __restrict__ rank,
                                    long long len, const int* __restrict__ owner, float* data)
{
    GRID_STRIDE(i, n)
    {
        const int r = row[i], c = col[i];
        const long long slot = (long long)rank[(long long)c - r + h - 1] * len + r;
        if (owner[slot] == (int)i) data[slot] = val[i];
    }
}

__global__ void k_block_heads(const unsigned long long* __restrict__ keys, long long n, int* head)
{
    GRID_STRIDE(i, n) head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// For each block (in (block row, block column) order): its block row and
// block column.
__global__ void k_block_list(const unsigned long long* __restrict__ keys, const int* __restrict__ head,
                             const int* __restrict__ bid, long long n, int colbits, int* brow, int* bcol)
{
    GRID_STRIDE(i, n)
    if (head[i]) {
        const int b = bid[i] - 1;
        brow[b] = (int)(keys[i] >> colbits);
        bcol[b] = (int)(keys[i] & ((1ULL << colbits) - 1));
    }
}

// col_id of block b: its first column / unit (4 for b4csr, 1 for bcsr)
__global__ void k_b4_colid(const int* __restrict__ bcol, long long nb, int bw, int unit, int* out)
{
    GRID_STRIDE(b, nb) out[b] = bcol[b] * bw / unit;
}

// Block formats: where an entry of block b lands. inner row hh, column
// w4 * 4 + w of the block.
struct B4csrPlace {
    long long len, plane;
    __device__ long long operator()(int, int, long long b, int hh, int w4, int w) const
    {
        return w4 * plane + hh * len + b * 4 + w;
    }
};
struct B4ellPlace {   // data[j*colsz + hh*f4 + w4*w4sz + r*4 + w] (include/matrix_storage.h:2178)
    long long f4, colsz, w4sz;
    __device__ long long operator()(int r, int j, long long, int hh, int w4, int w) const
    {
        return j * colsz + hh * f4 + w4 * w4sz + (long long)r * 4 + w;
    }
};
struct BcsrPlace {    // data[k*len + b], k = inner row * bw + inner column (include/matrix_storage.h:1728)
    long long len;
    int bw;
    __device__ long long operator()(int, int, long long b, int hh, int w4, int w) const
    {
        return ((long long)hh * bw + w4 * 4 + w) * len + b;
    }
};
struct BellPlace {    // data[r + k*len + j*colsz] (include/matrix_storage.h:1992)
    long long len, colsz;
    int bw;
    __device__ long long operator()(int r, int j, long long, int hh, int w4, int w) const
    {
        return (long long)r + ((long long)hh * bw + w4 * 4 + w) * len + j * colsz;
    }
};
struct SbellPlace {   // include/matrix_storage.h:2387
    const int* ptr;
    int sh, bs;
    long long colsz, w4sz, hsz;
    __device__ long long operator()(int r, int j, long long, int hh, int w4, int w) const
    {
        const int s = r / sh, lr = r - s * sh;
        return (long long)ptr[s] * bs + j * colsz + hh * hsz + w4 * w4sz + (long long)lr * 4 + w;
    }
};

template <class Place>
__global__ void k_block_scatter(const int* __restrict__ idx, const int* __restrict__ bid, const int* __restrict__ row,
                                const int* __restrict__ col, const float* __restrict__ val, long long n, int bw, int bh,
                                const int* __restrict__ brow, const int* __restrict__ bcol, const int* __restrict__ brp,
                                Place place, float* data)
{
    GRID_STRIDE(i, n)
    {
        const int e = idx[i];
        const int r = row[e], c = col[e];
        if (i + 1 < n) {
            const int e2 = idx[i + 1];
            if (row[e2] == r && col[e2] == c) continue;
        }
        const long long b = bid[i] - 1;
        const int br = brow[b];
        const int cc = c - bcol[b] * bw;
        data[place(br, (int)(b - brp[br]), b, r % bh, cc >> 2, cc & 3)] = val[e];
    }
}

// b4ell / bell col ids, slot (j, r): the first column of block j of block row
// r, over unit (4: float4 units for b4ell, 1: columns for bell), else the
// row's last (0 for an empty or missing row).
__global__ void k_b4ell_cols(const int* __restrict__ brp, const int* __restrict__ bcol, int nbr, int bw, int unit,
                             long long len, long long total, int* out)
{
    GRID_STRIDE(t, total)
    {
        const long long j = t / len, r = t - j * len;
        int c = 0;
        if (r < nbr) {
            const int a = brp[r], e = brp[r + 1];
            if (j < e - a) c = bcol[a + j] * bw / unit;
            else if (e > a) c = bcol[e - 1] * bw / unit;
        }
        out[t] = c;
    }
}

__global__ void k_sbell_cols(const int* __restrict__ ptr, int ns, const int* __restrict__ brp,
                             const int* __restrict__ bcol, int nbr, int sh, int bw, long long total, int* out)
{
    GRID_STRIDE(t, total)
    {
        const int s = slice_of(ptr, ns, t);
        const long long off = t - ptr[s];
        const long long j = off / sh;
        const long long r = (long long)s * sh + (off - j * sh);
        int c = 0;
        if (r < nbr) {
            const int a = brp[r], e = brp[r + 1];
            if (j < e - a) c = bcol[a + j] * bw / 4;
            else if (e > a) c = bcol[e - 1] * bw / 4;
        }
        out[t] = c;
    }
}

// ---------------------------------------------------------------------------
// Host steps
// ---------------------------------------------------------------------------

struct Coo {
    int h, w;
    long long n;
    const int* row;
    const int* col;
    const float* val;
};

bool coo_args_ok(const clspmv_coo_f32* m)
{
    if (!m || m->matinfo.width < 0 || m->matinfo.height < 0 || m->matinfo.nnz < 0) return false;
    if (m->matinfo.nnz > 0 && (!m->coo_row_id || !m->coo_col_id || !m->coo_data)) return false;
    return true;
}

bool block_shape_ok(unsigned int bw, unsigned int bh)
{
    return (bw == 4 || bw == 8) && (bh == 1 || bh == 2 || bh == 4 || bh == 8);
}

// Runs the range / order check; *flags as k_check_coo.
int check_coo(const Coo& c, cudaStream_t st, Allocs& S, int* flags)
{
    *flags = 0;
    if (c.n == 0) return CLSPMV_OK;
    int* f = S.get<int>(1);
    if (S.rc) return S.rc;
    int rc = cuda_status(cudaMemsetAsync(f, 0, sizeof(int), st));
    if (rc) return rc;
    k_check_coo<<<grid_for(c.n), kT, 0, st>>>(c.row, c.col, c.n, c.h, c.w, f);
    if ((rc = launched(st))) return rc;
    return read_back(f, flags, st);
}

// Stable radix sort of (key, position) pairs; on return *idx_out holds the
// positions in key order, and *keys_out the sorted keys.
int sort_pairs(unsigned long long* k0, unsigned long long* k1, int* v0, int* v1, long long n, int end_bit,
               cudaStream_t st, Allocs& S, unsigned long long** keys_out, int** idx_out)
{
    *keys_out = k0;
    *idx_out = v0;
    if (n <= 1 || end_bit == 0) return CLSPMV_OK;
    size_t tb = 0;
    int rc = cuda_status(cub::DeviceRadixSort::SortPairs(nullptr, tb, k0, k1, v0, v1, (int)n, 0, end_bit, st));
    if (rc) return rc;
    void* tmp = S.get<char>(tb);
    if (S.rc) return S.rc;
    rc = cuda_status(cub::DeviceRadixSort::SortPairs(tmp, tb, k0, k1, v0, v1, (int)n, 0, end_bit, st));
    if (rc) return rc;
    *keys_out = k1;
    *idx_out = v1;
    return CLSPMV_OK;
}

template <class T>
int exclusive_sum(const T* in, T* out, long long n, cudaStream_t st, Allocs& S)
{
    size_t tb = 0;
    int rc = cuda_status(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int)n, st));
    if (rc) return rc;
    void* tmp = S.get<char>(tb);
    if (S.rc) return S.rc;
    return cuda_status(cub::DeviceScan::ExclusiveSum(tmp, tb, in, out, (int)n, st));
}

template <class T>
int inclusive_sum(const T* in, T* out, long long n, cudaStream_t st, Allocs& S)
{
    size_t tb = 0;
    int rc = cuda_status(cub::DeviceScan::InclusiveSum(nullptr, tb, in, out, (int)n, st));
    if (rc) return rc;
    void* tmp = S.get<char>(tb);
    if (S.rc) return S.rc;
    return cuda_status(cub::DeviceScan::InclusiveSum(tmp, tb, in, out, (int)n, st));
}

int max_len(const int* rp, int nrows, cudaStream_t st, Allocs& S, int* out)
{
    *out = 0;
    if (nrows <= 0) return CLSPMV_OK;
    int* d = S.get<int>(1);
    if (S.rc) return S.rc;
    int rc = cuda_status(cudaMemsetAsync(d, 0, sizeof(int), st));
    if (rc) return rc;
    k_max_len<<<grid_for(nrows), kT, 0, st>>>(rp, nrows, d);
    if ((rc = launched(st))) return rc;
    return read_back(d, out, st);
}

// Slice pointer of slices of `sh` rows over row pointer rp (nrows rows):
// ptr[s + 1] = ptr[s] + longest row of slice s * sh. *total = ptr[ns].
int slice_ptr(const int* rp, int nrows, int sh, int ns, cudaStream_t st, Allocs& S, Allocs& O, int** ptr,
              long long* total)
{
    long long* w = S.get<long long>((size_t)ns + 1);
    long long* p64 = S.get<long long>((size_t)ns + 1);
    *ptr = O.get<int>((size_t)ns + 1);
    if (S.rc) return S.rc;
    if (O.rc) return O.rc;
    k_slice_slots<<<grid_for(ns + 1), kT, 0, st>>>(rp, nrows, sh, ns, w);
    int rc = launched(st);
    if (!rc) rc = exclusive_sum(w, p64, (long long)ns + 1, st, S);
    if (!rc) rc = read_back(p64 + ns, total, st);
    if (rc) return rc;
    if (*total > INT_MAX) return CLSPMV_ERR_UNSUPPORTED;   // the int slice pointer would overflow
    k_to_int<<<grid_for(ns + 1), kT, 0, st>>>(p64, (long long)ns + 1, *ptr);
    return launched(st);
}

int row_ptr(const int* ids, long long n, int nrows, cudaStream_t st, int* rp)
{
    k_lower_bounds<<<grid_for((long long)nrows + 1), kT, 0, st>>>(ids, n, nrows, rp);
    return launched(st);
}

Coo view(const clspmv_coo_f32* m)
{
    return Coo{m->matinfo.height, m->matinfo.width, (long long)m->matinfo.nnz, m->coo_row_id, m->coo_col_id,
               m->coo_data};
}

int finish(cudaStream_t st) { return cuda_status(cudaStreamSynchronize(st)); }

// Block rows of a sorted COO for bw x bh blocks: blocks in (block row, block
// column) order with their block row / column, the block row pointer, and
// for each entry in that order its COO position and 1-based block id.
struct Blocks {
    int nbr = 0;
    long long nb = 0;
    int* idx = nullptr;    // COO positions in block order
    int* bid = nullptr;    // 1-based block of each position
    int* brow = nullptr;   // per block
    int* bcol = nullptr;   // per block (block column index)
    int* brp = nullptr;    // nbr + 1
};

int make_blocks(const Coo& c, int bw, int bh, cudaStream_t st, Allocs& S, Blocks& B)
{
    B.nbr = (int)(c.h / bh + (c.h % bh ? 1 : 0));
    const long long nbc = c.w / bw + (c.w % bw ? 1 : 0);
    const int colbits = bits_for(nbc), rowbits = bits_for(B.nbr);
    B.brp = S.get<int>((size_t)B.nbr + 1);
    if (S.rc) return S.rc;
    int rc;
    if (c.n == 0) {
        rc = cuda_status(cudaMemsetAsync(B.brp, 0, sizeof(int) * ((size_t)B.nbr + 1), st));
        return rc;
    }
    unsigned long long* k0 = S.get<unsigned long long>(c.n);
    unsigned long long* k1 = S.get<unsigned long long>(c.n);
    int* v0 = S.get<int>(c.n);
    int* v1 = S.get<int>(c.n);
    int* head = S.get<int>(c.n);
    B.bid = S.get<int>(c.n);
    if (S.rc) return S.rc;
    k_block_keys<<<grid_for(c.n), kT, 0, st>>>(c.row, c.col, c.n, bw, bh, colbits, k0, v0);
    if ((rc = launched(st))) return rc;
    unsigned long long* keys;
    if ((rc = sort_pairs(k0, k1, v0, v1, c.n, colbits + rowbits, st, S, &keys, &B.idx))) return rc;
    k_block_heads<<<grid_for(c.n), kT, 0, st>>>(keys, c.n, head);
    if ((rc = launched(st))) return rc;
    if ((rc = inclusive_sum(head, B.bid, c.n, st, S))) return rc;
    int nb = 0;
    if ((rc = read_back(B.bid + (c.n - 1), &nb, st))) return rc;
    B.nb = nb;
    B.brow = S.get<int>((size_t)nb);
    B.bcol = S.get<int>((size_t)nb);
    if (S.rc) return S.rc;
    k_block_list<<<grid_for(c.n), kT, 0, st>>>(keys, head, B.bid, c.n, colbits, B.brow, B.bcol);
    if ((rc = launched(st))) return rc;
    return row_ptr(B.brow, B.nb, B.nbr, st, B.brp);
}

template <class Place>
int scatter_blocks(const Coo& c, const Blocks& B, int bw, int bh, Place place, float* data, cudaStream_t st)
{
    if (c.n == 0) return CLSPMV_OK;
    k_block_scatter<<<grid_for(c.n), kT, 0, st>>>(B.idx, B.bid, c.row, c.col, c.val, c.n, bw, bh, B.brow, B.bcol,
                                                  B.brp, place, data);
    return launched(st);
}

// Shared front of the converters that want a sorted COO: argument, range and
// order checks with the host converters' statuses.
int sorted_front(const Coo& c, cudaStream_t st, Allocs& S, bool shape_ok)
{
    int flags = 0;
    int rc = check_coo(c, st, S, &flags);
    if (rc) return rc;
    if (flags & 2) return CLSPMV_ERR_ARG;
    if (!shape_ok) return CLSPMV_ERR_UNSUPPORTED;
    if (flags & 1) return CLSPMV_ERR_NOT_SORTED;
    return CLSPMV_OK;
}

int dia_core(const clspmv_coo_f32* src, clspmv_dia_f32* dst, int alignment, cudaStream_t st, Allocs& O)
{
    if (!coo_args_ok(src) || !dst || alignment <= 0) return CLSPMV_ERR_ARG;
    const Coo c = view(src);
    Allocs S;
    int flags = 0;
    int rc = check_coo(c, st, S, &flags);
    if (rc) return rc;
    if (flags & 2) return CLSPMV_ERR_ARG;
    // dia_data[row] with row < aligned(min(w, h)): a taller-than-wide matrix
    // converts while every entry sits above that row, and is rejected when one
    // does not (as by clspmv_coo2dia_f32: the reference writes past its arrays)
    const long long len = aligned_len(std::min(c.w, c.h), alignment);
    if (c.h > c.w && c.n > 0) {
        int* f = S.get<int>(1);
        if (S.rc) return S.rc;
        if ((rc = cuda_status(cudaMemsetAsync(f, 0, sizeof(int), st)))) return rc;
        k_rows_at_least<<<grid_for(c.n), kT, 0, st>>>(c.row, c.n, len, f);
        if ((rc = launched(st))) return rc;
        int below = 0;
        if ((rc = read_back(f, &below, st))) return rc;
        if (below) return CLSPMV_ERR_ARG;
    }
    dst->matinfo = src->matinfo;
    dst->dia_length = std::min(c.w, c.h);
    dst->dia_length_aligned = (int)len;
    dst->dia_num = 0;
    dst->dia_offsets = nullptr;
    dst->dia_data = nullptr;
    const long long nd = c.h > 0 ? (long long)c.w + c.h - 1 : 0;
    int* flag = S.get<int>((size_t)nd + 1);
    int* rank = S.get<int>((size_t)nd + 1);
    if (S.rc) return S.rc;
    if ((rc = cuda_status(cudaMemsetAsync(flag, 0, sizeof(int) * ((size_t)nd + 1), st)))) return rc;
    if (c.n > 0) {
        k_dia_mark<<<grid_for(c.n), kT, 0, st>>>(c.row, c.col, c.n, c.h, flag);
        if ((rc = launched(st))) return rc;
    }
    if ((rc = exclusive_sum(flag, rank, nd + 1, st, S))) return rc;
    int D = 0;
    if ((rc = read_back(rank + nd, &D, st))) return rc;
    // The reference refuses at the discovery of a new diagonal when the count
    // found so far times the aligned length reaches 2 nnz
    // (include/matrix_storage.h:972): with D diagonals in all, iff
    // (D - 1) * len >= 2 nnz, leaving dia_num = the least k with k * len >= 2 nnz.
    if (D >= 1 && len > 0 && (long long)(D - 1) * len >= 2LL * c.n) {
        dst->dia_num = (int)((2LL * c.n + len - 1) / len);
        return CLSPMV_ERR_REFUSED;
    }
    int* off = O.get<int>((size_t)D);
    float* data = O.get<float>((size_t)D * (size_t)len);
    if (O.rc) return O.rc;
    if ((rc = cuda_status(cudaMemsetAsync(data, 0, sizeof(float) * (size_t)D * (size_t)len, st)))) return rc;
    if (nd > 0) {
        k_dia_offsets<<<grid_for(nd), kT, 0, st>>>(flag, rank, nd, c.h, off);
        if ((rc = launched(st))) return rc;
    }
    if (c.n > 0) {
        if (!(flags & 1)) {
            k_dia_scatter_sorted<<<grid_for(c.n), kT, 0, st>>>(c.row, c.col, c.val, c.n, c.h, rank, len, data);
            if ((rc = launched(st))) return rc;
        } else {
            int* owner = S.get<int>((size_t)D * (size_t)len);
            if (S.rc) return S.rc;
            if ((rc = cuda_status(cudaMemsetAsync(owner, 0xff, sizeof(int) * (size_t)D * (size_t)len, st)))) return rc;
            k_dia_claim<<<grid_for(c.n), kT, 0, st>>>(c.row, c.col, c.n, c.h, rank, len, owner);
            if ((rc = launched(st))) return rc;
            k_dia_scatter_owned<<<grid_for(c.n), kT, 0, st>>>(c.row, c.col, c.val, c.n, c.h, rank, len, owner, data);
            if ((rc = launched(st))) return rc;
        }
    }
    if ((rc = finish(st))) return rc;
    dst->dia_num = D;
    dst->dia_offsets = off;
    dst->dia_data = data;
    return CLSPMV_OK;
}

}  // namespace

extern "C" {

int clspmv_device_sort_coo_f32(clspmv_coo_f32* mat, clspmv_stream_t stream)
{
    if (!coo_args_ok(mat)) return CLSPMV_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const Coo c = view(mat);
    Allocs S;
    int flags = 0;
    int rc = check_coo(c, st, S, &flags);
    if (rc) return rc;
    if (flags & 2) return CLSPMV_ERR_ARG;
    if (!(flags & 1)) return CLSPMV_OK;
    const int colbits = bits_for(c.w), rowbits = bits_for(c.h);
    unsigned long long* k0 = S.get<unsigned long long>(c.n);
    unsigned long long* k1 = S.get<unsigned long long>(c.n);
    int* v0 = S.get<int>(c.n);
    int* v1 = S.get<int>(c.n);
    int* ti = S.get<int>(c.n);
    float* tf = S.get<float>(c.n);
    if (S.rc) return S.rc;
    k_coo_keys<<<grid_for(c.n), kT, 0, st>>>(c.row, c.col, c.n, colbits, k0, v0);
    if ((rc = launched(st))) return rc;
    unsigned long long* keys;
    int* idx;
    if ((rc = sort_pairs(k0, k1, v0, v1, c.n, colbits + rowbits, st, S, &keys, &idx))) return rc;
    k_gather<int><<<grid_for(c.n), kT, 0, st>>>(idx, mat->coo_row_id, c.n, ti);
    if ((rc = launched(st))) return rc;
    if ((rc = cuda_status(cudaMemcpyAsync(mat->coo_row_id, ti, sizeof(int) * c.n, cudaMemcpyDeviceToDevice, st)))) return rc;
    k_gather<int><<<grid_for(c.n), kT, 0, st>>>(idx, mat->coo_col_id, c.n, ti);
    if ((rc = launched(st))) return rc;
    if ((rc = cuda_status(cudaMemcpyAsync(mat->coo_col_id, ti, sizeof(int) * c.n, cudaMemcpyDeviceToDevice, st)))) return rc;
    k_gather<float><<<grid_for(c.n), kT, 0, st>>>(idx, mat->coo_data, c.n, tf);
    if ((rc = launched(st))) return rc;
    if ((rc = cuda_status(cudaMemcpyAsync(mat->coo_data, tf, sizeof(float) * c.n, cudaMemcpyDeviceToDevice, st)))) return rc;
    return finish(st);
}

int clspmv_device_coo2csr_f32(const clspmv_coo_f32* src, clspmv_csr_f32* dst, clspmv_stream_t stream)
{
    if (!coo_args_ok(src) || !dst) return CLSPMV_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const Coo c = view(src);
    Allocs S, O;
    int rc = sorted_front(c, st, S, true);
    if (rc) return rc;
    int* rp = O.get<int>((size_t)c.h + 1);
    int* col = O.get<int>((size_t)c.n);
    float* val = O.get<float>((size_t)c.n);
    if (O.rc) return O.rc;
    if ((rc = row_ptr(c.row, c.n, c.h, st, rp))) return rc;
    if (c.n > 0) {
        if ((rc = cuda_status(cudaMemcpyAsync(col, c.col, sizeof(int) * c.n, cudaMemcpyDeviceToDevice, st)))) return rc;
        if ((rc = cuda_status(cudaMemcpyAsync(val, c.val, sizeof(float) * c.n, cudaMemcpyDeviceToDevice, st)))) return rc;
    }
    if ((rc = finish(st))) return rc;
    O.keep = true;
    dst->matinfo = src->matinfo;
    dst->csr_row_ptr = rp;
    dst->csr_col_id = col;
    dst->csr_data = val;
    return CLSPMV_OK;
}

int clspmv_device_coo2dia_f32(const clspmv_coo_f32* src, clspmv_dia_f32* dst, int alignment, clspmv_stream_t stream)
{
    Allocs O;
    const int rc = dia_core(src, dst, alignment, (cudaStream_t)stream, O);
    if (!rc) O.keep = true;
    return rc;
}

int clspmv_device_coo2bdia_f32(const clspmv_coo_f32* src, clspmv_bdia_f32* dst, int alignment, clspmv_stream_t stream)
{
    if (!dst) return CLSPMV_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    Allocs O;
    clspmv_dia_f32 dia;
    int rc = dia_core(src, &dia, alignment, st, O);
    if (rc) return rc;
    // Bands are maximal runs of consecutive offsets (include/matrix_storage.h:
    // 1184-1236); the offsets are few, so the bands are found on the host.
    std::vector<int> offs((size_t)dia.dia_num);
    if (dia.dia_num > 0 &&
        (rc = cuda_status(cudaMemcpy(offs.data(), dia.dia_offsets, sizeof(int) * offs.size(), cudaMemcpyDeviceToHost))))
        return rc;
    std::vector<int> first, bptr(1, 0);
    for (size_t d = 0; d < offs.size(); d++) {
        if (d > 0 && offs[d] - offs[d - 1] == 1) bptr.back()++;
        else {
            first.push_back(offs[d]);
            bptr.push_back(bptr.back() + 1);
        }
    }
    int* boff = O.get<int>(first.size());
    int* bp = O.get<int>(bptr.size());
    if (O.rc) return O.rc;
    if (!first.empty() &&
        (rc = cuda_status(cudaMemcpy(boff, first.data(), sizeof(int) * first.size(), cudaMemcpyHostToDevice))))
        return rc;
    if ((rc = cuda_status(cudaMemcpy(bp, bptr.data(), sizeof(int) * bptr.size(), cudaMemcpyHostToDevice)))) return rc;
    O.keep = true;
    cudaFree(dia.dia_offsets);   // the DIA data array becomes the BDIA one
    dst->matinfo = dia.matinfo;
    dst->bdia_band_num = (int)first.size();
    dst->bdia_length = dia.dia_length;
    dst->bdia_length_aligned = dia.dia_length_aligned;
    dst->bdia_offsets = boff;
    dst->bdia_bptr = bp;
    dst->bdia_data = dia.dia_data;
    return CLSPMV_OK;
}

int clspmv_device_coo2ell_f32(const clspmv_coo_f32* src, clspmv_ell_f32* dst, int alignment, int ellnum,
                              clspmv_stream_t stream)
{
    if (!coo_args_ok(src) || !dst || alignment <= 0 || ellnum < 0) return CLSPMV_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const Coo c = view(src);
    Allocs S, O;
    int rc = sorted_front(c, st, S, true);
    if (rc) return rc;
    int* rp = S.get<int>((size_t)c.h + 1);
    if (S.rc) return S.rc;
    if ((rc = row_ptr(c.row, c.n, c.h, st, rp))) return rc;
    int maxlen = 0;
    if ((rc = max_len(rp, c.h, st, S, &maxlen))) return rc;
    // include/matrix_storage.h:1339-1394: ellnum 0 selects the longest row
    const int num = ellnum == 0 ? maxlen : ellnum;
    const long long len = aligned_len(c.h, alignment);
    dst->matinfo = src->matinfo;
    dst->ell_num = num;
    dst->ell_height_aligned = (int)len;
    dst->ell_col_id = nullptr;
    dst->ell_data = nullptr;
    if (maxlen > num) return ellnum > 0 ? CLSPMV_ERR_ARG : CLSPMV_ERR_REFUSED;
    if (len * num > (long long)INT_MAX) return CLSPMV_ERR_REFUSED;
    const long long total = len * num;
    int* col = O.get<int>((size_t)total);
    float* val = O.get<float>((size_t)total);
    if (O.rc) return O.rc;
    if (total > 0) {
        k_ell_fill<<<grid_for(total), kT, 0, st>>>(rp, c.col, c.val, c.h, len, total, col, val);
        if ((rc = launched(st))) return rc;
    }
    if ((rc = finish(st))) return rc;
    O.keep = true;
    dst->ell_col_id = col;
    dst->ell_data = val;
    return CLSPMV_OK;
}

int clspmv_device_coo2sell_f32(const clspmv_coo_f32* src, clspmv_sell_f32* dst, unsigned int slice_height,
                               clspmv_stream_t stream)
{
    if (!coo_args_ok(src) || !dst || slice_height == 0 || slice_height > (unsigned)INT_MAX) return CLSPMV_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const Coo c = view(src);
    Allocs S, O;
    int rc = sorted_front(c, st, S, true);
    if (rc) return rc;
    const int sh = (int)slice_height;
    const int ns = c.h / sh + (c.h % sh ? 1 : 0);
    int* rp = S.get<int>((size_t)c.h + 1);
    if (S.rc) return S.rc;
    if ((rc = row_ptr(c.row, c.n, c.h, st, rp))) return rc;
    int* ptr = nullptr;
    long long total = 0;
    if ((rc = slice_ptr(rp, c.h, sh, ns, st, S, O, &ptr, &total))) return rc;
    int* col = O.get<int>((size_t)total);
    float* val = O.get<float>((size_t)total);
    if (O.rc) return O.rc;
    if (total > 0) {
        k_sell_fill<<<grid_for(total), kT, 0, st>>>(ptr, ns, rp, c.col, c.val, c.h, sh, total, col, val);
        if ((rc = launched(st))) return rc;
    }
    if ((rc = finish(st))) return rc;
    O.keep = true;
    dst->matinfo = src->matinfo;
    dst->sell_slice_height = slice_height;
    dst->sell_slice_num = ns;
    dst->sell_slice_ptr = ptr;
    dst->sell_col_id = col;
    dst->sell_data = val;
    return CLSPMV_OK;
}

int clspmv_device_coo2b4csr_f32(const clspmv_coo_f32* src, clspmv_b4csr_f32* dst, unsigned int bwidth,
                                unsigned int bheight, int alignment, clspmv_stream_t stream)
{
    if (!coo_args_ok(src) || !dst || alignment <= 0) return CLSPMV_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const Coo c = view(src);
    Allocs S, O;
    int rc = sorted_front(c, st, S, block_shape_ok(bwidth, bheight));
    if (rc) return rc;
    const int bw = (int)bwidth, bh = (int)bheight, bs = bw * bh;
    dst->matinfo = src->matinfo;
    dst->b4csr_bwidth = bwidth;
    dst->b4csr_bheight = bheight;
    Blocks B;
    if ((rc = make_blocks(c, bw, bh, st, S, B))) return rc;
    // include/matrix_storage.h:1863: block count cap
    if ((size_t)B.nb > (size_t)CLSPMV_MAX_MEM_OBJ / ((size_t)bs * sizeof(float))) return CLSPMV_ERR_REFUSED;
    const long long len = aligned_len(B.nb * 4, alignment);
    const size_t ndata = (size_t)len * bh * (bw / 4);
    int* rp = O.get<int>((size_t)B.nbr + 1);
    int* colid = O.get<int>((size_t)B.nb);
    float* data = O.get<float>(ndata);
    if (O.rc) return O.rc;
    if ((rc = cuda_status(cudaMemcpyAsync(rp, B.brp, sizeof(int) * ((size_t)B.nbr + 1), cudaMemcpyDeviceToDevice, st))))
        return rc;
    if ((rc = cuda_status(cudaMemsetAsync(data, 0, sizeof(float) * ndata, st)))) return rc;
    if (B.nb > 0) {
        k_b4_colid<<<grid_for(B.nb), kT, 0, st>>>(B.bcol, B.nb, bw, 4, colid);
        if ((rc = launched(st))) return rc;
    }
    if ((rc = scatter_blocks(c, B, bw, bh, B4csrPlace{len, len * bh}, data, st))) return rc;
    if ((rc = finish(st))) return rc;
    O.keep = true;
    dst->b4csr_row_num = B.nbr;
    dst->b4csr_aligned_size = (int)len;
    dst->b4csr_block_num = (int)B.nb;
    dst->b4csr_row_ptr = rp;
    dst->b4csr_col_id = colid;
    dst->b4csr_data = data;
    return CLSPMV_OK;
}

int clspmv_device_coo2bcsr_f32(const clspmv_coo_f32* src, clspmv_bcsr_f32* dst, unsigned int bwidth,
                               unsigned int bheight, int alignment, clspmv_stream_t stream)
{
    if (!coo_args_ok(src) || !dst || bwidth == 0 || bheight == 0 || bwidth > (unsigned)INT_MAX ||
        bheight > (unsigned)INT_MAX || alignment <= 0)
        return CLSPMV_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const Coo c = view(src);
    Allocs S, O;
    int rc = sorted_front(c, st, S, true);
    if (rc) return rc;
    const int bw = (int)bwidth, bh = (int)bheight;
    const size_t bs = (size_t)bw * bh;
    dst->matinfo = src->matinfo;
    dst->bcsr_bwidth = bwidth;
    dst->bcsr_bheight = bheight;
    Blocks B;
    if ((rc = make_blocks(c, bw, bh, st, S, B))) return rc;
    const long long len = aligned_len(B.nb, alignment);
    const size_t ndata = (size_t)len * bs;
    int* rp = O.get<int>((size_t)B.nbr + 1);
    int* colid = O.get<int>((size_t)B.nb);
    float* data = O.get<float>(ndata);
    if (O.rc) return O.rc;
    if ((rc = cuda_status(cudaMemcpyAsync(rp, B.brp, sizeof(int) * ((size_t)B.nbr + 1), cudaMemcpyDeviceToDevice, st))))
        return rc;
    if (ndata && (rc = cuda_status(cudaMemsetAsync(data, 0, sizeof(float) * ndata, st)))) return rc;
    if (B.nb > 0) {
        k_b4_colid<<<grid_for(B.nb), kT, 0, st>>>(B.bcol, B.nb, bw, 1, colid);
        if ((rc = launched(st))) return rc;
    }
    if ((rc = scatter_blocks(c, B, bw, bh, BcsrPlace{len, bw}, data, st))) return rc;
    if ((rc = finish(st))) return rc;
    O.keep = true;
    dst->bcsr_row_num = B.nbr;
    dst->bcsr_aligned_size = (int)len;
    dst->bcsr_block_num = (int)B.nb;
    dst->bcsr_row_ptr = rp;
    dst->bcsr_col_id = colid;
    dst->bcsr_data = data;
    return CLSPMV_OK;
}

int clspmv_device_coo2bell_f32(const clspmv_coo_f32* src, clspmv_bell_f32* dst, unsigned int bwidth,
                               unsigned int bheight, int alignment, int ellnum, clspmv_stream_t stream)
{
    if (!coo_args_ok(src) || !dst || bwidth == 0 || bheight == 0 || bwidth > (unsigned)INT_MAX ||
        bheight > (unsigned)INT_MAX || alignment <= 0 || ellnum < 0)
        return CLSPMV_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const Coo c = view(src);
    Allocs S, O;
    int rc = sorted_front(c, st, S, true);
    if (rc) return rc;
    const int bw = (int)bwidth, bh = (int)bheight;
    const size_t bs = (size_t)bw * bh;
    dst->matinfo = src->matinfo;
    dst->bell_bwidth = bwidth;
    dst->bell_bheight = bheight;
    dst->bell_float4_aligned = 0;
    dst->bell_col_id = nullptr;
    dst->bell_data = nullptr;
    Blocks B;
    if ((rc = make_blocks(c, bw, bh, st, S, B))) return rc;
    int maxw = 0;
    if ((rc = max_len(B.brp, B.nbr, st, S, &maxw))) return rc;
    const int num = ellnum == 0 ? maxw : ellnum;
    const long long len = aligned_len(B.nbr, alignment);
    dst->bell_block_num = num;
    dst->bell_row_num = B.nbr;
    dst->bell_height_aligned = (int)len;
    if (maxw > num) return CLSPMV_ERR_ARG;   // a block row longer than ellnum (include/matrix_storage.h:1975)
    const size_t ncol = (size_t)len * num, colsz = (size_t)len * bs, ndata = colsz * num;
    int* col = O.get<int>(ncol);
    float* data = O.get<float>(ndata);
    if (O.rc) return O.rc;
    if (ndata && (rc = cuda_status(cudaMemsetAsync(data, 0, sizeof(float) * ndata, st)))) return rc;
    if (ncol > 0) {
        k_b4ell_cols<<<grid_for((long long)ncol), kT, 0, st>>>(B.brp, B.bcol, B.nbr, bw, 1, len, (long long)ncol, col);
        if ((rc = launched(st))) return rc;
    }
    if ((rc = scatter_blocks(c, B, bw, bh, BellPlace{len, (long long)colsz, bw}, data, st))) return rc;
    if ((rc = finish(st))) return rc;
    O.keep = true;
    dst->bell_col_id = col;
    dst->bell_data = data;
    return CLSPMV_OK;
}

int clspmv_device_coo2b4ell_f32(const clspmv_coo_f32* src, clspmv_b4ell_f32* dst, unsigned int bwidth,
                                unsigned int bheight, int alignment, int ellnum, clspmv_stream_t stream)
{
    if (!coo_args_ok(src) || !dst || alignment <= 0 || ellnum < 0) return CLSPMV_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const Coo c = view(src);
    Allocs S, O;
    int rc = sorted_front(c, st, S, block_shape_ok(bwidth, bheight));
    if (rc) return rc;
    const int bw = (int)bwidth, bh = (int)bheight, bs = bw * bh;
    dst->matinfo = src->matinfo;
    dst->b4ell_bwidth = bwidth;
    dst->b4ell_bheight = bheight;
    Blocks B;
    if ((rc = make_blocks(c, bw, bh, st, S, B))) return rc;
    int maxw = 0;
    if ((rc = max_len(B.brp, B.nbr, st, S, &maxw))) return rc;
    const int num = ellnum == 0 ? maxw : ellnum;
    // include/matrix_storage.h:2141: padded block count cap
    if ((size_t)B.nbr * (size_t)num > (size_t)CLSPMV_MAX_MEM_OBJ / ((size_t)bs * sizeof(float)))
        return CLSPMV_ERR_REFUSED;
    if (maxw > num) return CLSPMV_ERR_REFUSED;
    const long long len = aligned_len(B.nbr, alignment), f4 = aligned_len(4LL * B.nbr, alignment);
    const int w4n = bw / 4;
    const size_t ncol = (size_t)len * num, ndata = (size_t)f4 * bh * w4n * num;
    int* col = O.get<int>(ncol);
    float* data = O.get<float>(ndata);
    if (O.rc) return O.rc;
    if ((rc = cuda_status(cudaMemsetAsync(data, 0, sizeof(float) * ndata, st)))) return rc;
    if (ncol > 0) {
        k_b4ell_cols<<<grid_for((long long)ncol), kT, 0, st>>>(B.brp, B.bcol, B.nbr, bw, 4, len, (long long)ncol, col);
        if ((rc = launched(st))) return rc;
    }
    if ((rc = scatter_blocks(c, B, bw, bh, B4ellPlace{f4, f4 * w4n * bh, f4 * bh}, data, st))) return rc;
    if ((rc = finish(st))) return rc;
    O.keep = true;
    dst->b4ell_row_num = B.nbr;
    dst->b4ell_block_num = num;
    dst->b4ell_height_aligned = (int)len;
    dst->b4ell_float4_aligned = (int)f4;
    dst->b4ell_col_id = col;
    dst->b4ell_data = data;
    return CLSPMV_OK;
}

int clspmv_device_coo2sbell_f32(const clspmv_coo_f32* src, clspmv_sbell_f32* dst, unsigned int bwidth,
                                unsigned int bheight, unsigned int slice_height, clspmv_stream_t stream)
{
    if (!coo_args_ok(src) || !dst || slice_height == 0 || slice_height > (unsigned)INT_MAX) return CLSPMV_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const Coo c = view(src);
    Allocs S, O;
    int rc = sorted_front(c, st, S, block_shape_ok(bwidth, bheight));
    if (rc) return rc;
    const int bw = (int)bwidth, bh = (int)bheight, bs = bw * bh, sh = (int)slice_height;
    dst->matinfo = src->matinfo;
    dst->sbell_bwidth = bwidth;
    dst->sbell_bheight = bheight;
    dst->sbell_col_id = nullptr;
    dst->sbell_data = nullptr;
    Blocks B;
    if ((rc = make_blocks(c, bw, bh, st, S, B))) return rc;
    const int ns = B.nbr / sh + (B.nbr % sh ? 1 : 0);
    dst->sbell_slice_num = ns;
    dst->sbell_row_num = B.nbr;
    dst->sbell_slice_height = slice_height;
    dst->sbell_slice_ptr = nullptr;
    int* ptr = nullptr;
    long long total = 0;
    if ((rc = slice_ptr(B.brp, B.nbr, sh, ns, st, S, O, &ptr, &total))) return rc;
    // include/matrix_storage.h:2350: padded block count cap
    if ((size_t)total > (size_t)CLSPMV_MAX_MEM_OBJ / ((size_t)bs * sizeof(float))) return CLSPMV_ERR_REFUSED;
    const int w4n = bw / 4;
    int* col = O.get<int>((size_t)total);
    float* data = O.get<float>((size_t)total * bs);
    if (O.rc) return O.rc;
    if ((rc = cuda_status(cudaMemsetAsync(data, 0, sizeof(float) * (size_t)total * bs, st)))) return rc;
    if (total > 0) {
        k_sbell_cols<<<grid_for(total), kT, 0, st>>>(ptr, ns, B.brp, B.bcol, B.nbr, sh, bw, total, col);
        if ((rc = launched(st))) return rc;
    }
    const long long colsz = (long long)sh * w4n * bh * 4, w4sz = (long long)sh * bh * 4, hsz = (long long)sh * 4;
    if ((rc = scatter_blocks(c, B, bw, bh, SbellPlace{ptr, sh, bs, colsz, w4sz, hsz}, data, st))) return rc;
    if ((rc = finish(st))) return rc;
    O.keep = true;
    dst->sbell_slice_ptr = ptr;
    dst->sbell_col_id = col;
    dst->sbell_data = data;
    return CLSPMV_OK;
}

}  // extern "C"
