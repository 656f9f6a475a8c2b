// spmm_tc.cu — b4csr with 4 x 4 blocks times k >= 16 right-hand sides on the
// fifth-generation tensor cores: Y <- alpha * A * X + beta * Y with
// tcgen05.mma (kind::tf32), operands in shared memory, accumulators in
// tensor memory.
//
// The reference multiplies one vector per call with a work-group per block
// row (kernels/spmv_bcsr.cl); the dense contraction inside one 4 x 4 block,
//     Y[4r + i, j] += sum_c A_b[i][c] * X[4 bc + c, j],
// is 4 x 4 x k, so the only dimension wide enough for an MMA is the right-hand
// sides. They are the MMA's M (64 lanes of tensor memory, k <= 64 per pass).
// FP32 accuracy comes from splitting every value v into a TF32 head
// hi = rna(v) (10 explicit mantissa bits) and the exact remainder lo = v - hi:
// the block's four rows as (hi, lo) are N = 8, the block's four X columns as
// (hi, lo) are K = 8, and one MMA per block leaves
//     D[j, i]     = sum_c (x_hi + x_lo)[c][j] * a_hi[i][c]
//     D[j, 4 + i] = sum_c (x_hi + x_lo)[c][j] * a_lo[i][c]
// so y = D[j, i] + D[j, 4 + i] carries every product to about 2^-21 of
// |a x| (lo is rounded to TF32 once more: 2^-11 of 2^-11).
//
// Shared-memory operands (no swizzle, canonical core matrices of 8 rows x
// 16 bytes, both K-major):
//   A (M = 64 right-hand sides x K = 8): element (j, kk) at
//     (j / 8) * 256 + (kk / 4) * 128 + (j % 8) * 16 + (kk % 4) * 4; only
//     j < KC is written, the rest of the 2 KB a descriptor spans belongs to
//     the next block's slice and only feeds accumulator lanes that are never
//     read. Lane j of a slice loads X[4 bc + 0..3][j] (four coalesced scalar
//     loads, one per X row) and stores its head and remainder as two 16-byte
//     rows, so no transpose is needed. (MN-major TF32 operands without
//     swizzle, which would take the X rows as loaded, read as zeros on
//     sm_100a.)
//   B (K = 8 x N = 8): element (kk, n) at (kk / 4) * 128 + n * 16 +
//     (kk % 4) * 4, i.e. [hi rows | lo rows] twice (the x_hi and x_lo halves
//     of K see the same block).
// Accumulators: a tile of 32 block rows owns 8 tensor-memory columns per
// block row (256 columns per CTA, at most two CTAs per SM); right-hand side j
// sits in lane (j % 16) + 32 * (j / 16), the M = 64 layout, so warp w < 4
// reads right-hand sides 16w .. 16w + 15 back with tcgen05.ld.
//
// Pipeline per CTA (8 warps): each step gathers 32 blocks (4 per warp) — the
// block's column id, its four value rows and its 4 x KC slice of X, loaded a
// step ahead into registers — splits them into (hi, lo) while writing the
// stage's operands, and thread 0 issues the 32 MMAs and commits them to the
// stage's mbarrier, which the producers wait on before they reuse the stage.
// Every wait is bounded (about 2 s on %globaltimer); a wait that runs out
// ends the kernel cleanly, tensor memory released, and is counted in a device
// word that clspmv_tensor_timeouts reads.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include "clspmv_b200.h"
#include "api_internal.h"
#include "common.cuh"

using namespace clspmv;

namespace {

constexpr int kTcWarps = 8;
constexpr int kTcThreads = 32 * kTcWarps;
constexpr int kTcTileRows = 32;            // block rows per tile, 8 tensor-memory columns each
constexpr int kTcCols = 256;               // tensor-memory columns per CTA
constexpr int kTcPer = 4 * kTcWarps;       // blocks per pipeline step, 4 per warp
constexpr int kTcMaxKc = 64;               // right-hand sides per pass (MMA M = 64)
constexpr unsigned kFullMask = 0xffffffffu;

// Instruction descriptor: D F32 (bits 4-5 = 1), A TF32 (7-9 = 2), B TF32
// (10-12 = 2), A and B K-major (bits 15, 16 = 0), N / 8 = 1 (bits 17-22),
// M / 16 = 4 (bits 24-28).
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | (1u << 17) | (4u << 24);

__device__ unsigned int g_tc_timeouts;

// Pipeline stages: as many as keep two CTAs (2 x 256 of the 512
// tensor-memory columns) on an SM for k <= 32, three above.
template <int KC> constexpr int tc_stages() { return KC == 16 ? 3 : KC == 32 ? 2 : 3; }

template <int KC>
struct TcSmem {
    static constexpr int kStages = tc_stages<KC>();
    static constexpr int kATile = KC * 32;            // KC / 8 groups of 8 rows x 32 bytes
    static constexpr int kAStage = kTcPer * kATile;
    static constexpr int kAPad = 2048;                // an M = 64 descriptor spans 2 KB from its start
    static constexpr int kBTile = 256;
    static constexpr int kBStage = kTcPer * kBTile;
    static constexpr int kA = 0;
    static constexpr int kB = kA + kStages * kAStage + kAPad;
    static constexpr int kMeta = kB + kStages * kBStage;
    static constexpr int kPtr = kMeta + kStages * kTcPer * 4;
    static constexpr int kBar = (kPtr + (kTcTileRows + 1) * 4 + 7) / 8 * 8;
    static constexpr int kTmem = kBar + kStages * 8;
    static constexpr int kBytes = kTmem + 16;
    // at least 80 KB so that no third CTA (without tensor-memory columns) lands on an SM
    static constexpr int kLaunch = kBytes > 80 * 1024 ? kBytes : 80 * 1024;
    static constexpr int kPerSm = 2 * (kLaunch + 1024) <= 228 * 1024 ? 2 : 1;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ float tf32_rna(float v)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return __uint_as_float(r);
}

__device__ __forceinline__ void split4(float4 v, float4& hi, float4& lo)
{
    hi = make_float4(tf32_rna(v.x), tf32_rna(v.y), tf32_rna(v.z), tf32_rna(v.w));
    lo = make_float4(v.x - hi.x, v.y - hi.y, v.z - hi.z, v.w - hi.w);
}

// Shared-memory matrix descriptor, no swizzle: start address, leading (K)
// and stride (M / N) byte offsets in 16-byte units, version 1 at bit 46.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3fffu) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the completion of the mbarrier phase with this parity; false
// after about 2 s.
__device__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try(bar, parity))
        if (global_ns() - t0 > 2000000000ull) return false;
    return true;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 32 consecutive columns of this warp's 32 lanes, waited for in the same
// statement so no use of the registers can move above the wait.
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// One step's loads for one lane: for the warp's four blocks, KC / 8 (block,
// right-hand side) pairs e = lane + 32 i, each the four X rows of the block's
// slice at that right-hand side; lanes 0-15 also load row (lane & 3) of block
// (lane >> 2).
template <int KC>
struct StepLoads {
    float x[KC / 2];
    float4 v;
};

template <int KC>
__device__ __forceinline__ void load_step(StepLoads<KC>& f, int col_lane, int gw, int b1, const float* __restrict__ data,
                                          size_t len, const float* __restrict__ X, int ldx, int width, uint64_t pe,
                                          uint64_t pl)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < KC / 8; i++) {
        const int e = lane + 32 * i, q = e / KC, j = e % KC;
        const int c4 = __shfl_sync(kFullMask, col_lane, q);
        const bool ok = gw + q < b1;
        const float* xp = X + (size_t)(4 * c4) * ldx + j;
#pragma unroll
        for (int c = 0; c < 4; c++)
            f.x[4 * i + c] = (ok && (unsigned)(4 * c4 + c) < (unsigned)width) ? ld_x(xp + (size_t)c * ldx, pl) : 0.f;
    }
    f.v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (lane < 16 && gw + (lane >> 2) < b1)
        f.v = ld_stream_f4(data + (size_t)(lane & 3) * len + 4 * (size_t)(gw + (lane >> 2)), pe);
}

__device__ __forceinline__ int load_col(const int* __restrict__ col, int gw, int b1, uint64_t pe)
{
    const int lane = threadIdx.x & 31;
    return (lane < 4 && gw + lane < b1) ? ld_stream_i(col + gw + lane, pe) : 0;
}

template <int KC>
__global__ void __launch_bounds__(kTcThreads) k_b4csr_spmm_tc(int nbrow, int rows, int width, const int* __restrict__ ptr,
                                                              const int* __restrict__ col, const float* __restrict__ data,
                                                              size_t len, const float* __restrict__ X, int ldx,
                                                              float* __restrict__ Y, int ldy, float alpha, float beta,
                                                              int ntiles)
{
    using S = TcSmem<KC>;
    constexpr int kStages = S::kStages;
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = smem_addr(smem);
    int* meta = reinterpret_cast<int*>(smem + S::kMeta);
    int* sptr = reinterpret_cast<int*>(smem + S::kPtr);
    const uint32_t bar0 = sbase + S::kBar;

    if (tid == 0) {
        for (int s = 0; s < kStages; s++) mbar_init(bar0 + 8 * s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + S::kTmem),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + S::kTmem);

    const uint64_t pe = policy_evict_first(), pl = policy_evict_last();
    unsigned it = 0;     // steps this CTA has run; stage = it % kStages
    bool bad = false;    // a bounded wait ran out (the same on every thread)
    for (int tile = blockIdx.x; tile < ntiles && !bad; tile += gridDim.x) {
        const int br0 = tile * kTcTileRows;
        const int nbr = min(kTcTileRows, nbrow - br0);
        if (tid <= kTcTileRows) sptr[tid] = __ldg(ptr + br0 + min(tid, nbr));
        __syncthreads();
        const int b0 = sptr[0], b1 = sptr[nbr];
        const int nsteps = (b1 - b0 + kTcPer - 1) / kTcPer;

        StepLoads<KC> cur;
        int col_next = 0;
        if (nsteps > 0) {
            const int gw = b0 + 4 * warp;
            load_step<KC>(cur, load_col(col, gw, b1, pe), gw, b1, data, len, X, ldx, width, pe, pl);
            if (nsteps > 1) col_next = load_col(col, gw + kTcPer, b1, pe);
        }
        for (int step = 0; step < nsteps; step++, it++) {
            const int s = (int)(it % kStages);
            const unsigned use = it / kStages;
            bool late = false;
            if (use > 0) late = !mbar_wait(bar0 + 8 * s, (use - 1) & 1);   // the stage's previous MMAs are done
            late = __any_sync(kFullMask, late);   // the shuffles below need the whole warp
            const int gw = b0 + step * kTcPer + 4 * warp;
            unsigned char* as = smem + S::kA + s * S::kAStage;
            unsigned char* bs = smem + S::kB + s * S::kBStage;
            if (!late) {
#pragma unroll
                for (int i = 0; i < KC / 8; i++) {
                    const int e = lane + 32 * i, q = e / KC, j = e % KC;
                    if (gw + q < b1) {
                        float4 hi, lo;
                        split4(make_float4(cur.x[4 * i], cur.x[4 * i + 1], cur.x[4 * i + 2], cur.x[4 * i + 3]), hi, lo);
                        unsigned char* t = as + (4 * warp + q) * S::kATile + (j >> 3) * 256 + (j & 7) * 16;
                        *reinterpret_cast<float4*>(t) = hi;
                        *reinterpret_cast<float4*>(t + 128) = lo;
                    }
                }
                if (lane < 16 && gw + (lane >> 2) < b1) {
                    float4 hi, lo;
                    split4(cur.v, hi, lo);
                    unsigned char* t = bs + (4 * warp + (lane >> 2)) * S::kBTile + (lane & 3) * 16;
                    *reinterpret_cast<float4*>(t) = hi;
                    *reinterpret_cast<float4*>(t + 64) = lo;
                    *reinterpret_cast<float4*>(t + 128) = hi;
                    *reinterpret_cast<float4*>(t + 192) = lo;
                }
                if (lane < 4) {
                    const int g = gw + lane;
                    int m = 0;
                    if (g < b1) {
                        int lo_r = 0, hi_r = nbr - 1;   // last block row whose first block is <= g
                        while (lo_r < hi_r) {
                            const int mid = (lo_r + hi_r + 1) >> 1;
                            if (sptr[mid] <= g) lo_r = mid;
                            else hi_r = mid - 1;
                        }
                        m = lo_r | (sptr[lo_r] == g ? 256 : 0) | 512;
                    }
                    meta[s * kTcPer + 4 * warp + lane] = m;
                }
                // next step's loads go out before the barrier and land while the MMAs run
                if (step + 1 < nsteps) {
                    const int gn = gw + kTcPer;
                    load_step<KC>(cur, col_next, gn, b1, data, len, X, ldx, width, pe, pl);
                    if (step + 2 < nsteps) col_next = load_col(col, gn + kTcPer, b1, pe);
                }
            }
            fence_async_smem();
            if (__syncthreads_or(late)) {
                bad = true;
                break;
            }
            if (tid == 0) {
                tc_fence_after();
                // descriptors of the stage's first tiles; the next tiles are whole 16-byte steps further
                const uint64_t ad = smem_desc(sbase + S::kA + s * S::kAStage, 128, 256);
                const uint64_t bd = smem_desc(sbase + S::kB + s * S::kBStage, 128, 256);
                for (int b = 0; b < kTcPer; b++) {
                    const int m = meta[s * kTcPer + b];
                    if (m & 512)
                        tc_mma(tmem + (uint32_t)(m & 255) * 8, ad + (uint64_t)(b * (S::kATile >> 4)),
                               bd + (uint64_t)(b * (S::kBTile >> 4)), kIdesc, (m & 256) ? 0u : 1u);
                }
                tc_commit(bar0 + 8 * s);
            }
        }
        if (bad) break;

        // epilogue: all of the tile's MMAs are done once its last commit has arrived
        bool late = false;
        if (nsteps > 0) {
            const unsigned last = it - 1;
            late = !mbar_wait(bar0 + 8 * (last % kStages), (last / kStages) & 1);
        }
        if (__syncthreads_or(late)) {
            bad = true;
            break;
        }
        tc_fence_after();
        if (warp * 16 < KC) {   // warps 0-3: lane quarter w holds right-hand sides 16w .. 16w + 15
            const int j = warp * 16 + (lane & 15);
            for (int lr0 = 0; lr0 < nbr; lr0 += 4) {
                float d[32];
                tc_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)lr0 * 8, d);
                if (lane < 16) {
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int lr = lr0 + q;
                        if (lr < nbr) {
                            const bool has = sptr[lr + 1] > sptr[lr];
#pragma unroll
                            for (int i = 0; i < 4; i++) {
                                const long long row = 4LL * (br0 + lr) + i;
                                if (row < rows) {
                                    const float sum = has ? d[q * 8 + i] + d[q * 8 + 4 + i] : 0.f;
                                    float* yp = Y + (size_t)row * ldy + j;
                                    *yp = beta == 0.f ? alpha * sum : fmaf(alpha, sum, beta * *yp);
                                }
                            }
                        }
                    }
                }
            }
        }
        tc_fence_before();
        __syncthreads();   // tensor memory and the row-pointer cache are free for the next tile
    }

    if (bad && tid == 0) {
        atomicAdd(&g_tc_timeouts, 1u);
        // give MMAs still in flight a bounded chance to finish before the columns are released
        if (it > 0) mbar_wait(bar0 + 8 * ((it - 1) % kStages), ((it - 1) / kStages) & 1);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
}

int sm_count()
{
    static const int n = [] {
        int dev = 0, v = 148;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return v > 0 ? v : 148;
    }();
    return n;
}

template <int KC>
int launch_tc(const clspmv_b4csr_f32& m, const float* X, int ldx, float* Y, int ldy, float alpha, float beta,
              cudaStream_t st)
{
    using S = TcSmem<KC>;
    // the shared-memory limit is a per-device attribute of the function: set once per device
    static std::atomic<unsigned long long> attr_set{0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CLSPMV_ERR_CUDA;
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(attr_set.load() & bit)) {
        if (cudaFuncSetAttribute(k_b4csr_spmm_tc<KC>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kLaunch) !=
            cudaSuccess)
            return CLSPMV_ERR_CUDA;
        attr_set.fetch_or(bit);
    }
    const int ntiles = (m.b4csr_row_num + kTcTileRows - 1) / kTcTileRows;
    const int grid = std::max(1, std::min(ntiles, sm_count() * S::kPerSm));
    k_b4csr_spmm_tc<KC><<<grid, kTcThreads, S::kLaunch, st>>>(m.b4csr_row_num, m.matinfo.height, m.matinfo.width,
                                                              m.b4csr_row_ptr, m.b4csr_col_id, m.b4csr_data,
                                                              (size_t)m.b4csr_aligned_size, X, ldx, Y, ldy, alpha, beta,
                                                              ntiles);
    return after_launch(1);
}

}  // namespace

extern "C" {

int clspmv_b4csr_spmm_tc_f32(const clspmv_b4csr_f32* m, int k, const float* X, int ldx, float* Y, int ldy, float alpha,
                             float beta, clspmv_stream_t stream)
{
    if (!m || !X || !Y || !m->b4csr_row_ptr || k < 1 || ldx < k || ldy < k) return CLSPMV_ERR_ARG;
    if (m->b4csr_bwidth != 4 || m->b4csr_bheight != 4) return CLSPMV_ERR_UNSUPPORTED;
    if (k < 16 || k % 16 != 0 || k > 128) return CLSPMV_ERR_UNSUPPORTED;
    if (ldx % 4 != 0 || ((uintptr_t)X & 15) != 0 || ((uintptr_t)m->b4csr_data & 15) != 0 ||
        m->b4csr_aligned_size % 4 != 0)
        return CLSPMV_ERR_ALIGN;
    if (m->matinfo.height <= 0 || m->b4csr_row_num <= 0) return CLSPMV_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    for (int c0 = 0; c0 < k; c0 += kTcMaxKc) {
        const int kc = std::min(kTcMaxKc, k - c0);
        int rc;
        switch (kc) {
            case 16: rc = launch_tc<16>(*m, X + c0, ldx, Y + c0, ldy, alpha, beta, st); break;
            case 32: rc = launch_tc<32>(*m, X + c0, ldx, Y + c0, ldy, alpha, beta, st); break;
            case 48: rc = launch_tc<48>(*m, X + c0, ldx, Y + c0, ldy, alpha, beta, st); break;
            default: rc = launch_tc<64>(*m, X + c0, ldx, Y + c0, ldy, alpha, beta, st); break;
        }
        if (rc) return rc;
    }
    return CLSPMV_OK;
}

int clspmv_tensor_timeouts(unsigned int* count)
{
    if (!count) return CLSPMV_ERR_ARG;
    unsigned int zero = 0;
    if (cudaMemcpyFromSymbol(count, g_tc_timeouts, sizeof(unsigned int)) != cudaSuccess) return CLSPMV_ERR_CUDA;
    if (cudaMemcpyToSymbol(g_tc_timeouts, &zero, sizeof(unsigned int)) != cudaSuccess) return CLSPMV_ERR_CUDA;
    return CLSPMV_OK;
}

}  // extern "C"
