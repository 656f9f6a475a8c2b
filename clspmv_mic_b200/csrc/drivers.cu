// drivers.cu — the reference's benchmark drivers behind the C ABI.
//
// clSpMV ships one driver per format (src/spmv_<fmt>.cpp): convert the COO
// matrix, build every kernel variant, check each against the host COO
// product, time it and print the best. clspmv_run_method_f32 does the same
// for this library's kernels; the C++ spmv_<fmt>() names of the reference
// (compat.cpp) are thin calls into it. clspmv_bandwidth_test replaces
// method 0 (src/mem_bandwidth.cpp) and clspmv_cocktail_evaluate_f32 the
// Cocktail evaluate() (src/spmv_cocktail.cpp:1431-1455).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "clspmv_b200.h"
#include "api_internal.h"
#include "matrix_storage.h"
#include "spmv_serial.h"
#include "common.cuh"

using namespace clspmv;

namespace {

__global__ void k_copy4(const float4* __restrict__ a, float4* __restrict__ b, size_t n4)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}

__global__ void k_nothing() {}

// Random gathers x[idx[i]] with the SpMV kernels' load forms: indices
// streamed with 128-bit loads, x read with an L2 keep policy, through L1
// with allocation (GX = 0) or without (GX = 1), as ld_gx.
template <int GX>
__global__ void __launch_bounds__(kBlock) k_gather(const int* __restrict__ idx, const float* __restrict__ x,
                                                   float* __restrict__ out, long long n4)
{
    const uint64_t pol_s = policy_evict_first(), pol_x = policy_evict_last();
    float acc = 0.0f;
    for (long long i = blockIdx.x * (long long)kBlock + threadIdx.x; i < n4; i += (long long)gridDim.x * kBlock) {
        const int4 c = ld_stream_i4(idx + 4 * i, pol_s);
        acc += ld_gx<GX>(x + c.x, pol_x) + ld_gx<GX>(x + c.y, pol_x) + ld_gx<GX>(x + c.z, pol_x) + ld_gx<GX>(x + c.w, pol_x);
    }
    out[blockIdx.x * (long long)kBlock + threadIdx.x] = acc;
}

__global__ void k_fill_random(int* idx, long long n, int range, unsigned seed)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        unsigned long long h = (unsigned long long)i * 0x9E3779B97F4A7C15ull + seed;   // splitmix64 step
        h ^= h >> 30;
        h *= 0xBF58476D1CE4E5B9ull;
        h ^= h >> 27;
        h *= 0x94D049BB133111EBull;
        h ^= h >> 31;
        idx[i] = (int)(h % (unsigned long long)range);
    }
}

coo_matrix<int, float>* as_tmpl(const clspmv_coo_f32* c)
{
    return reinterpret_cast<coo_matrix<int, float>*>(const_cast<clspmv_coo_f32*>(c));
}

// two_vec_compare (src/util.cpp:93-131): L2 distance, and the largest
// difference of magnitudes, absolute and relative.
void compare(const std::vector<float>& ref, const std::vector<float>& got, clspmv_bench_variant& v)
{
    double sum = 0.0, maxd = 0.0, maxr = 0.0;
    for (size_t i = 0; i < ref.size(); i++) {
        const double d = (double)ref[i] - (double)got[i];
        sum += d * d;
        const float a = std::fabs(ref[i]), b = std::fabs(got[i]);
        const double diff = std::fabs((double)a - (double)b);
        const float mx = a > b ? a : b;
        if (diff > maxd) maxd = diff;
        if (mx > 0 && diff / mx > maxr) maxr = diff / mx;
    }
    v.distance = std::sqrt(sum);
    v.max_diff = maxd;
    v.max_diff_ratio = maxr;
}

// Device x, y and timing events for one driver run.
struct Session {
    const clspmv_coo_f32* coo = nullptr;
    int ntimes = 1;
    int verbose = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float* dx = nullptr;
    float* dy = nullptr;
    std::vector<float> ref, got;

    int open(const clspmv_coo_f32* c, int nt, int verb, bool arbitrary_x)
    {
        coo = c;
        ntimes = nt < 1 ? 1 : nt;
        verbose = verb;
        const int n = c->matinfo.width, m = c->matinfo.height;
        std::vector<float> x(n);
        if (arbitrary_x) initVectorArbitrary<int, float>(x.data(), n);
        else initVectorOne<int, float>(x.data(), n);
        ref.assign(m, 0.0f);
        coo_spmv<int, float>(as_tmpl(c), x.data(), ref.data(), n);   // spmv_only, src/util.cpp:85-91
        got.assign(m, 0.0f);
        int rc = cuda_status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        if (!rc) rc = cuda_status(cudaEventCreate(&e0));
        if (!rc) rc = cuda_status(cudaEventCreate(&e1));
        if (!rc) rc = cuda_status(cudaMalloc(&dx, sizeof(float) * ((size_t)n + 4)));
        if (!rc) rc = cuda_status(cudaMalloc(&dy, sizeof(float) * ((size_t)m + 4)));
        if (!rc) rc = cuda_status(cudaMemcpy(dx, x.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
        return rc;
    }

    void close()
    {
        if (dx) cudaFree(dx);
        if (dy) cudaFree(dy);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (st) cudaStreamDestroy(st);
    }

    // One variant: check from y = 0, 3 untimed runs, `ntimes` timed runs.
    template <class Launch>
    int run(Launch&& launch, clspmv_bench_variant& v)
    {
        const int m = coo->matinfo.height;
        int rc = cuda_status(cudaMemsetAsync(dy, 0, sizeof(float) * m, st));
        if (!rc) rc = launch(st);
        if (!rc) rc = cuda_status(cudaMemcpyAsync(got.data(), dy, sizeof(float) * m, cudaMemcpyDeviceToHost, st));
        if (!rc) rc = cuda_status(cudaStreamSynchronize(st));
        if (rc) return v.status = rc;
        compare(ref, got, v);
        for (int i = 0; !rc && i < 3; i++) rc = launch(st);
        if (!rc) rc = cuda_status(cudaEventRecord(e0, st));
        for (int i = 0; !rc && i < ntimes; i++) rc = launch(st);
        if (!rc) rc = cuda_status(cudaEventRecord(e1, st));
        if (!rc) rc = cuda_status(cudaEventSynchronize(e1));
        float ms = 0.0f;
        if (!rc) rc = cuda_status(cudaEventElapsedTime(&ms, e0, e1));
        if (rc) return v.status = rc;
        v.status = CLSPMV_OK;
        v.ms = (double)ms / ntimes;
        v.gflops = 2.0 * (double)coo->matinfo.nnz / (v.ms * 1e-3) / 1e9;
        if (verbose)
            printf("\nCorrectness Check: Distance %e max diff %e max diff ratio %e vec size %d\n", v.distance,
                   v.max_diff, v.max_diff_ratio, m);
        return CLSPMV_OK;
    }
};

const char* method_name(int method)
{
    switch (method) {
        case CLSPMV_METHOD_CSR_SCALAR: return "CSR scalar";
        case CLSPMV_METHOD_CSR_VECTOR: return "CSR vector";
        case CLSPMV_METHOD_BDIA: return "BDIA";
        case CLSPMV_METHOD_DIA: return "DIA";
        case CLSPMV_METHOD_ELL: return "ELL";
        case CLSPMV_METHOD_COO: return "COO";
        case CLSPMV_METHOD_BELL: return "BELL";
        case CLSPMV_METHOD_BCSR: return "BCSR";
        case CLSPMV_METHOD_SELL: return "SELL";
        case CLSPMV_METHOD_SBELL: return "SBELL";
        case CLSPMV_METHOD_CSR_MERGE: return "CSR merge";
    }
    return "?";
}

// Block shapes in the reference drivers' sweep order: width 4 then 8,
// height 1, 2, 4, 8 (src/spmv_bell.cpp:361-362).
const unsigned kShapes[8][2] = {{1, 4}, {2, 4}, {4, 4}, {8, 4}, {1, 8}, {2, 8}, {4, 8}, {8, 8}};

int run_csr(Session& s, int method, clspmv_bench_result& r)
{
    clspmv_csr_f32 csr, pad, dev;
    memset(&csr, 0, sizeof(csr));
    int rc = clspmv_coo2csr_f32(s.coo, &csr);
    if (rc) return rc;
    auto with_device = [&](const clspmv_csr_f32& host, auto&& body) {
        memset(&dev, 0, sizeof(dev));
        int rc2 = clspmv_upload_csr_f32(&host, &dev);
        if (!rc2) rc2 = body();
        clspmv_device_free_csr_f32(&dev);
        return rc2;
    };
    if (method == CLSPMV_METHOD_CSR_SCALAR) {
        // the reference times the plain and the 4-padded rows (src/spmv_csr_scalar.cpp:695)
        for (int padding : {1, 4}) {
            clspmv_bench_variant& v = r.v[r.nvariants++];
            v.param0 = padding;
            memset(&pad, 0, sizeof(pad));
            const clspmv_csr_f32* host = &csr;
            if (padding > 1) {
                const int prc = clspmv_pad_csr_f32(&csr, &pad, padding);
                if (prc) { v.status = prc; continue; }
                host = &pad;
            }
            v.status = with_device(*host, [&] {
                return s.run([&](cudaStream_t st) { return launch_csr_scalar(&dev, s.dx, s.dy, 1.0f, 1.0f, st, false); }, v);
            });
            if (padding > 1) clspmv_free_csr_f32(&pad);
        }
    } else if (method == CLSPMV_METHOD_CSR_VECTOR) {
        memset(&pad, 0, sizeof(pad));
        rc = clspmv_pad_csr_f32(&csr, &pad, 16);   // src/spmv_csr_vector.cpp:644
        if (!rc) {
            rc = with_device(pad, [&] {
                for (int lanes : {2, 4, 8, 16, 32}) {
                    clspmv_bench_variant& v = r.v[r.nvariants++];
                    v.param0 = lanes;
                    s.run([&](cudaStream_t st) { return launch_csr_vector(&dev, s.dx, s.dy, 1.0f, 1.0f, lanes, st, false); }, v);
                }
                return CLSPMV_OK;
            });
            clspmv_free_csr_f32(&pad);
        }
    } else {
        clspmv_bench_variant& v = r.v[r.nvariants++];
        v.status = with_device(csr, [&] {
            int* plan = nullptr;
            const int tiles = clspmv_csr_merge_tiles(dev.matinfo.height, dev.matinfo.nnz);
            int rc2 = cuda_status(cudaMalloc(&plan, sizeof(int) * 2 * ((size_t)tiles + 1)));
            if (!rc2) rc2 = launch_csr_merge_plan(&dev, plan, s.st);
            if (!rc2)
                rc2 = s.run([&](cudaStream_t st) { return launch_csr_merge(&dev, plan, s.dx, s.dy, 1.0f, 1.0f, st, false); }, v);
            if (plan) cudaFree(plan);
            return rc2;
        });
    }
    clspmv_free_csr_f32(&csr);
    return rc;
}

// Host conversion, upload, timed run and release of one variant.
template <class Host, class Convert, class Upload, class Launch, class FreeDev, class FreeHost>
void one_variant(Session& s, clspmv_bench_variant& v, Convert&& convert, Upload&& upload, Launch&& launch,
                 FreeDev&& free_dev, FreeHost&& free_host)
{
    Host host, dev;
    memset(&host, 0, sizeof(host));
    memset(&dev, 0, sizeof(dev));
    int rc = convert(&host);
    if (rc) { v.status = rc; return; }
    rc = upload(&host, &dev);
    if (!rc) rc = s.run([&](cudaStream_t st) { return launch(&dev, st); }, v);
    else v.status = rc;
    free_dev(&dev);
    free_host(&host);
}

void print_variant(const char* name, const clspmv_bench_variant& v, int index)
{
    if (v.status) {
        printf("%s variant %d (%d, %d) skipped: %s\n", name, index, v.param0, v.param1, clspmv_status_string(v.status));
        return;
    }
    printf("\n------------------------------------------------------------------------\n");
    printf("%s best time %f ms best method %d GFLOPS %f", name, v.ms, index, v.gflops);
    printf("\n------------------------------------------------------------------------\n");
}

}  // namespace

extern "C" {

int clspmv_run_method_f32(const clspmv_coo_f32* coo, int method, int ntimes, int verbose, clspmv_bench_result* out)
{
    if (!coo || coo->matinfo.height <= 0 || coo->matinfo.width <= 0 || coo->matinfo.nnz < 0) return CLSPMV_ERR_ARG;
    if (method < CLSPMV_METHOD_CSR_SCALAR || method > CLSPMV_METHOD_CSR_MERGE) return CLSPMV_ERR_ARG;
    if (!clspmv_is_sorted_coo_f32(coo)) return CLSPMV_ERR_NOT_SORTED;
    clspmv_bench_result r;
    memset(&r, 0, sizeof(r));
    r.method = method;
    r.best = -1;
    Session s;
    int rc = s.open(coo, ntimes, verbose, method == CLSPMV_METHOD_SBELL);
    if (rc) {
        s.close();
        return rc;
    }
    const char* name = method_name(method);
    const float one = 1.0f;
    switch (method) {
        case CLSPMV_METHOD_CSR_SCALAR:
        case CLSPMV_METHOD_CSR_VECTOR:
        case CLSPMV_METHOD_CSR_MERGE:
            rc = run_csr(s, method, r);
            break;
        case CLSPMV_METHOD_COO:
            one_variant<clspmv_coo_f32>(
                s, r.v[r.nvariants++], [&](clspmv_coo_f32* h) { return clspmv_coo2coo_f32(coo, h); },
                clspmv_upload_coo_f32,
                [&](const clspmv_coo_f32* d, cudaStream_t st) { return launch_coo(d, s.dx, s.dy, one, one, st, false); },
                clspmv_device_free_coo_f32, clspmv_free_coo_f32);
            break;
        case CLSPMV_METHOD_DIA:
            one_variant<clspmv_dia_f32>(
                s, r.v[r.nvariants++],
                [&](clspmv_dia_f32* h) { return clspmv_coo2dia_f32(coo, h, CLSPMV_GPU_ALIGNMENT); },
                clspmv_upload_dia_f32,
                [&](const clspmv_dia_f32* d, cudaStream_t st) { return launch_dia(d, s.dx, s.dy, one, one, st, false); },
                clspmv_device_free_dia_f32, clspmv_free_dia_f32);
            break;
        case CLSPMV_METHOD_BDIA:
            one_variant<clspmv_bdia_f32>(
                s, r.v[r.nvariants++],
                [&](clspmv_bdia_f32* h) { return clspmv_coo2bdia_f32(coo, h, CLSPMV_GPU_ALIGNMENT); },
                clspmv_upload_bdia_f32,
                [&](const clspmv_bdia_f32* d, cudaStream_t st) { return launch_bdia(d, s.dx, s.dy, one, one, st, false); },
                clspmv_device_free_bdia_f32, clspmv_free_bdia_f32);
            break;
        case CLSPMV_METHOD_ELL:
            one_variant<clspmv_ell_f32>(
                s, r.v[r.nvariants++],
                [&](clspmv_ell_f32* h) { return clspmv_coo2ell_f32(coo, h, CLSPMV_GPU_ALIGNMENT, 0); },
                clspmv_upload_ell_f32,
                [&](const clspmv_ell_f32* d, cudaStream_t st) { return launch_ell(d, s.dx, s.dy, one, one, st, false); },
                clspmv_device_free_ell_f32, clspmv_free_ell_f32);
            break;
        case CLSPMV_METHOD_SELL:
            for (unsigned sh : {(unsigned)CLSPMV_WARPSIZE, (unsigned)CLSPMV_SELL_GROUP_SIZE}) {
                clspmv_bench_variant& v = r.v[r.nvariants++];
                v.param0 = (int)sh;
                one_variant<clspmv_sell_f32>(
                    s, v, [&](clspmv_sell_f32* h) { return clspmv_coo2sell_f32(coo, h, sh); }, clspmv_upload_sell_f32,
                    [&](const clspmv_sell_f32* d, cudaStream_t st) { return launch_sell(d, s.dx, s.dy, one, one, st, false); },
                    clspmv_device_free_sell_f32, clspmv_free_sell_f32);
            }
            break;
        case CLSPMV_METHOD_BELL:
        case CLSPMV_METHOD_BCSR:
        case CLSPMV_METHOD_SBELL:
            for (const auto& shape : kShapes) {
                const unsigned bh = shape[0], bw = shape[1];
                clspmv_bench_variant& v = r.v[r.nvariants++];
                v.param0 = (int)bh;
                v.param1 = (int)bw;
                if (method == CLSPMV_METHOD_BELL)
                    one_variant<clspmv_b4ell_f32>(
                        s, v, [&](clspmv_b4ell_f32* h) { return clspmv_coo2b4ell_f32(coo, h, bw, bh, CLSPMV_GPU_ALIGNMENT, 0); },
                        clspmv_upload_b4ell_f32,
                        [&](const clspmv_b4ell_f32* d, cudaStream_t st) { return launch_b4ell(d, s.dx, s.dy, one, one, st, false); },
                        clspmv_device_free_b4ell_f32, clspmv_free_b4ell_f32);
                else if (method == CLSPMV_METHOD_BCSR)
                    one_variant<clspmv_b4csr_f32>(
                        s, v, [&](clspmv_b4csr_f32* h) { return clspmv_coo2b4csr_f32(coo, h, bw, bh, CLSPMV_GPU_ALIGNMENT); },
                        clspmv_upload_b4csr_f32,
                        [&](const clspmv_b4csr_f32* d, cudaStream_t st) { return launch_b4csr(d, s.dx, s.dy, one, one, st, false); },
                        clspmv_device_free_b4csr_f32, clspmv_free_b4csr_f32);
                else
                    one_variant<clspmv_sbell_f32>(
                        s, v, [&](clspmv_sbell_f32* h) { return clspmv_coo2sbell_f32(coo, h, bw, bh, CLSPMV_WARPSIZE); },
                        clspmv_upload_sbell_f32,
                        [&](const clspmv_sbell_f32* d, cudaStream_t st) { return launch_sbell(d, s.dx, s.dy, one, one, st, false); },
                        clspmv_device_free_sbell_f32, clspmv_free_sbell_f32);
            }
            break;
    }
    s.close();
    for (int i = 0; i < r.nvariants; i++) {
        const clspmv_bench_variant& v = r.v[i];
        if (verbose) print_variant(name, v, i);
        if (v.status == CLSPMV_OK && (r.best < 0 || v.ms < r.best_ms)) {
            r.best = i;
            r.best_ms = v.ms;
            r.best_gflops = v.gflops;
        }
    }
    if (verbose && r.best >= 0) {
        const clspmv_bench_variant& b = r.v[r.best];
        printf("\n------------------------------------------------------------------------\n");
        printf("Final %s best time %f ms GFLOPS %f variant %d (%d, %d)", name, r.best_ms, r.best_gflops, r.best,
               b.param0, b.param1);
        printf("\n------------------------------------------------------------------------\n");
    }
    if (out) *out = r;
    if (rc) return rc;
    if (r.best >= 0) return CLSPMV_OK;
    for (int i = 0; i < r.nvariants; i++)
        if (r.v[i].status != CLSPMV_ERR_REFUSED && r.v[i].status != CLSPMV_ERR_UNSUPPORTED) return r.v[i].status;
    return CLSPMV_ERR_REFUSED;
}

int clspmv_bandwidth_test(size_t bytes, int ntimes, int verbose, double* copy_gbs, double* launch_us)
{
    if (bytes < 16 || ntimes < 1) return CLSPMV_ERR_ARG;
    const size_t n4 = bytes / 16;
    float4 *a = nullptr, *b = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = cuda_status(cudaMalloc(&a, n4 * 16));
    if (!rc) rc = cuda_status(cudaMalloc(&b, n4 * 16));
    if (!rc) rc = cuda_status(cudaMemset(a, 0, n4 * 16));
    if (!rc) rc = cuda_status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (!rc) rc = cuda_status(cudaEventCreate(&e0));
    if (!rc) rc = cuda_status(cudaEventCreate(&e1));
    int sms = 148;
    if (!rc) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    float ms_copy = 0.0f, ms_empty = 0.0f;
    for (int pass = 0; !rc && pass < 2; pass++) {
        for (int i = 0; !rc && i < 3; i++) {   // warm-up
            if (pass == 0) k_copy4<<<sms * 8, 256, 0, st>>>(a, b, n4);
            else k_nothing<<<1, 32, 0, st>>>();
            rc = after_launch(1);
        }
        if (!rc) rc = cuda_status(cudaEventRecord(e0, st));
        for (int i = 0; !rc && i < ntimes; i++) {
            if (pass == 0) k_copy4<<<sms * 8, 256, 0, st>>>(a, b, n4);
            else k_nothing<<<1, 32, 0, st>>>();
            rc = after_launch(1);
        }
        if (!rc) rc = cuda_status(cudaEventRecord(e1, st));
        if (!rc) rc = cuda_status(cudaEventSynchronize(e1));
        if (!rc) rc = cuda_status(cudaEventElapsedTime(pass == 0 ? &ms_copy : &ms_empty, e0, e1));
    }
    if (!rc) {
        const double gbs = 2.0 * (double)(n4 * 16) / ((double)ms_copy / ntimes * 1e-3) / 1e9;
        const double us = (double)ms_empty / ntimes * 1e3;
        if (copy_gbs) *copy_gbs = gbs;
        if (launch_us) *launch_us = us;
        if (verbose)
            printf("\nCopy bandwidth %f GB/s over %zu bytes; launch overhead %f us (mean of %d)\n", gbs, n4 * 16, us,
                   ntimes);
    }
    if (a) cudaFree(a);
    if (b) cudaFree(b);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    return rc;
}

int clspmv_gather_test(int x_len, long long count, int ntimes, int verbose, double* gathers_per_s)
{
    if (x_len < 1 || count < 4 || ntimes < 1) return CLSPMV_ERR_ARG;
    const long long n4 = count / 4;
    int* idx = nullptr;
    float *x = nullptr, *out = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = sms * 8;
    int rc = cuda_status(cudaMalloc(&idx, sizeof(int) * 4 * n4));
    if (!rc) rc = cuda_status(cudaMalloc(&x, sizeof(float) * x_len));
    if (!rc) rc = cuda_status(cudaMalloc(&out, sizeof(float) * grid * kBlock));
    if (!rc) rc = cuda_status(cudaMemset(x, 0, sizeof(float) * x_len));
    if (!rc) rc = cuda_status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (!rc) rc = cuda_status(cudaEventCreate(&e0));
    if (!rc) rc = cuda_status(cudaEventCreate(&e1));
    if (!rc) {
        k_fill_random<<<grid, kBlock, 0, st>>>(idx, 4 * n4, x_len, 12345u);
        rc = after_launch(1);
    }
    // the load form the SpMV kernels use (CLSPMV_GATHER_FORM as in spmv_api.cu)
    const char* gf = getenv("CLSPMV_GATHER_FORM");
    auto gather = [&]() {
        if (gf && atoi(gf) == 1) k_gather<1><<<grid, kBlock, 0, st>>>(idx, x, out, n4);
        else k_gather<0><<<grid, kBlock, 0, st>>>(idx, x, out, n4);
        return after_launch(1);
    };
    for (int i = 0; !rc && i < 3; i++) rc = gather();
    if (!rc) rc = cuda_status(cudaEventRecord(e0, st));
    for (int i = 0; !rc && i < ntimes; i++) rc = gather();
    if (!rc) rc = cuda_status(cudaEventRecord(e1, st));
    if (!rc) rc = cuda_status(cudaEventSynchronize(e1));
    float ms = 0.0f;
    if (!rc) rc = cuda_status(cudaEventElapsedTime(&ms, e0, e1));
    if (!rc) {
        const double g = (double)(4 * n4) / ((double)ms / ntimes * 1e-3);
        if (gathers_per_s) *gathers_per_s = g;
        if (verbose) printf("\nRandom gathers from %d floats: %.1f G/s (%lld per launch)\n", x_len, g / 1e9, 4 * n4);
    }
    if (idx) cudaFree(idx);
    if (x) cudaFree(x);
    if (out) cudaFree(out);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    return rc;
}

int clspmv_cocktail_evaluate_f32(const clspmv_cocktail_f32* host, const float* vec, const float* res,
                                 const float* coores, int ntimes, int verbose, double* ms_out, double* gflops_out,
                                 double* max_diff_out)
{
    if (!host || !vec || !res || ntimes < 1) return CLSPMV_ERR_ARG;
    const int n = host->mat_width, m = host->mat_height;
    clspmv_cocktail_handle* h = nullptr;
    int rc = clspmv_cocktail_upload_f32(host, &h);
    if (rc) return rc;
    float *dx = nullptr, *dy = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    rc = cuda_status(cudaMalloc(&dx, sizeof(float) * ((size_t)n + 4)));
    if (!rc) rc = cuda_status(cudaMalloc(&dy, sizeof(float) * ((size_t)m + 4)));
    if (!rc) rc = cuda_status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (!rc) rc = cuda_status(cudaEventCreate(&e0));
    if (!rc) rc = cuda_status(cudaEventCreate(&e1));
    if (!rc) rc = cuda_status(cudaMemcpy(dx, vec, sizeof(float) * n, cudaMemcpyHostToDevice));
    if (!rc) rc = cuda_status(cudaMemcpy(dy, res, sizeof(float) * m, cudaMemcpyHostToDevice));
    // check_and_time (src/spmv_cocktail.cpp:1134-1154): one SpMV, compare, then time
    if (!rc) rc = clspmv_cocktail_spmv_f32(h, dx, dy, 1.0f, 1.0f, st);
    std::vector<float> got(m);
    if (!rc) rc = cuda_status(cudaMemcpyAsync(got.data(), dy, sizeof(float) * m, cudaMemcpyDeviceToHost, st));
    if (!rc) rc = cuda_status(cudaStreamSynchronize(st));
    if (!rc && coores) {
        clspmv_bench_variant v;
        memset(&v, 0, sizeof(v));
        compare(std::vector<float>(coores, coores + m), got, v);
        if (max_diff_out) *max_diff_out = v.max_diff;
        if (verbose)
            printf("\nCorrectness Check: Distance %e max diff %e max diff ratio %e vec size %d\n", v.distance,
                   v.max_diff, v.max_diff_ratio, m);
    }
    for (int i = 0; !rc && i < 3; i++) rc = clspmv_cocktail_spmv_f32(h, dx, dy, 1.0f, 1.0f, st);
    if (!rc) rc = cuda_status(cudaEventRecord(e0, st));
    for (int i = 0; !rc && i < ntimes; i++) rc = clspmv_cocktail_spmv_f32(h, dx, dy, 1.0f, 1.0f, st);
    if (!rc) rc = cuda_status(cudaEventRecord(e1, st));
    if (!rc) rc = cuda_status(cudaEventSynchronize(e1));
    float ms = 0.0f;
    if (!rc) rc = cuda_status(cudaEventElapsedTime(&ms, e0, e1));
    if (!rc) {
        const double per = (double)ms / ntimes;
        const double gf = 2.0 * (double)host->mat_nnz / (per * 1e-3) / 1e9;
        if (ms_out) *ms_out = per;
        if (gflops_out) *gflops_out = gf;
        if (verbose) printf("\nCocktail gpu time %lf ms GFLOPS %lf\n\n", per, gf);
    }
    if (dx) cudaFree(dx);
    if (dy) cudaFree(dy);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    clspmv_cocktail_free(h);
    return rc;
}

}  // extern "C"
