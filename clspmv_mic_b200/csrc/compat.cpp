// compat.cpp — the reference's C++ host API with its own names: util.h
// helpers (src/util.cpp), ReadMMF (src/fileio.cpp), the per-format
// benchmark drivers (src/spmv_<fmt>.cpp) and the Cocktail runtime calls
// (src/spmv_cocktail.cpp). Everything that touches the GPU goes through
// the C ABI of clspmv_b200.h.
#include <cuda_runtime.h>
#include <sys/time.h>

#include <algorithm>
#include <cassert>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "clspmv_b200.h"
#include "fileio.h"
#include "spmv_cocktail.h"
#include "spmv_drivers.h"
#include "spmv_serial.h"
#include "util.h"

namespace {
thread_local int g_compat_status = CLSPMV_OK;

int note(int rc, const char* where)
{
    g_compat_status = rc;
    if (rc)
        fprintf(stderr, "clspmv: %s failed: %s%s%s\n", where, clspmv_status_string(rc), rc == CLSPMV_ERR_CUDA ? ": " : "",
                rc == CLSPMV_ERR_CUDA ? clspmv_last_cuda_error() : "");
    return rc;
}

int cuda_rc(cudaError_t e) { return e == cudaSuccess ? CLSPMV_OK : CLSPMV_ERR_CUDA; }

clspmv_coo_f32* as_c(coo_matrix<int, float>* m) { return reinterpret_cast<clspmv_coo_f32*>(m); }
clspmv_cocktail_f32* as_c(cocktail<int, int, float>* m) { return reinterpret_cast<clspmv_cocktail_f32*>(m); }

// The reference drivers take any COO; the C ABI wants it sorted.
void run_driver(coo_matrix<int, float>* mat, int method, int ntimes)
{
    printMatInfo(mat);   // sorts an unsorted matrix, as the reference's drivers do through it
    note(clspmv_run_method_f32(as_c(mat), method, ntimes, 1, nullptr), "spmv driver");
}

// Lower-cased next whitespace-separated token of the header line.
std::string lower(const char* s)
{
    std::string t(s);
    for (char& c : t) c = (char)std::tolower((unsigned char)c);
    return t;
}

int read_mmf(const char* filename, coo_matrix<int, float>* mat)
{
    init_coo_matrix(*mat);
    FILE* f = fopen(filename, "r");
    if (!f) return CLSPMV_ERR_ARG;
    char tok[5][128];
    // "%%MatrixMarket matrix coordinate <field> <symmetry>"
    for (int i = 0; i < 5; i++)
        if (fscanf(f, "%127s", tok[i]) != 1) { fclose(f); return CLSPMV_ERR_ARG; }
    if (lower(tok[2]) != "coordinate") { fclose(f); return CLSPMV_ERR_UNSUPPORTED; }
    const std::string field = lower(tok[3]), sym = lower(tok[4]);
    if (field == "complex") { fclose(f); return CLSPMV_ERR_UNSUPPORTED; }
    const bool has_value = field == "real" || field == "integer" || field == "double";
    const bool symmetric = sym == "symmetric";
    // comment lines, then "height width nnz"
    char line[1100];
    long long height = -1, width = -1, nnz = -1;
    while (fgets(line, sizeof(line), f)) {
        const char* p = line;
        while (*p && std::isspace((unsigned char)*p)) p++;
        if (!*p || *p == '%') continue;
        if (sscanf(p, "%lld %lld %lld", &height, &width, &nnz) != 3) { fclose(f); return CLSPMV_ERR_ARG; }
        break;
    }
    if (height <= 0 || width <= 0 || nnz < 0 || height > 0x7fffffff || width > 0x7fffffff || (symmetric ? 2 * nnz : nnz) > 0x7fffffff) {
        fclose(f);
        return CLSPMV_ERR_ARG;
    }
    std::vector<int> r((size_t)nnz), c((size_t)nnz);
    std::vector<float> v((size_t)nnz, 1.0f);
    long long diag = 0;
    for (long long i = 0; i < nnz; i++) {
        long long ri, ci;
        if (fscanf(f, "%lld %lld", &ri, &ci) != 2 || ri < 1 || ri > height || ci < 1 || ci > width) {
            fclose(f);
            return CLSPMV_ERR_ARG;
        }
        if (has_value) {
            double d = 0.0;
            if (fscanf(f, "%lf", &d) != 1) { fclose(f); return CLSPMV_ERR_ARG; }
            v[i] = (float)d;
        }
        r[i] = (int)(ri - 1);
        c[i] = (int)(ci - 1);
        if (r[i] == c[i]) diag++;
    }
    fclose(f);
    const size_t total = symmetric ? (size_t)(2 * nnz - diag) : (size_t)nnz;
    mat->matinfo.height = (int)height;
    mat->matinfo.width = (int)width;
    mat->matinfo.nnz = (int)total;
    mat->coo_row_id = (int*)malloc(sizeof(int) * (total ? total : 1));
    mat->coo_col_id = (int*)malloc(sizeof(int) * (total ? total : 1));
    mat->coo_data = (float*)malloc(sizeof(float) * (total ? total : 1));
    if (!mat->coo_row_id || !mat->coo_col_id || !mat->coo_data) {
        free_coo_matrix(*mat);
        init_coo_matrix(*mat);
        return CLSPMV_ERR_ALLOC;
    }
    size_t k = 0;
    for (size_t i = 0; i < (size_t)nnz; i++) {
        mat->coo_row_id[k] = r[i];
        mat->coo_col_id[k] = c[i];
        mat->coo_data[k++] = v[i];
        if (symmetric && r[i] != c[i]) {   // mirrored entry right after its source, src/fileio.cpp:72-84
            mat->coo_row_id[k] = c[i];
            mat->coo_col_id[k] = r[i];
            mat->coo_data[k++] = v[i];
        }
    }
    if (!if_sorted_coo(mat)) sort_coo(mat);
    return CLSPMV_OK;
}

}  // namespace

// ---------------------------------------------------------------- util.h

double timestamp()
{
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}

int findPaddedSize(int realSize, int alignment)
{
    return realSize % alignment == 0 ? realSize : realSize + alignment - realSize % alignment;
}

void pad_csr(csr_matrix<int, float>* source, csr_matrix<int, float>* dest, int alignment)
{
    pad_csr<int, float>(source, dest, alignment);
}

double distance(float* vec1, float* vec2, int size)
{
    double sum = 0.0;
    for (int i = 0; i < size; i++) {
        const double d = (double)vec1[i] - (double)vec2[i];
        sum += d * d;
    }
    return std::sqrt(sum);
}

void spmv_only(coo_matrix<int, float>* mat, float* vec, float* coores)
{
    initVectorZero<int, float>(coores, mat->matinfo.height);
    coo_spmv<int, float>(mat, vec, coores, mat->matinfo.width);
}

void two_vec_compare(float* coovec, float* newvec, int size)
{
    double maxdiff = 0.0, maxratio = 0.0;
    int maxid = 0, shown = 0;
    for (int i = 0; i < size; i++) {
        const float a = std::fabs(coovec[i]), b = std::fabs(newvec[i]);
        const double diff = std::fabs((double)a - (double)b);
        const float mx = a > b ? a : b;
        if (diff > maxdiff) { maxdiff = diff; maxid = i; }
        if (mx > 0 && diff / mx > maxratio) maxratio = diff / mx;
        if (coovec[i] != newvec[i] && shown < 10) {
            printf("Error i %d coo res %f res %f \n", i, coovec[i], newvec[i]);
            shown++;
        }
    }
    if (size > 0) printf("Max diff id %d coo res %f res %f \n", maxid, coovec[maxid], newvec[maxid]);
    printf("\nCorrectness Check: Distance %e max diff %e max diff ratio %e vec size %d\n", distance(coovec, newvec, size),
           maxdiff, maxratio, size);
}

void correctness_check(coo_matrix<int, float>* mat, float* vec, float* res)
{
    std::vector<float> coores((size_t)mat->matinfo.height);
    spmv_only(mat, vec, coores.data());
    two_vec_compare(coores.data(), res, mat->matinfo.height);
}

void printMatInfo(coo_matrix<int, float>* mat)
{
    const int nnz = mat->matinfo.nnz, h = mat->matinfo.height;
    printf("\nMatInfo: Width %d Height %d NNZ %d\n", mat->matinfo.width, h, nnz);
    int minoff = mat->matinfo.width, maxoff = -mat->matinfo.width;
    int below = 0, near_below = 0, near_above = 0, above = 0;
    for (int i = 0; i < nnz; i++) {
        const int d = mat->coo_row_id[i] - mat->coo_col_id[i];
        minoff = std::min(minoff, d);
        maxoff = std::max(maxoff, d);
        if (d < -15) below++;
        else if (d < 0) near_below++;
        else if (d < 16) near_above++;
        else above++;
    }
    printf("Max Offset %d Min Offset %d\n", maxoff, minoff);
    printf("Histogram: <-15: %d -15~-1 %d < 0-15 %d > 16 %d\n", below, near_below, near_above, above);
    if (!if_sorted_coo(mat)) sort_coo(mat);
    // 16-float cache lines touched per row (a new line each time the column's line changes)
    long long sum = 0;
    int maxl = 0, minl = h > 0 ? 0x7fffffff : 0;
    for (int row = 0, i = 0; row < h; row++) {
        int lines = 0, last = -1;
        for (; i < nnz && mat->coo_row_id[i] == row; i++) {
            const int line = mat->coo_col_id[i] / 16;
            if (lines == 0 || line != last) { lines++; last = line; }
        }
        maxl = std::max(maxl, lines);
        minl = std::min(minl, lines);
        sum += lines;
    }
    printf("Cacheline usage per row: max %d min %d avg %f\n", maxl, minl, h ? (double)sum / (double)h : 0.0);
}

void rearrange_bell_4col(bell_matrix<int, float>* mat, int alignment)
{
    const int bw = (int)mat->bell_bwidth, bh = (int)mat->bell_bheight;
    const int blocks = mat->bell_block_num, rows = mat->bell_row_num, old_len = mat->bell_height_aligned;
    assert(bw % 4 == 0);
    const int w4n = bw / 4;
    const int len = findPaddedSize(4 * rows, alignment);
    std::vector<float> out((size_t)len * bh * w4n * blocks, 0.0f);
    // old: [block][h][w][row]; new: [block][w4][h][row*4 + w%4]
    for (int b = 0; b < blocks; b++)
        for (int hh = 0; hh < bh; hh++)
            for (int w = 0; w < bw; w++)
                for (int j = 0; j < rows; j++)
                    out[(size_t)b * len * w4n * bh + (size_t)(w / 4) * len * bh + (size_t)hh * len + (size_t)j * 4 + w % 4] =
                        mat->bell_data[(size_t)b * old_len * bw * bh + (size_t)hh * old_len * bw + (size_t)w * old_len + j];
    float* data = (float*)malloc(sizeof(float) * (out.size() ? out.size() : 1));
    std::copy(out.begin(), out.end(), data);
    free(mat->bell_data);
    mat->bell_data = data;
    mat->bell_float4_aligned = len;
    for (int i = 0; i < old_len * blocks; i++) mat->bell_col_id[i] /= 4;
}

// ---------------------------------------------------------------- fileio.h

void ReadMMF(char* filename, coo_matrix<int, float>* mat)
{
    const int rc = read_mmf(filename, mat);
    if (rc) fprintf(stderr, "ReadMMF: cannot read %s: %s\n", filename, clspmv_status_string(rc));
}

extern "C" int clspmv_read_mmf_f32(const char* filename, clspmv_coo_f32* out)
{
    if (!filename || !out) return CLSPMV_ERR_ARG;
    return read_mmf(filename, reinterpret_cast<coo_matrix<int, float>*>(out));
}

// ---------------------------------------------------------- spmv drivers

void spmv_csr_scalar(char*, coo_matrix<int, float>* mat, int, int ntimes, cl_device_type) { run_driver(mat, CLSPMV_METHOD_CSR_SCALAR, ntimes); }
void spmv_csr_vector(char*, coo_matrix<int, float>* mat, int, int ntimes, cl_device_type) { run_driver(mat, CLSPMV_METHOD_CSR_VECTOR, ntimes); }
void spmv_coo(char*, coo_matrix<int, float>* mat, int, int ntimes, cl_device_type) { run_driver(mat, CLSPMV_METHOD_COO, ntimes); }
void spmv_dia(char*, coo_matrix<int, float>* mat, int, int ntimes, cl_device_type) { run_driver(mat, CLSPMV_METHOD_DIA, ntimes); }
void spmv_bdia(char*, coo_matrix<int, float>* mat, int, int ntimes, cl_device_type) { run_driver(mat, CLSPMV_METHOD_BDIA, ntimes); }
void spmv_ell(char*, coo_matrix<int, float>* mat, int, int ntimes, cl_device_type) { run_driver(mat, CLSPMV_METHOD_ELL, ntimes); }
void spmv_sell(char*, coo_matrix<int, float>* mat, int, int ntimes, cl_device_type) { run_driver(mat, CLSPMV_METHOD_SELL, ntimes); }
void spmv_bell(char*, coo_matrix<int, float>* mat, int, int ntimes, cl_device_type) { run_driver(mat, CLSPMV_METHOD_BELL, ntimes); }
void spmv_sbell(char*, coo_matrix<int, float>* mat, int, int ntimes, cl_device_type) { run_driver(mat, CLSPMV_METHOD_SBELL, ntimes); }
void spmv_bcsr(char*, coo_matrix<int, float>* mat, int, int ntimes, cl_device_type) { run_driver(mat, CLSPMV_METHOD_BCSR, ntimes); }

void bandwidth_test(char*, cl_device_type, int)
{
    // the reference sweeps 32 KB .. 32 MB vectors (src/mem_bandwidth.cpp:22)
    for (size_t bytes = 32u << 10; bytes <= (32u << 20); bytes <<= 1)
        if (note(clspmv_bandwidth_test(bytes, 100, 1, nullptr, nullptr), "bandwidth_test")) return;
}

// ------------------------------------------------------- Cocktail runtime

int cocktail_last_status(void) { return g_compat_status; }

void init_cocktail_gpu(cocktail_gpu& mat) { memset(&mat, 0, sizeof(mat)); }

void free_cocktail_gpu(cocktail_gpu& mat)
{
    if (mat.vec) cudaFree(reinterpret_cast<void*>(mat.vec));
    if (mat.res) cudaFree(reinterpret_cast<void*>(mat.res));
    if (mat.handle) clspmv_cocktail_free(mat.handle);
    memset(&mat, 0, sizeof(mat));
}

void init_cocktail_kernels(cocktail_kernels& k) { memset(&k, 0, sizeof(k)); }

void free_cocktail_kernels(cocktail_kernels& k)
{
    if (k.cmdQueue) cudaStreamDestroy(reinterpret_cast<cudaStream_t>(k.cmdQueue));
    memset(&k, 0, sizeof(k));
}

void init_mat_kernels(cocktail<int, int, float>& cpumat, float* vec, float* res, cocktail_gpu& gpumat,
                      cocktail_kernels& kernels, bool /*use_tex*/)
{
    init_cocktail_gpu(gpumat);
    init_cocktail_kernels(kernels);
    cudaStream_t st = nullptr;
    int rc = cuda_rc(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    kernels.cmdQueue = reinterpret_cast<cl_command_queue>(st);
    if (!rc) rc = clspmv_cocktail_upload_f32(as_c(&cpumat), &gpumat.handle);
    void *x = nullptr, *y = nullptr;
    gpumat.vec_size = cpumat.mat_width;
    gpumat.res_size = cpumat.mat_height;
    if (!rc) rc = cuda_rc(cudaMalloc(&x, sizeof(float) * ((size_t)cpumat.mat_width + 4)));
    gpumat.vec = reinterpret_cast<cl_mem>(x);
    if (!rc) rc = cuda_rc(cudaMalloc(&y, sizeof(float) * ((size_t)cpumat.mat_height + 4)));
    gpumat.res = reinterpret_cast<cl_mem>(y);
    if (!rc && vec) rc = cuda_rc(cudaMemcpy(x, vec, sizeof(float) * cpumat.mat_width, cudaMemcpyHostToDevice));
    if (!rc && res) rc = cuda_rc(cudaMemcpy(y, res, sizeof(float) * cpumat.mat_height, cudaMemcpyHostToDevice));
#define COPY_FLAG(f) gpumat.f = cpumat.f;
    COPY_FLAG(ifusebdia) COPY_FLAG(ifusedia) COPY_FLAG(ifusesbell) COPY_FLAG(ifusebell) COPY_FLAG(ifusebcsr)
    COPY_FLAG(ifusesell) COPY_FLAG(ifuseell) COPY_FLAG(ifusecsr) COPY_FLAG(ifusecoo)
#undef COPY_FLAG
    kernels.handle = gpumat.handle;
    kernels.vec = gpumat.vec;
    kernels.res = gpumat.res;
    kernels.nnz = cpumat.mat_nnz;
    note(rc, "init_mat_kernels");
}

void free_mat_kernels(cocktail_gpu& gpumat, cocktail_kernels& kernels)
{
    if (kernels.cmdQueue) cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(kernels.cmdQueue));
    free_cocktail_kernels(kernels);
    free_cocktail_gpu(gpumat);
    g_compat_status = CLSPMV_OK;
}

void do_spmv(cocktail_kernels& kernels, cl_context&, cl_command_queue& cmdQueue, int ntimes)
{
    cudaStream_t st = reinterpret_cast<cudaStream_t>(cmdQueue);
    int rc = kernels.handle ? CLSPMV_OK : CLSPMV_ERR_ARG;
    for (int i = 0; !rc && i < ntimes; i++)
        rc = clspmv_cocktail_spmv_f32(kernels.handle, reinterpret_cast<const float*>(kernels.vec),
                                      reinterpret_cast<float*>(kernels.res), 1.0f, 1.0f, st);
    if (!rc) rc = cuda_rc(cudaStreamSynchronize(st));
    note(rc, "do_spmv");
}

namespace {
void copy_sync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cl_command_queue q, const char* where)
{
    cudaStream_t st = reinterpret_cast<cudaStream_t>(q);
    int rc = (dst && src) ? CLSPMV_OK : CLSPMV_ERR_ARG;
    if (!rc) rc = cuda_rc(cudaMemcpyAsync(dst, src, bytes, kind, st));
    if (!rc) rc = cuda_rc(cudaStreamSynchronize(st));
    note(rc, where);
}
}  // namespace

void cpy_vector_from_cpu(cocktail_gpu& g, cl_context&, cl_command_queue& q, float* vec, int n)
{
    copy_sync(g.vec, vec, sizeof(float) * (size_t)std::min(n, g.vec_size), cudaMemcpyHostToDevice, q, "cpy_vector_from_cpu");
}

void cpy_vector_from_gpu(cocktail_gpu& g, cl_context&, cl_command_queue& q, cl_mem vec, int n)
{
    copy_sync(g.vec, vec, sizeof(float) * (size_t)std::min(n, g.vec_size), cudaMemcpyDeviceToDevice, q, "cpy_vector_from_gpu");
}

void cpy_result_from_cpu(cocktail_gpu& g, cl_context&, cl_command_queue& q, float* res, int n)
{
    copy_sync(g.res, res, sizeof(float) * (size_t)std::min(n, g.res_size), cudaMemcpyHostToDevice, q, "cpy_result_from_cpu");
}

void cpy_result_from_gpu(cocktail_gpu& g, cl_context&, cl_command_queue& q, cl_mem res, int n)
{
    copy_sync(g.res, res, sizeof(float) * (size_t)std::min(n, g.res_size), cudaMemcpyDeviceToDevice, q, "cpy_result_from_gpu");
}

void cpy_result_to_cpu(cocktail_gpu& g, cl_context&, cl_command_queue& q, float* res, int n)
{
    copy_sync(res, g.res, sizeof(float) * (size_t)std::min(n, g.res_size), cudaMemcpyDeviceToHost, q, "cpy_result_to_cpu");
}

void cpy_result_to_gpu(cocktail_gpu& g, cl_context&, cl_command_queue& q, cl_mem res, int n)
{
    copy_sync(res, g.res, sizeof(float) * (size_t)std::min(n, g.res_size), cudaMemcpyDeviceToDevice, q, "cpy_result_to_gpu");
}

void check_and_time(cocktail_gpu& gpumat, cocktail_kernels& kernels, cl_context& context, cl_command_queue& cmdQueue,
                    float* result, float* coores, int res_size, int nnz)
{
    const int ntimes = 1000;   // src/spmv_cocktail.cpp:1136
    cpy_result_from_cpu(gpumat, context, cmdQueue, result, res_size);
    do_spmv(kernels, context, cmdQueue, 1);
    std::vector<float> got((size_t)res_size);
    cpy_result_to_cpu(gpumat, context, cmdQueue, got.data(), res_size);
    if (g_compat_status) return;
    two_vec_compare(coores, got.data(), res_size);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(cmdQueue);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    int rc = CLSPMV_OK;
    for (int i = 0; !rc && i < ntimes; i++)
        rc = clspmv_cocktail_spmv_f32(kernels.handle, reinterpret_cast<const float*>(kernels.vec),
                                      reinterpret_cast<float*>(kernels.res), 1.0f, 1.0f, st);
    cudaEventRecord(e1, st);
    if (!rc) rc = cuda_rc(cudaEventSynchronize(e1));
    float ms = 0.0f;
    if (!rc) rc = cuda_rc(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (note(rc, "check_and_time")) return;
    const double per = (double)ms / ntimes;
    printf("\nCocktail gpu time %lf ms GFLOPS %lf\n\n", per, 2.0 * (double)nnz / (per * 1e-3) / 1e9);
}

void output_cocktail_info(cocktail<int, int, float>& m)
{
    printf("\n*****************************\nCocktail matrix info\n*****************************\n");
    printf("Original Matrix Width %d Height %d nnz %d\n\n", m.mat_width, m.mat_height, m.mat_nnz);
    if (m.ifusebdia)
        printf("Use bdia\nImplementation no. %d\nNNZ %d\nBand num %d total diagonals %d\n------------------------------\n",
               m.bdia_meth_num, m.bdia.matinfo.nnz, m.bdia.bdia_band_num, m.bdia.bdia_bptr[m.bdia.bdia_band_num]);
    if (m.ifusedia)
        printf("Use dia\nImplementation no. %d\nNNZ %d\nNum of diagonals %d\n------------------------------\n",
               m.dia_meth_num, m.dia.matinfo.nnz, m.dia.dia_num);
    if (m.ifusesbell)
        printf("Use sbell\nImplementation no. %d\nNNZ %d\nblock height %d block width %d slice height %d\n"
               "------------------------------\n",
               m.sbell_meth_num, m.sbell.matinfo.nnz, m.sbell.sbell_bheight, m.sbell.sbell_bwidth, m.sbell.sbell_slice_height);
    if (m.ifusebell)
        printf("Use bell\nImplementation no. %d\nNNZ %d\nblock height %d block width %d block num %d\n"
               "------------------------------\n",
               m.bell_meth_num, m.bell.matinfo.nnz, m.bell.b4ell_bheight, m.bell.b4ell_bwidth, m.bell.b4ell_block_num);
    if (m.ifusebcsr)
        printf("Use bcsr\nImplementation no. %d\nNNZ %d\nblock height %d block width %d total blocks %d\n"
               "------------------------------\n",
               m.bcsr_meth_num, m.bcsr.matinfo.nnz, m.bcsr.b4csr_bheight, m.bcsr.b4csr_bwidth, m.bcsr.b4csr_block_num);
    if (m.ifusesell)
        printf("Use sell\nImplementation no. %d\nNNZ %d\nslice height %d slice num %d\n------------------------------\n",
               m.sell_meth_num, m.sell.matinfo.nnz, m.sell.sell_slice_height, m.sell.sell_slice_num);
    if (m.ifuseell)
        printf("Use ell\nImplementation no. %d\nNNZ %d\nell num %d\n------------------------------\n", m.ell_meth_num,
               m.ell.matinfo.nnz, m.ell.ell_num);
    if (m.ifusecsr)
        printf("Use csr\nImplementation no. %d\nNNZ %d\ngroup num %d\n------------------------------\n", m.csr_meth_num,
               m.csr.matinfo.nnz, m.csr_group_num);
    if (m.ifusecoo)
        printf("Use coo\nImplementation no. %d\nNNZ %d\ngroup num %d\n------------------------------\n", m.coo_meth_num,
               m.coo.matinfo.nnz, m.coo_group_num);
}

void evaluate(cocktail<int, int, float>& cpumat, float* vec, float* res, float* coores)
{
    output_cocktail_info(cpumat);
    cocktail_gpu gpumat;
    cocktail_kernels kernels;
    init_mat_kernels(cpumat, vec, res, gpumat, kernels, true);
    if (!g_compat_status)
        check_and_time(gpumat, kernels, kernels.context, kernels.cmdQueue, res, coores, cpumat.mat_height, cpumat.mat_nnz);
    const int rc = g_compat_status;
    free_mat_kernels(gpumat, kernels);
    g_compat_status = rc;
}
