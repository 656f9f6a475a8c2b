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
#include <cerrno>
#include <cstring>
#include <string>
#include <system_error>
#include <thread>
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

// The entry lines of a MatrixMarket file as whitespace-separated tokens,
// `per` of them per entry (row, column[, value]), parsed on several host
// threads: the text is cut into ranges at whitespace, each range's tokens are
// counted, and each range then converts its tokens knowing their global
// index. Integers go through strtoll and values through strtod, the
// conversions fscanf's %lld / %lf make, so every entry is the one fscanf
// would read. Tokens past nnz entries are ignored, as by fscanf.
int parse_entries(const std::vector<char>& text, long long nnz, int per, long long height, long long width,
                  std::vector<int>& r, std::vector<int>& c, std::vector<float>& v)
{
    const size_t n = text.size() - 1;   // text ends with '\0'
    auto space = [&](size_t i) { return i >= n || std::isspace((unsigned char)text[i]); };
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nt = (int)std::max<size_t>(1, std::min<size_t>((size_t)hw, n / (1u << 20) + 1));
    std::vector<size_t> cut((size_t)nt + 1, n);
    cut[0] = 0;
    for (int t = 1; t < nt; t++) {
        size_t b = std::max(cut[t - 1], n / nt * (size_t)t);
        while (!space(b)) b++;   // never inside a token
        cut[t] = b;
    }
    std::vector<long long> count((size_t)nt, 0), first((size_t)nt + 1, 0);
    std::vector<int> bad((size_t)nt, 0);
    auto run = [&](auto body) {
        std::vector<std::thread> th;
        try {
            for (int t = 1; t < nt; t++) th.emplace_back(body, t);
        } catch (const std::system_error&) {
            for (int t = (int)th.size() + 1; t < nt; t++) body(t);   // no more threads: the rest here
        }
        body(0);
        for (std::thread& x : th) x.join();
    };
    run([&](int t) {
        long long k = 0;
        for (size_t i = cut[t]; i < cut[t + 1]; i++)
            if (!space(i) && (i == cut[t] || space(i - 1))) k++;
        count[t] = k;
    });
    for (int t = 0; t < nt; t++) first[t + 1] = first[t] + count[t];
    if (first[nt] < nnz * per) return CLSPMV_ERR_ARG;   // the file ends before nnz entries
    run([&](int t) {
        long long tok = first[t];
        size_t i = cut[t];
        while (i < cut[t + 1] && tok < nnz * per) {
            while (i < cut[t + 1] && space(i)) i++;
            if (i >= cut[t + 1]) break;
            const char* s = text.data() + i;
            char* end = nullptr;
            const long long e = tok / per;
            const int field = (int)(tok % per);
            if (field < 2) {
                errno = 0;
                const long long x = std::strtoll(s, &end, 10);
                if (end == s || errno || (field == 0 ? (x < 1 || x > height) : (x < 1 || x > width))) bad[t] = 1;
                else (field == 0 ? r : c)[(size_t)e] = (int)(x - 1);
            } else {
                const double d = std::strtod(s, &end);
                if (end == s) bad[t] = 1;
                else v[(size_t)e] = (float)d;
            }
            if (bad[t]) return;
            if (!space((size_t)(end - text.data()))) {   // a token with trailing characters
                bad[t] = 1;
                return;
            }
            i = (size_t)(end - text.data());
            tok++;
        }
    });
    for (int t = 0; t < nt; t++)
        if (bad[t]) return CLSPMV_ERR_ARG;
    return CLSPMV_OK;
}

// Stable sort of (row, column) pairs with their values, as std::stable_sort
// by (row, column) would leave them: a stable counting sort by row, then a
// stable sort by column of each row not already in column order (files
// written column by column come out of the first step sorted).
void sort_entries(int* r, int* c, float* v, size_t n, int height)
{
    std::vector<size_t> start((size_t)height + 1, 0);
    for (size_t i = 0; i < n; i++) start[(size_t)r[i] + 1]++;
    for (int h = 0; h < height; h++) start[(size_t)h + 1] += start[(size_t)h];
    std::vector<unsigned> perm(n);
    {
        std::vector<size_t> fill(start.begin(), start.end() - 1);
        for (size_t i = 0; i < n; i++) perm[fill[(size_t)r[i]]++] = (unsigned)i;
    }
    // rows are independent: ranges of rows on separate host threads; short
    // rows by insertion (stable), long ones by std::stable_sort
    auto sort_rows = [&](int h0, int h1) {
        for (int h = h0; h < h1; h++) {
            unsigned* b = perm.data() + start[(size_t)h];
            const size_t len = start[(size_t)h + 1] - start[(size_t)h];
            bool ordered = true;
            for (size_t k = 1; k < len && ordered; k++) ordered = c[b[k - 1]] <= c[b[k]];
            if (ordered) continue;
            if (len <= 32) {
                for (size_t k = 1; k < len; k++) {
                    const unsigned x = b[k];
                    size_t j = k;
                    for (; j > 0 && c[b[j - 1]] > c[x]; j--) b[j] = b[j - 1];
                    b[j] = x;
                }
            } else {
                std::stable_sort(b, b + len, [&](unsigned x, unsigned y) { return c[x] < c[y]; });
            }
        }
    };
    const int nt = (int)std::max<size_t>(1, std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()),
                                                              n / (1u << 16) + 1));
    std::vector<int> cut((size_t)nt + 1, height);
    cut[0] = 0;
    for (int t = 1; t < nt; t++)   // about n / nt entries per range
        cut[t] = (int)(std::lower_bound(start.begin(), start.end(), n / nt * (size_t)t) - start.begin());
    for (int t = 1; t <= nt; t++) cut[t] = std::max(cut[t], cut[t - 1]);
    std::vector<std::thread> th;
    try {
        for (int t = 1; t < nt; t++) th.emplace_back(sort_rows, cut[t], cut[t + 1]);
    } catch (const std::system_error&) {
        for (int t = (int)th.size() + 1; t < nt; t++) sort_rows(cut[t], cut[t + 1]);
    }
    sort_rows(cut[0], cut[1]);
    for (std::thread& x : th) x.join();
    std::vector<int> tr(r, r + n), tc(c, c + n);
    std::vector<float> tv(v, v + n);
    for (size_t i = 0; i < n; i++) {
        r[i] = tr[perm[i]];
        c[i] = tc[perm[i]];
        v[i] = tv[perm[i]];
    }
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
    // the entry lines, whole, into memory
    std::vector<char> text;
    {
        const long here = ftell(f);
        size_t guess = 0;
        if (here >= 0 && fseek(f, 0, SEEK_END) == 0) {
            const long endpos = ftell(f);
            if (endpos > here) guess = (size_t)(endpos - here);
            fseek(f, here, SEEK_SET);
        }
        text.reserve(guess + 1);
        char chunk[1 << 16];
        size_t got;
        while ((got = fread(chunk, 1, sizeof(chunk), f)) > 0) text.insert(text.end(), chunk, chunk + got);
        text.push_back('\0');
    }
    fclose(f);
    std::vector<int> r((size_t)nnz), c((size_t)nnz);
    std::vector<float> v((size_t)nnz, 1.0f);
    const int rc = parse_entries(text, nnz, has_value ? 3 : 2, height, width, r, c, v);
    if (rc) return rc;
    std::vector<char>().swap(text);
    long long diag = 0;
    for (long long i = 0; i < nnz; i++) diag += r[(size_t)i] == c[(size_t)i];
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
    if (!if_sorted_coo(mat)) {
        // sort_entries counts rows in [0, height); a mirrored entry of a
        // non-square symmetric file has row = its column, which can reach
        // width - 1 >= height: such input takes sort_coo, which compares keys
        // and indexes nothing by row (the reference sorts it the same way)
        bool rows_in_range = true;
        for (size_t i = 0; i < total && rows_in_range; i++) rows_in_range = mat->coo_row_id[i] < height;
        if (rows_in_range) sort_entries(mat->coo_row_id, mat->coo_col_id, mat->coo_data, total, (int)height);
        else sort_coo(mat);
    }
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
