// cocktail_rt.cu — the Cocktail runtime: device residency of a partitioned
// matrix and y <- alpha * A * x + beta * y over all of its parts.
//
// The reference (src/spmv_cocktail.cpp) uploads each part into cl_mem
// buffers (cpy_<fmt>_mat, :304-1009), binds one kernel per part
// (set_cocktail_kernels, :1012-1085) and runs them one after another on an
// in-order queue, each reading and writing y (do_spmv, :1088-1132), then
// clFinish. Here each part's kernel runs on its own stream, forked from and
// joined back into the caller's stream with events, so the parts of one
// SpMV overlap on the GPU; every part adds alpha * A_p * x into y with
// red.global.add (beta is applied once, first). The fork/join is legal
// inside CUDA graph capture, so a caller can capture one SpMV and replay it
// without host round trips (the reference's A^k x loop, src/eval.cpp:19-72,
// synchronises after every step).
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include "clspmv_b200.h"
#include "api_internal.h"

using namespace clspmv;

struct clspmv_cocktail_handle {
    clspmv_cocktail_f32 dev;          // part structs with device pointers
    int* chunk_plan = nullptr;        // first row of every nonzero chunk of the CSR part
    int nparts = 0;
    FusedPlan* fused = nullptr;       // one persistent launch over all parts (two or more parts)
    clspmv_sell_plan* sell_plan = nullptr;   // the SELL part's length plan, when it reads well under the stored slots
    int schedule = CLSPMV_SCHEDULE_AUTO;
    int csr_lanes = 0;                // CSR part: 0 nonzero chunks, T > 0 CSR-vector with T lanes per row
    cudaStream_t streams[9] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[9] = {};
    // A^k x iteration: a graph of kIterUnroll steps, captured on `cap` for
    // one (x, y, alpha, beta) and replayed on the caller's stream
    cudaStream_t cap = nullptr;
    cudaGraphExec_t iter_exec = nullptr;
    const float* iter_x = nullptr;
    const float* iter_y = nullptr;
    float iter_alpha = 0.f, iter_beta = 0.f;
};

namespace {

enum Part { P_BDIA, P_DIA, P_SBELL, P_BELL, P_BCSR, P_SELL, P_ELL, P_CSR, P_COO, P_COUNT };

// CLSPMV_COCKTAIL_SELL_PLAN=0 keeps the padded SELL read for SELL parts (measurements)
bool sell_plan_disabled()
{
    static const bool v = [] {
        const char* e = getenv("CLSPMV_COCKTAIL_SELL_PLAN");
        return e && atoi(e) == 0;
    }();
    return v;
}

bool uses(const clspmv_cocktail_f32& c, int p)
{
    switch (p) {
        case P_BDIA: return c.ifusebdia;
        case P_DIA: return c.ifusedia;
        case P_SBELL: return c.ifusesbell;
        case P_BELL: return c.ifusebell;
        case P_BCSR: return c.ifusebcsr;
        case P_SELL: return c.ifusesell;
        case P_ELL: return c.ifuseell;
        case P_CSR: return c.ifusecsr;
        case P_COO: return c.ifusecoo;
    }
    return false;
}

int launch_part(const clspmv_cocktail_handle* h, int p, const float* x, float* y, float alpha, float beta, cudaStream_t st,
                bool atomic)
{
    const clspmv_cocktail_f32& d = h->dev;
    switch (p) {
        case P_BDIA: return launch_bdia(&d.bdia, x, y, alpha, beta, st, atomic);
        case P_DIA: return launch_dia(&d.dia, x, y, alpha, beta, st, atomic);
        case P_SBELL: return launch_sbell(&d.sbell, x, y, alpha, beta, st, atomic);
        case P_BELL: return launch_b4ell(&d.bell, x, y, alpha, beta, st, atomic);
        case P_BCSR: return launch_b4csr(&d.bcsr, x, y, alpha, beta, st, atomic);
        case P_SELL:
            if (h->sell_plan) return launch_sell_plan(&d.sell, h->sell_plan, x, y, alpha, beta, st, atomic);
            return launch_sell(&d.sell, x, y, alpha, beta, st, atomic);
        case P_ELL: return launch_ell(&d.ell, x, y, alpha, beta, st, atomic);
        case P_CSR:
            if (h->csr_lanes > 0) return launch_csr_vector(&d.csr, x, y, alpha, beta, h->csr_lanes, st, atomic);
            return launch_csr_chunk(&d.csr, h->chunk_plan, x, y, alpha, beta, st, atomic);
        case P_COO: return launch_coo(&d.coo, x, y, alpha, beta, st, atomic);
    }
    return CLSPMV_ERR_ARG;
}

void release(clspmv_cocktail_handle* h)
{
    clspmv_cocktail_f32& d = h->dev;
    if (d.ifusebdia) clspmv_device_free_bdia_f32(&d.bdia);
    if (d.ifusedia) clspmv_device_free_dia_f32(&d.dia);
    if (d.ifusesbell) clspmv_device_free_sbell_f32(&d.sbell);
    if (d.ifusebell) clspmv_device_free_b4ell_f32(&d.bell);
    if (d.ifusebcsr) clspmv_device_free_b4csr_f32(&d.bcsr);
    if (d.ifusesell) clspmv_device_free_sell_f32(&d.sell);
    if (d.ifuseell) clspmv_device_free_ell_f32(&d.ell);
    if (d.ifusecsr) clspmv_device_free_csr_f32(&d.csr);
    if (d.ifusecoo) clspmv_device_free_coo_f32(&d.coo);
    if (h->chunk_plan) cudaFree(h->chunk_plan);
    for (int i = 0; i < P_COUNT; i++) {
        if (h->streams[i]) cudaStreamDestroy(h->streams[i]);
        if (h->join[i]) cudaEventDestroy(h->join[i]);
    }
    if (h->fork) cudaEventDestroy(h->fork);
    if (h->sell_plan) clspmv_sell_plan_free(h->sell_plan);
    if (h->fused) fused_plan_free(h->fused);
    if (h->iter_exec) cudaGraphExecDestroy(h->iter_exec);
    if (h->cap) cudaStreamDestroy(h->cap);
}

constexpr int kIterUnroll = 16;   // steps per replayed graph

// n steps of the reference's loop (src/eval.cpp:44-50): y <- alpha*A*x + beta*y,
// then the first mat_height entries of x <- y (cpy_vector_from_gpu,
// src/spmv_cocktail.cpp:1510-1556), stream ordered, no host synchronisation.
int iterate_steps(clspmv_cocktail_handle* h, float* x, float* y, float alpha, float beta, int n, cudaStream_t st)
{
    const size_t bytes = sizeof(float) * (size_t)h->dev.mat_height;
    for (int i = 0; i < n; i++) {
        int rc = clspmv_cocktail_spmv_f32(h, x, y, alpha, beta, st);
        if (!rc && bytes) rc = cuda_status(cudaMemcpyAsync(x, y, bytes, cudaMemcpyDeviceToDevice, st));
        if (rc) return rc;
    }
    return CLSPMV_OK;
}

int iteration_graph(clspmv_cocktail_handle* h, float* x, float* y, float alpha, float beta)
{
    if (h->iter_exec && h->iter_x == x && h->iter_y == y && h->iter_alpha == alpha && h->iter_beta == beta)
        return CLSPMV_OK;
    if (h->iter_exec) {
        cudaGraphExecDestroy(h->iter_exec);
        h->iter_exec = nullptr;
    }
    int rc = CLSPMV_OK;
    if (!h->cap) rc = cuda_status(cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking));
    if (rc) return rc;
    if ((rc = cuda_status(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal)))) return rc;
    const int rc_steps = iterate_steps(h, x, y, alpha, beta, kIterUnroll, h->cap);
    cudaGraph_t g = nullptr;
    rc = cuda_status(cudaStreamEndCapture(h->cap, &g));   // always ends the capture
    if (rc_steps || rc) {
        if (g) cudaGraphDestroy(g);
        return rc_steps ? rc_steps : rc;
    }
    rc = cuda_status(cudaGraphInstantiate(&h->iter_exec, g, 0));
    cudaGraphDestroy(g);
    if (rc) {
        h->iter_exec = nullptr;
        return rc;
    }
    h->iter_x = x;
    h->iter_y = y;
    h->iter_alpha = alpha;
    h->iter_beta = beta;
    return CLSPMV_OK;
}

}  // namespace

extern "C" {

int clspmv_cocktail_upload_f32(const clspmv_cocktail_f32* host, clspmv_cocktail_handle** out)
{
    if (!host || !out) return CLSPMV_ERR_ARG;
    *out = nullptr;
    clspmv_cocktail_handle* h = new (std::nothrow) clspmv_cocktail_handle();
    if (!h) return CLSPMV_ERR_ALLOC;
    memset(&h->dev, 0, sizeof(h->dev));
    const clspmv_cocktail_f32& c = *host;
    clspmv_cocktail_f32& d = h->dev;
    // flags, variants and sizes are copied; arrays are uploaded part by part
    memcpy(&d, &c, offsetof(clspmv_cocktail_f32, bdia));
    d.ifusebdia = d.ifusedia = d.ifusesbell = d.ifusebell = d.ifusebcsr = false;
    d.ifusesell = d.ifuseell = d.ifusecsr = d.ifusecoo = false;
    int rc = CLSPMV_OK;
#define UP(flag, part, fn)                                  \
    if (!rc && c.flag) {                                    \
        rc = fn(&c.part, &d.part);                          \
        if (!rc) d.flag = true;                             \
    }
    UP(ifusebdia, bdia, clspmv_upload_bdia_f32)
    UP(ifusedia, dia, clspmv_upload_dia_f32)
    UP(ifusesbell, sbell, clspmv_upload_sbell_f32)
    UP(ifusebell, bell, clspmv_upload_b4ell_f32)
    UP(ifusebcsr, bcsr, clspmv_upload_b4csr_f32)
    UP(ifusesell, sell, clspmv_upload_sell_f32)
    UP(ifuseell, ell, clspmv_upload_ell_f32)
    UP(ifusecsr, csr, clspmv_upload_csr_f32)
    UP(ifusecoo, coo, clspmv_upload_coo_f32)
#undef UP
    if (!rc && d.ifusesell && !sell_plan_disabled()) {
        // SELL parts of uneven rows (slices padded to their longest row) take
        // the padding-free walk when its lines come to under 3/4 of the slots
        clspmv_sell_plan* sp = nullptr;
        if (clspmv_sell_plan_create(&d.sell, &sp) == CLSPMV_OK) {
            const long long slots = 8LL * (c.sell.sell_slice_ptr ? c.sell.sell_slice_ptr[c.sell.sell_slice_num] : 0);
            if (clspmv_sell_plan_line_bytes(sp) < slots * 3 / 4) h->sell_plan = sp;
            else clspmv_sell_plan_free(sp);
        }
        cudaGetLastError();
    }
    if (!rc && d.ifusecsr) {
        const int nplan = clspmv_csr_chunk_plan_size(d.csr.matinfo.nnz);
        rc = cuda_status(cudaMalloc(&h->chunk_plan, sizeof(int) * (size_t)(nplan > 0 ? nplan : 1)));
        if (!rc) rc = launch_csr_chunk_plan(&d.csr, h->chunk_plan, 0);
        if (!rc) rc = cuda_status(cudaStreamSynchronize(0));
    }
    for (int p = 0; !rc && p < P_COUNT; p++) {
        if (!uses(d, p)) continue;
        h->nparts++;
        rc = cuda_status(cudaStreamCreateWithFlags(&h->streams[p], cudaStreamNonBlocking));
        if (!rc) rc = cuda_status(cudaEventCreateWithFlags(&h->join[p], cudaEventDisableTiming));
    }
    if (!rc) rc = cuda_status(cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming));
    if (!rc && h->nparts >= 2) {
        // a part layout the fused kernel does not cover keeps the per-part launches
        const int frc = fused_plan_create(&h->dev, h->chunk_plan, &h->fused);
        if (frc != CLSPMV_ERR_UNSUPPORTED) rc = frc;
    }
    if (rc) {
        release(h);
        delete h;
        return rc;
    }
    *out = h;
    return CLSPMV_OK;
}

int clspmv_cocktail_spmv_f32(clspmv_cocktail_handle* h, const float* x, float* y, float alpha, float beta,
                             clspmv_stream_t stream)
{
    if (!h || !x || !y) return CLSPMV_ERR_ARG;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int rows = h->dev.mat_height;
    if (h->nparts == 0) return launch_prescale(y, rows, beta, st);
    if (h->nparts == 1) {
        for (int p = 0; p < P_COUNT; p++)
            if (uses(h->dev, p)) return launch_part(h, p, x, y, alpha, beta, st, false);
    }
    if (h->schedule == CLSPMV_SCHEDULE_FUSED) {
        if (!h->fused) return CLSPMV_ERR_UNSUPPORTED;
        if ((reinterpret_cast<uintptr_t>(x) & 15u) == 0) return fused_spmv(h->fused, x, y, alpha, beta, st);
    }
    int rc = launch_prescale(y, rows, beta, st);
    if (rc) return rc;
    rc = cuda_status(cudaEventRecord(h->fork, st));
    for (int p = 0; !rc && p < P_COUNT; p++) {
        if (!uses(h->dev, p)) continue;
        rc = cuda_status(cudaStreamWaitEvent(h->streams[p], h->fork, 0));
        if (!rc) rc = launch_part(h, p, x, y, alpha, 1.0f, h->streams[p], true);
        if (!rc) rc = cuda_status(cudaEventRecord(h->join[p], h->streams[p]));
        if (!rc) rc = cuda_status(cudaStreamWaitEvent(st, h->join[p], 0));
    }
    return rc;
}

int clspmv_cocktail_iterate_f32(clspmv_cocktail_handle* h, float* x, float* y, float alpha, float beta, int iterations,
                                clspmv_stream_t stream)
{
    if (!h || !x || !y || x == y || iterations < 0) return CLSPMV_ERR_ARG;
    if (h->dev.mat_width < h->dev.mat_height) return CLSPMV_ERR_ARG;   // x must hold a copy of y
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int full = iterations / kIterUnroll, rest = iterations % kIterUnroll;
    int rc = CLSPMV_OK;
    if (full > 0) {
        rc = iteration_graph(h, x, y, alpha, beta);
        for (int i = 0; !rc && i < full; i++) rc = cuda_status(cudaGraphLaunch(h->iter_exec, st));
        if (!rc) rc = after_launch(0);
    }
    if (!rc) rc = iterate_steps(h, x, y, alpha, beta, rest, st);
    return rc;
}

int clspmv_cocktail_set_schedule(clspmv_cocktail_handle* h, int schedule)
{
    if (!h || schedule < CLSPMV_SCHEDULE_AUTO || schedule > CLSPMV_SCHEDULE_PER_PART) return CLSPMV_ERR_ARG;
    if (schedule == CLSPMV_SCHEDULE_FUSED && !h->fused) return CLSPMV_ERR_UNSUPPORTED;
    h->schedule = schedule;
    if (h->iter_exec) {   // the cached iteration graph was captured under the old schedule
        cudaGraphExecDestroy(h->iter_exec);
        h->iter_exec = nullptr;
    }
    return CLSPMV_OK;
}

int clspmv_cocktail_fused_items(const clspmv_cocktail_handle* h) { return h ? fused_plan_items(h->fused) : -1; }

int clspmv_cocktail_sell_planned(const clspmv_cocktail_handle* h) { return h ? (h->sell_plan != nullptr) : -1; }

int clspmv_cocktail_set_csr_lanes(clspmv_cocktail_handle* h, int lanes)
{
    if (!h || !(lanes == 0 || lanes == 1 || lanes == 2 || lanes == 4 || lanes == 8 || lanes == 16 || lanes == 32))
        return CLSPMV_ERR_ARG;
    h->csr_lanes = lanes;
    if (h->iter_exec) {   // the cached iteration graph was captured with the old kernel
        cudaGraphExecDestroy(h->iter_exec);
        h->iter_exec = nullptr;
    }
    return CLSPMV_OK;
}

int clspmv_cocktail_device_view(const clspmv_cocktail_handle* h, clspmv_cocktail_f32* out)
{
    if (!h || !out) return CLSPMV_ERR_ARG;
    *out = h->dev;
    return CLSPMV_OK;
}

int clspmv_cocktail_free(clspmv_cocktail_handle* h)
{
    if (!h) return CLSPMV_ERR_ARG;
    release(h);
    delete h;
    return CLSPMV_OK;
}

}  // extern "C"
