// pg_noalloc.cu -- pg_sweep_noalloc: one value-iteration sweep that
// allocates no memory.
//
// Some callers cannot call cudaMalloc: a host that gives the solver a fixed
// device-memory budget carved out of its own pool, an embedding whose
// allocator owns the device, or code that must not allocate after start-up
// (cudaMalloc can synchronise the device and fail under fragmentation).  The
// staged API (pg_load_problem / pg_sweep) allocates its buffers itself, so
// those callers cannot use it.  This entry point takes every input and
// output as a device pointer the caller already holds and runs the cell-form
// sweep kernel on them; the only working memory the sweep needs -- one L1
// and one max-norm partial per thread block, plus the two reduced totals --
// lives in a fixed array compiled into the library.
//
// The working array is a file-scope __device__ variable, so every GPU that
// loads the library holds it (1 MiB) until the process exits.  Every call
// shares it and it keeps the last call's contents; each call writes every
// slot it reads before reading it and clears the two totals first.  Calls
// that overlap on the GPU (on different streams, or from different host
// threads) race on it.  The call is synchronous: it reads the two totals
// back and waits for its stream, so it must not be issued on a stream that
// is being captured into a CUDA graph.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "pg_kernels.h"
#include "pg_types.h"

namespace {

// Block partials the working array holds; the cell-form kernel runs one
// 128-thread block per 128 cells, so a grid may have at most
// 65536 * 128 = 8,388,608 cells.
constexpr int64_t kMaxParts = 65536;
constexpr int64_t kMaxCells = kMaxParts * pg::kCellThreads;

// [0, kMaxParts) L1 partials, [kMaxParts, 2 kMaxParts) max-norm partials,
// then the L1 total and the max-norm.  In host code this name stands for the
// variable; it is never a device address there.
static __device__ __align__(256) double g_sweep_scratch[2 * kMaxParts + 2];

// The array's device address in each CUDA context, looked up on the first
// call made with that context current.  The module holding the array is
// loaded once per context, so a caller that makes its own driver-API context
// current (cuCtxCreate) gets that context's copy, not the primary context's.
// The current context is read through the driver entry point the runtime
// hands out, so the library does not link libcuda itself.
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
std::mutex g_scratch_mu;
std::vector<std::pair<CUcontext, double*>> g_scratch_ptr;

// The context current on this thread (null when none is yet).
int current_context(CUcontext* ctx) {
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !f)
            return pg::set_last_error(PG_ECUDA, "cuCtxGetCurrent is not available from the driver");
        fn = reinterpret_cast<CtxGetCurrentFn>(f);
    }
    *ctx = nullptr;
    if (fn(ctx) != CUDA_SUCCESS)
        return pg::set_last_error(PG_ECUDA, "cuCtxGetCurrent failed");
    return PG_OK;
}

int scratch_on_current_device(double** out) {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    CUcontext cx = nullptr;
    int rc = current_context(&cx);
    if (rc) return rc;
    for (const auto& kv : g_scratch_ptr)
        if (cx && kv.first == cx) {
            *out = kv.second;
            return PG_OK;
        }
    // set-up: the array's address in the current context (the runtime makes
    // the current device's primary context current when no context is)
    double* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_sweep_scratch);
    if (e != cudaSuccess || p == nullptr)
        return pg::set_last_error(PG_ECUDA, std::string("cudaGetSymbolAddress(sweep scratch): ") +
                                                cudaGetErrorString(e));
    if (!cx) {
        rc = current_context(&cx);
        if (rc) return rc;
        if (!cx) return pg::set_last_error(PG_ECUDA, "no current CUDA context after set-up");
    }
    g_scratch_ptr.emplace_back(cx, p);
    *out = p;
    return PG_OK;
}

}  // namespace

extern "C" {

int pg_sweep_noalloc(const pg_grid6* g, const pg_model* m, const pg_params* p,
                     const uint8_t* occ_dev, const float* ctl_dev, int32_t nctl,
                     const float* v_in_dev, float* v_out_dev, int32_t phase, void* stream,
                     double* delta, double* maxnorm) {
    using pg::set_last_error;
    if (!g || !m || !p || !occ_dev || !ctl_dev || !v_in_dev || !v_out_dev)
        return set_last_error(PG_EINVAL, "null argument");
    if ((const void*)v_in_dev == (const void*)v_out_dev)
        return set_last_error(PG_EINVAL, "v_in and v_out must be different buffers (Jacobi sweep)");
    int64_t ncells = 1;
    for (int k = 0; k < 6; ++k) {
        if (g->n[k] < 2)
            return set_last_error(PG_EINVAL, "every axis needs at least 2 samples (Grid6)");
        if (!(g->step[k] > 0.0f) || !std::isfinite(g->lo[k]))
            return set_last_error(PG_EINVAL, "grid steps must be positive and origins finite");
        if (ncells <= kMaxCells) ncells *= g->n[k];
    }
    if (ncells > kMaxCells)
        return set_last_error(
            PG_EINVAL, "pg_sweep_noalloc takes grids of at most 8388608 cells (its fixed working "
                       "array holds 65536 block partials); use pg_load_problem/pg_sweep for "
                       "larger grids");
    if (nctl < 2)
        return set_last_error(PG_EINVAL, "the control table needs coast plus at least one command");
    if (nctl > 32767) return set_last_error(PG_EINVAL, "the control table holds at most 32767 controls");
    if (!(p->cap > 0.0f)) return set_last_error(PG_EINVAL, "value_cap must be positive");
    if (p->nsub < 1) return set_last_error(PG_EINVAL, "substeps must be >= 1");
    if (p->checks < 1) return set_last_error(PG_EINVAL, "sweep_checks must be >= 1");
    if (!(p->dt > 0.0f)) return set_last_error(PG_EINVAL, "dt must be positive");

    double* scratch = nullptr;
    int rc = scratch_on_current_device(&scratch);
    if (rc) return rc;

    pg::KParams kp{};
    kp.g = *g;
    kp.m = *m;
    kp.p = *p;
    kp.P = (int64_t)g->n[0] * g->n[1];
    kp.nplanes = (int64_t)g->n[2] * g->n[3] * g->n[4] * g->n[5];
    kp.ncells = ncells;
    kp.nctl = nctl;
    kp.phase = phase;
    kp.xoff = 0;
    kp.n1g = g->n[0];
    kp.ux0 = 0;
    kp.ux1 = g->n[0];
    pg::SweepBufs sb{scratch, scratch + kMaxParts, kMaxParts, scratch + 2 * kMaxParts};

    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(sb.out, 0, 2 * sizeof(double), st);
    int64_t launches = 0;
    if (e == cudaSuccess)
        e = pg::launch_cellform(PG_STORE_F32, false, v_in_dev, v_out_dev, occ_dev, nullptr, kp,
                                ctl_dev, sb, nullptr, st, &launches);
    double res[2] = {0.0, 0.0};
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(res, sb.out, sizeof(res), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return set_last_error(PG_ECUDA, std::string("pg_sweep_noalloc: ") + cudaGetErrorString(e));
    if (delta) *delta = res[0];
    if (maxnorm) *maxnorm = res[1];
    return PG_OK;
}

}  // extern "C"
