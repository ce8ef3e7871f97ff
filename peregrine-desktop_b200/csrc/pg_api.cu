// pg_api.cu -- the C ABI of libperegrine_hjb.so (include/peregrine_hjb.h).
//
// A context owns one CUDA stream and the device buffers of one loaded
// problem: two value buffers (Jacobi ping-pong), the occupancy in (h, x, y)
// order, the control table, the Int8 warm-start policy and the per-block
// reduction partials.  The sweep loop of solve_value! (Run.jl:1434-1474) runs
// here: one sweep kernel and one fixed-order reduction per sweep, a 16-byte
// read of the two convergence numbers, the seed re-assertion, the stop rule.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <algorithm>
#include <thread>
#include <vector>

#include "pg_kernels.h"
#include "pg_types.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define PG_CUDA(call)                                                                    \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(e_ == cudaErrorMemoryAllocation ? PG_ENOMEM : PG_ECUDA,          \
                        std::string(#call) + ": " + cudaGetErrorString(e_));             \
    } while (0)

size_t elem_bytes(int storage) {
    switch (storage) {
        case PG_STORE_F32: return 4;
        case PG_STORE_F16: return 2;
        case PG_STORE_BF16: return 2;
        case PG_STORE_Q16: return 2;
        case PG_STORE_F64: return 8;
    }
    return 0;
}

// substeps_for on the host, same float arithmetic as the device
// (PeregrineSolver.jl:985-989).
int32_t host_substeps_for(float tau, const pg_params& p) {
    if (p.hmax <= 0.0f) return p.nsub;
    volatile float q = tau / p.hmax;
    float qq = q < 1.0e4f ? q : 1.0e4f;
    int32_t k = (int32_t)qq + 1;
    return k < 1 ? 1 : (k > 64 ? 64 : k);
}

}  // namespace

struct pg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ev_wait = nullptr;  // the per-sweep residual copy, for bounded waits
    double wait_timeout_s = 0.0;    // 0: wait for each sweep without a limit
    int64_t launches = 0;

    bool loaded = false;
    pg::KParams kp{};
    int base_storage = PG_STORE_F32;  // storage the problem was loaded with
    int storage = PG_STORE_F32;       // storage of V right now (polish switches it)
    bool stencil_ok = false;
    std::string stencil_why;
    std::vector<float> ctl_h;

    void* V[2] = {nullptr, nullptr};
    int cur = 0;
    uint8_t* occ_d = nullptr;
    float* ctl_d = nullptr;
    int32_t* order_d = nullptr;
    std::vector<int32_t> order_h;
    uint32_t* mask_d = nullptr;  // admissibility bits of the masked stencil
    uint32_t* recs_d = nullptr;  // its per-(plane, control) records
    bool mask_ok = false;
    bool blend_ok = false;   // the blend-then-shift tiling fits (shared memory, row width)
    bool gather_ok = false;  // the 64-corner masked gather fits its shared memory
    uint16_t* gord_d = nullptr;  // per plane, its controls in corner-group order
    uint32_t* tmask_d = nullptr; // admissibility per (plane, tile, control) in tile order
    size_t tmask_cap = 0;
    bool rblend_ok = false;      // the register-resident blend can run (tables, tiling)
    int8_t* pol_d = nullptr;
    double* part_sum = nullptr;
    double* part_max = nullptr;
    int64_t nparts = 0;
    double* red_d = nullptr;
    double* red_h = nullptr;  // pinned [2]
    int64_t* tidx_d = nullptr;
    int64_t tidx_cap = 0;
    int64_t ntidx = 0;
    int16_t* argmin_d = nullptr;
    uint8_t* enc_d = nullptr;
    size_t enc_cap = 0;
    unsigned long long* counts_d = nullptr;
    float* stage_d = nullptr;  // row-major f32 staging for get/set
    size_t stage_cap = 0;

    bool slab = false;           // loaded as an x slab (pg_load_slab): row stencil only

    void free_values() {
        for (int i = 0; i < 2; ++i) {
            if (V[i]) cudaFree(V[i]);
            V[i] = nullptr;
        }
    }
    void free_problem() {
        free_values();
        if (occ_d) cudaFree(occ_d);
        if (ctl_d) cudaFree(ctl_d);
        if (order_d) cudaFree(order_d);
        order_d = nullptr;
        if (mask_d) cudaFree(mask_d);
        mask_d = nullptr;
        if (recs_d) cudaFree(recs_d);
        recs_d = nullptr;
        mask_ok = false;
        blend_ok = false;
        gather_ok = false;
        if (gord_d) cudaFree(gord_d);
        gord_d = nullptr;
        if (tmask_d) cudaFree(tmask_d);
        tmask_d = nullptr;
        tmask_cap = 0;
        rblend_ok = false;
        if (pol_d) cudaFree(pol_d);
        if (part_sum) cudaFree(part_sum);
        if (part_max) cudaFree(part_max);
        if (tidx_d) cudaFree(tidx_d);
        if (argmin_d) cudaFree(argmin_d);
        if (enc_d) cudaFree(enc_d);
        if (stage_d) cudaFree(stage_d);
        occ_d = nullptr; ctl_d = nullptr; pol_d = nullptr; part_sum = nullptr;
        part_max = nullptr; tidx_d = nullptr; argmin_d = nullptr; enc_d = nullptr;
        stage_d = nullptr;
        tidx_cap = 0; enc_cap = 0; stage_cap = 0; nparts = 0; ntidx = 0;
        loaded = false;
    }
};

namespace {

int check_ctx(pg_ctx* ctx, bool need_problem) {
    if (!ctx) return fail(PG_EINVAL, "null context");
    if (need_problem && !ctx->loaded) return fail(PG_ESTATE, "no problem loaded");
    if (cudaSetDevice(ctx->device) != cudaSuccess)
        return fail(PG_ECUDA, "cudaSetDevice failed");
    return PG_OK;
}

int ensure_stage(pg_ctx* ctx) {
    size_t need = (size_t)ctx->kp.ncells * sizeof(float);
    if (ctx->stage_cap >= need) return PG_OK;
    if (ctx->stage_d) cudaFree(ctx->stage_d);
    ctx->stage_d = nullptr;
    ctx->stage_cap = 0;
    PG_CUDA(cudaMalloc(&ctx->stage_d, need));
    ctx->stage_cap = need;
    return PG_OK;
}

// Make V buffers match `storage` (reallocating when the polish phase left
// them in FP32).
int ensure_values(pg_ctx* ctx, int storage) {
    if (ctx->V[0] && ctx->storage == storage) return PG_OK;
    ctx->free_values();
    const size_t bytes = (size_t)ctx->kp.ncells * elem_bytes(storage);
    size_t fr = 0, tot = 0;
    PG_CUDA(cudaMemGetInfo(&fr, &tot));
    if (2 * bytes > fr)
        return fail(PG_ENOMEM, "the whole-grid solve needs " +
                                   std::to_string(2.0 * bytes / (1 << 30)) +
                                   " GiB of device memory for V but only " +
                                   std::to_string((double)fr / (1 << 30)) + " GiB is free");
    for (int i = 0; i < 2; ++i) PG_CUDA(cudaMalloc(&ctx->V[i], bytes));
    ctx->storage = storage;
    ctx->cur = 0;
    return PG_OK;
}

// Register-resident blend tiling.  A block of rblock threads (a multiple of
// 32, at most 512) sweeps a tile of rtile_x rows: its first rgroups * Ny
// threads own one column of four window rows each, so the window of
// rtile_x + 3 rows needs 4 rgroups >= rtile_x + 3.  rows = 0 picks the tile
// height: for each candidate (the most rows that rgroups groups allow,
// balanced over the plane) the work per tile cell and control -- window
// cells blended, plus cells shifted, plus idle threads -- and the resident
// warps per SM (128 registers a thread); the cheapest with at least 12
// warps per SM, else the cheapest.  rows < 0, or a tiling that cannot run,
// leaves it at 0 (not eligible).  The controls a block stages at once
// (rchunk) are all of them when they fit the shared memory that the blocks
// the registers allow on an SM share (228 KB, less 1 KB reserved and the
// static shared memory per block, checked with the occupancy calculator),
// else as many as fit, with fewer blocks per SM only when fewer than 16
// would fit.
namespace {
struct RTile {
    int32_t tx = 0, groups = 0, block = 0;
    double cost = 0.0;
    int warps = 0;
};
RTile r_candidate(int32_t n1, int32_t n2, int32_t tx) {
    RTile c;
    if (tx < 1 || tx > n1) return c;
    const int32_t groups = (tx + 3 + 3) / 4;
    const int64_t block = 32 * (((int64_t)groups * n2 + 31) / 32);
    if (block > 512) return c;
    const int32_t live = (tx + 3) / 4;
    c.tx = tx;
    c.groups = groups;
    c.block = (int32_t)std::max<int64_t>(64, block);
    // instructions per thread and control: ~50 to blend four window cells,
    // ~55 to shift four cells, ~10 for a thread that only waits
    c.cost = (50.0 * groups * n2 + 55.0 * live * n2 + 10.0 * (c.block - (int64_t)groups * n2)) /
             ((double)tx * n2);
    c.warps = (512 / c.block) * (c.block / 32);
    return c;
}
}  // namespace

void r_tiling(pg::KParams& kp, int32_t rows) {
    const int32_t n1 = kp.g.n[0], n2 = kp.g.n[1];
    kp.rtile_x = kp.rtiles_x = kp.rblock = kp.rgroups = kp.rchunk = 0;
    if (rows < 0 || n2 < 1 || n2 > 512 || kp.nctl < 1 || kp.nctl > (int)pg::kCtlMaskHost) return;
    RTile pick;
    if (rows > 0) {
        pick = r_candidate(n1, n2, rows);
    } else {
        auto better = [](const RTile& a, const RTile& b) {  // a better than b
            if (b.tx == 0) return a.tx != 0;
            if (a.tx == 0) return false;
            const bool aw = a.warps >= 12, bw = b.warps >= 12;
            if (aw != bw) return aw;
            return a.cost < b.cost;
        };
        for (int32_t groups = 1; groups * n2 <= 512; ++groups) {
            const int32_t txmax = std::min<int32_t>(n1, 4 * groups - 3);
            if (txmax < 1) continue;
            const int32_t nt = (n1 + txmax - 1) / txmax;
            const RTile c = r_candidate(n1, n2, (n1 + nt - 1) / nt);
            if (better(c, pick)) pick = c;
        }
    }
    // the packed row entries hold window byte offsets in 16 bits
    if (pick.tx == 0 || (int64_t)16 * pick.groups * pg::stencil_r_row_stride_host(n2) > 0xffff) return;
    kp.rtile_x = pick.tx;
    kp.rtiles_x = (n1 + pick.tx - 1) / pick.tx;
    kp.rgroups = pick.groups;
    kp.rblock = pick.block;
    // controls staged at once: as many as fit the blocks that the registers
    // allow on an SM (up to four), with fewer blocks only when fewer than 16
    // controls would fit
    const size_t per = pg::stencil_r_ctl_smem_bytes(kp, pick.tx);
    kp.rchunk = 1;
    const size_t fixed = pg::stencil_r_smem_bytes(kp) - per + 32;  // + the areas' rounding
    const int bps = std::min(4, 512 / pick.block);
    // a chunk's y increments are staged into the window buffers
    const int64_t ybuf = (int64_t)16 * pick.groups * pg::stencil_r_row_stride_host(n2) /
                         std::max(1, pg::stencil_r_ninc_host(kp.nsub));
    int32_t chunk = 0;
    for (int b = bps; b >= 1; --b) {
        // 228 KB per SM less 1 KB reserved per block; the occupancy
        // calculator has the last word (the kernel's static shared memory)
        const size_t lim = std::min<size_t>((size_t)pg::kRSmemMax, 228 * 1024 / b - 1024);
        int64_t c = lim > fixed ? (int64_t)((lim - fixed) / per) : 0;
        c = std::min<int64_t>({c, (int64_t)kp.nctl, ybuf});
        for (; c >= 1; --c) {
            kp.rchunk = (int32_t)c;
            if (pg::stencil_r_blocks_per_sm(pick.block, pg::stencil_r_smem_bytes(kp)) >= b) break;
        }
        chunk = (int32_t)std::max<int64_t>(c, 0);
        // as many blocks per SM as the registers allow, while a block still
        // stages a useful number of controls at once
        if (chunk >= std::min(kp.nctl, 16)) break;
    }
    if (chunk < 1) {
        kp.rtile_x = kp.rtiles_x = kp.rblock = kp.rgroups = kp.rchunk = 0;
        return;
    }
    kp.rchunk = chunk;
}

// Whether the register-resident blend's tiling is set and runs.
bool r_smem_fits(const pg::KParams& kp) {
    return kp.rtile_x > 0 && pg::stencil_r_shape_ok(kp) &&
           pg::stencil_r_smem_bytes(kp) <= (size_t)pg::kRSmemMax;
}

// Planes of row-order mask words that fit a staging buffer of `bytes`.
int64_t mask_chunk_planes(const pg::KParams& kp, size_t bytes) {
    const size_t per = pg::stencil_mask_bytes(kp) / (size_t)kp.nplanes;
    const int64_t c = (int64_t)(bytes / std::max<size_t>(per, 1));
    return std::max<int64_t>(1, std::min<int64_t>(c, kp.nplanes));
}

// (Re)builds the tile-order mask of the register-resident blend for the
// current tiling and sets rblend_ok.  From the row-order mask when the
// context keeps it; otherwise the records and the row-order words are made
// again by k_stencil_prep a chunk of planes at a time into a staging buffer
// of at most 4 GiB, and each chunk regrouped before the next.  The blend
// stays off (the re-reading blend, or the row stencil, runs) when the tile
// mask does not fit in device memory with 2 GiB to spare.
int build_r_tables(pg_ctx* ctx) {
    pg::KParams& kp = ctx->kp;
    ctx->rblend_ok = false;
    if (!ctx->recs_d || !ctx->gord_d || !r_smem_fits(kp)) return PG_OK;
    const size_t need = pg::stencil_tmask_bytes(kp);
    if (need > ctx->tmask_cap) {
        PG_CUDA(cudaStreamSynchronize(ctx->stream));
        if (ctx->tmask_d) cudaFree(ctx->tmask_d);
        ctx->tmask_d = nullptr;
        ctx->tmask_cap = 0;
        size_t fr = 0, tot = 0;
        PG_CUDA(cudaMemGetInfo(&fr, &tot));
        if (need + ((size_t)2 << 30) > fr || cudaMalloc(&ctx->tmask_d, need) != cudaSuccess) {
            cudaGetLastError();
            ctx->tmask_d = nullptr;
            return PG_OK;
        }
        ctx->tmask_cap = need;
    }
    if (ctx->mask_d) {
        cudaError_t e = pg::launch_stencil_tmask(ctx->mask_d, kp, 0, kp.nplanes, ctx->tmask_d,
                                                 ctx->stream, &ctx->launches);
        if (e != cudaSuccess)
            return fail(PG_ECUDA, std::string("tile mask: ") + cudaGetErrorString(e));
    } else {
        size_t fr = 0, tot = 0;
        PG_CUDA(cudaMemGetInfo(&fr, &tot));
        const size_t spare = fr > ((size_t)2 << 30) ? fr - ((size_t)2 << 30) : 0;
        const int64_t chunk = mask_chunk_planes(kp, std::min(spare, (size_t)4 << 30));
        const size_t cb = pg::stencil_mask_bytes(kp) / (size_t)kp.nplanes * (size_t)chunk;
        uint32_t* tmp = nullptr;
        if (cb > spare || cudaMalloc(&tmp, cb) != cudaSuccess) {
            cudaGetLastError();
            return PG_OK;
        }
        cudaError_t e = cudaSuccess;
        for (int64_t p0 = 0; p0 < kp.nplanes && e == cudaSuccess; p0 += chunk) {
            const int64_t np = std::min<int64_t>(chunk, kp.nplanes - p0);
            e = pg::launch_stencil_prep(ctx->occ_d, kp, ctx->ctl_d, tmp, ctx->recs_d, p0, np,
                                        ctx->stream, &ctx->launches);
            if (e == cudaSuccess)
                e = pg::launch_stencil_tmask(tmp, kp, p0, np, ctx->tmask_d, ctx->stream,
                                             &ctx->launches);
        }
        cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
        cudaFree(tmp);
        if (e == cudaSuccess) e = e2;
        if (e != cudaSuccess)
            return fail(PG_ECUDA, std::string("tile mask from chunks: ") + cudaGetErrorString(e));
    }
    ctx->rblend_ok = true;
    return PG_OK;
}

int pick_kernel(pg_ctx* ctx, int32_t kernel, int* out) {
    if (kernel == PG_KERNEL_AUTO) kernel = ctx->stencil_ok ? PG_KERNEL_STENCIL : PG_KERNEL_CELLFORM;
    if ((kernel == PG_KERNEL_STENCIL || kernel == PG_KERNEL_STENCIL_EXACT) && !ctx->stencil_ok)
        return fail(PG_EUNSUPPORTED, "the stencil kernel cannot run this scheme: " + ctx->stencil_why);
    if (kernel == PG_KERNEL_STENCIL_ROWS && !ctx->stencil_ok)
        return fail(PG_EUNSUPPORTED, "the stencil kernel cannot run this scheme: " + ctx->stencil_why);
    if ((kernel == PG_KERNEL_STENCIL_GATHER || kernel == PG_KERNEL_STENCIL_BLEND) && !ctx->stencil_ok)
        return fail(PG_EUNSUPPORTED, "the stencil kernel cannot run this scheme: " + ctx->stencil_why);
    if (kernel < PG_KERNEL_STENCIL || kernel > PG_KERNEL_STENCIL_BLEND)
        return fail(PG_EINVAL, "unknown kernel " + std::to_string(kernel));
    *out = kernel;
    return PG_OK;
}

// One Jacobi sweep V[cur] -> V[1-cur]; does NOT read the residual back.
int sweep_async(pg_ctx* ctx, int kernel, int32_t phase, bool esc, int16_t* argmin_d,
                bool use_pol) {
    ctx->kp.phase = phase;
    pg::SweepBufs sb{ctx->part_sum, ctx->part_max, ctx->nparts, ctx->red_d};
    const void* vin = ctx->V[ctx->cur];
    void* vout = ctx->V[1 - ctx->cur];
    cudaError_t e;
    const bool r_ok = ctx->rblend_ok && ctx->storage != PG_STORE_F64;
    const bool b_ok = ctx->mask_ok && ctx->blend_ok && ctx->storage != PG_STORE_F64;
    if (ctx->storage == PG_STORE_Q16 &&
        (esc || !((kernel == PG_KERNEL_STENCIL && (r_ok || b_ok)) ||
                  (kernel == PG_KERNEL_STENCIL_BLEND && b_ok))))
        return fail(PG_EUNSUPPORTED, "Q16 storage is swept by the blend-then-shift kernels only");
    if (ctx->slab && (esc || kernel == PG_KERNEL_CELLFORM))
        return fail(PG_EUNSUPPORTED, "a slab is swept by the row stencil (PG_KERNEL_STENCIL_ROWS, "
                                     "PG_KERNEL_STENCIL_EXACT or PG_KERNEL_STENCIL)");
    if (kernel == PG_KERNEL_STENCIL_BLEND && !esc && !b_ok)
        return fail(PG_EUNSUPPORTED, "the blend-then-shift kernel cannot run this table (its "
                                     "tiling, shared memory, or FP64 storage)");
    if (esc || kernel == PG_KERNEL_CELLFORM)
        e = pg::launch_cellform(ctx->storage, esc, vin, vout, ctx->occ_d,
                                use_pol ? ctx->pol_d : nullptr, ctx->kp, ctx->ctl_d, sb, argmin_d,
                                ctx->stream, &ctx->launches);
    else if (kernel == PG_KERNEL_STENCIL && r_ok)
        e = pg::launch_stencil_r(ctx->storage, vin, vout, ctx->occ_d, ctx->recs_d, ctx->tmask_d,
                                 ctx->kp, ctx->gord_d, sb, argmin_d, ctx->stream, &ctx->launches);
    else if ((kernel == PG_KERNEL_STENCIL || kernel == PG_KERNEL_STENCIL_BLEND) && b_ok)
        e = pg::launch_stencil_b(ctx->storage, vin, vout, ctx->occ_d, ctx->mask_d, ctx->recs_d,
                                 ctx->kp, ctx->order_d, sb, argmin_d, ctx->stream,
                                 &ctx->launches);
    else if (kernel == PG_KERNEL_STENCIL && ctx->storage == PG_STORE_F64 && ctx->mask_ok &&
             ctx->kp.btile_x > 0)
        e = pg::launch_stencil_d(vin, vout, ctx->occ_d, ctx->mask_d, ctx->recs_d, ctx->kp, sb,
                                 argmin_d, ctx->stream, &ctx->launches);
    else if ((kernel == PG_KERNEL_STENCIL || kernel == PG_KERNEL_STENCIL_GATHER) && ctx->mask_ok &&
             ctx->gather_ok && ctx->storage != PG_STORE_F64)
        e = pg::launch_stencil_u(ctx->storage, vin, vout, ctx->occ_d, ctx->mask_d, ctx->recs_d,
                                 ctx->kp, ctx->order_d, sb, argmin_d, ctx->stream,
                                 &ctx->launches);
    else
        e = pg::launch_stencil(ctx->storage, kernel == PG_KERNEL_STENCIL_EXACT, vin, vout,
                               ctx->occ_d, ctx->kp, ctx->ctl_d, ctx->order_d, sb, argmin_d,
                               ctx->stream, &ctx->launches);
    if (e != cudaSuccess) return fail(PG_ECUDA, std::string("sweep launch: ") + cudaGetErrorString(e));
    ctx->cur = 1 - ctx->cur;
    return PG_OK;
}

// Waits for the context stream up to the context's time limit (none when
// it is 0): polls the event recorded after the last queued work.  On
// PG_ETIMEOUT the work is still queued or running; the context stays usable
// once it finishes (pg_destroy waits for it).
int wait_stream(pg_ctx* ctx) {
    if (!(ctx->wait_timeout_s > 0.0)) {
        PG_CUDA(cudaStreamSynchronize(ctx->stream));
        return PG_OK;
    }
    PG_CUDA(cudaEventRecord(ctx->ev_wait, ctx->stream));
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaEventQuery(ctx->ev_wait);
        if (e == cudaSuccess) return PG_OK;
        if (e != cudaErrorNotReady)
            return fail(PG_ECUDA, std::string("sweep wait: ") + cudaGetErrorString(e));
        const double el =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > ctx->wait_timeout_s)
            return fail(PG_ETIMEOUT, "a sweep did not finish within the context's wait limit of " +
                                         std::to_string(ctx->wait_timeout_s) + " s");
        std::this_thread::sleep_for(std::chrono::microseconds(el < 1e-3 ? 20 : 200));
    }
}

int read_residual(pg_ctx* ctx, double* d, double* dm) {
    PG_CUDA(cudaMemcpyAsync(ctx->red_h, ctx->red_d, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream));
    int rc = wait_stream(ctx);
    if (rc) return rc;
    *d = ctx->red_h[0];
    *dm = ctx->red_h[1];
    return PG_OK;
}

int reseed(pg_ctx* ctx) {
    if (ctx->ntidx <= 0) return PG_OK;
    cudaError_t e = pg::launch_seed_only(ctx->storage, ctx->V[ctx->cur], ctx->kp, ctx->tidx_d,
                                         ctx->ntidx, ctx->stream);
    ctx->launches += 1;
    if (e != cudaSuccess) return fail(PG_ECUDA, std::string("seed: ") + cudaGetErrorString(e));
    return PG_OK;
}

// The iteration of solve_value! / solve_escape! (Run.jl:1441-1472, 1509-1528)
int iterate(pg_ctx* ctx, int kernel, bool esc, int32_t iters, double tol, int stop_rule,
            bool use_pol, int32_t progress_every, int32_t it0, pg_progress_cb cb, void* user,
            int32_t* done_out, double* d_out, double* dm_out, double* kms, bool* converged) {
    const pg_params& p = ctx->kp.p;
    const int32_t nctl = ctx->kp.nctl;
    int quiet_needed = 1;
    if (p.ncoarse > 0) {
        int q = (nctl - 1 + p.ncoarse - 1) / p.ncoarse;
        quiet_needed = q > 1 ? q : 1;
    }
    double d = INFINITY, dm = INFINITY;
    int quiet = 0;
    int32_t done = 0;
    *converged = false;
    for (int32_t it = 1; it <= iters; ++it) {
        PG_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
        int rc = sweep_async(ctx, kernel, it0 + it - 1, esc, nullptr, use_pol);
        if (rc) return rc;
        PG_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
        if (!esc) {
            rc = reseed(ctx);
            if (rc) return rc;
        }
        rc = read_residual(ctx, &d, &dm);
        if (rc) return rc;
        float ms = 0.0f;
        PG_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        *kms += ms;
        done = it;
        const double crit = stop_rule == PG_STOP_MAXNORM ? dm : d;
        quiet = crit <= tol ? quiet + 1 : 0;
        const bool stop = quiet >= quiet_needed;
        const bool report = progress_every > 0 ? (it % progress_every == 0 || it == 1 || stop)
                                               : (it % 5 == 0 || it == 1 || stop);
        if (cb && report && cb(user, it0 + it, d, dm)) {
            *done_out = done; *d_out = d; *dm_out = dm;
            return fail(PG_ECANCELLED, "cancelled by the progress callback");
        }
        if (stop) { *converged = true; break; }
    }
    *done_out = done;
    *d_out = d;
    *dm_out = dm;
    return PG_OK;
}

}  // namespace

namespace pg {
int set_last_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace pg

extern "C" {

int32_t pg_abi_version(void) { return PG_ABI_VERSION; }

const char* pg_last_error(void) { return g_err.c_str(); }

void pg_default_opts(pg_solve_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->stop_rule = PG_STOP_L1_QUIET;
    o->storage = PG_STORE_F32;
    o->kernel = PG_KERNEL_AUTO;
    o->warm_start = 0;
    o->polish_sweeps = 64;
    o->progress_every = 0;
}

int pg_create(pg_ctx** out, int device) {
    if (!out) return fail(PG_EINVAL, "null output pointer");
    int n = 0;
    PG_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n)
        return fail(PG_EINVAL, "device " + std::to_string(device) + " out of range (" +
                                   std::to_string(n) + " visible)");
    PG_CUDA(cudaSetDevice(device));
    pg_ctx* c = new pg_ctx();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_wait, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&c->red_d, 2 * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&c->red_h, 2 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->counts_d, 2 * sizeof(unsigned long long)) != cudaSuccess) {
        delete c;
        return fail(PG_ECUDA, "context creation failed");
    }
    *out = c;
    return PG_OK;
}

int pg_destroy(pg_ctx* ctx) {
    if (!ctx) return PG_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->free_problem();
    if (ctx->red_d) cudaFree(ctx->red_d);
    if (ctx->red_h) cudaFreeHost(ctx->red_h);
    if (ctx->counts_d) cudaFree(ctx->counts_d);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->ev_wait) cudaEventDestroy(ctx->ev_wait);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return PG_OK;
}

}  // extern "C"

namespace {

// An x slab of a table: interior rows [x0, x1) with `halo` rows either side.
struct SlabSpec {
    int32_t x0, x1, halo;
};

int load_impl(pg_ctx* ctx, const pg_grid6* g_in, const pg_model* m, const pg_params* p,
              const uint8_t* occ, const float* ctl, int32_t nctl, int32_t storage,
              const SlabSpec* slab) {
    int rc = check_ctx(ctx, false);
    if (rc) return rc;
    if (!g_in || !m || !p || !occ || !ctl) return fail(PG_EINVAL, "null argument");
    const pg_grid6* g = g_in;
    pg_grid6 gl;
    int32_t xa = 0;
    if (slab) {
        const int32_t n1 = g_in->n[0];
        if (slab->x0 < 0 || slab->x1 > n1 || slab->x0 >= slab->x1 || slab->halo < 0)
            return fail(PG_EINVAL, "a slab needs 0 <= x0 < x1 <= Nx and halo >= 0");
        if (storage != PG_STORE_F32)
            return fail(PG_EUNSUPPORTED, "slabs are swept in FP32 storage");
        xa = std::max(0, slab->x0 - slab->halo);
        const int32_t xb = std::min(n1, slab->x1 + slab->halo);
        if (xb - xa < 2) return fail(PG_EINVAL, "a slab needs at least 2 rows with its halo");
        gl = *g_in;
        gl.n[0] = xb - xa;
        g = &gl;
    }
    for (int k = 0; k < 6; ++k)
        if (g->n[k] < 2)
            return fail(PG_EINVAL, "every axis needs at least 2 samples (Grid6)");
    for (int k = 0; k < 6; ++k)
        if (!(g->step[k] > 0.0f) || !std::isfinite(g->lo[k]))
            return fail(PG_EINVAL, "grid steps must be positive and origins finite");
    if (nctl < 2) return fail(PG_EINVAL, "the control table needs coast plus at least one command");
    if (nctl > 32767) return fail(PG_EINVAL, "the control table holds at most 32767 controls");
    if (elem_bytes(storage) == 0) return fail(PG_EINVAL, "unknown storage");
    if (storage == PG_STORE_Q16 && !(p->cap < 32.0f))
        return fail(PG_EUNSUPPORTED, "Q16 storage holds values below 32 s; value_cap is larger");
    if (!(p->cap > 0.0f)) return fail(PG_EINVAL, "value_cap must be positive");
    if (p->nsub < 1) return fail(PG_EINVAL, "substeps must be >= 1");
    if (p->checks < 1) return fail(PG_EINVAL, "sweep_checks must be >= 1");
    if (!(p->dt > 0.0f)) return fail(PG_EINVAL, "dt must be positive");

    ctx->free_problem();
    pg::KParams& kp = ctx->kp;
    std::memset(&kp, 0, sizeof(kp));
    kp.g = *g;
    kp.m = *m;
    kp.p = *p;
    kp.P = (int64_t)g->n[0] * g->n[1];
    kp.nplanes = (int64_t)g->n[2] * g->n[3] * g->n[4] * g->n[5];
    kp.ncells = kp.P * kp.nplanes;
    kp.nctl = nctl;
    kp.xoff = xa;
    kp.n1g = g_in->n[0];
    kp.ux0 = slab ? slab->x0 - xa : 0;
    kp.ux1 = slab ? slab->x1 - xa : g->n[0];
    // Stencil tiling: a block takes whole planes (x rows split only past 4096
    // four-cell segments), and the block size is the multiple of 32 in
    // [96, 256] that leaves the fewest idle threads in the last pass.
    {
        const int32_t spr = (g->n[1] + 3) / 4;
        const int64_t segs_plane = (int64_t)g->n[0] * spr;
        const int64_t ntile = (segs_plane + 4095) / 4096;
        int32_t tx = (int32_t)((g->n[0] + ntile - 1) / ntile);
        kp.tile_x = tx;
        kp.tiles_x = (g->n[0] + tx - 1) / tx;
        const int64_t segs = (int64_t)tx * spr;
        int best_bs = 256;
        int64_t best_waste = -1;
        if (segs < 96) {
            best_bs = (int)(32 * ((segs + 31) / 32));
        } else {
            for (int bs = 256; bs >= 96; bs -= 32) {
                const int64_t waste = ((segs + bs - 1) / bs) * bs - segs;
                if (best_waste < 0 || waste < best_waste) { best_waste = waste; best_bs = bs; }
            }
        }
        kp.block = best_bs;
    }
    // Masked stencil: blocks of 2 rows x 4 columns per thread, whole planes
    // per block up to 2048 such blocks.
    {
        const int64_t rbn = (g->n[0] + 1) / 2, cbn = (g->n[1] + 3) / 4;
        const int64_t ntile = (rbn * cbn + 2047) / 2048;
        const int32_t rows_per_tile = (int32_t)(2 * ((rbn + ntile - 1) / ntile));
        kp.utile_x = rows_per_tile;
        kp.utiles_x = (g->n[0] + rows_per_tile - 1) / rows_per_tile;
        const int64_t segs = (int64_t)((rows_per_tile + 1) / 2) * cbn;
        int best_bs = 256;
        int64_t best_waste = -1;
        if (segs < 96) {
            best_bs = (int)(32 * ((segs + 31) / 32));
        } else {
            for (int bs = 256; bs >= 96; bs -= 32) {
                const int64_t waste = ((segs + bs - 1) / bs) * bs - segs;
                if (best_waste < 0 || waste < best_waste) { best_waste = waste; best_bs = bs; }
            }
        }
        kp.ublock = best_bs;
    }
    // Blend-then-shift: a block takes whole rows of one plane, at most
    // 1024 cells (4 per thread), as few tiles per plane as that allows.
    if (g->n[1] <= pg::kBMaxTileCells) {
        int32_t tx = std::min<int32_t>(g->n[0], pg::kBMaxTileCells / g->n[1]);
        const int32_t nt = (g->n[0] + tx - 1) / tx;
        tx = (g->n[0] + nt - 1) / nt;
        const int64_t cells = (int64_t)tx * g->n[1];
        int64_t th = 32 * (((cells + 2) / 3 + 31) / 32);
        th = std::max<int64_t>(64, std::min<int64_t>(256, th));
        kp.btile_x = tx;
        kp.btiles_x = nt;
        kp.bblock = (int32_t)th;
    }
    r_tiling(kp, 0);
    kp.nsub = host_substeps_for(p->cfl <= 0.0f ? p->dt : p->tau_max, *p);
    kp.nchk = p->checks;

    // Which schemes the position-invariant stencil reproduces exactly.
    ctx->stencil_ok = true;
    ctx->stencil_why.clear();
    auto no = [&](const char* why) {
        if (ctx->stencil_ok) ctx->stencil_why = why;
        ctx->stencil_ok = false;
    };
    if (p->cfl > 0.0f) no("cfl > 0 (per-cell horizon)");
    if (p->ntau > 1) no("tau_levels > 1 (horizon ladder)");
    if (p->ncoarse > 0 && p->ncoarse < nctl - 1) no("control_scan rotates a partial slice");
    if (p->rounds > 0) no("refine_rounds > 0 (pattern search)");
    if (p->adaptive_checks) no("adaptive_checks");
    if (p->nearest) no("nearest");
    if (p->simplex) no("simplex (Kuhn) interpolation");
    if (kp.nsub > pg::kStencilMaxSub) no("more than 16 substeps");
    if (p->checks > pg::kStencilMaxChk) no("more than 4 swept probes");
    if (kp.ncells / kp.tiles_x > (int64_t)1 << 40) no("grid too large");

    ctx->ctl_h.assign(ctl, ctl + 3 * nctl);
    ctx->base_storage = storage;
    rc = ensure_values(ctx, storage);
    if (rc) { ctx->free_problem(); return rc; }

    // the whole table's occupancy, also for a slab (its sweep reads it at
    // global rows)
    const int32_t nx = g_in->n[0], ny = g->n[1], nh = g->n[2];
    std::vector<uint8_t> occ_hxy((size_t)nx * ny * nh);
    for (int32_t i = 0; i < nx; ++i)
        for (int32_t j = 0; j < ny; ++j)
            for (int32_t k = 0; k < nh; ++k)
                occ_hxy[((size_t)k * nx + i) * ny + j] = occ[((size_t)i * ny + j) * nh + k] ? 1 : 0;
    PG_CUDA(cudaMalloc(&ctx->occ_d, occ_hxy.size()));
    PG_CUDA(cudaMemcpyAsync(ctx->occ_d, occ_hxy.data(), occ_hxy.size(), cudaMemcpyHostToDevice,
                            ctx->stream));
    PG_CUDA(cudaMalloc(&ctx->ctl_d, sizeof(float) * 3 * nctl));
    PG_CUDA(cudaMemcpyAsync(ctx->ctl_d, ctl, sizeof(float) * 3 * nctl, cudaMemcpyHostToDevice,
                            ctx->stream));
    // The stencil visits controls in (u1, u2, u3) order, so consecutive
    // controls land on neighbouring successor planes and reuse them from L1;
    // its tie-break on the table index keeps the result order-independent.
    ctx->order_h.resize(nctl);
    for (int32_t k = 0; k < nctl; ++k) ctx->order_h[k] = k;
    std::stable_sort(ctx->order_h.begin(), ctx->order_h.end(), [&](int32_t a, int32_t b) {
        for (int c = 0; c < 3; ++c) {
            const float ua = ctl[a + c * nctl], ub = ctl[b + c * nctl];
            if (ua != ub) return ua < ub;
        }
        return a < b;
    });
    PG_CUDA(cudaMalloc(&ctx->order_d, sizeof(int32_t) * nctl));
    PG_CUDA(cudaMemcpyAsync(ctx->order_d, ctx->order_h.data(), sizeof(int32_t) * nctl,
                            cudaMemcpyHostToDevice, ctx->stream));
    ctx->nparts = pg::cellform_blocks(kp.ncells);
    const int64_t sb = pg::stencil_blocks(kp);
    if (sb > ctx->nparts) ctx->nparts = sb;
    const int64_t ub = kp.nplanes * kp.utiles_x;
    if (ub > ctx->nparts) ctx->nparts = ub;
    const int64_t bb = kp.nplanes * kp.btiles_x;
    if (bb > ctx->nparts) ctx->nparts = bb;
    const int64_t rb = kp.nplanes * kp.rtiles_x;
    if (rb > ctx->nparts) ctx->nparts = rb;
    PG_CUDA(cudaMalloc(&ctx->part_sum, sizeof(double) * ctx->nparts));
    PG_CUDA(cudaMalloc(&ctx->part_max, sizeof(double) * ctx->nparts));
    // The admissibility decisions of the masked stencils, made once here and
    // read by every sweep: the per-(plane, control) records, the row-order
    // mask (the re-reading blend, the 64-corner gather, the adjoint) and the
    // tile-order mask with the corner-group order (the register-resident
    // blend).  Everything is kept when it leaves 4 GiB free.  Otherwise the
    // register-resident blend alone is kept when its records and tile mask
    // fit (the row-order mask is then made a chunk of planes at a time and
    // dropped), else the row-order mask alone; with neither, the row stencil
    // decides per sweep.
    // FP64 storage keeps the row-order mask and records only: its sweep is
    // the precision oracle, which takes the FP32 solver's decisions.  A slab
    // runs the row stencil, which decides every probe per sweep.
    if (ctx->stencil_ok && !slab) {
        const size_t mb = pg::stencil_mask_bytes(kp), rb = pg::stencil_recs_bytes(kp);
        const size_t gb = (size_t)kp.nplanes * kp.nctl * sizeof(uint16_t);
        const bool r_able = storage != PG_STORE_F64 && r_smem_fits(kp);
        const size_t tb = r_able ? pg::stencil_tmask_bytes(kp) : 0;
        const size_t G = (size_t)1 << 30;
        size_t fr = 0, tot = 0;
        PG_CUDA(cudaMemGetInfo(&fr, &tot));
        bool keep_rows = mb + rb + (r_able ? gb + tb : 0) + 4 * G < fr;
        bool r_only = !keep_rows && r_able && rb + gb + tb + 6 * G < fr;
        if (!keep_rows && !r_only) keep_rows = mb + rb + 4 * G < fr;
        cudaError_t e = cudaSuccess;
        if (keep_rows || r_only) {
            if (cudaMalloc(&ctx->recs_d, rb) != cudaSuccess ||
                (keep_rows && cudaMalloc(&ctx->mask_d, mb) != cudaSuccess)) {
                cudaGetLastError();
                if (ctx->recs_d) cudaFree(ctx->recs_d);
                ctx->recs_d = nullptr;
                ctx->mask_d = nullptr;
                keep_rows = r_only = false;
            }
        }
        if (keep_rows) {
            e = pg::launch_stencil_prep(ctx->occ_d, kp, ctx->ctl_d, ctx->mask_d, ctx->recs_d, 0,
                                        kp.nplanes, ctx->stream, &ctx->launches);
            if (e != cudaSuccess) return fail(PG_ECUDA, std::string("prep: ") + cudaGetErrorString(e));
            ctx->mask_ok = true;
            ctx->blend_ok = storage != PG_STORE_F64 && kp.btile_x > 0 &&
                            pg::stencil_b_smem_bytes(kp) <= 200 * 1024;
            ctx->gather_ok = storage != PG_STORE_F64 && pg::stencil_u_smem_bytes(kp) <= 200 * 1024;
        }
        if ((keep_rows || r_only) && r_able) {
            size_t fr2 = 0, tot2 = 0;
            PG_CUDA(cudaMemGetInfo(&fr2, &tot2));
            if (gb + tb + 2 * G < fr2 && cudaMalloc(&ctx->gord_d, gb) == cudaSuccess) {
                // the records first (made by the chunked prep when no
                // row-order mask is kept), then the group order
                if (!keep_rows) {
                    int rc2 = build_r_tables(ctx);
                    if (rc2) return rc2;
                }
                e = pg::launch_stencil_group(ctx->recs_d, kp, ctx->order_d, ctx->gord_d,
                                             ctx->stream, &ctx->launches);
                if (e != cudaSuccess)
                    return fail(PG_ECUDA, std::string("group: ") + cudaGetErrorString(e));
                if (keep_rows) {
                    int rc2 = build_r_tables(ctx);
                    if (rc2) return rc2;
                }
            } else {
                cudaGetLastError();
                ctx->gord_d = nullptr;
            }
        }
        if (!ctx->mask_ok && !ctx->rblend_ok && ctx->recs_d) {
            cudaFree(ctx->recs_d);
            ctx->recs_d = nullptr;
        }
    }
    PG_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->loaded = true;
    ctx->slab = slab != nullptr;
    return PG_OK;
}

}  // namespace

extern "C" {

int pg_load_problem(pg_ctx* ctx, const pg_grid6* g, const pg_model* m, const pg_params* p,
                    const uint8_t* occ, const float* ctl, int32_t nctl, int32_t storage) {
    return load_impl(ctx, g, m, p, occ, ctl, nctl, storage, nullptr);
}

int pg_load_slab(pg_ctx* ctx, const pg_grid6* g, const pg_model* m, const pg_params* p,
                 const uint8_t* occ, const float* ctl, int32_t nctl, int32_t x0, int32_t x1,
                 int32_t halo, int32_t* row0, int32_t* rows) {
    const SlabSpec sl{x0, x1, halo};
    int rc = load_impl(ctx, g, m, p, occ, ctl, nctl, PG_STORE_F32, &sl);
    if (rc) return rc;
    if (row0) *row0 = ctx->kp.xoff;
    if (rows) *rows = ctx->kp.g.n[0];
    return PG_OK;
}

int pg_get_rows(pg_ctx* ctx, int32_t r0, int32_t r1, void* out, int32_t on_device) {
    int rc = check_ctx(ctx, true);
    if (rc) return rc;
    if (!out) return fail(PG_EINVAL, "null argument");
    if (ctx->storage != PG_STORE_F32) return fail(PG_EUNSUPPORTED, "row copies read FP32 storage");
    if (r0 < 0 || r1 > ctx->kp.g.n[0] || r1 < r0) return fail(PG_EINVAL, "rows out of range");
    const size_t bytes = (size_t)(r1 - r0) * (size_t)(ctx->kp.ncells / ctx->kp.g.n[0]) * 4;
    if (bytes == 0) return PG_OK;
    void* dst = out;
    if (!on_device) {
        rc = ensure_stage(ctx);
        if (rc) return rc;
        dst = ctx->stage_d;
    }
    PG_CUDA(pg::launch_slab_out(4, ctx->V[ctx->cur], dst, ctx->kp, r0, r1, ctx->stream));
    if (!on_device)
        PG_CUDA(cudaMemcpyAsync(out, ctx->stage_d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    PG_CUDA(cudaStreamSynchronize(ctx->stream));
    return PG_OK;
}

int pg_set_rows(pg_ctx* ctx, int32_t r0, int32_t r1, const void* in, int32_t on_device) {
    int rc = check_ctx(ctx, true);
    if (rc) return rc;
    if (!in) return fail(PG_EINVAL, "null argument");
    if (ctx->storage != PG_STORE_F32) return fail(PG_EUNSUPPORTED, "row copies write FP32 storage");
    if (r0 < 0 || r1 > ctx->kp.g.n[0] || r1 < r0) return fail(PG_EINVAL, "rows out of range");
    const size_t bytes = (size_t)(r1 - r0) * (size_t)(ctx->kp.ncells / ctx->kp.g.n[0]) * 4;
    if (bytes == 0) return PG_OK;
    const void* src = in;
    if (!on_device) {
        rc = ensure_stage(ctx);
        if (rc) return rc;
        PG_CUDA(cudaMemcpyAsync(ctx->stage_d, in, bytes, cudaMemcpyHostToDevice, ctx->stream));
        src = ctx->stage_d;
    }
    PG_CUDA(pg::launch_slab_in(4, src, ctx->V[ctx->cur], ctx->kp, ctx->stream, r0, r1));
    PG_CUDA(cudaStreamSynchronize(ctx->stream));
    return PG_OK;
}

int pg_solve(pg_ctx* ctx, const int64_t* tidx, int64_t ntidx, int32_t iters, double tol,
             const pg_solve_opts* opts_in, pg_solve_result* res, pg_progress_cb cb, void* user) {
    auto t0 = std::chrono::steady_clock::now();
    int rc = check_ctx(ctx, true);
    if (rc) return rc;
    pg_solve_opts opts;
    if (opts_in) opts = *opts_in;
    else pg_default_opts(&opts);
    if (ntidx < 0 || (ntidx > 0 && !tidx)) return fail(PG_EINVAL, "bad seed list");
    if (iters < 0) return fail(PG_EINVAL, "iterations must be >= 0");
    for (int64_t t = 0; t < ntidx; ++t)
        if (tidx[t] < 0 || tidx[t] >= ctx->kp.ncells)
            return fail(PG_EINVAL, "seed index " + std::to_string(tidx[t]) + " outside the grid");
    int kernel = 0;
    rc = pick_kernel(ctx, opts.warm_start && opts.kernel == PG_KERNEL_AUTO ? PG_KERNEL_CELLFORM
                                                                          : opts.kernel,
                     &kernel);
    if (rc) return rc;
    if (opts.warm_start && kernel != PG_KERNEL_CELLFORM)
        return fail(PG_EUNSUPPORTED, "the warm-start policy needs the cell-form kernel");
    rc = ensure_values(ctx, ctx->base_storage);
    if (rc) return rc;

    if (ntidx > ctx->tidx_cap) {
        if (ctx->tidx_d) cudaFree(ctx->tidx_d);
        ctx->tidx_d = nullptr;
        PG_CUDA(cudaMalloc(&ctx->tidx_d, sizeof(int64_t) * ntidx));
        ctx->tidx_cap = ntidx;
    }
    if (ntidx > 0)
        PG_CUDA(cudaMemcpyAsync(ctx->tidx_d, tidx, sizeof(int64_t) * ntidx, cudaMemcpyHostToDevice,
                                ctx->stream));
    ctx->ntidx = ntidx;
    if (opts.warm_start) {
        if (!ctx->pol_d) PG_CUDA(cudaMalloc(&ctx->pol_d, (size_t)ctx->kp.ncells * 3));
        PG_CUDA(cudaMemsetAsync(ctx->pol_d, 0, (size_t)ctx->kp.ncells * 3, ctx->stream));
    }
    ctx->cur = 0;
    cudaError_t e = pg::launch_fill_seed(ctx->storage, ctx->V[0], ctx->kp, ctx->tidx_d, ntidx,
                                         ctx->stream);
    ctx->launches += ntidx > 0 ? 2 : 1;
    if (e != cudaSuccess) return fail(PG_ECUDA, std::string("fill: ") + cudaGetErrorString(e));

    int32_t done = 0, pdone = 0;
    double d = INFINITY, dm = INFINITY, kms = 0.0;
    bool conv = false;
    rc = iterate(ctx, kernel, false, iters, tol, opts.stop_rule, opts.warm_start != 0,
                 opts.progress_every, 0, cb, user, &done, &d, &dm, &kms, &conv);
    if (rc) return rc;

    // 16-bit storage: continue in FP32 from the converged 16-bit table until
    // the same stop rule holds at FP32 resolution.
    if ((ctx->storage == PG_STORE_F16 || ctx->storage == PG_STORE_BF16 ||
         ctx->storage == PG_STORE_Q16) && opts.polish_sweeps > 0) {
        const size_t bytes = (size_t)ctx->kp.ncells * 4;
        void* nv[2] = {nullptr, nullptr};
        PG_CUDA(cudaMalloc(&nv[0], bytes));
        if (cudaMalloc(&nv[1], bytes) != cudaSuccess) {
            cudaFree(nv[0]);
            return fail(PG_ENOMEM, "no room for the FP32 polish buffers");
        }
        e = pg::launch_convert_to_f32(ctx->storage, ctx->V[ctx->cur], (float*)nv[0],
                                      ctx->kp.ncells, ctx->stream);
        ctx->launches += 1;
        if (e != cudaSuccess) { cudaFree(nv[0]); cudaFree(nv[1]); return fail(PG_ECUDA, "convert"); }
        PG_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->free_values();
        ctx->V[0] = nv[0];
        ctx->V[1] = nv[1];
        ctx->cur = 0;
        ctx->storage = PG_STORE_F32;
        double d2 = d, dm2 = dm;
        bool conv2 = false;
        // Plain value iteration (V <- T V) for the polish: the 16-bit table's
        // rounding error has both signs, and a cell rounded below the fixed
        // point must be allowed back up (stencil kernels; the cell-form
        // kernel keeps the reference's lower-only update).
        ctx->kp.relax = 1;
        rc = iterate(ctx, kernel, false, opts.polish_sweeps, tol, opts.stop_rule,
                     opts.warm_start != 0, opts.progress_every, done, cb, user, &pdone, &d2, &dm2,
                     &kms, &conv2);
        ctx->kp.relax = 0;
        if (rc) return rc;
        d = d2;
        dm = dm2;
    }
    if (res) {
        res->iterations = done + pdone;
        res->polish_iterations = pdone;
        res->last_delta = d;
        res->last_maxnorm = dm;
        res->kernel_ms = kms;
        res->cell_controls = (int64_t)(done + pdone) * ctx->kp.ncells * ctx->kp.nctl;
        res->elapsed_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return PG_OK;
}

int pg_get_value(pg_ctx* ctx, float* V_out) {
    int rc = check_ctx(ctx, true);
    if (rc) return rc;
    if (!V_out) return fail(PG_EINVAL, "null output");
    rc = ensure_stage(ctx);
    if (rc) return rc;
    cudaError_t e = pg::launch_to_rowmajor(ctx->storage, ctx->V[ctx->cur], ctx->stage_d, ctx->kp,
                                           ctx->stream);
    ctx->launches += 1;
    if (e != cudaSuccess) return fail(PG_ECUDA, "to_rowmajor");
    PG_CUDA(cudaMemcpyAsync(V_out, ctx->stage_d, (size_t)ctx->kp.ncells * 4, cudaMemcpyDeviceToHost,
                            ctx->stream));
    PG_CUDA(cudaStreamSynchronize(ctx->stream));
    return PG_OK;
}

int pg_set_value(pg_ctx* ctx, const float* V_in) {
    int rc = check_ctx(ctx, true);
    if (rc) return rc;
    if (!V_in) return fail(PG_EINVAL, "null input");
    rc = ensure_stage(ctx);
    if (rc) return rc;
    PG_CUDA(cudaMemcpyAsync(ctx->stage_d, V_in, (size_t)ctx->kp.ncells * 4, cudaMemcpyHostToDevice,
                            ctx->stream));
    cudaError_t e = pg::launch_from_rowmajor(ctx->storage, ctx->stage_d, ctx->V[ctx->cur], ctx->kp,
                                             ctx->stream);
    ctx->launches += 1;
    if (e != cudaSuccess) return fail(PG_ECUDA, "from_rowmajor");
    PG_CUDA(cudaStreamSynchronize(ctx->stream));
    return PG_OK;
}

int pg_sweep(pg_ctx* ctx, int32_t phase, int32_t kernel, double* delta, double* maxnorm,
             int16_t* argmin_out) {
    int rc = check_ctx(ctx, true);
    if (rc) return rc;
    int k = 0;
    rc = pick_kernel(ctx, kernel, &k);
    if (rc) return rc;
    if (argmin_out && !ctx->argmin_d)
        PG_CUDA(cudaMalloc(&ctx->argmin_d, (size_t)ctx->kp.ncells * sizeof(int16_t)));
    rc = sweep_async(ctx, k, phase, false, argmin_out ? ctx->argmin_d : nullptr, false);
    if (rc) return rc;
    double d = 0, dm = 0;
    rc = read_residual(ctx, &d, &dm);
    if (rc) return rc;
    if (delta) *delta = d;
    if (maxnorm) *maxnorm = dm;
    if (argmin_out) {
        PG_CUDA(cudaMemcpyAsync(argmin_out, ctx->argmin_d, (size_t)ctx->kp.ncells * sizeof(int16_t),
                                cudaMemcpyDeviceToHost, ctx->stream));
        PG_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return PG_OK;
}

int pg_escape_sweep(pg_ctx* ctx, int32_t phase, double* delta) {
    int rc = check_ctx(ctx, true);
    if (rc) return rc;
    rc = sweep_async(ctx, PG_KERNEL_CELLFORM, phase, true, nullptr, false);
    if (rc) return rc;
    double d = 0, dm = 0;
    rc = read_residual(ctx, &d, &dm);
    if (rc) return rc;
    if (delta) *delta = d;
    return PG_OK;
}

int pg_solve_escape(pg_ctx* ctx, int32_t iters, double tol, pg_solve_result* res,
                    pg_progress_cb cb, void* user) {
    auto t0 = std::chrono::steady_clock::now();
    int rc = check_ctx(ctx, true);
    if (rc) return rc;
    int32_t done = 0;
    double d = INFINITY, dm = INFINITY, kms = 0.0;
    bool conv = false;
    rc = iterate(ctx, PG_KERNEL_CELLFORM, true, iters, tol, PG_STOP_L1_QUIET, false, 0, 0, cb,
                 user, &done, &d, &dm, &kms, &conv);
    if (rc) return rc;
    if (res) {
        std::memset(res, 0, sizeof(*res));
        res->iterations = done;
        res->last_delta = d;
        res->last_maxnorm = dm;
        res->kernel_ms = kms;
        res->cell_controls = (int64_t)done * ctx->kp.ncells * ctx->kp.nctl;
        res->elapsed_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return PG_OK;
}

int pg_encode(pg_ctx* ctx, int32_t dtype, double scale, double escape_scale, int64_t lo,
              int64_t n, uint8_t* out, int64_t* reached, int64_t* escaped) {
    int rc = check_ctx(ctx, true);
    if (rc) return rc;
    if (dtype < PG_DTYPE_U8 || dtype > PG_DTYPE_F32) return fail(PG_EINVAL, "unknown dtype");
    if (lo < 0 || n < 0 || lo + n > ctx->kp.ncells) return fail(PG_EINVAL, "range outside the grid");
    if (n == 0) {
        if (reached) *reached = 0;
        if (escaped) *escaped = 0;
        return PG_OK;
    }
    if (!out) return fail(PG_EINVAL, "null output");
    if ((dtype == PG_DTYPE_U8 || dtype == PG_DTYPE_U16) && !(scale > 0.0))
        return fail(PG_EINVAL, "scale must be positive");
    const size_t eb = dtype == PG_DTYPE_U8 ? 1 : (dtype == PG_DTYPE_F32 ? 4 : 2);
    const size_t need = (size_t)n * eb;
    if (ctx->enc_cap < need) {
        if (ctx->enc_d) cudaFree(ctx->enc_d);
        ctx->enc_d = nullptr;
        ctx->enc_cap = 0;
        PG_CUDA(cudaMalloc(&ctx->enc_d, need));
        ctx->enc_cap = need;
    }
    PG_CUDA(cudaMemsetAsync(ctx->counts_d, 0, 2 * sizeof(unsigned long long), ctx->stream));
    cudaError_t e = pg::launch_encode(ctx->storage, ctx->V[ctx->cur], ctx->kp, dtype, scale,
                                      escape_scale, lo, n, ctx->enc_d, ctx->counts_d, ctx->stream);
    ctx->launches += 1;
    if (e != cudaSuccess) return fail(PG_ECUDA, "encode launch");
    unsigned long long cnt[2] = {0, 0};
    PG_CUDA(cudaMemcpyAsync(out, ctx->enc_d, need, cudaMemcpyDeviceToHost, ctx->stream));
    PG_CUDA(cudaMemcpyAsync(cnt, ctx->counts_d, sizeof(cnt), cudaMemcpyDeviceToHost, ctx->stream));
    PG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (reached) *reached = (int64_t)cnt[0];
    if (escaped) *escaped = (int64_t)cnt[1];
    return PG_OK;
}

int pg_time_sweeps(pg_ctx* ctx, int32_t warmup, int32_t steps, int32_t kernel,
                   double* ms_per_sweep) {
    int rc = check_ctx(ctx, true);
    if (rc) return rc;
    if (steps < 1 || warmup < 0) return fail(PG_EINVAL, "steps must be >= 1");
    int k = 0;
    rc = pick_kernel(ctx, kernel, &k);
    if (rc) return rc;
    for (int32_t i = 0; i < warmup; ++i) {
        rc = sweep_async(ctx, k, i, false, nullptr, false);
        if (rc) return rc;
    }
    PG_CUDA(cudaStreamSynchronize(ctx->stream));
    PG_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    for (int32_t i = 0; i < steps; ++i) {
        rc = sweep_async(ctx, k, warmup + i, false, nullptr, false);
        if (rc) return rc;
    }
    PG_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    PG_CUDA(cudaEventSynchronize(ctx->ev1));
    float ms = 0.0f;
    PG_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (ms_per_sweep) *ms_per_sweep = (double)ms / steps;
    return PG_OK;
}

int pg_adjoint(pg_ctx* ctx, const float* dl_dv, int32_t dl_dv_on_device, int32_t iters,
               double tol, double* grad18, pg_adjoint_result* res) {
    int rc = check_ctx(ctx, true);
    if (rc) return rc;
    if (!dl_dv || !grad18) return fail(PG_EINVAL, "null argument");
    if (!ctx->stencil_ok || !ctx->mask_ok)
        return fail(PG_EUNSUPPORTED, "the adjoint needs the plain scheme with the masked stencil's "
                                     "records (" + (ctx->stencil_ok ? std::string("not enough device "
                                     "memory for them") : ctx->stencil_why) + ")");
    if (ctx->storage != PG_STORE_F32)
        return fail(PG_EUNSUPPORTED, "the adjoint runs on an FP32 table");
    const pg::KParams& kp = ctx->kp;
    const int64_t n = kp.ncells;
    if (!ctx->argmin_d)
        PG_CUDA(cudaMalloc(&ctx->argmin_d, (size_t)n * sizeof(int16_t)));
    double* lam[2] = {nullptr, nullptr};
    float* c = nullptr;
    uint8_t* active = nullptr;
    double* grad_d = nullptr;
    auto release = [&]() {
        if (lam[0]) cudaFree(lam[0]);
        if (lam[1]) cudaFree(lam[1]);
        if (c) cudaFree(c);
        if (active) cudaFree(active);
        if (grad_d) cudaFree(grad_d);
    };
    auto cuda_fail = [&](cudaError_t e, const char* what) {
        release();
        return fail(e == cudaErrorMemoryAllocation ? PG_ENOMEM : PG_ECUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
    };
    cudaError_t e = cudaMalloc(&lam[0], (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&lam[1], (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&c, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&active, (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&grad_d, pg::kNThetaHost * sizeof(double));
    if (e != cudaSuccess) return cuda_fail(e, "adjoint buffers");

    // the policy: one sweep with argmin into the spare buffer, V untouched
    pg::SweepBufs sb{ctx->part_sum, ctx->part_max, ctx->nparts, ctx->red_d};
    const void* vin = ctx->V[ctx->cur];
    void* spare = ctx->V[1 - ctx->cur];
    if (ctx->rblend_ok)
        e = pg::launch_stencil_r(ctx->storage, vin, spare, ctx->occ_d, ctx->recs_d, ctx->tmask_d,
                                 kp, ctx->gord_d, sb, ctx->argmin_d, ctx->stream, &ctx->launches);
    else if (ctx->blend_ok)
        e = pg::launch_stencil_b(ctx->storage, vin, spare, ctx->occ_d, ctx->mask_d, ctx->recs_d,
                                 kp, ctx->order_d, sb, ctx->argmin_d, ctx->stream, &ctx->launches);
    else if (ctx->gather_ok)
        e = pg::launch_stencil_u(ctx->storage, vin, spare, ctx->occ_d, ctx->mask_d, ctx->recs_d,
                                 kp, ctx->order_d, sb, ctx->argmin_d, ctx->stream, &ctx->launches);
    else
        e = pg::launch_stencil(ctx->storage, false, vin, spare, ctx->occ_d, kp, ctx->ctl_d,
                               ctx->order_d, sb, ctx->argmin_d, ctx->stream, &ctx->launches);
    if (e != cudaSuccess) return cuda_fail(e, "policy sweep");

    double dm0 = 0.0;
    // c = dL/dV in the device layout
    if (dl_dv_on_device) {
        e = pg::launch_from_rowmajor(PG_STORE_F32, dl_dv, c, kp, ctx->stream);
    } else {
        rc = ensure_stage(ctx);
        if (rc) { release(); return rc; }
        e = cudaMemcpyAsync(ctx->stage_d, dl_dv, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) e = pg::launch_from_rowmajor(PG_STORE_F32, ctx->stage_d, c, kp, ctx->stream);
    }
    ctx->launches += 1;
    if (e == cudaSuccess)
        e = pg::launch_adj_active((const float*)vin, ctx->argmin_d, ctx->occ_d, ctx->mask_d,
                                  ctx->recs_d, kp, active, ctx->stream);
    ctx->launches += 1;
    double nact = 0.0;
    if (e == cudaSuccess) e = pg::launch_adj_count(active, n, sb, ctx->stream);
    ctx->launches += 2;
    if (e != cudaSuccess) return cuda_fail(e, "adjoint set-up");
    rc = read_residual(ctx, &nact, &dm0);
    if (rc) { release(); return rc; }
    // lambda_0 = c, and the first sweep's output starts from c
    if (e == cudaSuccess) e = pg::launch_adj_start(c, lam[0], lam[1], n, sb, ctx->stream);
    ctx->launches += 2;
    if (e != cudaSuccess) return cuda_fail(e, "adjoint set-up");
    double cn = 0.0, dm = 0.0;
    rc = read_residual(ctx, &cn, &dm);
    if (rc) { release(); return rc; }

    // lambda <- c + P^T lambda until quiet; the step kernel measures the
    // change and resets the older buffer to c for the next sweep
    int cur = 0, done = 0;
    double r = INFINITY, kms = 0.0;
    for (int32_t it = 1; it <= iters && cn > 0.0; ++it) {
        double* lin = lam[cur];
        double* lout = lam[1 - cur];
        PG_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
        e = pg::launch_adj_scatter(lin, lout, ctx->argmin_d, active, ctx->recs_d, kp, ctx->stream);
        if (e == cudaSuccess) e = pg::launch_adj_step(lout, lin, c, n, sb, ctx->stream);
        ctx->launches += 3;
        if (e != cudaSuccess) return cuda_fail(e, "adjoint sweep");
        PG_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
        rc = read_residual(ctx, &r, &dm);
        if (rc) { release(); return rc; }
        float ms = 0.0f;
        PG_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        kms += ms;
        cur = 1 - cur;
        done = it;
        if (r <= tol * cn) break;
    }

    // dL/dtheta = lambda^T g_theta
    e = cudaMemsetAsync(grad_d, 0, pg::kNThetaHost * sizeof(double), ctx->stream);
    if (e == cudaSuccess)
        e = pg::launch_adj_grad((const float*)vin, lam[cur], ctx->argmin_d, active, ctx->recs_d, kp,
                                ctx->ctl_d, grad_d, ctx->stream);
    ctx->launches += 1;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(grad18, grad_d, pg::kNThetaHost * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint gradient");
    if (res) {
        std::memset(res, 0, sizeof(*res));
        res->iterations = done;
        res->last_residual = r;
        res->c_norm = cn;
        res->kernel_ms = kms;
        res->active_cells = (int32_t)nact;
    }
    release();
    return PG_OK;
}

int pg_set_tile_rows(pg_ctx* ctx, int32_t rows) {
    int rc = check_ctx(ctx, true);
    if (rc) return rc;
    pg::KParams& kp = ctx->kp;
    const int32_t n1 = kp.g.n[0], n2 = kp.g.n[1];
    const bool b_fits = (int64_t)rows * n2 <= pg::kBMaxTileCells;
    const bool r_fits = (int64_t)((rows + 6) / 4) * n2 <= pg::kRMaxWindowHost / 4;
    if (rows < 1 || rows > n1 || !(b_fits || r_fits))
        return fail(PG_EINVAL, "tile rows must be in [1, Nx] with rows * Ny <= 1024 or "
                               "ceil((rows + 3) / 4) * Ny <= 512");
    const int32_t nt = (n1 + rows - 1) / rows;
    const int64_t need = kp.nplanes * nt;
    if (need > ctx->nparts) {
        double *ps = nullptr, *pm = nullptr;
        PG_CUDA(cudaMalloc(&ps, sizeof(double) * need));
        if (cudaMalloc(&pm, sizeof(double) * need) != cudaSuccess) {
            cudaFree(ps);
            return fail(PG_ENOMEM, "no room for the partials of that tiling");
        }
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->part_sum);
        cudaFree(ctx->part_max);
        ctx->part_sum = ps;
        ctx->part_max = pm;
        ctx->nparts = need;
    }
    if (b_fits) {
        const int64_t cells = (int64_t)rows * n2;
        int64_t th = 32 * (((cells + 2) / 3 + 31) / 32);
        th = std::max<int64_t>(64, std::min<int64_t>(256, th));
        kp.btile_x = rows;
        kp.btiles_x = nt;
        kp.bblock = (int32_t)th;
    } else {
        kp.btile_x = kp.btiles_x = kp.bblock = 0;
    }
    ctx->blend_ok = ctx->mask_ok && ctx->storage != PG_STORE_F64 && b_fits &&
                    pg::stencil_b_smem_bytes(kp) <= 200 * 1024;
    r_tiling(kp, r_fits ? rows : -1);
    return build_r_tables(ctx);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// batched solves
// ---------------------------------------------------------------------------

struct pg_batch {
    int device = 0;
    int storage = PG_STORE_F32;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<pg_ctx*> tabs;
    std::vector<std::vector<int64_t>> seeds;
    std::vector<int32_t> sweeps;
    std::vector<double> last_max;
    pg::BatchTable* tabs_d = nullptr;
    double* part_sum = nullptr;
    double* part_max = nullptr;
    double* out_d = nullptr;
    double* out_h = nullptr;
    int32_t* done_d = nullptr;
    int32_t* done_h = nullptr;
    int64_t cap_items = 0;
    int cap_tabs = 0;

    void free_bufs() {
        if (tabs_d) cudaFree(tabs_d);
        if (part_sum) cudaFree(part_sum);
        if (part_max) cudaFree(part_max);
        if (out_d) cudaFree(out_d);
        if (out_h) cudaFreeHost(out_h);
        if (done_d) cudaFree(done_d);
        if (done_h) cudaFreeHost(done_h);
        tabs_d = nullptr; part_sum = part_max = out_d = out_h = nullptr;
        done_d = done_h = nullptr;
        cap_items = 0;
        cap_tabs = 0;
    }
};

namespace {

// Descriptors of every table at storage `st` (the V buffers of each
// context, its masks and records), ordered by the tables' block size so each
// block size is one contiguous item range; perm[k] = the table of
// descriptor k; smem_out = the largest shared memory.
struct BatchGroup {
    int64_t first, count;
    int threads;
    bool any_vec, any_scalar;
    bool off32;  // every table of the group has fewer than 2^32 cells
};

// The batch runs the register-resident item when every table can (its
// tables and tile-order mask are built), else the re-reading blend item.
bool batch_uses_r(const pg_batch* b) {
    for (const pg_ctx* c : b->tabs)
        if (!c->rblend_ok) return false;
    return !b->tabs.empty();
}

int batch_descriptors(pg_batch* b, int st, std::vector<pg::BatchTable>& d, std::vector<int>& perm,
                      std::vector<BatchGroup>& groups, int64_t* nitems, size_t* smem_out) {
    d.clear();
    groups.clear();
    const int ntab = (int)b->tabs.size();
    const bool use_r = batch_uses_r(b);
    for (const pg_ctx* c : b->tabs)
        if (!use_r && !c->blend_ok)
            return fail(PG_EUNSUPPORTED, "the batch's tables cannot share one blend-then-shift "
                                         "sweep (mixed eligibility of the two kernels)");
    auto threads_of = [&](const pg_ctx* c) { return use_r ? c->kp.rblock : c->kp.bblock; };
    perm.resize(ntab);
    for (int t = 0; t < ntab; ++t) perm[t] = t;
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int c) {
        return threads_of(b->tabs[a]) < threads_of(b->tabs[c]);
    });
    int64_t item = 0;
    size_t smem = 0;
    const int vn = 16 / (int)elem_bytes(st);
    for (int k = 0; k < ntab; ++k) {
        pg_ctx* c = b->tabs[perm[k]];
        pg::BatchTable t{};
        t.V[0] = c->V[0];
        t.V[1] = c->V[1];
        t.occ = c->occ_d;
        t.mask = c->mask_d;
        t.recs = c->recs_d;
        t.order = c->order_d;
        t.tmask = c->tmask_d;
        t.gord = c->gord_d;
        t.kp = c->kp;
        t.kp.tile_x = use_r ? c->kp.rtile_x : c->kp.btile_x;
        t.kp.tiles_x = use_r ? c->kp.rtiles_x : c->kp.btiles_x;
        t.item0 = item;
        t.nitems = c->kp.nplanes * t.kp.tiles_x;
        t.vec = c->kp.g.n[1] % vn == 0 ? 1 : 0;
        if (groups.empty() || groups.back().threads != threads_of(c))
            groups.push_back(BatchGroup{item, 0, threads_of(c), false, false, true});
        groups.back().count += t.nitems;
        if (c->kp.ncells > (int64_t)0xffffffffLL) groups.back().off32 = false;
        (t.vec ? groups.back().any_vec : groups.back().any_scalar) = true;
        item += t.nitems;
        smem = std::max(smem, use_r ? pg::stencil_r_smem_bytes(c->kp)
                                    : pg::stencil_b_smem_bytes(c->kp));
        d.push_back(t);
    }
    *nitems = item;
    *smem_out = smem;
    return PG_OK;
}

// Sweep every not-yet-converged table, two sweeps per step, until each has
// a step whose second sweep moved no cell by more than tol, or max_sweeps.
int batch_phase(pg_batch* b, int st, int32_t max_sweeps, double tol, bool use_graph,
                double* kms, int32_t* steps_sweeps) {
    std::vector<pg::BatchTable> d;
    std::vector<int> perm;
    std::vector<BatchGroup> groups;
    int64_t nitems = 0;
    size_t smem = 0;
    int drc = batch_descriptors(b, st, d, perm, groups, &nitems, &smem);
    if (drc) return drc;
    const int ntab = (int)b->tabs.size();
    if (nitems > b->cap_items || ntab > b->cap_tabs) {
        b->free_bufs();
        PG_CUDA(cudaMalloc(&b->tabs_d, sizeof(pg::BatchTable) * ntab));
        PG_CUDA(cudaMalloc(&b->part_sum, sizeof(double) * nitems));
        PG_CUDA(cudaMalloc(&b->part_max, sizeof(double) * nitems));
        PG_CUDA(cudaMalloc(&b->out_d, sizeof(double) * 2 * ntab));
        PG_CUDA(cudaMallocHost(&b->out_h, sizeof(double) * 2 * ntab));
        PG_CUDA(cudaMalloc(&b->done_d, sizeof(int32_t) * ntab));
        PG_CUDA(cudaMallocHost(&b->done_h, sizeof(int32_t) * ntab));
        b->cap_items = nitems;
        b->cap_tabs = ntab;
    }
    PG_CUDA(cudaMemcpyAsync(b->tabs_d, d.data(), sizeof(pg::BatchTable) * ntab,
                            cudaMemcpyHostToDevice, b->stream));
    for (int k = 0; k < ntab; ++k) b->done_h[k] = 0;
    PG_CUDA(cudaMemcpyAsync(b->done_d, b->done_h, sizeof(int32_t) * ntab, cudaMemcpyHostToDevice,
                            b->stream));
    int sms = 0;
    PG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    const bool use_r = batch_uses_r(b);
    std::vector<int> grids;
    for (const BatchGroup& gr : groups) {
        const int per_sm = use_r ? pg::r_batch_blocks_per_sm(st, smem, gr.threads)
                                 : pg::batch_blocks_per_sm(st, smem, gr.threads);
        if (per_sm <= 0) return fail(PG_EUNSUPPORTED, "the batched sweep does not fit on an SM");
        grids.push_back((int)std::min<int64_t>(gr.count, (int64_t)sms * per_sm));
    }

    auto step = [&](cudaStream_t s) -> cudaError_t {
        cudaError_t e = cudaSuccess;
        for (int parity = 0; parity < 2 && e == cudaSuccess; ++parity) {
            for (size_t g = 0; g < groups.size() && e == cudaSuccess; ++g)
                e = use_r ? pg::launch_stencil_r_batch(st, b->tabs_d, ntab, groups[g].first,
                                                       groups[g].count, groups[g].threads, parity,
                                                       b->done_d, b->part_sum, b->part_max, smem,
                                                       grids[g], s)
                          : pg::launch_stencil_b_batch(st, b->tabs_d, ntab, groups[g].first,
                                                       groups[g].count, groups[g].threads, parity,
                                                       b->done_d, b->part_sum, b->part_max, smem,
                                                       grids[g], groups[g].any_vec,
                                                       groups[g].any_scalar, groups[g].off32, s);
            if (e == cudaSuccess)
                e = pg::launch_reduce_batch(b->tabs_d, ntab, b->part_sum, b->part_max, b->out_d, s);
        }
        return e;
    };
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (use_graph) {
        PG_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = step(b->stream);
        cudaError_t e2 = cudaStreamEndCapture(b->stream, &graph);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            return fail(PG_ECUDA, "graph capture of the batched sweep failed");
        }
        e = cudaGraphInstantiate(&exec, graph, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(graph);
            return fail(PG_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
    }
    int rc = PG_OK;
    int32_t done_sw = 0;
    while (done_sw < max_sweeps) {
        cudaError_t e = cudaEventRecord(b->ev0, b->stream);
        if (e == cudaSuccess) e = use_graph ? cudaGraphLaunch(exec, b->stream) : step(b->stream);
        if (e == cudaSuccess) e = cudaEventRecord(b->ev1, b->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(b->out_h, b->out_d, sizeof(double) * 2 * ntab,
                                cudaMemcpyDeviceToHost, b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, b->ev0, b->ev1);
        if (e != cudaSuccess) {
            rc = fail(PG_ECUDA, std::string("batched sweep: ") + cudaGetErrorString(e));
            break;
        }
        *kms += ms;
        done_sw += 2;
        int left = 0;
        for (int k = 0; k < ntab; ++k) {
            if (b->done_h[k]) continue;
            const int t = perm[k];
            b->sweeps[t] += 2;
            b->last_max[t] = b->out_h[2 * k + 1];
            if (b->last_max[t] <= tol) b->done_h[k] = 1;
            else ++left;
        }
        if (!left) break;
        e = cudaMemcpyAsync(b->done_d, b->done_h, sizeof(int32_t) * ntab, cudaMemcpyHostToDevice,
                            b->stream);
        if (e != cudaSuccess) {
            rc = fail(PG_ECUDA, std::string("batched sweep: ") + cudaGetErrorString(e));
            break;
        }
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    *steps_sweeps = done_sw;
    return rc;
}

}  // namespace

extern "C" {

int pg_batch_create(pg_batch** out, int device, int32_t storage) {
    if (!out) return fail(PG_EINVAL, "null output pointer");
    if (storage != PG_STORE_F32 && storage != PG_STORE_F16 && storage != PG_STORE_BF16 &&
        storage != PG_STORE_Q16)
        return fail(PG_EUNSUPPORTED, "batched solves store V in FP32, FP16, BF16 or Q16");
    PG_CUDA(cudaSetDevice(device));
    pg_batch* b = new pg_batch();
    b->device = device;
    b->storage = storage;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess) {
        delete b;
        return fail(PG_ECUDA, "batch creation failed");
    }
    *out = b;
    return PG_OK;
}

int pg_batch_destroy(pg_batch* b) {
    if (!b) return PG_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    for (pg_ctx* c : b->tabs) pg_destroy(c);
    b->free_bufs();
    cudaEventDestroy(b->ev0);
    cudaEventDestroy(b->ev1);
    cudaStreamDestroy(b->stream);
    delete b;
    return PG_OK;
}

int pg_batch_add(pg_batch* b, const pg_grid6* g, const pg_model* m, const pg_params* p,
                 const uint8_t* occ, const int64_t* tidx, int64_t ntidx, const float* ctl,
                 int32_t nctl, int32_t tile_rows, int32_t* index) {
    if (!b) return fail(PG_EINVAL, "null batch");
    if (ntidx < 0 || (ntidx > 0 && !tidx)) return fail(PG_EINVAL, "bad seed list");
    pg_ctx* c = nullptr;
    int rc = pg_create(&c, b->device);
    if (rc) return rc;
    rc = pg_load_problem(c, g, m, p, occ, ctl, nctl, b->storage);
    if (!rc && tile_rows > 0) rc = pg_set_tile_rows(c, tile_rows);
    if (!rc && !(c->stencil_ok && ((c->mask_ok && c->blend_ok) || c->rblend_ok)))
        rc = fail(PG_EUNSUPPORTED, "a batched table must run a blend-then-shift sweep (" +
                                       (c->stencil_ok ? std::string("its records do not fit")
                                                      : c->stencil_why) + ")");
    for (int64_t t = 0; !rc && t < ntidx; ++t)
        if (tidx[t] < 0 || tidx[t] >= c->kp.ncells)
            rc = fail(PG_EINVAL, "seed index outside the grid");
    if (rc) {
        pg_destroy(c);
        return rc;
    }
    b->tabs.push_back(c);
    b->seeds.emplace_back(tidx, tidx + ntidx);
    b->sweeps.push_back(0);
    b->last_max.push_back(INFINITY);
    if (index) *index = (int32_t)b->tabs.size() - 1;
    return PG_OK;
}

int pg_batch_solve(pg_batch* b, int32_t iters, double tol, int32_t polish_sweeps,
                   int32_t use_graph, pg_batch_result* res) {
    auto t0 = std::chrono::steady_clock::now();
    if (!b || b->tabs.empty()) return fail(PG_EINVAL, "empty batch");
    PG_CUDA(cudaSetDevice(b->device));
    const int ntab = (int)b->tabs.size();
    // seed every table into V[0]
    for (int t = 0; t < ntab; ++t) {
        pg_ctx* c = b->tabs[t];
        c->kp.relax = 0;
        int rc = ensure_values(c, c->base_storage);
        if (rc) return rc;
        const int64_t nt = (int64_t)b->seeds[t].size();
        if (nt > c->tidx_cap) {
            if (c->tidx_d) cudaFree(c->tidx_d);
            c->tidx_d = nullptr;
            PG_CUDA(cudaMalloc(&c->tidx_d, sizeof(int64_t) * nt));
            c->tidx_cap = nt;
        }
        if (nt > 0)
            PG_CUDA(cudaMemcpyAsync(c->tidx_d, b->seeds[t].data(), sizeof(int64_t) * nt,
                                    cudaMemcpyHostToDevice, c->stream));
        c->ntidx = nt;
        c->cur = 0;
        cudaError_t e = pg::launch_fill_seed(c->storage, c->V[0], c->kp, c->tidx_d, nt, c->stream);
        c->launches += 1;
        if (e != cudaSuccess) return fail(PG_ECUDA, std::string("fill: ") + cudaGetErrorString(e));
        PG_CUDA(cudaStreamSynchronize(c->stream));
        b->sweeps[t] = 0;
        b->last_max[t] = INFINITY;
    }
    double kms = 0.0;
    int32_t sw = 0, psw = 0;
    int rc = batch_phase(b, b->storage, iters, tol, use_graph != 0, &kms, &sw);
    if (rc) return rc;
    int32_t conv = 0;
    for (int t = 0; t < ntab; ++t) conv += b->last_max[t] <= tol ? 1 : 0;
    // 16-bit storage: continue every table in FP32 with plain value iteration
    if (b->storage != PG_STORE_F32 && polish_sweeps > 0) {
        for (int t = 0; t < ntab; ++t) {
            pg_ctx* c = b->tabs[t];
            const size_t bytes = (size_t)c->kp.ncells * 4;
            void* nv[2] = {nullptr, nullptr};
            PG_CUDA(cudaMalloc(&nv[0], bytes));
            if (cudaMalloc(&nv[1], bytes) != cudaSuccess) {
                cudaFree(nv[0]);
                return fail(PG_ENOMEM, "no room for the FP32 polish buffers");
            }
            cudaError_t e = pg::launch_convert_to_f32(c->storage, c->V[0], (float*)nv[0],
                                                      c->kp.ncells, c->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
            if (e != cudaSuccess) {
                cudaFree(nv[0]);
                cudaFree(nv[1]);
                return fail(PG_ECUDA, "convert");
            }
            c->free_values();
            c->V[0] = nv[0];
            c->V[1] = nv[1];
            c->cur = 0;
            c->storage = PG_STORE_F32;
            c->kp.relax = 1;
        }
        rc = batch_phase(b, PG_STORE_F32, polish_sweeps, tol, use_graph != 0, &kms, &psw);
        for (pg_ctx* c : b->tabs) c->kp.relax = 0;
        if (rc) return rc;
        conv = 0;
        for (int t = 0; t < ntab; ++t) conv += b->last_max[t] <= tol ? 1 : 0;
    }
    if (res) {
        std::memset(res, 0, sizeof(*res));
        res->tables = ntab;
        res->converged = conv;
        res->sweeps = sw;
        res->polish_sweeps = psw;
        res->graph = use_graph ? 1 : 0;
        res->kernel_ms = kms;
        int64_t cc = 0;
        for (int t = 0; t < ntab; ++t)
            cc += (int64_t)b->sweeps[t] * b->tabs[t]->kp.ncells * b->tabs[t]->kp.nctl;
        res->cell_controls = cc;
        res->elapsed_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return PG_OK;
}

int pg_batch_table(pg_batch* b, int32_t table, int32_t* sweeps, double* last_maxnorm,
                   pg_ctx** ctx) {
    if (!b || table < 0 || table >= (int32_t)b->tabs.size())
        return fail(PG_EINVAL, "no such table in the batch");
    if (sweeps) *sweeps = b->sweeps[table];
    if (last_maxnorm) *last_maxnorm = b->last_max[table];
    if (ctx) *ctx = b->tabs[table];
    return PG_OK;
}

int pg_set_wait_timeout(pg_ctx* ctx, double seconds) {
    if (!ctx) return fail(PG_EINVAL, "null context");
    if (!(seconds >= 0.0) || !std::isfinite(seconds))
        return fail(PG_EINVAL, "the wait limit must be a finite number of seconds >= 0");
    ctx->wait_timeout_s = seconds;
    return PG_OK;
}

int pg_launch_count(pg_ctx* ctx, int64_t* launches) {
    if (!ctx || !launches) return fail(PG_EINVAL, "null argument");
    *launches = ctx->launches;
    return PG_OK;
}

}  // extern "C"

// ---- self-test probes ------------------------------------------------------

namespace {
// Device copies of a probe's host inputs and its output, freed on scope exit.
struct ProbeBufs {
    std::vector<void*> ptrs;
    ~ProbeBufs() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T> cudaError_t put(T** d, const T* h, int64_t n) {
        cudaError_t e = cudaMalloc((void**)d, (size_t)std::max<int64_t>(n, 1) * sizeof(T));
        if (e != cudaSuccess) return e;
        ptrs.push_back(*d);
        return h ? cudaMemcpy(*d, h, (size_t)n * sizeof(T), cudaMemcpyHostToDevice) : cudaSuccess;
    }
};
}  // namespace

extern "C" {

int pg_probe_step(int device, const pg_model* m, int32_t rk2, const float* states,
                  const float* controls, const float* dt, const int32_t* nsub, int64_t n,
                  float* out_states) {
    if (!m || (n > 0 && (!states || !controls || !dt || !nsub || !out_states)))
        return fail(PG_EINVAL, "null argument");
    if (n < 0) return fail(PG_EINVAL, "negative count");
    for (int64_t i = 0; i < n; ++i)
        if (nsub[i] < 1 || nsub[i] > 1 << 20) return fail(PG_EINVAL, "nsub out of range");
    if (n == 0) return PG_OK;
    PG_CUDA(cudaSetDevice(device));
    ProbeBufs b;
    float *s_d, *u_d, *dt_d, *o_d;
    int32_t* ns_d;
    PG_CUDA(b.put(&s_d, states, 6 * n));
    PG_CUDA(b.put(&u_d, controls, 3 * n));
    PG_CUDA(b.put(&dt_d, dt, n));
    PG_CUDA(b.put(&ns_d, nsub, n));
    PG_CUDA(b.put<float>(&o_d, nullptr, 6 * n));
    PG_CUDA(pg::launch_probe_step(*m, rk2, s_d, u_d, dt_d, ns_d, n, o_d, 0));
    PG_CUDA(cudaMemcpy(out_states, o_d, (size_t)6 * n * sizeof(float), cudaMemcpyDeviceToHost));
    return PG_OK;
}

int pg_probe_traction_gain(int device, const float* controls, float knee, int64_t n,
                           float* gain) {
    if (n > 0 && (!controls || !gain)) return fail(PG_EINVAL, "null argument");
    if (n < 0) return fail(PG_EINVAL, "negative count");
    if (n == 0) return PG_OK;
    PG_CUDA(cudaSetDevice(device));
    ProbeBufs b;
    float *u_d, *o_d;
    PG_CUDA(b.put(&u_d, controls, 3 * n));
    PG_CUDA(b.put<float>(&o_d, nullptr, n));
    PG_CUDA(pg::launch_probe_gain(u_d, knee, n, o_d, 0));
    PG_CUDA(cudaMemcpy(gain, o_d, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost));
    return PG_OK;
}

int pg_probe_interp(pg_ctx* ctx, const float* states, int64_t n, int32_t kuhn, int32_t nearest,
                    int32_t vclamp, float cap, float* values, float* grads) {
    int rc = check_ctx(ctx, true);
    if (rc) return rc;
    if (n > 0 && (!states || !values)) return fail(PG_EINVAL, "null argument");
    if (n < 0) return fail(PG_EINVAL, "negative count");
    if (ctx->storage == PG_STORE_F64)
        return fail(PG_EUNSUPPORTED, "the interpolation probe reads FP32 or 16-bit storage");
    if (n == 0) return PG_OK;
    PG_CUDA(cudaStreamSynchronize(ctx->stream));
    ProbeBufs b;
    float *s_d, *o_d, *g_d = nullptr;
    PG_CUDA(b.put(&s_d, states, 6 * n));
    PG_CUDA(b.put<float>(&o_d, nullptr, n));
    if (grads) PG_CUDA(b.put<float>(&g_d, nullptr, 6 * n));
    PG_CUDA(pg::launch_probe_interp(ctx->storage, ctx->V[ctx->cur], ctx->kp, s_d, n, kuhn,
                                    nearest, vclamp, cap, o_d, g_d, ctx->stream));
    ctx->launches += 1;
    PG_CUDA(cudaStreamSynchronize(ctx->stream));
    PG_CUDA(cudaMemcpy(values, o_d, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost));
    if (grads)
        PG_CUDA(cudaMemcpy(grads, g_d, (size_t)6 * n * sizeof(float), cudaMemcpyDeviceToHost));
    return PG_OK;
}

int pg_solve_value(pg_ctx* ctx, const pg_grid6* g, const pg_model* m, const pg_params* p,
                   const uint8_t* occ, const int64_t* tidx, int64_t ntidx, const float* ctl,
                   int32_t nctl, int32_t iters, double tol, const pg_solve_opts* opts,
                   float* V_out, pg_solve_result* res, pg_progress_cb cb, void* user) {
    pg_solve_opts o;
    if (opts) o = *opts;
    else pg_default_opts(&o);
    int rc = pg_load_problem(ctx, g, m, p, occ, ctl, nctl, o.storage);
    if (rc) return rc;
    rc = pg_solve(ctx, tidx, ntidx, iters, tol, &o, res, cb, user);
    if (rc) return rc;
    if (V_out) return pg_get_value(ctx, V_out);
    return PG_OK;
}

}  // extern "C"
