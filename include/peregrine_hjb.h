/*
 * peregrine_hjb.h -- C ABI of libperegrine_hjb.so, the B200 (sm_100a)
 * minimum-time value-table solver.
 *
 * This library replaces the value-iteration solve that Peregrine-Desktop's
 * `solver/solve.jl` drives through `solve_value!` (solver/src/Run.jl:1434-1474)
 * and the CUDA.jl sweep kernels behind it (solver/src/Gpu.jl:5-37). It is a
 * plain C interface: POD structs, pointers and sizes, no C++ or torch types.
 *
 * Conventions
 *   - Every entry point returns an int status: PG_OK (0) or a negative PG_E*
 *     code.  The message of the last failure on the calling thread is
 *     available from pg_last_error().  No exception ever crosses the ABI.
 *   - Flat cell indices are 0-based and follow the table's row-major order
 *     ((((ix*Ny+iy)*Nh+ih)*Nvx+ivx)*Nvy+ivy)*Nw+iw (docs/TABLE_FORMAT.md §4).
 *     The reference passes 1-based indices (`seeds = tcells .+ 1`,
 *     Run.jl:1853); this ABI does not add the 1.
 *   - The caller owns every host buffer; a context owns its device buffers.
 *     One context per host thread; each context has its own CUDA stream.
 *   - Progress callbacks run on the calling thread, between sweeps.
 */
#ifndef PEREGRINE_HJB_H
#define PEREGRINE_HJB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PG_ABI_VERSION 1

/* status codes */
#define PG_OK            0
#define PG_EINVAL       -1   /* bad argument (the reference's `error(...)`)   */
#define PG_ECUDA        -2   /* a CUDA runtime call failed                     */
#define PG_ENOMEM       -3   /* device allocation failed or would not fit      */
#define PG_ETIMEOUT     -4   /* a bounded device wait gave up                  */
#define PG_ESTATE       -5   /* call out of order (no problem loaded, ...)     */
#define PG_EUNSUPPORTED -6   /* option combination not implemented             */
#define PG_ECANCELLED   -7   /* the progress callback asked to stop            */

/* Grid6 (solver/src/PeregrineSolver.jl:47-51): samples per axis, axis origin
 * and step.  Axis 2 (heading) is periodic with lo = -pi, step = 2pi/n. */
typedef struct pg_grid6 {
    int32_t n[6];
    float lo[6];
    float step[6];
} pg_grid6;

/* Model (PeregrineSolver.jl:100-109): row-major 3x3 blocks. */
typedef struct pg_model {
    float B[9];     /* control                          */
    float A[9];     /* velocity                         */
    float q[3];     /* omega^2                          */
    float S[9];     /* Coulomb, multiplies csign(v)     */
    float D[9];     /* quadratic drag, multiplies |v|v  */
    float c[3];     /* constant                         */
    float eps[3];   /* Coulomb smoothing band           */
    float knee;     /* traction knee; <= 0 or NaN disables saturation */
} pg_model;

/* Params (PeregrineSolver.jl:897-916).  Booleans are int32 0/1. */
typedef struct pg_params {
    float dt;
    int32_t nsub;
    int32_t checks;
    int32_t adaptive_checks;
    int32_t nearest;
    float cap;
    int32_t ntau;
    float tau_ratio;
    float cfl;
    float tau_min;
    float tau_max;
    float hmax;
    int32_t ncoarse;
    int32_t rounds;
    float delta0;
    int32_t rk2;
    int32_t vclamp;
    int32_t simplex;
} pg_params;

/* Stop rule.  L1_QUIET is the reference's: total improvement of a sweep
 * <= tol for ceil((nctl-1)/ncoarse) consecutive sweeps (Run.jl:1441-1471).
 * MAXNORM stops on the largest single-cell change instead. */
#define PG_STOP_L1_QUIET 0
#define PG_STOP_MAXNORM  1

/* Storage of V on the device.  Arithmetic is FP32 for F32/F16/BF16 and FP64
 * for F64 (the FP64 device oracle). */
#define PG_STORE_F32  0
#define PG_STORE_F16  1
#define PG_STORE_BF16 2
#define PG_STORE_F64  3
/* Q16: unsigned 16-bit fixed point, V = code * 2^-11 s (0.49 ms steps,
 * 0..32 s; value_cap must be below 32 s).  Swept by the blend-then-shift
 * kernel only; a 16-bit storage like F16/BF16, with the FP32 polish. */
#define PG_STORE_Q16  4

/* Sweep kernel selection. */
#define PG_KERNEL_AUTO     0  /* stencil when the scheme allows it, else cellform */
#define PG_KERNEL_STENCIL  1  /* position-invariant stencil (plain scheme)     */
#define PG_KERNEL_CELLFORM 2  /* one thread per cell, the full cell_update     */
#define PG_KERNEL_STENCIL_EXACT 3 /* stencil with the reference's rounding order */
#define PG_KERNEL_STENCIL_ROWS  4 /* stencil deciding every probe per sweep (no mask) */
#define PG_KERNEL_STENCIL_GATHER 5 /* masked stencil gathering all 64 corners per cell */
#define PG_KERNEL_STENCIL_BLEND  6 /* masked stencil, blend-then-shift re-reading the
                                      corner planes per control (PG_KERNEL_STENCIL runs
                                      the register-resident blend where it fits; both
                                      give bit-identical tables) */

/* Table dtypes (solver/src/Pipeline.jl:620-625). */
#define PG_DTYPE_U8  0
#define PG_DTYPE_U16 1
#define PG_DTYPE_F16 2
#define PG_DTYPE_F32 3

typedef struct pg_solve_opts {
    int32_t stop_rule;      /* PG_STOP_*                                         */
    int32_t storage;        /* PG_STORE_*                                        */
    int32_t kernel;         /* PG_KERNEL_*                                       */
    int32_t warm_start;     /* keep the Int8 warm-start policy (Run.jl:1784)     */
    int32_t polish_sweeps;  /* 16-bit storage: max FP32 sweeps after convergence */
    int32_t progress_every; /* callback cadence; 0 = reference cadence (it%5, 1, last) */
    int32_t reserved[6];
} pg_solve_opts;

typedef struct pg_solve_result {
    int32_t iterations;     /* sweeps run (16-bit phase + polish)                */
    int32_t polish_iterations;
    double last_delta;      /* L1 total improvement of the last sweep            */
    double last_maxnorm;    /* largest single-cell improvement of the last sweep */
    double kernel_ms;       /* device time of the sweeps (CUDA events)           */
    double elapsed_ms;      /* host wall time of the call                        */
    int64_t cell_controls;  /* lookaheads evaluated over all sweeps (all cells)  */
} pg_solve_result;

/* Return nonzero to cancel the solve (PG_ECANCELLED). */
typedef int (*pg_progress_cb)(void* user, int32_t iter, double delta, double maxnorm);

typedef struct pg_ctx pg_ctx;

/* ------------------------------------------------------------------ */
/* library                                                             */
/* ------------------------------------------------------------------ */
int32_t pg_abi_version(void);
const char* pg_last_error(void);
void pg_default_opts(pg_solve_opts* opts);

/* Create a context on CUDA device `device`; its own stream. */
int pg_create(pg_ctx** out, int device);
int pg_destroy(pg_ctx* ctx);

/* ------------------------------------------------------------------ */
/* one-shot solve: the drop-in for solve_value!                        */
/*   solve_value!(V, occ, g, m, tidx, ctl, nctl, p; iters, tol, ...)   */
/*   (solver/src/Run.jl:1434-1474)                                     */
/* occ: Nx*Ny*Nh bytes, index (ix*Ny+iy)*Nh+ih (Pipeline.jl:393-398).  */
/* ctl: planar [u1(nctl) u2(nctl) u3(nctl)] (Run.jl:283-285).          */
/* tidx: 0-based seeded target cells.  V_out: ncells floats, row-major */
/* (may be NULL to keep V on the device for pg_get_value/pg_encode).   */
/* ------------------------------------------------------------------ */
int pg_solve_value(pg_ctx* ctx, const pg_grid6* g, const pg_model* m,
                   const pg_params* p, const uint8_t* occ,
                   const int64_t* tidx, int64_t ntidx,
                   const float* ctl, int32_t nctl,
                   int32_t iters, double tol, const pg_solve_opts* opts,
                   float* V_out, pg_solve_result* res,
                   pg_progress_cb cb, void* user);

/* ------------------------------------------------------------------ */
/* staged use: load the problem once, then solve / sweep / read        */
/* ------------------------------------------------------------------ */

/* Upload grid, model, params, occupancy and control table and allocate the
 * device value buffers for `storage`.  Replaces the allocations of
 * run_solve (Run.jl:1776-1784). */
int pg_load_problem(pg_ctx* ctx, const pg_grid6* g, const pg_model* m,
                    const pg_params* p, const uint8_t* occ,
                    const float* ctl, int32_t nctl, int32_t storage);

/* Load one x slab of a table: its interior rows [x0, x1) and `halo` rows
 * either side (clipped to the table), FP32 storage.  Sweeps (pg_sweep,
 * pg_solve with the row stencil) update the interior only and pass the halo
 * through; every coordinate, range test and occupancy lookup uses the global
 * row, so a slab sweep equals the whole-table sweep on its interior as long
 * as the halo covers one backup's reach in x.  occ is the whole table's; the
 * context's rows are the global rows [*row0, *row0 + *rows), seeds passed
 * to pg_solve are indices into that slab's row-major order.  For tables
 * split over several GPUs (and for the reference's tiles, Tiles.jl:311-340). */
int pg_load_slab(pg_ctx* ctx, const pg_grid6* g, const pg_model* m, const pg_params* p,
                 const uint8_t* occ, const float* ctl, int32_t nctl, int32_t x0, int32_t x1,
                 int32_t halo, int32_t* row0, int32_t* rows);

/* Rows [r0, r1) of the loaded table (the slab's rows for a slab), FP32
 * row-major, to or from a host buffer, or a device buffer on the context's
 * device when on_device is nonzero (for a halo exchange over NCCL). */
int pg_get_rows(pg_ctx* ctx, int32_t r0, int32_t r1, void* out, int32_t on_device);
int pg_set_rows(pg_ctx* ctx, int32_t r0, int32_t r1, const void* in, int32_t on_device);

/* Seed and iterate on the loaded problem (solve_value!, Run.jl:1434-1474). */
int pg_solve(pg_ctx* ctx, const int64_t* tidx, int64_t ntidx, int32_t iters,
             double tol, const pg_solve_opts* opts, pg_solve_result* res,
             pg_progress_cb cb, void* user);

/* Device V <-> host, row-major f32 (the reference's Array(V), Run.jl:1954). */
int pg_get_value(pg_ctx* ctx, float* V_out);
int pg_set_value(pg_ctx* ctx, const float* V_in);

/* One Jacobi sweep V <- min(V, T V) on the loaded problem, `phase` as in
 * sweep_gpu! (Gpu.jl:27-37).  delta = L1 total improvement, maxnorm = the
 * largest single-cell improvement.  When `argmin_out` is non-NULL it gets,
 * per cell (row-major), the index of the winning control in the control
 * table, or -1 for a blocked cell. */
int pg_sweep(pg_ctx* ctx, int32_t phase, int32_t kernel, double* delta,
             double* maxnorm, int16_t* argmin_out);

/* One escape sweep (Gpu.jl:51-80 semantics, Jacobi) on the loaded V. */
int pg_escape_sweep(pg_ctx* ctx, int32_t phase, double* delta);

/* Escape pass driver (solve_escape!, Run.jl:1503-1530). */
int pg_solve_escape(pg_ctx* ctx, int32_t iters, double tol,
                    pg_solve_result* res, pg_progress_cb cb, void* user);

/* Encode V[lo, lo+n) (row-major) on the device into a host buffer
 * (encode_into!, Pipeline.jl:698-780).  out must hold n*elem_bytes. */
int pg_encode(pg_ctx* ctx, int32_t dtype, double scale, double escape_scale,
              int64_t lo, int64_t n, uint8_t* out, int64_t* reached,
              int64_t* escaped);

/* Device-timed sweeps on the loaded, seeded problem: runs `warmup` untimed
 * and `steps` timed sweeps with CUDA events on the context stream and
 * returns the mean milliseconds per sweep.  No host copies inside. */
int pg_time_sweeps(pg_ctx* ctx, int32_t warmup, int32_t steps, int32_t kernel,
                   double* ms_per_sweep);

/* A limit on each wait for a sweep in the solve loops (pg_solve,
 * pg_solve_value, pg_solve_escape, pg_sweep): when the sweep and its
 * residual copy have not finished `seconds` after the host starts waiting,
 * the call returns PG_ETIMEOUT instead of blocking; the queued work still
 * completes on the device, and pg_destroy waits for it.  0 (the default)
 * waits without a limit.  The reference blocks in CUDA.synchronize after
 * every sweep (solver/src/Gpu.jl:33-36); this bounds that wait. */
int pg_set_wait_timeout(pg_ctx* ctx, double seconds);

/* Number of this library's kernel launches since the context was created. */
int pg_launch_count(pg_ctx* ctx, int64_t* launches);

/* Rows of one plane per tile of the blend-then-shift sweeps (the tile
 * shape the autotuner picks): 1 <= rows <= Nx, and rows * Ny <= 1024 (the
 * re-reading blend) or ceil((rows + 3) / 4) * Ny <= 512 (the register-
 * resident blend: its window has 3 more rows than the tile, and a thread
 * owns four window rows of one column); a kernel whose limit the rows
 * exceed is not used.  No counterpart in the reference (its kernel has one
 * thread per cell). */
int pg_set_tile_rows(pg_ctx* ctx, int32_t rows);

/* ------------------------------------------------------------------ */
/* batched solves: many independent tables swept side by side: per     */
/* sweep one persistent launch for each block size among the tables    */
/* (one launch when they share it), captured in a CUDA graph.  The     */
/* reference                                                            */
/* solves its targets one after another (Run.jl:1851-1958); this is the */
/* same per-table solve_value!, run side by side.                       */
/* ------------------------------------------------------------------ */

typedef struct pg_batch pg_batch;

typedef struct pg_batch_result {
    int32_t tables;
    int32_t converged;      /* tables whose last max-norm change <= tol      */
    int32_t sweeps;         /* batched sweeps of the storage phase           */
    int32_t polish_sweeps;  /* batched FP32 sweeps after a 16-bit phase      */
    int32_t graph;          /* 1 when the sweeps ran as a CUDA graph         */
    double kernel_ms;       /* device time of the batched sweeps             */
    double elapsed_ms;      /* host wall time of the call                    */
    int64_t cell_controls;  /* lookaheads of the tables' own sweeps          */
} pg_batch_result;

/* storage: PG_STORE_F32, F16 or BF16 for every table of the batch. */
int pg_batch_create(pg_batch** out, int device, int32_t storage);
int pg_batch_destroy(pg_batch* b);
/* Add one table (arguments as pg_load_problem + its seeds); tile_rows > 0
 * overrides the blend tiling (pg_set_tile_rows).  The table must run the
 * plain scheme with the blend-then-shift sweep. */
int pg_batch_add(pg_batch* b, const pg_grid6* g, const pg_model* m,
                 const pg_params* p, const uint8_t* occ, const int64_t* tidx,
                 int64_t ntidx, const float* ctl, int32_t nctl,
                 int32_t tile_rows, int32_t* index);
/* Seed every table and sweep them all, two Jacobi sweeps per step, until
 * each table's max-norm change is <= tol or `iters` sweeps ran; then, for
 * 16-bit storage, up to polish_sweeps FP32 sweeps of plain value iteration
 * (target cells pinned) under the same rule. */
int pg_batch_solve(pg_batch* b, int32_t iters, double tol,
                   int32_t polish_sweeps, int32_t use_graph,
                   pg_batch_result* res);
/* Sweeps and last max-norm change of one table, and its context (owned by
 * the batch; pg_get_value / pg_encode on it read the table). */
int pg_batch_table(pg_batch* b, int32_t table, int32_t* sweeps,
                   double* last_maxnorm, pg_ctx** ctx);

/* ------------------------------------------------------------------ */
/* adjoint: gradient of a loss on the converged table                  */
/* ------------------------------------------------------------------ */

typedef struct pg_adjoint_result {
    int32_t iterations;     /* adjoint sweeps run                              */
    int32_t active_cells;   /* cells whose backup depends on the model         */
    double last_residual;   /* L1 change of lambda in the last sweep           */
    double c_norm;          /* L1 norm of dL/dV                                */
    double kernel_ms;       /* device time of the adjoint sweeps               */
} pg_adjoint_result;

/* dL/dtheta for the 18 model entries theta = (B00 B11 B22, A00 A11 A22,
 * q0 q1 q2, S00 S11 S22, D00 D11 D22, c0 c1 c2) of the loaded problem, at
 * its current (converged) FP32 table, given dl_dv = dL/dV (ncells floats,
 * row-major; a device pointer when dl_dv_on_device, else host).  The policy
 * is the table's argmin (one extra sweep that leaves V unchanged); the
 * adjoint lambda = dL/dV + P^T lambda is iterated (in FP64; 16 bytes of
 * device memory per cell for the two iterates) until its L1 change is at
 * most tol * |dL/dV|_1 or `iters` sweeps ran.  Plain scheme with the masked
 * stencil's records only (PG_EUNSUPPORTED otherwise).  No counterpart in
 * the reference, which never differentiates its tables. */
int pg_adjoint(pg_ctx* ctx, const float* dl_dv, int32_t dl_dv_on_device,
               int32_t iters, double tol, double* grad18,
               pg_adjoint_result* res);

/* On-chip ceilings of `device`, measured: shared-memory read bandwidth
 * (GB/s, all SMs), read bandwidth of an L2-resident 64 MiB buffer (GB/s) and
 * FP32 FMA throughput (TFLOP/s).  No counterpart in the reference: the
 * secondary rooflines of the sweep (on-chip bytes and FMAs per lookahead) are
 * quoted against these.  Any output may be NULL to skip that probe. */
int pg_measure_peaks(int device, double* smem_gbs, double* l2_gbs,
                     double* fma_tflops);

/* ------------------------------------------------------------------ */
/* out of core: a table larger than device memory, a tile of x rows at   */
/* a time (solve_value_ooc!, solver/src/OutOfCore.jl:412-584; tiles and */
/* halo from the reach, solver/src/Tiles.jl:104-187, 311-315, 446-476).  */
/* ------------------------------------------------------------------ */

typedef struct pg_ooc_opts {
    int32_t tile_rows;      /* interior x rows per tile; 0: the most that fit */
    int32_t halo_rows;      /* x rows loaded each side; 0: the reach plus two */
    int32_t tile_sweeps;    /* sweeps per tile residency (tile_sweeps, 4)     */
    int32_t jacobi;         /* 1: each round reads the last round's table (two
                               host tables; with tile_sweeps = 1 a round is one
                               whole-table Jacobi sweep); 0: tiles are written
                               back in place (one host table)                 */
    int32_t kernel;         /* PG_KERNEL_STENCIL_ROWS or PG_KERNEL_STENCIL_EXACT */
    int32_t storage;        /* PG_STORE_F32, F16 or BF16: the host table's type */
    int32_t stop_rule;      /* PG_STOP_MAXNORM (max over a round) or L1_QUIET */
    int32_t allow_starved_halo; /* 1: accept a halo below the reach (tests)   */
    int64_t device_budget_bytes; /* 0: free device memory less 2 GiB          */
    int32_t reserved[4];
} pg_ooc_opts;

typedef struct pg_ooc_result {
    int32_t rounds;         /* rounds run (each sweeps every tile tile_sweeps times) */
    int32_t tiles_per_round;
    int32_t tile_rows;      /* interior rows per tile                          */
    int32_t halo_rows;      /* halo rows per side                              */
    int32_t reach_rows;     /* the largest successor offset in x, in rows      */
    int32_t reserved;
    double last_delta;      /* L1 change of the last round / tile_sweeps       */
    double last_maxnorm;    /* largest single-cell change of the last round    */
    double kernel_ms;       /* device time of the rounds (compute stream)      */
    double elapsed_ms;      /* host wall time of the call                      */
    int64_t h2d_bytes;      /* table bytes moved to the device                 */
    int64_t d2h_bytes;      /* and back                                        */
    int64_t launches;       /* sweep kernel launches                           */
} pg_ooc_result;

void pg_default_ooc_opts(pg_ooc_opts* opts);

/* The largest successor offset in x over every (plane, control) of the plain
 * scheme, in rows (one backup's reach; a tile or slab halo needs reach + 2,
 * the rule of solver/src/Tiles.jl:311-315).  Measured on `device`. */
int pg_reach_rows(int device, const pg_grid6* g, const pg_model* m, const pg_params* p,
                  const float* ctl, int32_t nctl, int32_t* reach);

/* Solve with the table on the host: V_host holds ncells values of
 * opts->storage in the table's row-major order and is written in full (the
 * solve starts from value_cap with the seeds at zero, as solve_value! does).
 * Runs `rounds` rounds or until the stop rule's measure of a round is <= tol.
 * The plain scheme only.  A halo below the reach is refused with PG_EINVAL
 * (the reference refuses a halo that is too small, Run.jl:1688-1691). */
int pg_solve_ooc(int device, const pg_grid6* g, const pg_model* m, const pg_params* p,
                 const uint8_t* occ, const int64_t* tidx, int64_t ntidx, const float* ctl,
                 int32_t nctl, int32_t rounds, double tol, const pg_ooc_opts* opts,
                 void* V_host, pg_ooc_result* res, pg_progress_cb cb, void* user);

/* ------------------------------------------------------------------ */
/* self-test probes: the device's own implementations of the           */
/* reference's functions, evaluated on caller-given inputs (host       */
/* buffers).  The reference's self-test calls the same functions       */
/* directly (solver/src/SelfTest.jl:208-258, 407-564); on this library */
/* they exist only on the device, so these entry points expose them.   */
/* ------------------------------------------------------------------ */

/* step_state (rk2 = 0) or step_state_rk2 (PeregrineSolver.jl:203-279) of n
 * states (x, y, h, vx, vy, w; body-frame velocity) under held commands
 * (u1, u2, u3) for dt[i] in nsub[i] substeps; a diverged state comes back as
 * NaN in every component (the reference's NANSTATE). */
int pg_probe_step(int device, const pg_model* m, int32_t rk2, const float* states,
                  const float* controls, const float* dt, const int32_t* nsub, int64_t n,
                  float* out_states);

/* traction_gain (PeregrineSolver.jl:126-136) of n commands. */
int pg_probe_traction_gain(int device, const float* controls, float knee, int64_t n,
                           float* gain);

/* interp (kuhn = 0; PeregrineSolver.jl:399-466) or interp_kuhn (kuhn = 1;
 * 571-665) of the context's current V at n states (field-frame velocity),
 * with the given cap, nearest and vclamp flags; grads (may be NULL) gets the
 * Kuhn gradient, 6 per state. */
int pg_probe_interp(pg_ctx* ctx, const float* states, int64_t n, int32_t kuhn, int32_t nearest,
                    int32_t vclamp, float cap, float* values, float* grads);

/* One Jacobi sweep that allocates nothing.  No counterpart in the reference:
 * it is for callers that cannot call cudaMalloc (a host that owns all device
 * memory through its own pool or a fixed budget, or code that must not
 * allocate after start-up), which the staged calls above cannot serve
 * because they allocate their own buffers.
 *
 * Runs the cell-form sweep (the scheme pg_sweep runs with
 * PG_KERNEL_CELLFORM on FP32 storage, phase as there) on device buffers the
 * caller holds, on the current CUDA device and on `stream` (NULL: the
 * default stream), and waits for it to finish:
 *   v_in_dev, v_out_dev  float[ncells], different buffers, plane-major:
 *                        index (((ih*Nvx+ivx)*Nvy+ivy)*Nw+iw)*Nx*Ny + ix*Ny + iy
 *   occ_dev              uint8[Nh*Nx*Ny], index (ih*Nx+ix)*Ny+iy, nonzero = occupied
 *   ctl_dev              float[3*nctl], the u1 column, then u2, then u3
 * delta / maxnorm (may be NULL) receive the sweep's L1 and max decrease.
 *
 * Its only working memory is a 1 MiB array compiled into the library, which
 * every GPU that loads the library holds until the process exits; grids of
 * more than 8,388,608 cells are refused with PG_EINVAL.  Every call shares
 * the array and it keeps the last call's contents: each call clears or
 * writes every slot it reads, and calls that overlap on the GPU race on it.
 * The first call in a CUDA context looks up the array's device address in
 * that context (set-up, with the device current); each context gets its own
 * copy of the array.  The call is synchronous -- it copies the two totals to
 * the host and waits for `stream` -- so it must not be called on a stream
 * that is being captured into a CUDA graph.
 * Calls no cudaMalloc, cudaFree or other allocating routine. */
int pg_sweep_noalloc(const pg_grid6* g, const pg_model* m, const pg_params* p,
                     const uint8_t* occ_dev, const float* ctl_dev, int32_t nctl,
                     const float* v_in_dev, float* v_out_dev, int32_t phase,
                     void* stream, double* delta, double* maxnorm);

#ifdef __cplusplus
}
#endif

#endif /* PEREGRINE_HJB_H */
