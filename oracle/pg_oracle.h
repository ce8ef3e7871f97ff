/*
 * pg_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement, in plain C, of the value-iteration hot path of
 * Peregrine-Desktop's solver (solver/src/PeregrineSolver.jl, Pipeline.jl,
 * Run.jl).  It is the checker the CUDA path is measured against and the
 * timed CPU baseline; no product code links it.
 *
 * Floating point: FP32 throughout like the reference, compiled with
 * -ffp-contract=off so every a*b+c rounds twice exactly as Julia does on the
 * CPU.  sin, cos and tanh of a Float32 are evaluated in double and rounded
 * once, which is how Julia's Float32 kernels behave (they evaluate in
 * Float64); the reference pins no library version, so bit parity of these
 * three functions with Julia itself is unpinned.
 *
 * Value arrays here are in the table's row-major order, ω fastest.
 */
#ifndef PG_ORACLE_H
#define PG_ORACLE_H

#include <stdint.h>

typedef struct og_grid {
    int32_t n[6];
    float lo[6];
    float step[6];
} og_grid;

typedef struct og_model {
    float B[9], A[9], q[3], S[9], D[9], c[3], eps[3], knee;
} og_model;

typedef struct og_params {
    float dt;
    int32_t nsub, checks, adaptive_checks, nearest;
    float cap;
    int32_t ntau;
    float tau_ratio, cfl, tau_min, tau_max, hmax;
    int32_t ncoarse, rounds;
    float delta0;
    int32_t rk2, vclamp, simplex;
} og_params;

typedef struct og_state { float x, y, h, vx, vy, w; } og_state;

/* PeregrineSolver.jl:53-60 */
void og_grid_make(og_grid* g, const int32_t n[6], const double lo[6], const double hi[6]);
/* PeregrineSolver.jl:126-136 */
float og_traction_gain(float u1, float u2, float u3, float knee);
/* PeregrineSolver.jl:166-171 */
void og_body_accel(const og_model* m, float u1r, float u2r, float u3r,
                   float vx, float vy, float w, float out[3]);
/* PeregrineSolver.jl:203-223, 254-279 */
og_state og_step_state(const og_model* m, og_state s, float u1r, float u2r, float u3r,
                       float dt, int32_t nsub);
og_state og_step_state_rk2(const og_model* m, og_state s, float u1r, float u2r,
                           float u3r, float dt, int32_t nsub);
/* PeregrineSolver.jl:318-346; returns count, writes planar [u1|u2|u3] */
int og_control_set(int level, float* out, int max);
/* PeregrineSolver.jl:399-466 */
float og_interp(const float* V, const og_grid* g, og_state s, int nearest, float cap,
                int vclamp);
/* PeregrineSolver.jl:571-665; grad may be NULL */
float og_interp_kuhn(const float* V, const og_grid* g, og_state s, float cap,
                     int vclamp, float grad[6]);
/* PeregrineSolver.jl:954-989 */
float og_cfl_tau(const og_grid* g, const og_model* m, float vfx, float vfy, float w,
                 const og_params* p);
int32_t og_substeps_for(float tau, const og_params* p);
/* PeregrineSolver.jl:1100-1153 (esc = the escape pass's views of V and occ) */
float og_lookahead(const float* V, const uint8_t* occ, const og_grid* g,
                   const og_model* m, og_state s, float u1, float u2, float u3,
                   float tau, int32_t nsub, const og_params* p, int esc,
                   int esc_blocked);
/* PeregrineSolver.jl:1205-1344; pol is the Int8 policy (3 per cell) or NULL */
float og_cell_update(int64_t idx, const float* V, const uint8_t* occ, const int8_t* pol,
                     const og_grid* g, const og_model* m, const float* ctl, int32_t nctl,
                     const og_params* p, int32_t phase, int esc, float ub[3]);

/* One Jacobi sweep over cells [lo, hi): Vout = min(Vin, T Vin) with the
 * reference's update rule (Pipeline.jl:552-568, "write only if lower").
 * pol is updated in place (a cell reads only its own entry).  total gets the
 * L1 improvement, maxd the largest; argmin (may be NULL) the winning control
 * index per cell or -1 for blocked cells.  threads <= 0 uses all cores. */
void og_sweep_jacobi(const float* Vin, float* Vout, const uint8_t* occ, int8_t* pol,
                     const og_grid* g, const og_model* m, const float* ctl,
                     int32_t nctl, const og_params* p, int32_t phase, int64_t lo,
                     int64_t hi, int threads, double* total, double* maxd,
                     int16_t* argmin);
/* Every control's lookahead value (coast first, then the table in order, as
 * the plain scheme's cell_update scans them, PeregrineSolver.jl:1246-1275)
 * for the n listed cells: out[i*nctl + k].  Blocked cells get cap for every
 * control.  Plain scheme only (one horizon, no warm start, no pattern
 * search); used to tell tied argmins from decided ones. */
void og_cell_lookaheads(const float* V, const uint8_t* occ, const og_grid* g,
                        const og_model* m, const float* ctl, int32_t nctl,
                        const og_params* p, const int64_t* cells, int64_t n, int threads,
                        float* out);
/* og_sweep_jacobi over cells [lo, hi) writing only that slab:
 * Vout_slab[idx - lo] (hi - lo floats); no policy, no argmin. */
void og_sweep_jacobi_slab(const float* Vin, float* Vout_slab, const uint8_t* occ,
                          const og_grid* g, const og_model* m, const float* ctl, int32_t nctl,
                          const og_params* p, int32_t phase, int64_t lo, int64_t hi, int threads,
                          double* total, double* maxd);
/* The reference's own in-place sweep order (Pipeline.jl:552-568), serial so it
 * is deterministic. */
double og_sweep_inplace(float* V, const uint8_t* occ, int8_t* pol, const og_grid* g,
                        const og_model* m, const float* ctl, int32_t nctl,
                        const og_params* p, int32_t phase, int rev);
/* Escape sweep, Jacobi (Pipeline.jl:580-597 update rule). */
void og_sweep_escape_jacobi(const float* Vin, float* Vout, const uint8_t* occ,
                            const og_grid* g, const og_model* m, const float* ctl,
                            int32_t nctl, const og_params* p, int32_t phase, int threads,
                            double* total);

/* solve_value! (Run.jl:1434-1474) with Jacobi sweeps (jacobi=1) or the
 * reference's in-place alternating sweeps (jacobi=0).  stop_rule 0 = L1 quiet,
 * 1 = max-norm. */
int og_solve_value(float* V, const uint8_t* occ, int8_t* pol, const og_grid* g,
                   const og_model* m, const int64_t* tidx, int64_t ntidx,
                   const float* ctl, int32_t nctl, const og_params* p, int32_t iters,
                   double tol, int stop_rule, int jacobi, int threads,
                   double* last_delta, double* last_maxd);

/* target_cells (Pipeline.jl:504-536): 0-based flat indices, unique, sorted
 * in the reference's loop order.  Returns the count (or -needed if max is
 * too small). */
int64_t og_target_cells(const og_grid* g, const float s[6], const float tol[6],
                        int64_t* out, int64_t max);

/* encode_into! (Pipeline.jl:698-780); dtype 0=u8 1=u16 2=f16 3=f32 */
int og_encode(const float* V, int64_t n, int dtype, double scale, float cap,
              double escape_scale, uint8_t* out, int64_t* reached, int64_t* escaped);

/* build_occupancy (Pipeline.jl:287-399).  polys: npoly polygons, vertex
 * counts in nverts, xy pairs concatenated in pts.  robot may be NULL (point
 * robot).  bounds may be NULL (no wall).  Output Nx*Ny*Nh bytes in
 * (i*Ny+j)*Nh+k order. */
void og_build_occupancy(const og_grid* g, int npoly, const int* nverts, const double* pts,
                        double margin_cm, int nrobot, const double* robot, int substeps,
                        double clearance_cm, const double* bounds, double wall_clearance_cm,
                        uint8_t* out);

/* FP64 reference gradient of a loss on the converged table (pg_oracle_grad.c):
 * V, pol (-1 = blocked), c = dL/dV row-major; grad gets dL/dtheta for
 * theta = diagonals of B, A, q, S, D, c (18).  Returns 0, or -1 if out of
 * memory. */
int og_adjoint_grad_f64(const double* V, const int16_t* pol, const uint8_t* occ, const og_grid* g,
                        const og_model* m, const float* ctl, int32_t nctl, const og_params* p,
                        const double* c, int32_t iters, double tol, int threads, double* grad,
                        int32_t* iters_done, int64_t* nactive);

#endif
