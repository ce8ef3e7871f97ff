// pg_kernels.h -- host-side launchers of the sweep, seed, layout and encode
// kernels (pg_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "pg_types.h"

namespace pg {

cudaError_t launch_fill_seed(int storage, void* V, const KParams& kp, const int64_t* tidx_dev,
                             int64_t nt, cudaStream_t st);
cudaError_t launch_seed_only(int storage, void* V, const KParams& kp, const int64_t* tidx_dev,
                             int64_t nt, cudaStream_t st);
cudaError_t launch_to_rowmajor(int storage, const void* V, float* out, const KParams& kp,
                               cudaStream_t st);
cudaError_t launch_from_rowmajor(int storage, const float* in, void* V, const KParams& kp,
                                 cudaStream_t st);
cudaError_t launch_convert_to_f32(int storage, const void* in, float* out, int64_t n,
                                  cudaStream_t st);
cudaError_t launch_cellform(int storage, bool esc, const void* Vin, void* Vout,
                            const uint8_t* occ, int8_t* pol, const KParams& kp, const float* ctl,
                            const SweepBufs& sb, int16_t* argmin, cudaStream_t st,
                            int64_t* launches);
cudaError_t launch_stencil(int storage, bool exact, const void* Vin, void* Vout,
                           const uint8_t* occ, const KParams& kp, const float* ctl,
                           const int32_t* order, const SweepBufs& sb, int16_t* argmin,
                           cudaStream_t st, int64_t* launches);
cudaError_t launch_encode(int storage, const void* V, const KParams& kp, int32_t dtype,
                          double scale, double escape_scale, int64_t lo, int64_t n, uint8_t* out,
                          unsigned long long* counts, cudaStream_t st);

// Records of the planes [plane0, plane0 + nplanes) into recs (indexed by
// plane), their row-order mask words into `mask` (plane plane0 first).
cudaError_t launch_stencil_prep(const uint8_t* occ, const KParams& kp, const float* ctl,
                                uint32_t* mask, uint32_t* recs, int64_t plane0, int64_t nplanes,
                                cudaStream_t st, int64_t* launches);
cudaError_t launch_stencil_u(int storage, const void* Vin, void* Vout, const uint8_t* occ,
                             const uint32_t* mask, const uint32_t* recs, const KParams& kp,
                             const int32_t* order, const SweepBufs& sb, int16_t* argmin,
                             cudaStream_t st, int64_t* launches);
cudaError_t launch_stencil_b(int storage, const void* Vin, void* Vout, const uint8_t* occ,
                             const uint32_t* mask, const uint32_t* recs, const KParams& kp,
                             const int32_t* order, const SweepBufs& sb, int16_t* argmin,
                             cudaStream_t st, int64_t* launches);
size_t stencil_b_smem_bytes(const KParams& kp);
cudaError_t launch_stencil_group(const uint32_t* recs, const KParams& kp, const int32_t* order,
                                 uint16_t* gord, cudaStream_t st, int64_t* launches);
cudaError_t launch_stencil_r(int storage, const void* Vin, void* Vout, const uint8_t* occ,
                             const uint32_t* recs, const uint32_t* tmask, const KParams& kp,
                             const uint16_t* gord, const SweepBufs& sb, int16_t* argmin,
                             cudaStream_t st, int64_t* launches);
// The FP64 precision oracle of the plain sweep: FP32 decisions (mask,
// records), FP64 value arithmetic and storage; the blend tiling.
cudaError_t launch_stencil_d(const void* Vin, void* Vout, const uint8_t* occ,
                             const uint32_t* mask, const uint32_t* recs, const KParams& kp,
                             const SweepBufs& sb, int16_t* argmin, cudaStream_t st,
                             int64_t* launches);
// Tile-order mask of the planes [plane0, plane0 + nplanes) from their row-order
// words in `mask` (plane plane0 first).
cudaError_t launch_stencil_tmask(const uint32_t* mask, const KParams& kp, int64_t plane0,
                                 int64_t nplanes, uint32_t* tmask, cudaStream_t st,
                                 int64_t* launches);
size_t stencil_r_smem_bytes(const KParams& kp);
// whether kp's register-resident tiling (rtile_x, rgroups, rblock, rchunk)
// is one k_stencil_r can run
bool stencil_r_shape_ok(const KParams& kp);
// resident blocks per SM of k_stencil_r (FP32) with this block size and
// dynamic shared memory, on the current device (0 when it cannot run)
int stencil_r_blocks_per_sm(int threads, size_t smem);
// k_stencil_r's window row stride (floats) for Ny = n2, and its increments
// staged per control and axis for nsub substeps
int32_t stencil_r_row_stride_host(int32_t n2);
int32_t stencil_r_ninc_host(int nsub);
// shared memory one staged control takes in a k_stencil_r block of tile_x rows
size_t stencil_r_ctl_smem_bytes(const KParams& kp, int32_t tile_x);
size_t stencil_tmask_bytes(const KParams& kp);
cudaError_t launch_stencil_b_batch(int storage, const BatchTable* tabs, int ntab, int64_t first,
                                   int64_t count, int threads, int parity, const int32_t* done,
                                   double* part_sum, double* part_max, size_t smem, int grid,
                                   bool any_vec, bool any_scalar, bool off32, cudaStream_t st);
cudaError_t launch_reduce_batch(const BatchTable* tabs, int ntab, const double* part_sum,
                                const double* part_max, double* out, cudaStream_t st);
int batch_blocks_per_sm(int storage, size_t smem, int threads);
cudaError_t launch_stencil_r_batch(int storage, const BatchTable* tabs, int ntab, int64_t first,
                                   int64_t count, int threads, int parity, const int32_t* done,
                                   double* part_sum, double* part_max, size_t smem, int grid,
                                   cudaStream_t st);
int r_batch_blocks_per_sm(int storage, size_t smem, int threads);
cudaError_t launch_adj_active(const float* V, const int16_t* pol, const uint8_t* occ,
                              const uint32_t* mask, const uint32_t* recs, const KParams& kp,
                              uint8_t* active, cudaStream_t st);
cudaError_t launch_adj_scatter(const double* lam_in, double* lam_out, const int16_t* pol,
                               const uint8_t* active, const uint32_t* recs, const KParams& kp,
                               cudaStream_t st);
cudaError_t launch_adj_start(const float* c, double* l0, double* l1, int64_t n, const SweepBufs& sb,
                             cudaStream_t st);
cudaError_t launch_adj_step(const double* lout, double* lin, const float* c, int64_t n,
                            const SweepBufs& sb, cudaStream_t st);
cudaError_t launch_adj_count(const uint8_t* a, int64_t n, const SweepBufs& sb, cudaStream_t st);
cudaError_t launch_adj_grad(const float* V, const double* lam, const int16_t* pol,
                            const uint8_t* active, const uint32_t* recs, const KParams& kp,
                            const float* ctl, double* grad, cudaStream_t st);
size_t stencil_u_smem_bytes(const KParams& kp);
size_t stencil_recs_bytes(const KParams& kp);
size_t stencil_mask_bytes(const KParams& kp);

// x slabs: row-major store rows <-> device layout (bits unchanged; 4- or
// 2-byte words), device rows [row0, row1) (slab_in: all rows by default).
cudaError_t launch_slab_in(int elem_bytes, const void* rm, void* V, const KParams& kp,
                           cudaStream_t st, int32_t row0 = 0, int32_t row1 = -1);
cudaError_t launch_slab_out(int elem_bytes, const void* V, void* rm, const KParams& kp,
                            int32_t row0, int32_t row1, cudaStream_t st);
// acc[0] += red[0]; acc[1] = max(acc[1], red[1]) (one thread)
cudaError_t launch_accum(const double* red, double* acc, cudaStream_t st);
// The largest successor reach in x over every (plane, control), in cells
// (atomic max into *out, which the caller zeroes).
cudaError_t launch_reach(const KParams& kp, const float* ctl, int32_t* out, cudaStream_t st);

cudaError_t launch_probe_step(const pg_model& m, int32_t rk2, const float* states,
                              const float* controls, const float* dt, const int32_t* nsub,
                              int64_t n, float* out, cudaStream_t st);
cudaError_t launch_probe_gain(const float* controls, float knee, int64_t n, float* out,
                              cudaStream_t st);
cudaError_t launch_probe_interp(int storage, const void* V, const KParams& kp, const float* states,
                                int64_t n, int32_t kuhn, int32_t nearest, int32_t vclamp,
                                float cap, float* out, float* grads, cudaStream_t st);

int64_t cellform_blocks(int64_t ncells);
int64_t stencil_blocks(const KParams& kp);
size_t stencil_smem(int storage, bool exact, const KParams& kp);

}  // namespace pg
