// pg_types.h -- internal types shared by the kernels and the C-ABI layer.
#pragma once

#include <cstdint>
#include <string>

#include "peregrine_hjb.h"

namespace pg {

// Largest substep count / probe count the stencil kernel stages in shared
// memory.  Schemes beyond these run on the cell-form kernel.
constexpr int kStencilMaxSub = 16;
constexpr int kStencilMaxChk = 4;
constexpr int kStencilThreads = 256;
constexpr int kCellThreads = 128;
// Blend-then-shift sweep: cells per thread, cells per block at most.
constexpr int kBCells = 4;
constexpr int kBMaxTileCells = 1024;
// register-resident blend: window cells per block, and per thread
constexpr int kRMaxWindowHost = 2048;
constexpr int kRCellsPerThread = 4;
// register-resident blend: dynamic shared memory a block may take (the
// sm_100 maximum per block, 227 KB, less 2 KB for the kernels' static
// shared memory)
constexpr int kRSmemMax = 225 * 1024;
// register-resident blend: controls per plane at most (14-bit indices in
// the group order)
constexpr int kCtlMaskHost = 0x3fff;
// Model entries the adjoint differentiates (diagonals of B, A, S, D; q; c).
constexpr int kNThetaHost = 18;

// Q16 storage: V = u * kQ16Step seconds, u an unsigned 16-bit code.
struct Q16 {
    uint16_t u;
};
constexpr float kQ16Step = 1.0f / 2048.0f;
constexpr float kQ16Scale = 2048.0f;

// Everything a sweep kernel needs besides the arrays, passed by value.
struct KParams {
    pg_grid6 g;
    pg_model m;
    pg_params p;
    int64_t P;        // Nx*Ny, one (h, v) plane
    int64_t nplanes;  // Nh*Nvx*Nvy*Nw
    int64_t ncells;
    int32_t nctl;
    int32_t tile_x;   // stencil: x rows per block
    int32_t tiles_x;  // stencil: blocks per plane
    int32_t nsub;     // stencil: substeps of the single horizon
    int32_t nchk;     // stencil: swept probes per lookahead
    int32_t block;    // stencil: threads per block
    int32_t utile_x;  // masked stencil: x rows per block
    int32_t utiles_x; // masked stencil: blocks per plane
    int32_t ublock;   // masked stencil: threads per block
    int32_t btile_x;  // blend-then-shift: x rows per block (0: not eligible)
    int32_t btiles_x; // blend-then-shift: blocks per plane
    int32_t bblock;   // blend-then-shift: threads per block
    int32_t rtile_x;  // register-resident blend: x rows per block (0: not eligible)
    int32_t rtiles_x; // register-resident blend: blocks per plane
    int32_t rblock;   // register-resident blend: threads per block (a multiple of 32)
    int32_t rgroups;  // register-resident blend: row groups of 4 window rows; the
                      // first rgroups * Ny threads of a block own one column each
    int32_t rchunk;   // register-resident blend: controls staged in shared memory at once
    int32_t relax;    // 0: V' = min(V, T V), the reference's update; 1: V' = T V except
                      // where V = 0 (target cells, which stay pinned)
    int32_t phase;
    // x slabs (the row stencil only): the device table holds the global rows
    // [xoff, xoff + g.n[0]) of a table of n1g rows; rows [ux0, ux1) of the
    // slab are swept, the others (the halo) pass through unchanged.  Whole
    // tables: xoff = 0, n1g = g.n[0], [ux0, ux1) = [0, g.n[0]).
    int32_t xoff, n1g, ux0, ux1;
};

// Per-sweep reduction buffers: one partial per block, reduced in a fixed
// order so the convergence signal is bit-for-bit reproducible.
struct SweepBufs {
    double* part_sum;
    double* part_max;
    int64_t nparts;
    double* out;  // [2]: L1 total, max-norm
};

// One table of a batched sweep: its buffers, its work items in the batch's
// numbering and its kernel parameters (tile_x / tiles_x = the blend tiling).
struct BatchTable {
    const void* V[2];
    const uint8_t* occ;
    const uint32_t* mask;
    const uint32_t* recs;
    const int32_t* order;
    const uint32_t* tmask;   // register-resident sweep: tile-order mask
    const uint16_t* gord;    // register-resident sweep: group order
    int64_t item0, nitems;
    int32_t vec;
    int32_t pad;
    KParams kp;
};
static_assert(sizeof(BatchTable) % 4 == 0, "BatchTable is copied as 32-bit words");

// Records msg as the text pg_last_error returns on this thread; returns code.
int set_last_error(int code, const std::string& msg);

}  // namespace pg
