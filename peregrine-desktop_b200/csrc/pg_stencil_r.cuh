// pg_stencil_r.cuh -- the plain scheme's sweep as blend-then-shift with the
// corner planes held in registers (included inside namespace pg by
// pg_kernels.cu, after pg_stencil_b.cuh, whose records, mask, shared-memory
// helpers and storage unpacking it shares).
//
// k_stencil_b re-reads the 16 corner planes of every control from L2.  But
// the controls of one destination plane land on very few distinct corner
// sets: the successor's (h, v) moves by at most a cell or two over one
// lookahead, so the 125 controls of the benchmark grid fall into about two
// groups that share the same 16 corner planes and the same nominal x offset
// (and about 23 distinct planes in all, against 2000 plane reads).  So:
//
//   k_stencil_group (once per solve) sorts each plane's controls by their
//   (corner planes, x offset) and flags the first control of each group;
//   controls that no cell of the plane admits go last, flagged;
//
//   k_stencil_tmask (once per tiling) regroups the admissibility mask per
//   (plane, tile, control) in the order the sweep's threads read it;
//
//   k_stencil_r: block = plane, its tiles of TX rows one after another.
//   Thread (g, j) of the first G * Ny owns column j of the four window rows
//   4g .. 4g+3 and of the tile cells in those rows.  Once per plane the
//   block stages its controls' weights, tau, offsets and substep increments
//   into shared memory with asynchronous copies and computes every
//   control's per-column successor corners and fractions; per tile it
//   stages the controls' mask words and computes their per-row successor
//   corners and fractions (all of it per tile, a chunk of controls at a
//   time, when the controls do not all fit).  It walks the controls in
//   group order, two per step while both are in one group.  At the first
//   control of a group each thread loads the 16 corner values of its four
//   window cells into registers; for every control it blends them with the
//   control's 16 weights (16 FMAs per window cell, two cells per packed
//   fma.rn.f32x2, the two controls' chains interleaved, nothing re-read)
//   into the shared window; one barrier per step; then it shifts: its four
//   cells lie in consecutive rows of one column, and the successor rows of
//   consecutive rows are nearly always consecutive too, so the four
//   bilinear steps read five window rows (ten values) instead of eight, the
//   column entry once, the row entries and the mask words as one vector
//   each.
//
// The arithmetic is k_stencil_b's, operation for operation: the same FMA
// chain over the corners in record order, the same per-row / per-column
// successor corners and fractions, the same bilinear step; the results are
// bit-identical to it.  The window has one padding column (a copy of the
// last column), so the upper column corner needs no clamp.

// Two FP32 lanes in one 64-bit register, and the packed FMA of sm_100
// (fma.rn.f32x2: an IEEE fma per lane, the same result as two fmaf).
__device__ __forceinline__ uint64_t pk2(float a, float b) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void upk2(uint64_t v, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// Controls of a plane in group order: entry = control | kGroupFirst on the
// first control of a group | kCtlInadmissible when no cell of the plane
// admits it (those come last).
constexpr uint16_t kGroupFirst = 0x8000u;
constexpr uint16_t kCtlInadmissible = 0x4000u;
constexpr uint16_t kCtlMask = 0x3fffu;
static_assert(kCtlMask == kCtlMaskHost, "the host's control limit is the group order's");
static_assert(kRMaxWindowHost == 4 * 512, "window cells per block: 4 per thread, 512 threads");

// Threads per block at most and the minimum resident blocks for KR window
// cells per thread: 16 KR corner registers per thread, so KR = 4 keeps 64 of
// them and allows up to 512 threads (128 registers each).
template <int KR> struct RShape;
template <> struct RShape<4> { static constexpr int kMaxThreads = 512, kMinBlocks = 1; };

__host__ __device__ inline size_t stencil_group_smem(int nctl) {
    return (size_t)nctl * (17 * sizeof(int32_t) + 2 * sizeof(int32_t));
}

// Block = plane.  Key of a control: (not admissible anywhere, its 16 corner
// planes, its x offset); rank = number of controls with a smaller key, or
// the same key and an earlier place in `order` (the (u1, u2, u3) order).
__global__ void __launch_bounds__(128)
    k_stencil_group(const uint32_t* __restrict__ recs, KParams kp, const int32_t* __restrict__ order,
                    uint16_t* __restrict__ gord) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nctl = kp.nctl;
    int32_t* key = reinterpret_cast<int32_t*>(smem_raw);  // [nctl][17]: planes, ox
    int32_t* pos = key + (size_t)nctl * 17;               // [nctl] place in order
    int32_t* srt = pos + nctl;                            // [nctl] sorted controls
    const int64_t pl = blockIdx.x;
    const uint32_t* prec = recs + (size_t)pl * nctl * kURec;
    for (int k = threadIdx.x; k < nctl; k += blockDim.x) pos[__ldg(order + k)] = k;
    for (int i = threadIdx.x; i < nctl * 17; i += blockDim.x) {
        const int u = i / 17, f = i - u * 17;
        const uint32_t* rec = prec + (size_t)u * kURec;
        const bool ok = rec[kUNT + 18] != 0u;
        // inadmissible controls share one key that sorts after every other
        key[i] = ok ? (int32_t)(f < 16 ? rec[kUNT + f] : rec[kUNT + 16]) : 0x7fffffff;
    }
    __syncthreads();
    for (int u = threadIdx.x; u < nctl; u += blockDim.x) {
        const int32_t* ku = key + u * 17;
        int rank = 0;
        for (int v = 0; v < nctl; ++v) {
            if (v == u) continue;
            const int32_t* kv = key + v * 17;
            int cmp = 0;
            for (int f = 0; f < 17 && cmp == 0; ++f) cmp = (kv[f] > ku[f]) - (kv[f] < ku[f]);
            if (cmp < 0 || (cmp == 0 && pos[v] < pos[u])) ++rank;
        }
        srt[rank] = u;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < nctl; r += blockDim.x) {
        const int u = srt[r];
        bool first = r == 0;
        if (!first) {
            const int32_t *a = key + u * 17, *b = key + srt[r - 1] * 17;
            for (int f = 0; f < 17 && !first; ++f) first = a[f] != b[f];
        }
        const bool ok = key[u * 17] != 0x7fffffff;
        gord[(size_t)pl * nctl + r] =
            (uint16_t)((uint32_t)u | (first ? kGroupFirst : 0u) | (ok ? 0u : kCtlInadmissible));
    }
}

// The successor's lower corner li and fraction t of one row (row = true,
// idx = the row) or one column, rounded as the reference rounds them: x +
// inc_1 + ... + inc_nsub one add at a time, then (x' - lo) / step and its
// floor (PeregrineSolver.jl:248-279, 399-431).  li is clamped to
// [-2, n + 2]: successors off the table are never admissible, and the clamp
// only keeps their (unused) indices small.  Reads the grid from the kernel
// parameters, so it costs no registers for the grid.
__device__ __forceinline__ void succ_li_t(const pg_grid6& g, const float* inc, int nsub, bool row,
                                          int32_t idx, int32_t n1, int32_t n2, int32_t* li,
                                          float* t) {
    typedef Ar<float> R_;
    const float lo = row ? g.lo[0] : g.lo[1];
    const float st = row ? g.step[0] : g.step[1];
    float xn = R_::add(lo, R_::mul((float)idx, st));  // axisvalue
    for (int k = 0; k < nsub; ++k) xn = R_::add(xn, inc[k]);
    const float f = R_::div(R_::sub(xn, lo), st);
    const float fl = floorf(f);
    *t = R_::sub(f, fl);
    *li = (int32_t)fminf(fmaxf(fl, -2.0f), (float)(row ? n1 + 2 : n2 + 2));
}

// Row groups of a tile of tile_x rows that hold cells (four rows each), the
// warps whose threads own those cells, and the mask words per (plane, tile,
// control): four per such warp (one per row of the group, bit = lane).
__host__ __device__ inline int32_t stencil_r_live_groups(int32_t tile_x) { return (tile_x + 3) >> 2; }
__host__ __device__ inline int32_t stencil_r_live_warps(int32_t tile_x, int32_t n2) {
    return (stencil_r_live_groups(tile_x) * n2 + 31) >> 5;
}
__host__ __device__ inline int32_t tile_mask_stride(int32_t tile_x, int32_t n2) {
    return 4 * stencil_r_live_warps(tile_x, n2);
}

// The admissibility mask regrouped per (plane, tile, control) in thread
// order, from the per-row layout of k_stencil_prep, for the planes [plane0,
// plane0 + nplanes) whose row-order words `mask` holds (plane plane0 first):
// word 4 w + q holds, in bit l, the cell of thread t = 32 w + l in row
// 4 (t / Ny) + q of the tile, column t % Ny (0 past the tile's rows).
__global__ void k_stencil_tmask(const uint32_t* __restrict__ mask, KParams kp, int32_t tile_x,
                                int32_t tiles_x, int32_t tstride, int64_t plane0, int64_t nplanes,
                                uint32_t* __restrict__ tmask) {
    const int32_t n1 = kp.g.n[0], n2 = kp.g.n[1], W = mask_words(n2);
    const int nctl = kp.nctl;
    const int64_t total = nplanes * tiles_x * nctl * tstride;
    uint32_t* out = tmask + (size_t)plane0 * tiles_x * nctl * tstride;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = i / tstride;
        const int32_t wq = (int32_t)(i - r * tstride);
        const int32_t w = wq >> 2, q = wq & 3;
        const int32_t u = (int32_t)(r % nctl);
        r /= nctl;
        const int32_t xt = (int32_t)(r % tiles_x);
        const int64_t pl = r / tiles_x;
        const int32_t x0 = xt * tile_x;
        const int32_t nr = min(tile_x, n1 - x0);
        const uint32_t* mrow = mask + ((size_t)pl * nctl + u) * n1 * W;
        uint32_t word = 0;
        // the warp's 32 threads: runs of consecutive columns of one row,
        // each taken from at most two of the row's words
        const int32_t t0 = 32 * w, t1 = t0 + 32;
        int32_t t = t0;
        while (t < t1) {
            const int32_t g = t / n2, j = t - g * n2;
            const int32_t len = min(t1 - t, n2 - j);  // 1..32
            const int32_t a = 4 * g + q;
            if (a < nr) {
                const uint32_t* rw = mrow + (x0 + a) * W;
                const int32_t wi = j >> 5;
                const uint32_t lo = __ldg(rw + wi);
                const uint32_t hi = (wi + 1 < W) ? __ldg(rw + wi + 1) : 0u;
                const uint32_t bits = __funnelshift_r(lo, hi, (uint32_t)(j & 31));
                const uint32_t keep = len >= 32 ? 0xffffffffu : ((1u << len) - 1u);
                word |= (bits & keep) << (t - t0);
            }
            t += len;
        }
        out[i] = word;
    }
}

// Window row stride in floats: at least Ny + 1 (one padding column), and,
// when Ny is a multiple of 4, such that rows four apart differ by Ny mod 32
// banks -- a warp whose lanes straddle two row groups (the end of row 4g,
// the start of row 4g + 4) then touches each bank once.
__host__ __device__ inline int32_t stencil_r_row_stride(int32_t n2) {
    int32_t sb = n2 + 1;
    if ((n2 & 3) == 0)
        while (((4 * sb - n2) & 31) != 0) ++sb;
    return sb;
}

// Shared memory of one k_stencil_r block: the plane's group order (all
// controls); per staged control a parameter area of kRInc + NI words --
// the 16 weights, each duplicated into an FP32 pair for the packed blend
// (words 0-31: staged raw into words 16-31, then spread), tau, tx, ty,
// next, ox, oy, ok, nsub (words 32-39; next = 1 when the following control
// starts a new corner group), and its x substep position increments (NI
// words from word 40) --, its mask words for the current tile,
// its row entries for the current tile (per live row group: the four rows'
// x fractions, and their window offsets in bytes packed two to a word, bit
// 0 of the first set when the four successor rows are consecutive) and its
// column entries (per
// column: the lower column's byte offset and the y fraction); then four
// window buffers (two controls a step, double-buffered) of 4 G rows of
// stencil_r_row_stride(Ny) floats.  The y increments, needed once per plane
// for the column entries, are staged into the window buffers (NI words per
// control), which are idle until the first blend.
constexpr int kRTau = 32, kRNext = 35, kROx = 36, kRInc = 40;
__host__ __device__ inline int32_t stencil_r_ninc(int nsub) { return (nsub + 3) & ~3; }
__host__ __device__ inline size_t stencil_r_ctl_bytes(int tile_x, int n2, int nsub) {
    return (size_t)(kRInc + stencil_r_ninc(nsub)) * 4 + (size_t)tile_mask_stride(tile_x, n2) * 4 +
           (size_t)stencil_r_live_groups(tile_x) * 24 + (size_t)n2 * 8;
}
__host__ __device__ inline size_t stencil_r_smem(int nctl, int chunk, int tile_x, int n2, int groups,
                                                 int nsub) {
    const size_t ord = (size_t)((nctl + 7) & ~7) * 2;
    const size_t per = (size_t)(kRInc + stencil_r_ninc(nsub)) * 4 +
                       (size_t)tile_mask_stride(tile_x, n2) * 4 +
                       (size_t)stencil_r_live_groups(tile_x) * 16;
    const size_t rofs = ((size_t)chunk * stencil_r_live_groups(tile_x) * 8 + 15) & ~(size_t)15;
    const size_t cent = ((size_t)chunk * n2 * 8 + 15) & ~(size_t)15;
    return ord + (size_t)chunk * per + rofs + cent +
           4 * (size_t)(4 * groups) * stencil_r_row_stride(n2) * sizeof(float);
}

// v0c + tx * (v1c - v0c) for the two columns, then the y step: the bilinear
// step of k_stencil_b (whose packed form computes the same IEEE operations
// per lane).
__device__ __forceinline__ float r_bilerp(float lo0, float lo1, float hi0, float hi1, float tx,
                                          float ty) {
    const float m0 = fmaf(tx, hi0 - lo0, lo0);
    const float m1 = fmaf(tx, hi1 - lo1, lo1);
    return fmaf(ty, m1 - m0, m0);
}

// The four blended window values of a thread (rows 4g .. 4g+3 of its
// column, two packed pairs) into the window at bw, and into the padding
// column when the thread's column is the last.
__device__ __forceinline__ void r_store_window(float* bw, const uint64_t* a2, int32_t SB, bool jlast) {
    float v0, v1, v2, v3;
    upk2(a2[0], v0, v1);
    upk2(a2[1], v2, v3);
    bw[0] = v0;
    bw[SB] = v1;
    bw[2 * SB] = v2;
    bw[3 * SB] = v3;
    if (jlast) {
        bw[1] = v0;
        bw[SB + 1] = v1;
        bw[2 * SB + 1] = v2;
        bw[3 * SB + 1] = v3;
    }
}

// Phase 2 of one control for a thread's four cells (rows 4g .. 4g+3 of its
// column): shift, admissibility, tau, min -- computed for every row of the
// group (dead rows read row 0 and have no mask bit), kept where the control
// is admissible.  wu: the control's parameter area; B: its window; rt, rp:
// its row group's x fractions and packed window offsets; cc: its column
// entry; mk: the warp's four mask words; lbit: the thread's bit in them
// (1 << lane); u: its table index (argmin only).
template <bool ARGMIN>
__device__ __forceinline__ void r_shift(const float* wu, const float* B, const float4* rt,
                                        const uint2* rp, const int2 cc, const uint32_t* mk,
                                        int32_t SB4, uint32_t lbit, float cap, int u, float* best,
                                        int* bk) {
    const float tau = wu[kRTau];
    const uint2 ro = *rp;
    const float4 rf = *rt;
    const uint4 m4 = *reinterpret_cast<const uint4*>(mk);
    const float ty = __int_as_float(cc.y);
    const float tx[4] = {rf.x, rf.y, rf.z, rf.w};
    const uint32_t mw[4] = {m4.x, m4.y, m4.z, m4.w};
    const unsigned char* Bc = reinterpret_cast<const unsigned char*>(B) + cc.x;
    float val[4];
    if (ro.x & 1u) {
        // consecutive successor rows: five window rows serve the four cells
        const unsigned char* p = Bc + (ro.x & 0xfffeu);
        float v[5][2];
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            v[r][0] = *reinterpret_cast<const float*>(p + r * SB4);
            v[r][1] = *reinterpret_cast<const float*>(p + r * SB4 + 4);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            val[q] = r_bilerp(v[q][0], v[q][1], v[q + 1][0], v[q + 1][1], tx[q], ty);
    } else {
        const uint32_t offs[4] = {ro.x & 0xffffu, ro.x >> 16, ro.y & 0xffffu, ro.y >> 16};
        const int32_t SB = SB4 >> 2;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float* p = reinterpret_cast<const float*>(Bc + offs[q]);
            val[q] = r_bilerp(p[0], p[1], p[SB], p[SB + 1], tx[q], ty);
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const bool adm = (mw[q] & lbit) != 0u;
        if constexpr (ARGMIN) {
            const float cvl = adm ? fminf(tau + fminf(val[q], cap), cap) : cap;
            // equal values go to the lower table index, which is what the
            // reference's strict < in table order keeps
            if (cvl < best[q] || (cvl == best[q] && u < bk[q])) {
                best[q] = cvl;
                bk[q] = u;
            }
        } else {
            // best <= cap throughout, so min(best, min(tau + min(val, cap),
            // cap)) is min(best, tau + val) for finite values
            if (adm) best[q] = fminf(best[q], tau + val[q]);
        }
    }
}

// The tiles [t0, t1) of plane pl (tiles of kp.tile_x rows x all columns);
// their residual partials go to slots slot0, slot0 + 1, ...  Needs
// blockDim.x a multiple of 32 and >= kp.rgroups * Ny, and tile_x + 3 <=
// 4 kp.rgroups.  Threads past rgroups * Ny only help with the staging.  When
// one chunk holds every admissible control, the controls' parameters, the
// column entries and the duplicated weights are made once for all the tiles;
// per tile only the mask words and the row entries change.
template <typename S, bool ARGMIN, int KR>
__device__ __forceinline__ void stencil_r_plane(
    const S* __restrict__ Vin, S* __restrict__ Vout, const uint8_t* __restrict__ occ,
    const uint32_t* __restrict__ recs, const uint32_t* __restrict__ tmask, const KParams& kp,
    const uint16_t* __restrict__ gord, double* part_sum, double* part_max, int16_t* argmin,
    int64_t pl, int32_t t0, int32_t t1, int64_t slot0, unsigned char* smem_raw) {
    static_assert(KR == 4, "a thread owns four window rows of one column");
    __shared__ int s_nadm;
    const int nctl = kp.nctl;
    const int32_t n1 = kp.g.n[0], n2 = kp.g.n[1];
    const int32_t TX = kp.tile_x;
    const int32_t G = kp.rgroups;
    const int32_t CH = kp.rchunk;
    const int T = blockDim.x;
    const int tid = threadIdx.x;
    const int32_t SB = stencil_r_row_stride(n2);  // window row stride in floats
    const int32_t SB4 = 4 * SB;                   // and in bytes
    const int32_t GL = stencil_r_live_groups(TX);
    const int32_t TS = tile_mask_stride(TX, n2);
    const int32_t NI = stencil_r_ninc(kp.nsub);
    const int32_t RW = kRInc + NI;
    const int32_t bsz = 4 * G * SB;  // floats per window buffer
    uint16_t* ord = reinterpret_cast<uint16_t*>(smem_raw);
    float* wt = reinterpret_cast<float*>(smem_raw + (size_t)((nctl + 7) & ~7) * 2);  // [CH][RW]
    uint32_t* msk = reinterpret_cast<uint32_t*>(wt + CH * RW);                        // [CH][TS]
    float4* rtx = reinterpret_cast<float4*>(msk + CH * TS);  // [CH][GL]: x fractions
    uint2* rofs = reinterpret_cast<uint2*>(rtx + CH * GL);    // [CH][GL]: packed offsets
    int2* cent = reinterpret_cast<int2*>(rofs + ((CH * GL + 1) & ~1));  // [CH][Ny], 16-B aligned
    float* Bbuf = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(cent) +
                                           (((size_t)CH * n2 * 8 + 15) & ~(size_t)15));
    const Layout L = make_layout(kp);
    const float cap = kp.p.cap;
    const int64_t P = L.P;
    int32_t pq6[4];
    {
        int64_t pp = pl;
        pq6[3] = (int32_t)(pp % L.n[5]); pp /= L.n[5];
        pq6[2] = (int32_t)(pp % L.n[4]); pp /= L.n[4];
        pq6[1] = (int32_t)(pp % L.n[3]); pp /= L.n[3];
        pq6[0] = (int32_t)pp;
    }
    const uint32_t* prec = recs + (size_t)pl * nctl * kURec;

    // this thread: column j of the window rows 4g .. 4g+3 (act) and of the
    // tile's cells in those rows (cel)
    const int32_t g = tid / n2;
    const int32_t j = tid - g * n2;
    const bool act = g < G;
    const bool cel = g < GL;
    const int wid = tid >> 5, nw = T >> 5;
    const uint32_t lane = (uint32_t)tid & 31u;
    const uint32_t lbit = 1u << lane;  // the thread's bit in its warp's mask words
    const bool jlast = j == n2 - 1;
    const int32_t wofs = 4 * g * SB + j;  // this thread's first window cell

    // the group order; admissible controls first, nadm of them
    if (tid == 0) s_nadm = nctl;
    for (int i = tid; i < nctl; i += T) ord[i] = __ldg(gord + (size_t)pl * nctl + i);
    __syncthreads();
    for (int i = tid; i < nctl; i += T)
        if ((ord[i] & kCtlInadmissible) && (i == 0 || !(ord[i - 1] & kCtlInadmissible)))
            s_nadm = i;
    __syncthreads();
    const int nadm = s_nadm;
    // one chunk holds every admissible control: its parameters, column
    // entries and weights stay for all the plane's tiles
    const bool keep = nadm <= CH;

    // a chunk's per-control parameters, a warp per control: its record's
    // words 0-15 (w[16]) into words 16-31, words 16-19 (tau, tx, ty, -) and
    // kUNT+16..19 (ox, oy, ok, nsub) into words 32-39, its first NI x
    // increments from word 40 and its first NI y increments into the window
    // buffers, as 16-byte asynchronous copies
    auto stage_params = [&](int c0, int ch) {
        const int32_t pieces = NI / 2, half = NI / 4;
        for (int lp = wid; lp < ch; lp += nw) {
            const uint32_t* rec = prec + (size_t)(ord[c0 + lp] & kCtlMask) * kURec;
            for (int c = (int)lane; c < 6 + pieces; c += 32) {
                if (c < 6) {
                    cp_async16(wt + lp * RW + 16 + 4 * c, rec + (c < 5 ? 4 * c : kUNT + 16));
                } else {
                    const int32_t k = c - 6;
                    if (k < half)
                        cp_async16(wt + lp * RW + kRInc + 4 * k, rec + kUInc + 4 * k);
                    else
                        cp_async16(Bbuf + lp * NI + 4 * (k - half),
                                   rec + kUInc + kStencilMaxSub + 4 * (k - half));
                }
            }
        }
    };
    // a chunk's column entries (a warp per control, a lane per column) --
    // the lower column's byte offset and the y fraction
    auto make_columns = [&](int ch) {
        for (int lp = wid; lp < ch; lp += nw) {
            for (int k = (int)lane; k < n2; k += 32) {
                int32_t li;
                float t;
                succ_li_t(kp.g, Bbuf + lp * NI, kp.nsub, false, k, n1, n2, &li, &t);
                cent[lp * n2 + k] = make_int2(min(max(li, 0), n2 - 1) * 4, __float_as_int(t));
            }
        }
    };
    // a chunk's duplicated weight pairs and next-group flags (a thread per
    // control)
    auto spread_weights = [&](int c0, int ch) {
        for (int lp = tid; lp < ch; lp += T) {
            float* a = wt + lp * RW;
            float w[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) w[c] = a[16 + c];
#pragma unroll
            for (int c = 0; c < 16; ++c) { a[2 * c] = w[c]; a[2 * c + 1] = w[c]; }
            const int p1 = c0 + lp + 1;
            a[kRNext] = __int_as_float((p1 < nadm && (ord[p1] & kGroupFirst)) ? 1 : 0);
        }
    };

    uint64_t cv[2][16];  // the group's corner values, rows (4g, 4g+1) and (4g+2, 4g+3) paired
    int buf = 0;
    for (int32_t xt = t0; xt < t1; ++xt) {
        const int32_t x0 = xt * TX;
        const int32_t nr = min(TX, n1 - x0);
        const uint8_t* occ_h = occ + ((int64_t)pq6[0] * n1 + x0) * n2;
        const uint32_t* tmt = tmask + (size_t)(pl * kp.tiles_x + xt) * nctl * TS;
        float best[4];
        int bk[ARGMIN ? 4 : 1];
        uint32_t live = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            best[q] = cap;
            if constexpr (ARGMIN) bk[q] = 0x7fffffff;
            const int32_t a = 4 * g + q;
            if (cel && a < nr && occ_h[a * n2 + j] == 0) live |= 1u << q;
        }
        // corner values of the group that the control at position p starts:
        // the planes of its record, rows from its x offset
        auto load_group = [&](int p) {
            const uint32_t* rec = prec + (size_t)(ord[p] & kCtlMask) * kURec;
            const int32_t wbase = x0 + (int32_t)__ldg(rec + kUNT + 16) - 1;
            const S* base[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int32_t r = min(max(wbase + 4 * g + k, 0), n1 - 1);
                base[k] = Vin + (int64_t)r * n2 + j;
            }
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                const int64_t off = (int64_t)__ldg(rec + kUNT + c) * P;
                cv[0][c] = pk2(Conv<S>::ld(base[0] + off), Conv<S>::ld(base[1] + off));
                cv[1][c] = pk2(Conv<S>::ld(base[2] + off), Conv<S>::ld(base[3] + off));
            }
        };
        if (nadm > 0 && act) load_group(0);

        for (int c0 = 0; c0 < nadm; c0 += CH) {
            const int ch = min(CH, nadm - c0);
            const bool fresh = !keep || xt == t0;  // this chunk's parameters are not staged yet
            if (fresh) stage_params(c0, ch);
            // the tile's mask words of the chunk's controls, a warp per control
            for (int lp = wid; lp < ch; lp += nw) {
                const uint32_t* tm = tmt + (size_t)(ord[c0 + lp] & kCtlMask) * TS;
                for (int c = (int)lane; c < TS / 4; c += 32) cp_async16(msk + lp * TS + 4 * c, tm + 4 * c);
            }
            cp_async_commit();
            cp_async_wait_all();
            __syncthreads();
            if (fresh) make_columns(ch);
            // the tile's row entries, a thread per (control, live row group):
            // the four rows' window offsets (the lower corner's row from the
            // window base, in bytes; bit 0 of the first set when the four rows
            // are in the tile and their successor rows consecutive) and x
            // fractions
            for (int i = tid; i < ch * GL; i += T) {
                const int lp = i / GL, k = i - lp * GL;
                const float* a = wt + lp * RW;
                const int32_t wbase = x0 + __float_as_int(a[kROx]) - 1;
                int32_t off[4];
                float t[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int32_t row = 4 * k + q;
                    off[q] = 0;
                    t[q] = 0.0f;
                    if (row < nr) {
                        int32_t li;
                        succ_li_t(kp.g, a + kRInc, kp.nsub, true, x0 + row, n1, n2, &li, &t[q]);
                        off[q] = min(max(li - wbase, 0), nr + 1) * SB4;
                    }
                }
                const bool cons = 4 * k + 3 < nr && off[1] == off[0] + SB4 &&
                                  off[2] == off[0] + 2 * SB4 && off[3] == off[0] + 3 * SB4;
                rofs[i] = make_uint2((uint32_t)(off[0] | (cons ? 1 : 0)) | ((uint32_t)off[1] << 16),
                                     (uint32_t)off[2] | ((uint32_t)off[3] << 16));
                rtx[i] = make_float4(t[0], t[1], t[2], t[3]);
            }
            // (the weight pairs and flags occupy words 0-31 and 35, which the
            // two passes above do not read)
            if (fresh) spread_weights(c0, ch);
            __syncthreads();
            // the controls two at a time (one barrier per pair) while the second
            // stays in the first's corner group, else one: blend into the pair's
            // two window buffers -- the two FMA chains of each control
            // interleaved, four independent chains per thread --, one barrier,
            // then shift both
            int lp = 0;
            while (lp < ch) {
                const bool two = lp + 1 < ch && __float_as_int(wt[lp * RW + kRNext]) == 0;
                const float* wa = wt + lp * RW;
                const float* wb = wa + RW;
                float* BA = Bbuf + (2 * buf) * bsz;
                float* BB = BA + bsz;
                buf ^= 1;
                if (act) {
                    if (two) {
                        uint64_t a2[2] = {0ull, 0ull}, b2[2] = {0ull, 0ull};
    #pragma unroll
                        for (int c4 = 0; c4 < 4; ++c4) {
                            // (w, w) pairs of corners 4 c4 .. 4 c4 + 3
                            const ulonglong2 pa = reinterpret_cast<const ulonglong2*>(wa)[2 * c4];
                            const ulonglong2 qa = reinterpret_cast<const ulonglong2*>(wa)[2 * c4 + 1];
                            const ulonglong2 pb = reinterpret_cast<const ulonglong2*>(wb)[2 * c4];
                            const ulonglong2 qb = reinterpret_cast<const ulonglong2*>(wb)[2 * c4 + 1];
    #pragma unroll
                            for (int k = 0; k < 2; ++k) {
                                a2[k] = fma2(pa.x, cv[k][4 * c4 + 0], a2[k]);
                                b2[k] = fma2(pb.x, cv[k][4 * c4 + 0], b2[k]);
                            }
    #pragma unroll
                            for (int k = 0; k < 2; ++k) {
                                a2[k] = fma2(pa.y, cv[k][4 * c4 + 1], a2[k]);
                                b2[k] = fma2(pb.y, cv[k][4 * c4 + 1], b2[k]);
                            }
    #pragma unroll
                            for (int k = 0; k < 2; ++k) {
                                a2[k] = fma2(qa.x, cv[k][4 * c4 + 2], a2[k]);
                                b2[k] = fma2(qb.x, cv[k][4 * c4 + 2], b2[k]);
                            }
    #pragma unroll
                            for (int k = 0; k < 2; ++k) {
                                a2[k] = fma2(qa.y, cv[k][4 * c4 + 3], a2[k]);
                                b2[k] = fma2(qb.y, cv[k][4 * c4 + 3], b2[k]);
                            }
                        }
                        r_store_window(BA + wofs, a2, SB, jlast);
                        r_store_window(BB + wofs, b2, SB, jlast);
                    } else {
                        uint64_t a2[2] = {0ull, 0ull};
    #pragma unroll
                        for (int c4 = 0; c4 < 4; ++c4) {
                            const ulonglong2 pa = reinterpret_cast<const ulonglong2*>(wa)[2 * c4];
                            const ulonglong2 qa = reinterpret_cast<const ulonglong2*>(wa)[2 * c4 + 1];
    #pragma unroll
                            for (int k = 0; k < 2; ++k) {
                                a2[k] = fma2(pa.x, cv[k][4 * c4 + 0], a2[k]);
                                a2[k] = fma2(pa.y, cv[k][4 * c4 + 1], a2[k]);
                                a2[k] = fma2(qa.x, cv[k][4 * c4 + 2], a2[k]);
                                a2[k] = fma2(qa.y, cv[k][4 * c4 + 3], a2[k]);
                            }
                        }
                        r_store_window(BA + wofs, a2, SB, jlast);
                    }
                    // the corner values are free now: if the control after this
                    // step starts a new group, its loads fly during the barrier
                    // and the shifts
                    const int last = two ? lp + 1 : lp;
                    if (__float_as_int(wt[last * RW + kRNext]) != 0) load_group(c0 + last + 1);
                }
                __syncthreads();
                if (cel) {
                    r_shift<ARGMIN>(wa, BA, rtx + lp * GL + g, rofs + lp * GL + g,
                                    cent[lp * n2 + j], msk + lp * TS + 4 * wid, SB4, lbit, cap,
                                    ARGMIN ? (int)(ord[c0 + lp] & kCtlMask) : 0, best, bk);
                    if (two)
                        r_shift<ARGMIN>(wb, BB, rtx + (lp + 1) * GL + g, rofs + (lp + 1) * GL + g,
                                        cent[(lp + 1) * n2 + j], msk + (lp + 1) * TS + 4 * wid, SB4,
                                        lbit, cap, ARGMIN ? (int)(ord[c0 + lp + 1] & kCtlMask) : 0,
                                        best, bk);
                }
                lp += two ? 2 : 1;
            }
            __syncthreads();  // the chunk's shared data is read; the next chunk may stage
        }
        if constexpr (ARGMIN) {
            // controls no cell of the plane admits: ties at the cap go to the
            // lower table index
            for (int p = nadm; p < nctl; ++p) {
                const int u = ord[p] & kCtlMask;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (best[q] == cap && u < bk[q]) bk[q] = u;
            }
        }

        // write the tile's V' and its residual partials
        const S* Vp0 = Vin + pl * P + (int64_t)x0 * n2;
        S* Vo0 = Vout + pl * P + (int64_t)x0 * n2;
        double dsum = 0.0, dmax = 0.0;
        if (cel) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int32_t a = 4 * g + q;
                if (a >= nr) break;
                const int32_t e = a * n2 + j;
                const S ov = Vp0[e];
                const float old = (float)Conv<S>::val(ov);
                const bool lv = (live >> q) & 1u;
                if constexpr (ARGMIN)
                    argmin[L.rowmajor(x0 + a, j, pq6[0], pq6[1], pq6[2], pq6[3])] =
                        lv ? (int16_t)bk[q] : (int16_t)-1;
                if (lv && (best[q] < old || (kp.relax && old > 0.0f && best[q] != old))) {
                    const S nv = Conv<S>::template st<float>(best[q]);
                    const float nvT = (float)Conv<S>::val(nv);
                    Vo0[e] = nv;
                    const double d = fabs((double)old - (double)nvT);
                    dsum += d;
                    dmax = fmax(dmax, d);
                } else {
                    Vo0[e] = ov;
                }
            }
        }
        block_partial_at(dsum, dmax, part_sum, part_max, slot0 + (xt - t0));
    }
}

// The single-table sweep: block = plane, all its tiles.
template <typename S, bool ARGMIN, int KR>
__global__ void __launch_bounds__(RShape<KR>::kMaxThreads, RShape<KR>::kMinBlocks)
    k_stencil_r(const S* __restrict__ Vin, S* __restrict__ Vout, const uint8_t* __restrict__ occ,
                const uint32_t* __restrict__ recs, const uint32_t* __restrict__ tmask, KParams kp,
                const uint16_t* __restrict__ gord, double* part_sum, double* part_max,
                int16_t* argmin) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    stencil_r_plane<S, ARGMIN, KR>(Vin, Vout, occ, recs, tmask, kp, gord, part_sum, part_max,
                                   argmin, blockIdx.x, 0, kp.tiles_x,
                                   (int64_t)blockIdx.x * kp.tiles_x, smem_raw);
}

// Many tables in one launch, as k_stencil_b_batch (pg_stencil_b.cuh) but
// with the register-resident item: a persistent grid walks the items
// [first, first + count) of the tables sharing one block size; items of a
// table whose `done` flag is set only clear their residual slot.
template <typename S, int KR>
__global__ void __launch_bounds__(RShape<KR>::kMaxThreads, RShape<KR>::kMinBlocks)
    k_stencil_r_batch(const BatchTable* __restrict__ tabs, int ntab, int64_t first, int64_t count,
                      int parity, const int32_t* __restrict__ done, double* part_sum,
                      double* part_max) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) BatchTable tb;
    __shared__ int cur;
    if (threadIdx.x == 0) cur = -1;
    for (int64_t it = first + blockIdx.x; it < first + count; it += gridDim.x) {
        int lo = 0, hi = ntab - 1;  // the table owning item `it`
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tabs[mid].item0 <= it) lo = mid;
            else hi = mid - 1;
        }
        __syncthreads();  // the previous item's shared memory is free
        if (lo != cur) {
            constexpr int nw = (int)(sizeof(BatchTable) / 4);
            const uint32_t* src = reinterpret_cast<const uint32_t*>(tabs + lo);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&tb);
            for (int k = threadIdx.x; k < nw; k += blockDim.x) dst[k] = src[k];
            __syncthreads();
            if (threadIdx.x == 0) cur = lo;
        }
        if (done[lo]) {
            if (threadIdx.x == 0) { part_sum[it] = 0.0; part_max[it] = 0.0; }
            continue;
        }
        const S* vin = static_cast<const S*>(tb.V[parity]);
        S* vout = const_cast<S*>(static_cast<const S*>(tb.V[1 - parity]));
        const int64_t item = it - tb.item0;  // (plane, tile)
        const int64_t pl = item / tb.kp.tiles_x;
        const int32_t xt = (int32_t)(item - pl * tb.kp.tiles_x);
        stencil_r_plane<S, false, KR>(vin, vout, tb.occ, tb.recs, tb.tmask, tb.kp, tb.gord,
                                      part_sum, part_max, nullptr, pl, xt, xt + 1, it, smem_raw);
    }
}
