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
//   controls that no cell of the plane admits go last;
//
//   k_stencil_tmask (once per tiling) regroups the admissibility mask per
//   (plane, tile, control) in tile order;
//
//   k_stencil_r copies a block's per-control data (weights, tau, offsets,
//   substep increments, mask words) into shared memory with asynchronous
//   copies, computes from the staged increments every control's per-row and
//   per-column successor corners and fractions (which k_stencil_b
//   recomputes per control; here many independent chains per thread, once
//   per block), loads at the first control of each group the 16 corner
//   values of each of its window cells into registers (KR cells per
//   thread), and for every control of the group blends them with the
//   control's 16 weights -- 16 FMAs per window cell from registers, nothing
//   re-read -- into the shared window, then shifts exactly as k_stencil_b
//   does.
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
// a - b per lane, IEEE round to nearest (sub.rn.f32x2)
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// Controls of a plane in group order: entry = control | kGroupFirst on the
// first control of a group.
constexpr uint16_t kGroupFirst = 0x8000u;
static_assert(kRMaxWindowHost == 4 * 512, "window cells per block: 4 per thread, 512 threads");

// Threads per block at most and the minimum resident blocks for KR window
// cells per thread: 16 KR corner registers per thread, so KR = 2 keeps 64
// registers and up to 1024 threads; KR = 4, 128 registers and 512 threads.
template <int KR> struct RShape;
template <> struct RShape<2> { static constexpr int kMaxThreads = 1024, kMinBlocks = 1; };
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
        gord[(size_t)pl * nctl + r] = (uint16_t)u | (first ? kGroupFirst : 0u);
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

// Words of one tile's admissibility bits in tile order (bit e of the tile =
// cell e = a * n2 + j of its rows), rounded up to whole 16-byte pieces: the
// stride of one (plane, tile, control)'s words in the tile-order mask.
__host__ __device__ inline int32_t tile_mask_stride(int32_t tile_x, int32_t n2) {
    return ((tile_x * n2 + 31) / 32 + 3) & ~3;
}

// The admissibility mask regrouped per (plane, tile, control) in tile order,
// from the per-row layout of k_stencil_prep, for the planes [plane0,
// plane0 + nplanes) whose row-order words `mask` holds (plane plane0 first);
// tstride words per control, zero past the tile's cells.
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
        const int32_t w = (int32_t)(i - r * tstride);
        const int32_t u = (int32_t)(r % nctl);
        r /= nctl;
        const int32_t xt = (int32_t)(r % tiles_x);
        const int64_t pl = r / tiles_x;
        const int32_t x0 = xt * tile_x;
        const int32_t ncell = min(tile_x, n1 - x0) * n2;
        const uint32_t* mrow = mask + ((size_t)pl * nctl + u) * n1 * W;
        uint32_t word = 0;
        // bits 32w .. 32w+31 of the tile: runs of consecutive columns of one
        // row, each taken from at most two of the row's words
        const int32_t e0 = 32 * w, e1 = min(e0 + 32, ncell);
        int32_t e = e0;
        int32_t a = e / n2, j = e - a * n2;
        while (e < e1) {
            const int32_t len = min(e1 - e, n2 - j);  // 1..32
            const uint32_t* rw = mrow + (x0 + a) * W;
            const int32_t wi = j >> 5;
            const uint32_t lo = __ldg(rw + wi);
            const uint32_t hi = (wi + 1 < W) ? __ldg(rw + wi + 1) : 0u;
            const uint32_t bits = __funnelshift_r(lo, hi, (uint32_t)(j & 31));
            const uint32_t keep = len >= 32 ? 0xffffffffu : ((1u << len) - 1u);
            word |= (bits & keep) << (e - e0);
            e += len;
            j = 0;
            ++a;
        }
        out[i] = word;
    }
}

// Shared memory of one k_stencil_r block of `threads` threads (a multiple of
// 32) with KR cells per thread: the plane's group order; per control a
// parameter area of kRWt + 2 NI words -- staged as its record's weights,
// tau, offsets, admissibility and substeps (24 words) and its substep
// position increments (x, then y, NI words each), and once the successor
// entries are made, rewritten as the 16 weights each duplicated into an
// FP32 pair (32 words) and the 8 parameter words; its mask words (one per
// warp and cell slot, a warp's KR words together, zero past the tile's);
// its successor entries (the tile's rows, then every column); and two
// padded window buffers with room for every thread's KR window slots (slots
// past the window land in scratch rows).
constexpr int kRWt = 24;  // as staged: w[16], tau, tx, ty, -, ox, oy, ok, nsub
// as rewritten: (w, w) pairs in words 0-31, then tau, tx, ty, -, ox, oy, ok, nsub
constexpr int kRTau = 32, kROx = 36, kROk = 38;
// x and y increments per control: at least 8 each, so that the parameter
// area holds the rewritten 40 words
__host__ __device__ inline int32_t stencil_r_ninc(int nsub) {
    const int32_t n = (nsub + 3) & ~3;
    return n > 8 ? n : 8;
}
__host__ __device__ inline int32_t stencil_r_window_rows(int tile_x, int n2, int threads, int kr) {
    const int32_t slots = (kr * threads + n2 - 1) / n2;
    return slots > tile_x + 3 ? slots : tile_x + 3;
}
__host__ __device__ inline size_t stencil_r_smem(int nctl, int tile_x, int n2, int threads, int kr,
                                                 int nsub) {
    return (size_t)((nctl + 7) & ~7) * 2 + (size_t)nctl * kRWt * 4 +
           (size_t)nctl * 2 * stencil_r_ninc(nsub) * 4 + (size_t)nctl * kr * (threads / 32) * 4 +
           (size_t)nctl * (tile_x + n2) * sizeof(int2) +
           2 * (size_t)stencil_r_window_rows(tile_x, n2, threads, kr) * (n2 + 1) * sizeof(float);
}

// One work item = (plane, tile of kp.tile_x rows x all columns); block =
// item.  Needs (tile_x + 3) * n2 <= KR * blockDim.x and blockDim.x a
// multiple of 32.  The block first stages what its controls need into
// shared memory; the control loop then reads nothing else but the corner
// values at the start of each group.
template <typename S, bool ARGMIN, int KR>
__device__ __forceinline__ void stencil_r_item(
    const S* __restrict__ Vin, S* __restrict__ Vout, const uint8_t* __restrict__ occ,
    const uint32_t* __restrict__ recs, const uint32_t* __restrict__ tmask, const KParams& kp,
    const uint16_t* __restrict__ gord, double* part_sum, double* part_max, int16_t* argmin,
    int64_t item, int64_t slot, unsigned char* smem_raw) {
    const int nctl = kp.nctl;
    const int32_t n1 = kp.g.n[0], n2 = kp.g.n[1];
    const int32_t TX = kp.tile_x;
    const int T = blockDim.x;
    const int tid = threadIdx.x;
    const int32_t SB = n2 + 1;  // window row stride (one padding column)
    const int32_t bsz = stencil_r_window_rows(TX, n2, T, KR) * SB;
    const int32_t mwq = T >> 5;          // mask words per cell slot
    const int32_t MWS = KR * mwq;        // mask words per control in shared memory
    const int32_t TS = tile_mask_stride(TX, n2);  // mask words per control in the tile mask
    const int32_t NI = stencil_r_ninc(kp.nsub);   // increments per axis in shared memory
    const int32_t ecs = TX + n2;  // successor entries per control
    const int32_t RW = kRWt + 2 * NI;    // parameter words per control
    uint16_t* ord = reinterpret_cast<uint16_t*>(smem_raw);
    float* wt = reinterpret_cast<float*>(ord + ((nctl + 7) & ~7));  // [nctl][RW]
    uint32_t* msk = reinterpret_cast<uint32_t*>(wt + nctl * RW);    // [nctl][MWS]
    // [nctl][ecs]: TX rows (window offset, x fraction), n2 columns (column,
    // y fraction)
    int2* ent = reinterpret_cast<int2*>(msk + nctl * MWS);
    float* Bbuf = reinterpret_cast<float*>(ent + (size_t)nctl * ecs);
    const Layout L = make_layout(kp);
    const float cap = kp.p.cap;
    const int64_t P = L.P;
    const int64_t pl = item / kp.tiles_x;
    const int32_t xt = (int32_t)(item - pl * kp.tiles_x);
    const int32_t x0 = xt * TX;
    const int32_t nr = min(TX, n1 - x0);
    const int32_t ncell = nr * n2;
    int32_t pq6[4];
    {
        int64_t pp = pl;
        pq6[3] = (int32_t)(pp % L.n[5]); pp /= L.n[5];
        pq6[2] = (int32_t)(pp % L.n[4]); pp /= L.n[4];
        pq6[1] = (int32_t)(pp % L.n[3]); pp /= L.n[3];
        pq6[0] = (int32_t)pp;
    }
    const uint32_t* prec = recs + (size_t)pl * nctl * kURec;

    // stage the block's per-control data with asynchronous copies, waited
    // for once below: per control its record's words 0-19 (w[16], tau, tx,
    // ty, -) and kUNT+16..19 (ox, oy, ok, nsub) as six 16-byte pieces, its
    // first NI x and y increments, and its mask words (zero past the tile's)
    for (int i = tid; i < nctl; i += T) ord[i] = __ldg(gord + (size_t)pl * nctl + i);
    for (int i = tid; i < nctl * 6; i += T) {
        const int u = i / 6, c = i - u * 6;
        cp_async16(wt + u * RW + 4 * c, prec + (size_t)u * kURec + (c < 5 ? 4 * c : kUNT + 16));
    }
    {
        const int32_t pieces = NI / 2;  // 16-byte pieces per control: NI/4 for x, NI/4 for y
        for (int i = tid; i < nctl * pieces; i += T) {
            const int u = i / pieces, c = i - u * pieces;
            const int32_t half = NI / 4;
            const int32_t src = c < half ? kUInc + 4 * c : kUInc + kStencilMaxSub + 4 * (c - half);
            cp_async16(wt + u * RW + kRWt + 4 * c, prec + (size_t)u * kURec + src);
        }
    }
    {
        // tile word tw = q * mwq + w (cell slot q, warp w) lands at w * KR + q,
        // so that a warp's KR words are one vector; words past the tile's are 0
        const uint32_t* src = tmask + (size_t)(pl * kp.tiles_x + xt) * nctl * TS;
        for (int i = tid; i < nctl * TS; i += T) {
            const int u = i / TS, tw = i - u * TS;
            const int32_t q = tw / mwq, w = tw - q * mwq;
            cp_async4(msk + u * MWS + w * KR + q, src + (size_t)u * TS + tw);
        }
        for (int i = tid; i < nctl * MWS; i += T) {
            const int u = i / MWS, r = i - u * MWS;
            const int32_t w = r / KR, q = r - w * KR;
            if (q * mwq + w >= TS) msk[i] = 0u;
        }
    }
    cp_async_commit();

    // this thread's tile cells e = tid + q*T: (row a, column j) packed
    const uint8_t* occ_h = occ + ((int64_t)pq6[0] * n1 + x0) * n2;
    float best[KR];
    int bk[ARGMIN ? KR : 1];
    int32_t caj[KR];  // a << 16 | j
    uint32_t live = 0;
#pragma unroll
    for (int q = 0; q < KR; ++q) {
        const int32_t e = tid + q * T;
        best[q] = cap;
        if constexpr (ARGMIN) bk[q] = 0x7fffffff;
        // slots past the tile read cell (0, 0) and are never kept
        const int32_t a = e < ncell ? e / n2 : 0;
        caj[q] = e < ncell ? (a << 16) | (e - a * n2) : 0;
        if (e < ncell && occ_h[e] == 0) live |= 1u << q;
    }
    // this thread's window slots w = tid + k*T: their offset in the padded
    // window (slots past the window fall in its scratch rows); bit k of
    // wlast: slot k is in the last column
    int32_t wsb[KR];
    uint32_t wlast = 0;
#pragma unroll
    for (int k = 0; k < KR; ++k) {
        const int32_t w = tid + k * T;
        const int32_t a = w / n2, j = w - a * n2;
        wsb[k] = a * SB + j;
        if (j == n2 - 1) wlast |= 1u << k;
    }
    // the warp's mask words in a control's words; its bit is the lane
    const int32_t mw0 = (tid >> 5) * KR;
    const uint32_t lane = (uint32_t)tid & 31u;
    cp_async_wait_all();
    __syncthreads();

    // every admissible control's successor entries from its staged
    // increments: rows (the window offset of the lower corner, the x
    // fraction), then columns (the lower column, the y fraction).  Many
    // independent chains per thread, all from shared memory.
    for (int32_t i = tid; i < nctl * ecs; i += T) {
        const int u = i / ecs;
        const int32_t k = i - u * ecs;
        if (__float_as_uint(wt[u * RW + 22]) == 0u || (k >= nr && k < TX)) continue;
        const bool row = k < TX;
        int32_t li;
        float t;
        succ_li_t(kp.g, wt + u * RW + kRWt + (row ? 0 : NI), kp.nsub, row,
                  row ? x0 + k : k - TX, n1, n2, &li, &t);
        if (row) {
            const int32_t wbase = x0 + __float_as_int(wt[u * RW + 20]) - 1;
            ent[i] = make_int2(min(max(li - wbase, 0), nr + 1) * SB, __float_as_int(t));
        } else {
            ent[i] = make_int2(min(max(li, 0), n2 - 1), __float_as_int(t));
        }
    }
    __syncthreads();
    // the increments are spent: rewrite each control's parameter area as
    // its weights duplicated into FP32 pairs for the packed blend, then the
    // eight parameter words (each thread its own controls, so no barrier
    // between reading and writing one)
    for (int u = tid; u < nctl; u += T) {
        float* a = wt + u * RW;
        float w[16], par[8];
#pragma unroll
        for (int c = 0; c < 16; ++c) w[c] = a[c];
#pragma unroll
        for (int c = 0; c < 8; ++c) par[c] = a[16 + c];
#pragma unroll
        for (int c = 0; c < 16; ++c) { a[2 * c] = w[c]; a[2 * c + 1] = w[c]; }
#pragma unroll
        for (int c = 0; c < 8; ++c) a[kRTau + c] = par[c];
    }
    __syncthreads();

    static_assert(KR % 2 == 0, "window slots are paired for the packed FMA");
    uint64_t cv[KR / 2][16];  // the group's corner values, slots 2i and 2i+1 paired
    // corner values of the group that control uu starts: the planes of its
    // record, rows from its x offset
    auto load_group = [&](int uu) {
        const int u = ord[uu] & 0x7fff;
        const int32_t wbase = x0 + __float_as_int(wt[u * RW + kROx]) - 1;
        const uint32_t* rec = prec + (size_t)u * kURec;
        const S* base[KR];
#pragma unroll
        for (int k = 0; k < KR; ++k) {
            const int32_t a = wsb[k] / SB, j = wsb[k] - a * SB;
            const int32_t r = min(max(wbase + a, 0), n1 - 1);
            base[k] = Vin + (int64_t)r * n2 + j;
        }
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            const int64_t off = (int64_t)__ldg(rec + kUNT + c) * P;
#pragma unroll
            for (int k = 0; k < KR; k += 2)
                cv[k / 2][c] = pk2(Conv<S>::ld(base[k] + off), Conv<S>::ld(base[k + 1] + off));
        }
    };
    // the first control starts a group; inadmissible controls come last and
    // their records' corner planes are never read
    if (__float_as_uint(wt[(ord[0] & 0x7fff) * RW + kROk]) != 0u) load_group(0);
    int buf = 0;
    for (int uu = 0; uu < nctl; ++uu) {
        const uint32_t ent_u = ord[uu];
        const int u = (int)(ent_u & 0x7fffu);
        const float* wu = wt + u * RW;
        if (__float_as_uint(wu[kROk]) == 0u) {
            // no cell of the plane admits this control (block-uniform)
            if constexpr (ARGMIN) {
#pragma unroll
                for (int q = 0; q < KR; ++q)
                    if (best[q] == cap && u < bk[q]) bk[q] = u;
            }
            continue;
        }
        float* B = Bbuf + buf * bsz;
        buf ^= 1;

        // phase 1: blend, 16 FMAs per window slot from registers
        {
            uint64_t acc2[KR / 2];
#pragma unroll
            for (int k = 0; k < KR / 2; ++k) acc2[k] = 0ull;
#pragma unroll
            for (int c4 = 0; c4 < 4; ++c4) {
                // (w, w) pairs of corners 4 c4 .. 4 c4 + 3
                const ulonglong2 wa = reinterpret_cast<const ulonglong2*>(wu)[2 * c4];
                const ulonglong2 wb = reinterpret_cast<const ulonglong2*>(wu)[2 * c4 + 1];
#pragma unroll
                for (int k = 0; k < KR / 2; ++k) {
                    acc2[k] = fma2(wa.x, cv[k][4 * c4 + 0], acc2[k]);
                    acc2[k] = fma2(wa.y, cv[k][4 * c4 + 1], acc2[k]);
                    acc2[k] = fma2(wb.x, cv[k][4 * c4 + 2], acc2[k]);
                    acc2[k] = fma2(wb.y, cv[k][4 * c4 + 3], acc2[k]);
                }
            }
            float acc[KR];
#pragma unroll
            for (int k = 0; k < KR / 2; ++k) upk2(acc2[k], acc[2 * k], acc[2 * k + 1]);
#pragma unroll
            for (int k = 0; k < KR; ++k) {
                B[wsb[k]] = acc[k];
                // the padding column repeats the last one
                if ((wlast >> k) & 1u) B[wsb[k] + 1] = acc[k];
            }
        }
        // the corner values are free now: if the next control starts a new
        // group, its loads fly during this control's barrier and phase 2
        if (uu + 1 < nctl && (ord[uu + 1] & kGroupFirst) &&
            __float_as_uint(wt[(ord[uu + 1] & 0x7fff) * RW + kROk]) != 0u)
            load_group(uu + 1);
        __syncthreads();

        // phase 2: shift, admissibility, tau, min -- computed for every cell
        // slot (entries are clamped into the window, dead slots read cell
        // (0, 0)), kept where the control is admissible.  The mask has no
        // bit for an occupied cell or a slot past the tile, so it alone
        // decides; the bilinear step takes the two row lerps as one packed
        // FMA (the same IEEE operations per lane as k_stencil_b's).
        const float tau = wu[kRTau];
        const int2* ri = ent + (size_t)u * ecs;
        const int2* ci = ri + TX;
        uint32_t mw[KR];  // the warp's mask words of this control, one vector load
        {
            const uint32_t* mu = msk + u * MWS + mw0;
            if constexpr (KR == 4) {
                const uint4 m4 = *reinterpret_cast<const uint4*>(mu);
                mw[0] = m4.x; mw[1] = m4.y; mw[2] = m4.z; mw[3] = m4.w;
            } else {
#pragma unroll
                for (int q = 0; q < KR; ++q) mw[q] = mu[q];
            }
        }
#pragma unroll
        for (int q = 0; q < KR; ++q) {
            // warp-uniform: slots no lane of the warp has a cell in
            if ((tid & ~31) + q * T >= ncell) break;
            const int32_t a = caj[q] >> 16, j = caj[q] & 0xffff;
            const bool adm = (mw[q] >> lane) & 1u;
            const int2 rr = ri[a];
            const int2 cc = ci[j];
            const float tx = __int_as_float(rr.y), ty = __int_as_float(cc.y);
            const float* p = B + rr.x + cc.x;
            const uint64_t lo = pk2(p[0], p[1]), hi = pk2(p[SB], p[SB + 1]);
            float m0, m1;  // v0c + tx * (v1c - v0c) for columns c = 0, 1
            upk2(fma2(pk2(tx, tx), sub2(hi, lo), lo), m0, m1);
            const float val = fmaf(ty, m1 - m0, m0);
            if constexpr (ARGMIN) {
                const float cvl = adm ? fminf(tau + fminf(val, cap), cap) : cap;
                // equal values go to the lower table index, which is what
                // the reference's strict < in table order keeps
                if (cvl < best[q] || (cvl == best[q] && u < bk[q])) {
                    best[q] = cvl;
                    bk[q] = u;
                }
            } else {
                // best <= cap throughout, so min(best, min(tau + min(val,
                // cap), cap)) is min(best, tau + val) for finite values
                if (adm) best[q] = fminf(best[q], tau + val);
            }
        }
    }

    // write V' and the residual partials
    const S* Vp0 = Vin + pl * P + (int64_t)x0 * n2;
    S* Vo0 = Vout + pl * P + (int64_t)x0 * n2;
    double dsum = 0.0, dmax = 0.0;
#pragma unroll
    for (int q = 0; q < KR; ++q) {
        const int32_t e = tid + q * T;
        if (e >= ncell) break;
        const S ov = Vp0[e];
        const float old = (float)Conv<S>::val(ov);
        const bool lv = (live >> q) & 1u;
        if constexpr (ARGMIN)
            argmin[L.rowmajor(x0 + (caj[q] >> 16), caj[q] & 0xffff, pq6[0], pq6[1], pq6[2],
                              pq6[3])] = lv ? (int16_t)bk[q] : (int16_t)-1;
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
    block_partial_at(dsum, dmax, part_sum, part_max, slot);
}

// The single-table sweep: one block per work item.
template <typename S, bool ARGMIN, int KR>
__global__ void __launch_bounds__(RShape<KR>::kMaxThreads, RShape<KR>::kMinBlocks)
    k_stencil_r(const S* __restrict__ Vin, S* __restrict__ Vout, const uint8_t* __restrict__ occ,
                const uint32_t* __restrict__ recs, const uint32_t* __restrict__ tmask, KParams kp,
                const uint16_t* __restrict__ gord, double* part_sum, double* part_max,
                int16_t* argmin) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    stencil_r_item<S, ARGMIN, KR>(Vin, Vout, occ, recs, tmask, kp, gord, part_sum, part_max,
                                  argmin, blockIdx.x, blockIdx.x, smem_raw);
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
        stencil_r_item<S, false, KR>(vin, vout, tb.occ, tb.recs, tb.tmask, tb.kp, tb.gord,
                                     part_sum, part_max, nullptr, it - tb.item0, it, smem_raw);
    }
}
