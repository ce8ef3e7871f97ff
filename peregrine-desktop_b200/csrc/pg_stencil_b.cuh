// pg_stencil_b.cuh -- the plain scheme's sweep as blend-then-shift
// (included inside namespace pg by pg_kernels.cu, after pg_stencil_u.cuh,
// whose records and admissibility mask it reads).
//
// The reference interpolates each lookahead over 64 corners: 16 (h, v)
// corner planes times a bilinear (x, y) footprint (PeregrineSolver.jl:
// 399-466).  Within one destination plane a control's successor lands on
// the same 16 corner planes with the same weights from every cell, and sits
// at (almost) the same (x, y) offset, so the interpolation separates:
//
//   phase 1 (blend)  B[r][j] = sum_c w_c * V[plane_c][r][j] over the window
//                    rows r = x0+ox-1 .. x1+ox+1 of the block's tile -- every
//                    cell reads the same aligned element of all 16 planes,
//                    so the loads are contiguous 16-byte vectors;
//   phase 2 (shift)  each cell reads B at its successor's lower (x, y) corner
//                    and the three neighbours from shared memory and
//                    finishes the bilinear step; the admissibility bit, tau
//                    and the min follow as in the reference's cell_update.
//
// The successor's x coordinate is rounded as the reference rounds it --
// x + inc_1 + ... + inc_nsub one add at a time, then (x' - lo) / step
// (PeregrineSolver.jl:248-279, 399-431) -- and that depends on the row only
// (y on the column only), so phase 1 also computes, per control, each row's
// lower corner and fraction and each column's.  They differ from the
// plane's nominal offset (ox, oy) by at most one cell, which the window's
// extra rows absorb.
//
// Per cell-control that is ~19 aligned vector-lane loads and 6 shared-memory
// reads instead of 64 shifted gathers.  FP32 arithmetic with FMAs; the
// result differs from the reference's by the rounding order of the
// interpolation sum, never in a corner, a fraction or an admissibility
// decision (those are the mask's).  Each control's 304-byte record is
// copied into shared memory with cp.async one control ahead, so its latency
// hides behind the previous control's work and the block's shared memory
// (and with it the L1 capacity left for the corner planes) stays small.

// Elements of S in one 16-byte load.
template <typename S> struct BVec { static constexpr int N = 16 / sizeof(S); };

template <typename S> struct BUnpack;
template <> struct BUnpack<float> {
    static __device__ __forceinline__ void fma(const uint4 q, float w, float (&a)[4]) {
        a[0] = fmaf(w, __uint_as_float(q.x), a[0]);
        a[1] = fmaf(w, __uint_as_float(q.y), a[1]);
        a[2] = fmaf(w, __uint_as_float(q.z), a[2]);
        a[3] = fmaf(w, __uint_as_float(q.w), a[3]);
    }
};
template <> struct BUnpack<__half> {
    static __device__ __forceinline__ void fma(const uint4 q, float w, float (&a)[8]) {
        const uint32_t v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&v[k]));
            a[2 * k] = fmaf(w, f.x, a[2 * k]);
            a[2 * k + 1] = fmaf(w, f.y, a[2 * k + 1]);
        }
    }
};
template <> struct BUnpack<__nv_bfloat16> {
    static __device__ __forceinline__ void fma(const uint4 q, float w, float (&a)[8]) {
        const uint32_t v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            a[2 * k] = fmaf(w, __uint_as_float(v[k] << 16), a[2 * k]);
            a[2 * k + 1] = fmaf(w, __uint_as_float(v[k] & 0xffff0000u), a[2 * k + 1]);
        }
    }
};

template <> struct BUnpack<Q16> {
    static __device__ __forceinline__ void fma(const uint4 q, float w, float (&a)[8]) {
        const uint32_t v[4] = {q.x, q.y, q.z, q.w};
        const float ws = w * kQ16Step;  // an exact power-of-two scaling
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            a[2 * k] = fmaf(ws, (float)(v[k] & 0xffffu), a[2 * k]);
            a[2 * k + 1] = fmaf(ws, (float)(v[k] >> 16), a[2 * k + 1]);
        }
    }
};

// Shared memory of one block: two record slots, the control order, two
// window buffers, two sets of per-row / per-column successor corners and
// three slots of the tile's admissibility-mask rows.
__host__ __device__ inline size_t stencil_b_smem(int nctl, int tile_x, int n2) {
    return 2 * (size_t)kURec * 4 + (size_t)((nctl + 3) & ~3) * 4 +
           2 * (size_t)(tile_x + 3) * n2 * sizeof(float) +
           2 * (size_t)(tile_x + n2) * 2 * sizeof(int32_t) +
           3 * (size_t)tile_x * mask_words(n2) * sizeof(uint32_t);
}

// 16-byte global -> shared copy that completes asynchronously (cp.async).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// One work item = (plane, tile of kp.tile_x rows x all columns), item
// number `item` of the table; its residual partial goes to slot `slot`.
// VEC: n2 is a multiple of the 16-byte vector width, so window rows are
// whole vectors.  OFF32: the table has fewer than 2^32 cells, so element
// offsets of the corner planes fit 32-bit arithmetic (5.5 % faster on the
// medium planes).  Called by every thread of the block.
template <typename S, bool ARGMIN, bool VEC, bool OFF32>
__device__ __forceinline__ void stencil_b_item(
    const S* __restrict__ Vin, S* __restrict__ Vout, const uint8_t* __restrict__ occ,
    const uint32_t* __restrict__ mask, const uint32_t* __restrict__ recs, const KParams& kp,
    const int32_t* __restrict__ order, double* part_sum, double* part_max, int16_t* argmin,
    int64_t item, int64_t slot, unsigned char* smem_raw) {
    typedef Ar<float> R_;
    constexpr int VN = BVec<S>::N;
    const int nctl = kp.nctl;
    const int32_t n1 = kp.g.n[0], n2 = kp.g.n[1], W = mask_words(n2);
    const int32_t TX = kp.tile_x;
    const int64_t bsz = (int64_t)(TX + 3) * n2;
    uint32_t* rslot = reinterpret_cast<uint32_t*>(smem_raw);  // [2][kURec]
    int32_t* ord = reinterpret_cast<int32_t*>(rslot + 2 * kURec);
    float* Bbuf = reinterpret_cast<float*>(ord + ((nctl + 3) & ~3));
    // per control: (window row, x fraction) of each tile row and (lower
    // column, y fraction) of each column, double-buffered like the window
    int2* rinfo = reinterpret_cast<int2*>(Bbuf + 2 * bsz);
    int2* cinfo = rinfo + 2 * TX;
    // per control: the tile rows of its admissibility mask, three slots --
    // the prefetch for control uu+1 must not overwrite the slot that a
    // thread still in control uu-1's phase 2 reads
    uint32_t* mslot = reinterpret_cast<uint32_t*>(cinfo + 2 * n2);
    const int32_t mstride = TX * W;
    const Layout L = make_layout(kp);
    GridT<float> g;
    load_grid(g, kp.g);
    const float cap = kp.p.cap;
    const int64_t P = L.P;
    const int64_t pl = item / kp.tiles_x;
    const int32_t xt = (int32_t)(item - pl * kp.tiles_x);
    const int32_t x0 = xt * TX;
    const int32_t nr = min(TX, n1 - x0);
    const int32_t ncell = nr * n2;
    const int32_t nw = nr + 3;  // window rows x0+ox-1 .. x0+ox+nr+1
    const int T = blockDim.x;
    const int tid = threadIdx.x;
    int32_t pq6[4];
    {
        int64_t pp = pl;
        pq6[3] = (int32_t)(pp % L.n[5]); pp /= L.n[5];
        pq6[2] = (int32_t)(pp % L.n[4]); pp /= L.n[4];
        pq6[1] = (int32_t)(pp % L.n[3]); pp /= L.n[3];
        pq6[0] = (int32_t)pp;
    }
    const uint32_t* prec = recs + (size_t)pl * nctl * kURec;

    // this thread's cells: e = tid + q*T, (row a, column j) of the tile
    const uint8_t* occ_h = occ + ((int64_t)pq6[0] * n1 + x0) * n2;
    float best[kBCells];
    int bk[ARGMIN ? kBCells : 1];
    int32_t ca[kBCells], cj[kBCells], cm[kBCells];  // row, column, mask word
    uint32_t live = 0;
#pragma unroll
    for (int q = 0; q < kBCells; ++q) {
        const int32_t e = tid + q * T;
        best[q] = cap;
        if constexpr (ARGMIN) bk[q] = 0x7fffffff;
        ca[q] = e / n2;
        cj[q] = e - ca[q] * n2;
        cm[q] = ca[q] * W + (cj[q] >> 5);
        if (e < ncell && occ_h[e] == 0) live |= 1u << q;
    }
    const uint32_t* mplane = mask + ((size_t)pl * nctl * n1 + x0) * W;
    const int32_t nmw = nr * W;  // mask words of the tile per control
    // mask words are copied by the threads after the first warp (which
    // copies the record)
    const int32_t mt = tid >= 32 ? tid - 32 : tid + T - 32;
    for (int i = tid; i < nctl; i += T) ord[i] = __ldg(order + i);
    __syncthreads();
    constexpr int kRecVec = kURec / 4;  // 16-byte pieces of a record
    if (tid < kRecVec)
        cp_async16(rslot + 4 * tid, prec + (size_t)ord[0] * kURec + 4 * tid);
    for (int32_t k = mt; k < nmw; k += T)
        cp_async4(mslot + k, mplane + (size_t)ord[0] * n1 * W + k);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();

    int buf = 0;
    for (int uu = 0; uu < nctl; ++uu) {
        const int u = ord[uu];
        const uint32_t* rec = rslot + (uu & 1) * kURec;
        // prefetch the next control's record into the other slot; it is
        // waited for at this control's barrier
        const int ms = uu % 3;
        if (uu + 1 < nctl) {
            const int un = ord[uu + 1];
            if (tid < kRecVec)
                cp_async16(rslot + ((uu + 1) & 1) * kURec + 4 * tid,
                           prec + (size_t)un * kURec + 4 * tid);
            uint32_t* md = mslot + (ms == 2 ? 0 : ms + 1) * mstride;
            const uint32_t* msrc = mplane + (size_t)un * n1 * W;
            for (int32_t k = mt; k < nmw; k += T) cp_async4(md + k, msrc + k);
        }
        cp_async_commit();
        // (ox, oy, ok, nsub)
        const int4 oi = *reinterpret_cast<const int4*>(rec + kUNT + 16);
        if (oi.z == 0) {
            // no cell of the plane admits this control (block-uniform)
            if constexpr (ARGMIN) {
#pragma unroll
                for (int q = 0; q < kBCells; ++q)
                    if (best[q] == cap && u < bk[q]) bk[q] = u;
            }
            cp_async_wait_all();
            __syncthreads();
            continue;
        }
        const float tau = __uint_as_float(rec[16]);
        const int32_t wbase = x0 + oi.x - 1;
        float* B = Bbuf + buf * bsz;
        int2* ri = rinfo + buf * TX;
        int2* ci = cinfo + buf * n2;
        buf ^= 1;

        // phase 1a: blend the 16 corner planes over the window rows
        if constexpr (VEC) {
            const int32_t nv = n2 / VN;
            const int32_t items = nw * nv;
            for (int32_t it = tid; it < items; it += T) {
                const int32_t k = it / nv;
                const int32_t jv = it - k * nv;
                const int32_t r = min(max(wbase + k, 0), n1 - 1);
                const S* base = Vin + (int64_t)r * n2 + (int64_t)jv * VN;
                float acc[VN];
#pragma unroll
                for (int t = 0; t < VN; ++t) acc[t] = 0.0f;
#pragma unroll 2
                for (int c4 = 0; c4 < 4; ++c4) {
                    const float4 w = reinterpret_cast<const float4*>(rec)[c4];
                    const int4 pq = reinterpret_cast<const int4*>(rec + kUNT)[c4];
                    uint4 q0, q1, q2, q3;
                    if constexpr (OFF32) {
                        const uint32_t P32 = (uint32_t)P;
                        q0 = __ldg(reinterpret_cast<const uint4*>(base + (uint32_t)pq.x * P32));
                        q1 = __ldg(reinterpret_cast<const uint4*>(base + (uint32_t)pq.y * P32));
                        q2 = __ldg(reinterpret_cast<const uint4*>(base + (uint32_t)pq.z * P32));
                        q3 = __ldg(reinterpret_cast<const uint4*>(base + (uint32_t)pq.w * P32));
                    } else {
                        q0 = __ldg(reinterpret_cast<const uint4*>(base + (int64_t)pq.x * P));
                        q1 = __ldg(reinterpret_cast<const uint4*>(base + (int64_t)pq.y * P));
                        q2 = __ldg(reinterpret_cast<const uint4*>(base + (int64_t)pq.z * P));
                        q3 = __ldg(reinterpret_cast<const uint4*>(base + (int64_t)pq.w * P));
                    }
                    BUnpack<S>::fma(q0, w.x, acc);
                    BUnpack<S>::fma(q1, w.y, acc);
                    BUnpack<S>::fma(q2, w.z, acc);
                    BUnpack<S>::fma(q3, w.w, acc);
                }
                float4* dst = reinterpret_cast<float4*>(B + (int64_t)k * n2 + (int64_t)jv * VN);
#pragma unroll
                for (int t = 0; t < VN / 4; ++t)
                    dst[t] = make_float4(acc[4 * t], acc[4 * t + 1], acc[4 * t + 2], acc[4 * t + 3]);
            }
        } else {
            const int32_t items = nw * n2;
            for (int32_t it = tid; it < items; it += T) {
                const int32_t k = it / n2;
                const int32_t j = it - k * n2;
                const int32_t r = min(max(wbase + k, 0), n1 - 1);
                const int64_t off = (int64_t)r * n2 + j;
                float acc = 0.0f;
#pragma unroll 4
                for (int c = 0; c < 16; ++c) {
                    const float w = __uint_as_float(rec[c]);
                    const int32_t pc = (int32_t)rec[kUNT + c];
                    acc = fmaf(w, (float)Conv<S>::ld(Vin + (int64_t)pc * P + off), acc);
                }
                B[it] = acc;
            }
        }
        // phase 1b: the successor's lower corner and fraction per row and
        // per column, rounded as the reference rounds them
        for (int32_t it = tid; it < nr + n2; it += T) {
            const bool row = it < nr;
            const int32_t idx = row ? x0 + it : it - nr;
            const float* inc = reinterpret_cast<const float*>(rec + kUInc) + (row ? 0 : kStencilMaxSub);
            // constant axis indices keep the grid in registers
            const float x = row ? axisvalue(g, 0, idx) : axisvalue(g, 1, idx);
            const float lo = row ? g.lo[0] : g.lo[1];
            const float st = row ? g.step[0] : g.step[1];
            float xn = x;
            for (int k = 0; k < oi.w; ++k) xn = R_::add(xn, inc[k]);
            const float f = R_::div(R_::sub(xn, lo), st);
            const float fl = floorf(f);
            const float t = R_::sub(f, fl);
            // successors off the table are never admissible; the clamps only
            // keep their (unused) indices inside the window
            const float flc = fminf(fmaxf(fl, -2.0f), (float)(row ? n1 + 2 : n2 + 2));
            const int32_t li = (int32_t)flc;
            if (row)
                ri[it] = make_int2(min(max(li - wbase, 0), nw - 2), __float_as_int(t));
            else
                ci[it - nr] = make_int2(min(max(li, 0), n2 - 1), __float_as_int(t));
        }
        cp_async_wait_all();
        __syncthreads();

        // phase 2: shift, admissibility, tau, min (the record slot is not
        // read here: the next prefetch may already be filling it)
        const uint32_t* mctl = mslot + ms * mstride;
#pragma unroll
        for (int q = 0; q < kBCells; ++q) {
            if (tid + q * T >= ncell) break;
            float cv = cap;
            const bool adm =
                ((live >> q) & 1u) && ((mctl[cm[q]] >> (cj[q] & 31)) & 1u);
            if (adm) {
                const int2 rr = ri[ca[q]];
                const int2 cc = ci[cj[q]];
                const float tx = __int_as_float(rr.y), ty = __int_as_float(cc.y);
                const int32_t j0 = cc.x;
                const int32_t j1 = min(j0 + 1, n2 - 1);
                const float* b0 = B + (int64_t)rr.x * n2;
                const float* b1 = b0 + n2;
                const float v00 = b0[j0], v01 = b0[j1], v10 = b1[j0], v11 = b1[j1];
                const float m0 = fmaf(tx, v10 - v00, v00);
                const float m1 = fmaf(tx, v11 - v01, v01);
                const float val = fmaf(ty, m1 - m0, m0);
                cv = fminf(tau + fminf(val, cap), cap);
            }
            if constexpr (ARGMIN) {
                // equal values go to the lower table index, which is what
                // the reference's strict < in table order keeps
                if (cv < best[q] || (cv == best[q] && u < bk[q])) {
                    best[q] = cv;
                    bk[q] = u;
                }
            } else {
                best[q] = fminf(best[q], cv);
            }
        }
    }

    // write V' and the residual partials
    const S* Vp0 = Vin + pl * P + (int64_t)x0 * n2;
    S* Vo0 = Vout + pl * P + (int64_t)x0 * n2;
    double dsum = 0.0, dmax = 0.0;
#pragma unroll
    for (int q = 0; q < kBCells; ++q) {
        const int32_t e = tid + q * T;
        if (e >= ncell) break;
        const S ov = Vp0[e];
        const float old = (float)Conv<S>::val(ov);
        const bool lv = (live >> q) & 1u;
        if constexpr (ARGMIN)
            argmin[L.rowmajor(x0 + ca[q], cj[q], pq6[0], pq6[1], pq6[2], pq6[3])] =
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
    block_partial_at(dsum, dmax, part_sum, part_max, slot);
}

// The single-table sweep: one block per work item.  Five resident blocks
// per SM (48 registers) measured 3.7 % faster than four on the medium planes.
template <typename S, bool ARGMIN, bool VEC, bool OFF32>
__global__ void __launch_bounds__(256, 5)
    k_stencil_b(const S* __restrict__ Vin, S* __restrict__ Vout, const uint8_t* __restrict__ occ,
                const uint32_t* __restrict__ mask, const uint32_t* __restrict__ recs, KParams kp,
                const int32_t* __restrict__ order, double* part_sum, double* part_max,
                int16_t* argmin) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    stencil_b_item<S, ARGMIN, VEC, OFF32>(Vin, Vout, occ, mask, recs, kp, order, part_sum, part_max,
                                   argmin, blockIdx.x, blockIdx.x, smem_raw);
}

// Many tables in one launch (BatchTable, pg_types.h).  Work items of all
// tables are numbered contiguously (table t owns items [item0, item0 +
// nitems)); a persistent grid walks the items [first, first + count) -- the
// tables sharing one block size -- and items of a table whose `done` flag is
// set only clear their residual slot.  The two value buffers of a table
// alternate with `parity`.

template <typename S, bool VEC, bool OFF32>
__global__ void __launch_bounds__(256, 4)
    k_stencil_b_batch(const BatchTable* __restrict__ tabs, int ntab, int64_t first, int64_t count,
                      int parity, const int32_t* __restrict__ done, double* part_sum,
                      double* part_max) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // the current table's descriptor, in shared memory so that its many
    // fields are read from there rather than held in registers
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
        // tables of the other vector class and converged tables only clear
        // their slot (the other class has its own launch)
        if (done[lo] || (tb.vec != 0) != VEC) {
            if (threadIdx.x == 0 && done[lo]) { part_sum[it] = 0.0; part_max[it] = 0.0; }
            continue;
        }
        const S* vin = static_cast<const S*>(tb.V[parity]);
        S* vout = const_cast<S*>(static_cast<const S*>(tb.V[1 - parity]));
        stencil_b_item<S, false, VEC, OFF32>(vin, vout, tb.occ, tb.mask, tb.recs, tb.kp, tb.order,
                                             part_sum, part_max, nullptr, it - tb.item0, it,
                                             smem_raw);
    }
}

// Per-table (sum, max) of the residual partials: block t reduces table t's
// slots in a fixed order into out[2t], out[2t+1].
__global__ void k_reduce_batch(const BatchTable* __restrict__ tabs, const double* part_sum,
                               const double* part_max, double* out) {
    __shared__ double ss[256], sm[256];
    const BatchTable& tb = tabs[blockIdx.x];
    double s = 0.0, m = 0.0;
    for (int64_t i = threadIdx.x; i < tb.nitems; i += blockDim.x) {
        s += part_sum[tb.item0 + i];
        m = fmax(m, part_max[tb.item0 + i]);
    }
    ss[threadIdx.x] = s;
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int w = blockDim.x >> 1; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            ss[threadIdx.x] += ss[threadIdx.x + w];
            sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[2 * blockIdx.x] = ss[0];
        out[2 * blockIdx.x + 1] = sm[0];
    }
}
