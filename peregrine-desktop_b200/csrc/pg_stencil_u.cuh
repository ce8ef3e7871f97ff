// pg_stencil_u.cuh -- the plain scheme's sweep with every V-independent
// quantity computed once per solve (included inside namespace pg by
// pg_kernels.cu).
//
// Whether a lookahead is admissible -- the successor is finite and inside
// the velocity envelope, every swept probe lands on a free cell of the field,
// the successor's (x, y) is on the table (PeregrineSolver.jl:1106-1144 and
// the range tests of interp, 419-431) -- depends on the grid, the model and
// the occupancy, never on V; so do the successor's (h, v) corners and
// weights.  k_stencil_prep decides admissibility once per solve for every
// (plane, control, cell), with the reference's rounding, into one bit, and
// stores one record per (plane, control) with what the sweep needs.
//
// k_stencil_u is the sweep.  With the decisions out of the way, the
// interpolation weights of a (plane, control) pair are uniform across the
// plane: the successor sits at a fixed offset (the sum of the substep
// position increments) from every cell, so its x/y fractions and its 16
// (h, v) corners and weights are one set per pair.  A thread owns RX rows x
// R columns of cells; per control it gathers an (RX+1) x (R+1) window from
// each of the 16 corner planes with 16-byte loads, shared by its RX*R cells.
// FP32 arithmetic with FMAs; the value differs from the reference's per-cell
// rounding by a few ulp of the interpolation weights, never in a decision.

constexpr int kURX = 2;  // rows per thread

// Mask words per (plane, control, row): ceil(Ny / 32).
__host__ __device__ inline int32_t mask_words(int32_t n2) { return (n2 + 31) / 32; }

// Record per (plane, control), 76 words, 16-byte aligned:
//   float: w[16] (the (h, v)-corner weights), tau, tx, ty, -
//   int:   plane[16], ox, oy, ok, nsub
//   float: incx[16], incy[16] (the field-frame position increment of each
//          substep, which the reference adds to x and y one at a time)
//   float: tt[4], the successor's (h, vx, vy, w) fractions the weights are
//          products of (the FP64 sweep forms its weights from them)
// Every vector load on a record is aligned to its size: the record is 304
// bytes, (tau, tx, ty, -) sits at byte 64 and (ox, oy) at byte 144.
constexpr int kUNT = 20;
constexpr int kUNI = 20;
constexpr int kUInc = 40;
constexpr int kUTT = kUInc + 2 * kStencilMaxSub;
constexpr int kURec = kUTT + 4;

__host__ __device__ inline size_t stencil_u_smem(int nctl) {
    return (size_t)nctl * (kURec * 4 + 4) + 64;
}
__host__ __device__ inline size_t stencil_prep_smem(int nctl, int nsub) {
    return (size_t)nctl * nsub * 2 * sizeof(float) + (size_t)nctl * (kStencilMaxChk + 1) * 4 + 64;
}
// The column table of k_stencil_prep: one word per (control, column).
__host__ __device__ inline size_t stencil_prep_tab_smem(int nctl, int n2) {
    return (size_t)nctl * n2 * sizeof(uint32_t);
}
constexpr uint32_t kPrepColOff = 0xffffffffu;

// Once per solve.  Block = plane.  Phase A integrates each control once and
// writes its sweep record; phase B walks (control, row, 32-column word) items
// and decides admissibility per cell exactly as lookahead does.  With
// `coltab` (columns <= 255), what depends on the column only -- the swept
// probes' y cells and whether they and the successor's y stay on the table
// -- is decided once per (control, column) into a shared word of four probe
// columns (kPrepColOff: off the table), and the per-row walk only adds the x
// side and the occupancy lookups.  The decisions are the same either way.
__global__ void __launch_bounds__(256)
    k_stencil_prep(const uint8_t* __restrict__ occ, KParams kp, const float* __restrict__ ctl,
                   uint32_t* __restrict__ mask, uint32_t* __restrict__ recs, int coltab,
                   int64_t plane0) {
    typedef Ar<float> R_;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nctl = kp.nctl, nsub = kp.nsub, nchk = kp.nchk;
    float* sx = reinterpret_cast<float*>(smem_raw);    // [nctl][nsub] x increments
    float* sy = sx + (size_t)nctl * nsub;              // [nctl][nsub] y increments
    int32_t* sck = reinterpret_cast<int32_t*>(sy + (size_t)nctl * nsub);  // [nctl][4]
    int32_t* sok = sck + (size_t)nctl * kStencilMaxChk;                   // [nctl]
    const Layout L = make_layout(kp);
    GridT<float> g;
    load_grid(g, kp.g);
    // block = plane plane0 + blockIdx.x; its mask rows go to `mask` at the
    // block's place (mask holds the planes from plane0 on)
    const int64_t pl = plane0 + blockIdx.x;
    const int64_t ml = blockIdx.x;
    int32_t i3, i4, i5, i6;
    {
        int64_t q = pl;
        i6 = (int32_t)(q % L.n[5]); q /= L.n[5];
        i5 = (int32_t)(q % L.n[4]); q /= L.n[4];
        i4 = (int32_t)(q % L.n[3]); q /= L.n[3];
        i3 = (int32_t)q;
    }
    for (int u = threadIdx.x; u < nctl; u += blockDim.x) {
        Transition<float> t;
        transition(kp, g, i3, i4, i5, i6, ctl, u, t);
        for (int k = 0; k < nsub; ++k) {
            sx[u * nsub + k] = t.incx[k];
            sy[u * nsub + k] = t.incy[k];
        }
        for (int sc = 0; sc < kStencilMaxChk; ++sc) sck[u * kStencilMaxChk + sc] = t.ck[sc];
        sok[u] = t.ok ? 1 : 0;
        // the sweep record: successor offset in cells, its fractions, the
        // (h, v) corners with the x fraction folded into their weights
        uint32_t* rec = recs + ((size_t)pl * nctl + u) * kURec;
        const float dxc = t.sumx / g.step[0], dyc = t.sumy / g.step[1];
        const float fx = floorf(dxc), fy = floorf(dyc);
        const float tx = dxc - fx, ty = dyc - fy;
        for (int c = 0; c < 16; ++c) {
            rec[c] = __float_as_uint(corner_weight(t, c));
            rec[kUNT + c] = (uint32_t)corner_plane(g, t, c);
        }
        rec[16] = __float_as_uint(t.tau);
        rec[17] = __float_as_uint(tx);
        rec[18] = __float_as_uint(ty);
        rec[19] = 0u;
        rec[kUNT + 16] = (uint32_t)(t.ok ? (int32_t)fx : 0);
        rec[kUNT + 17] = (uint32_t)(t.ok ? (int32_t)fy : 0);
        rec[kUNT + 18] = t.ok ? 1u : 0u;
        rec[kUNT + 19] = (uint32_t)nsub;
        for (int k = 0; k < 4; ++k) rec[kUTT + k] = __float_as_uint(t.ok ? t.tt[k] : 0.0f);
        for (int k = 0; k < kStencilMaxSub; ++k) {
            rec[kUInc + k] = __float_as_uint(t.ok && k < nsub ? t.incx[k] : 0.0f);
            rec[kUInc + kStencilMaxSub + k] = __float_as_uint(t.ok && k < nsub ? t.incy[k] : 0.0f);
        }
    }
    __syncthreads();
    const int32_t n1 = L.n[0], n2 = L.n[1], W = mask_words(n2);
    const float lo0 = g.lo[0], lo1 = g.lo[1], st0 = g.step[0], st1 = g.step[1];
    const float rs0 = 1.0f / st0, rs1 = 1.0f / st1;
    const float hx = (float)(n1 - 1), hy = (float)(n2 - 1);
    float ap[kStencilMaxChk];
    for (int sc = 0; sc < kStencilMaxChk; ++sc)
        ap[sc] = R_::div((float)(sc + 1), (float)(nchk > 0 ? nchk : 1));
    const uint8_t* occ_h = occ + (int64_t)i3 * n1 * n2;
    const int64_t items = (int64_t)nctl * n1 * W;
    if (coltab) {
        uint32_t* tab = reinterpret_cast<uint32_t*>(smem_raw + stencil_prep_smem(nctl, nsub));
        for (int32_t it = threadIdx.x; it < nctl * n2; it += blockDim.x) {
            const int u = it / n2;
            const int32_t j = it - u * n2;
            uint32_t word = kPrepColOff;
            if (sok[u]) {
                const float y = axisvalue(g, 1, j);
                float yn = y;
                for (int k = 0; k < nsub; ++k) yn = R_::add(yn, sy[u * nsub + k]);
                const float dy = R_::sub(yn, y);
                bool ok = true;
                uint32_t packed = 0;
                for (int sc = 0; sc < nchk && ok; ++sc) {
                    int32_t cj = 0;
                    ok = probe_coord(R_::sub(R_::add(y, R_::mul(dy, ap[sc])), lo1), st1, rs1, hy, &cj);
                    packed |= (uint32_t)cj << (8 * sc);
                }
                float f2;
                if (ok) ok = succ_coord<true>(R_::sub(yn, lo1), st1, rs1, hy, &f2);
                if (ok) word = packed;
            }
            tab[it] = word;
        }
        __syncthreads();
        for (int64_t it = threadIdx.x; it < items; it += blockDim.x) {
            const int u = (int)(it / ((int64_t)n1 * W));
            const int32_t rem = (int32_t)(it - (int64_t)u * n1 * W);
            const int32_t i1 = rem / W, w = rem - i1 * W;
            uint32_t bits = 0;
            if (sok[u]) {
                const float x = axisvalue(g, 0, i1);
                float xn = x;
                for (int k = 0; k < nsub; ++k) xn = R_::add(xn, sx[u * nsub + k]);
                const float dx = R_::sub(xn, x);
                bool xok = true;
                int32_t ci[kStencilMaxChk];
                for (int sc = 0; sc < kStencilMaxChk; ++sc) {
                    ci[sc] = 0;
                    if (sc < nchk && xok)
                        xok = probe_coord(R_::sub(R_::add(x, R_::mul(dx, ap[sc])), lo0), st0, rs0,
                                          hx, &ci[sc]);
                }
                float f1;
                if (xok) xok = succ_coord<true>(R_::sub(xn, lo0), st0, rs0, hx, &f1);
                if (xok) {
                    const uint8_t* orow[kStencilMaxChk];
                    for (int sc = 0; sc < kStencilMaxChk; ++sc)
                        orow[sc] = sc < nchk
                                       ? occ + ((int64_t)sck[u * kStencilMaxChk + sc] * n1 + ci[sc]) * n2
                                       : occ;
                    const uint32_t* trow = tab + (size_t)u * n2;
                    for (int b = 0; b < 32; ++b) {
                        const int32_t j = w * 32 + b;
                        if (j >= n2) break;
                        if (occ_h[(int64_t)i1 * n2 + j]) continue;
                        const uint32_t yw = trow[j];
                        if (yw == kPrepColOff) continue;
                        bool ok = true;
                        for (int sc = 0; sc < nchk && ok; ++sc)
                            ok = orow[sc][(yw >> (8 * sc)) & 0xffu] == 0;
                        if (ok) bits |= 1u << b;
                    }
                }
            }
            mask[((ml * nctl + u) * n1 + i1) * W + w] = bits;
        }
        return;
    }
    for (int64_t it = threadIdx.x; it < items; it += blockDim.x) {
        const int u = (int)(it / ((int64_t)n1 * W));
        const int32_t rem = (int32_t)(it - (int64_t)u * n1 * W);
        const int32_t i1 = rem / W, w = rem - i1 * W;
        uint32_t bits = 0;
        if (sok[u]) {
            const float x = axisvalue(g, 0, i1);
            float xn = x;
            for (int k = 0; k < nsub; ++k) xn = R_::add(xn, sx[u * nsub + k]);
            const float dx = R_::sub(xn, x);
            bool xok = true;
            int32_t ci[kStencilMaxChk];
            for (int sc = 0; sc < kStencilMaxChk; ++sc) {
                ci[sc] = 0;
                if (sc < nchk && xok)
                    xok = probe_coord(R_::sub(R_::add(x, R_::mul(dx, ap[sc])), lo0), st0, rs0, hx,
                                      &ci[sc]);
            }
            float f1;
            if (xok) xok = succ_coord<true>(R_::sub(xn, lo0), st0, rs0, hx, &f1);
            if (xok) {
                for (int b = 0; b < 32; ++b) {
                    const int32_t j = w * 32 + b;
                    if (j >= n2) break;
                    if (occ_h[(int64_t)i1 * n2 + j]) continue;
                    const float y = axisvalue(g, 1, j);
                    float yn = y;
                    for (int k = 0; k < nsub; ++k) yn = R_::add(yn, sy[u * nsub + k]);
                    const float dy = R_::sub(yn, y);
                    bool ok = true;
                    for (int sc = 0; sc < nchk && ok; ++sc) {
                        int32_t cj = 0;
                        ok = probe_coord(R_::sub(R_::add(y, R_::mul(dy, ap[sc])), lo1), st1, rs1, hy, &cj);
                        if (ok)
                            ok = occ[((int64_t)sck[u * kStencilMaxChk + sc] * n1 + ci[sc]) * n2 + cj] == 0;
                    }
                    float f2;
                    if (ok) ok = succ_coord<true>(R_::sub(yn, lo1), st1, rs1, hy, &f2);
                    if (ok) bits |= 1u << b;
                }
            }
        }
        mask[((ml * nctl + u) * n1 + i1) * W + w] = bits;
    }
}

// Storage element IDX of a run of 16-byte words, as float; IDX is a
// compile-time constant so the selection costs no instructions.
template <typename S> struct VecElem;
template <> struct VecElem<float> {
    static constexpr int VEC = 4;
    template <int IDX, int NV>
    static __device__ __forceinline__ float get(const uint4 (&w)[NV]) {
        const uint4 q = w[IDX / 4];
        const uint32_t b = (IDX % 4 == 0) ? q.x : (IDX % 4 == 1) ? q.y : (IDX % 4 == 2) ? q.z : q.w;
        return __uint_as_float(b);
    }
};
template <> struct VecElem<__half> {
    static constexpr int VEC = 8;
    template <int IDX, int NV>
    static __device__ __forceinline__ float get(const uint4 (&w)[NV]) {
        const uint4 q = w[IDX / 8];
        constexpr int c = (IDX % 8) / 2;
        const uint32_t b = (c == 0) ? q.x : (c == 1) ? q.y : (c == 2) ? q.z : q.w;
        return __half2float(__ushort_as_half((unsigned short)((IDX % 2) ? (b >> 16) : (b & 0xffffu))));
    }
};
template <> struct VecElem<__nv_bfloat16> {
    static constexpr int VEC = 8;
    template <int IDX, int NV>
    static __device__ __forceinline__ float get(const uint4 (&w)[NV]) {
        const uint4 q = w[IDX / 8];
        constexpr int c = (IDX % 8) / 2;
        const uint32_t b = (c == 0) ? q.x : (c == 1) ? q.y : (c == 2) ? q.z : q.w;
        return __uint_as_float((IDX % 2) ? (b & 0xffff0000u) : (b << 16));
    }
};

// Where window column k (0..R) sits in the loaded span of R+VEC elements.
//   MODE 0 (inner column block): the span starts PARAM elements before it.
//   MODE 1 (left edge, successor offset -PARAM < 0): columns left of the
//          grid clamp to column 0, the span's first element.
//   MODE 2 (right edge, offset PARAM >= 0): the span is the row's last
//          R+VEC elements; columns past the grid clamp to its last one.
template <int MODE, int PARAM, int R, int VEC>
__host__ __device__ constexpr int span_index(int k) {
    return MODE == 0 ? PARAM + k
         : MODE == 1 ? (k - PARAM < 0 ? 0 : k - PARAM)
         : (VEC + PARAM + k < R + VEC - 1 ? VEC + PARAM + k : R + VEC - 1);
}

// Accumulate the 16 (h, v) corners of one control: m[a][k] over window rows
// a (0..RX-1, already combined with row a+1 along x) and columns k (0..R).
template <typename S, int RX, int R, int MODE, int PARAM>
__device__ __forceinline__ void gather_vec(const S* __restrict__ Vin, int64_t P,
                                           const int32_t* irec, const float* rec, float tx,
                                           const int32_t* roff, int32_t c0,
                                           float (&m)[RX][R + 1]) {
    constexpr int VEC = VecElem<S>::VEC;
    constexpr int NV = (R + VEC) / VEC;
#pragma unroll 2
    for (int c = 0; c < 16; ++c) {
        const int32_t pq = irec[c];
        const float wa = rec[c] * (1.0f - tx), wb = rec[c] * tx;
        const S* Vc = Vin + (int64_t)pq * P + c0;
        float v[RX + 1][R + 1];
#pragma unroll
        for (int a = 0; a <= RX; ++a) {
            const uint4* src = reinterpret_cast<const uint4*>(Vc + roff[a]);
            uint4 w[NV];
#pragma unroll
            for (int t = 0; t < NV; ++t) w[t] = __ldg(src + t);
#pragma unroll
            for (int k = 0; k <= R; ++k) {
                switch (k) {
#define PG_VE(K) case K: if constexpr (K <= R) v[a][K] = VecElem<S>::template get<span_index<MODE, PARAM, R, VEC>(K), NV>(w); break;
                    PG_VE(0) PG_VE(1) PG_VE(2) PG_VE(3) PG_VE(4) PG_VE(5) PG_VE(6) PG_VE(7) PG_VE(8)
#undef PG_VE
                }
            }
        }
#pragma unroll
        for (int a = 0; a < RX; ++a)
#pragma unroll
            for (int k = 0; k <= R; ++k) m[a][k] = fmaf(wa, v[a][k], fmaf(wb, v[a + 1][k], m[a][k]));
    }
}

// Any columns (clamped to the row), one load per value.
template <typename S, int RX, int R>
__device__ __forceinline__ void gather_scalar(const S* __restrict__ Vin, int64_t P,
                                              const int32_t* irec, const float* rec, float tx,
                                              const int32_t* roff, const int32_t* coff,
                                              float (&m)[RX][R + 1]) {
#pragma unroll 2
    for (int c = 0; c < 16; ++c) {
        const int32_t pq = irec[c];
        const float wa = rec[c] * (1.0f - tx), wb = rec[c] * tx;
        const S* Vc = Vin + (int64_t)pq * P;
        float v[RX + 1][R + 1];
#pragma unroll
        for (int a = 0; a <= RX; ++a)
#pragma unroll
            for (int k = 0; k <= R; ++k) v[a][k] = (float)Conv<S>::ld(Vc + roff[a] + coff[k]);
#pragma unroll
        for (int a = 0; a < RX; ++a)
#pragma unroll
            for (int k = 0; k <= R; ++k) m[a][k] = fmaf(wa, v[a][k], fmaf(wb, v[a + 1][k], m[a][k]));
    }
}

template <typename S, int RX, int R, bool ARGMIN>
__global__ void __launch_bounds__(256, 2)
    k_stencil_u(const S* __restrict__ Vin, S* __restrict__ Vout, const uint8_t* __restrict__ occ,
                const uint32_t* __restrict__ mask, const uint32_t* __restrict__ recs, KParams kp,
                const int32_t* __restrict__ order, double* part_sum, double* part_max,
                int16_t* argmin) {
    constexpr int VEC = VecElem<S>::VEC;
    constexpr int NV = (R + VEC) / VEC;
    static_assert(R % VEC == 0, "the window width must be a multiple of the vector width");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nctl = kp.nctl;
    uint32_t* srec = reinterpret_cast<uint32_t*>(smem_raw);
    int32_t* ord = reinterpret_cast<int32_t*>(srec + (size_t)nctl * kURec);
    const Layout L = make_layout(kp);
    const float cap = kp.p.cap;
    const int64_t pl = blockIdx.x / kp.tiles_x;
    const int32_t xt = (int32_t)(blockIdx.x - pl * kp.tiles_x);
    const int32_t n1 = L.n[0], n2 = L.n[1], W = mask_words(n2);
    int32_t pq6[4];  // (h, vx, vy, w) of this plane
    {
        int64_t pp = pl;
        pq6[3] = (int32_t)(pp % L.n[5]); pp /= L.n[5];
        pq6[2] = (int32_t)(pp % L.n[4]); pp /= L.n[4];
        pq6[1] = (int32_t)(pp % L.n[3]); pp /= L.n[3];
        pq6[0] = (int32_t)pp;
    }

    // the plane's records, staged with 16-byte copies
    {
        const uint4* src = reinterpret_cast<const uint4*>(recs + (size_t)pl * nctl * kURec);
        uint4* dst = reinterpret_cast<uint4*>(srec);
        const int n4 = nctl * kURec / 4;
        for (int i = threadIdx.x; i < n4; i += blockDim.x) dst[i] = __ldg(src + i);
        for (int u = threadIdx.x; u < nctl; u += blockDim.x) ord[u] = order[u];
    }
    __syncthreads();

    const int32_t x0 = xt * kp.tile_x;
    const int32_t x1 = min(x0 + kp.tile_x, n1);
    const int32_t rb_n = (x1 - x0 + RX - 1) / RX;
    const int32_t cb_n = (n2 + R - 1) / R;
    // Inner column blocks first, then all left edges, then all right edges,
    // so that whole warps take one gather variant.
    const bool vec_ok = (n2 % R) == 0 && cb_n >= 3;
    const int32_t n_inner = vec_ok ? rb_n * (cb_n - 2) : 0;
    const int32_t nseg = rb_n * cb_n;
    const int64_t P = L.P;
    const S* __restrict__ Vp0 = Vin + pl * P;
    const uint8_t* occ_h = occ + (int64_t)pq6[0] * n1 * n2;
    const uint32_t* mplane = mask + (size_t)pl * nctl * n1 * W;
    double dsum = 0.0, dmax = 0.0;

    for (int seg = threadIdx.x; seg < nseg; seg += blockDim.x) {
        int32_t rb, cb, mode;
        if (seg < n_inner) {
            rb = seg / (cb_n - 2);
            cb = 1 + (seg - rb * (cb_n - 2));
            mode = 0;
        } else if (vec_ok) {
            const int32_t e = seg - n_inner;
            if (e < rb_n) { rb = e; cb = 0; mode = 1; }
            else { rb = e - rb_n; cb = cb_n - 1; mode = 2; }
        } else {
            rb = seg / cb_n;
            cb = seg - rb * cb_n;
            mode = 3;  // scalar
        }
        const int32_t i1 = x0 + rb * RX;
        const int32_t j0 = cb * R;
        float best[RX][R];
        int bk[ARGMIN ? RX : 1][ARGMIN ? R : 1];
        uint32_t live = 0;
#pragma unroll
        for (int a = 0; a < RX; ++a)
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int32_t i = i1 + a, j = j0 + r;
                if (i < x1 && j < n2 && occ_h[(int64_t)i * n2 + j] == 0) live |= 1u << (a * R + r);
                best[a][r] = cap;
                if constexpr (ARGMIN) bk[a][r] = 0x7fffffff;
            }
        if (live) {
            const int32_t wj = j0 >> 5, sh = j0 & 31;
            const uint32_t bmask = R >= 32 ? 0xffffffffu : ((1u << R) - 1u);
            for (int uu = 0; uu < nctl; ++uu) {
                const int u = ord[uu];
                const uint32_t* mrow = mplane + ((size_t)u * n1 + i1) * W + wj;
                uint32_t vb[RX];
                uint32_t vany = 0;
#pragma unroll
                for (int a = 0; a < RX; ++a) {
                    vb[a] = (i1 + a < x1) ? (__ldg(mrow + (size_t)a * W) >> sh) & bmask : 0u;
                    vany |= vb[a];
                }
                if (!vany) {
                    if constexpr (ARGMIN) {
#pragma unroll
                        for (int a = 0; a < RX; ++a)
#pragma unroll
                            for (int r = 0; r < R; ++r)
                                if (best[a][r] == cap && u < bk[a][r]) bk[a][r] = u;
                    }
                    continue;
                }
                const float* rec = reinterpret_cast<const float*>(srec + (size_t)u * kURec);
                const int32_t* irec = reinterpret_cast<const int32_t*>(srec + (size_t)u * kURec + kUNT);
                const float4 tt = *reinterpret_cast<const float4*>(rec + 16);
                // (ox, oy) at record word 36: 8-byte aligned for the int2 load
                const int2 oo = *reinterpret_cast<const int2*>(irec + 16);
                const float tau = tt.x, tx = tt.y, ty = tt.z;
                const int32_t ox = oo.x, oy = oo.y;
                int32_t roff[RX + 1];
#pragma unroll
                for (int a = 0; a <= RX; ++a) roff[a] = min(max(i1 + a + ox, 0), n1 - 1) * n2;
                float m[RX][R + 1];
#pragma unroll
                for (int a = 0; a < RX; ++a)
#pragma unroll
                    for (int k = 0; k <= R; ++k) m[a][k] = 0.0f;
                // every lane of a warp shares `mode` (apart from the few warps
                // straddling two groups) and `oy`, so these branches are uniform
                if (mode == 0 && oy >= -VEC && oy < VEC) {
                    const int mis = oy & (VEC - 1);
                    const int32_t c0 = j0 + oy - mis;
                    switch (mis) {
#define PG_GV(MM) case MM: if constexpr (MM < VEC) gather_vec<S, RX, R, 0, MM>(Vin, P, irec, rec, tx, roff, c0, m); break;
                        PG_GV(0) PG_GV(1) PG_GV(2) PG_GV(3) PG_GV(4) PG_GV(5) PG_GV(6) PG_GV(7)
#undef PG_GV
                    }
                } else if (mode == 1 && oy >= -VEC && oy < VEC) {
                    if (oy >= 0) {
                        const int mis = oy & (VEC - 1);
                        switch (mis) {
#define PG_GV(MM) case MM: if constexpr (MM < VEC) gather_vec<S, RX, R, 0, MM>(Vin, P, irec, rec, tx, roff, oy - MM, m); break;
                            PG_GV(0) PG_GV(1) PG_GV(2) PG_GV(3) PG_GV(4) PG_GV(5) PG_GV(6) PG_GV(7)
#undef PG_GV
                        }
                    } else {
                        switch (-oy) {
#define PG_GV(MM) case MM: if constexpr (MM >= 1 && MM <= VEC) gather_vec<S, RX, R, 1, MM>(Vin, P, irec, rec, tx, roff, 0, m); break;
                            PG_GV(1) PG_GV(2) PG_GV(3) PG_GV(4) PG_GV(5) PG_GV(6) PG_GV(7) PG_GV(8)
#undef PG_GV
                        }
                    }
                } else if (mode == 2 && oy >= -VEC && oy < VEC) {
                    if (oy < 0) {
                        const int mis = oy & (VEC - 1);
                        switch (mis) {
#define PG_GV(MM) case MM: if constexpr (MM < VEC) gather_vec<S, RX, R, 0, MM>(Vin, P, irec, rec, tx, roff, j0 + oy - MM, m); break;
                            PG_GV(0) PG_GV(1) PG_GV(2) PG_GV(3) PG_GV(4) PG_GV(5) PG_GV(6) PG_GV(7)
#undef PG_GV
                        }
                    } else {
                        switch (oy) {
#define PG_GV(MM) case MM: if constexpr (MM < VEC) gather_vec<S, RX, R, 2, MM>(Vin, P, irec, rec, tx, roff, n2 - NV * VEC, m); break;
                            PG_GV(0) PG_GV(1) PG_GV(2) PG_GV(3) PG_GV(4) PG_GV(5) PG_GV(6) PG_GV(7)
#undef PG_GV
                        }
                    }
                } else {
                    int32_t coff[R + 1];
#pragma unroll
                    for (int k = 0; k <= R; ++k) coff[k] = min(max(j0 + k + oy, 0), n2 - 1);
                    gather_scalar<S, RX, R>(Vin, P, irec, rec, tx, roff, coff, m);
                }
#pragma unroll
                for (int a = 0; a < RX; ++a)
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const float val = fmaf(ty, m[a][r + 1] - m[a][r], m[a][r]);
                        const float cv = ((vb[a] >> r) & 1u) ? fminf(tau + fminf(val, cap), cap) : cap;
                        if constexpr (ARGMIN) {
                            // equal values go to the lower table index, which is
                            // what the reference's strict < in table order keeps
                            if (cv < best[a][r] || (cv == best[a][r] && u < bk[a][r])) {
                                best[a][r] = cv;
                                bk[a][r] = u;
                            }
                        } else {
                            best[a][r] = fminf(best[a][r], cv);
                        }
                    }
            }
        }
#pragma unroll
        for (int a = 0; a < RX; ++a)
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int32_t i = i1 + a, j = j0 + r;
                if (i >= x1 || j >= n2) continue;
                const int64_t didx = pl * P + (int64_t)i * n2 + j;
                const S ov = Vp0[(int64_t)i * n2 + j];
                const float old = (float)Conv<S>::val(ov);
                const bool lv = (live >> (a * R + r)) & 1u;
                if constexpr (ARGMIN)
                    argmin[L.rowmajor(i, j, pq6[0], pq6[1], pq6[2], pq6[3])] = lv ? (int16_t)bk[a][r] : (int16_t)-1;
                if (lv && (best[a][r] < old || (kp.relax && old > 0.0f && best[a][r] != old))) {
                    const S nv = Conv<S>::template st<float>(best[a][r]);
                    const float nvT = (float)Conv<S>::val(nv);
                    Vout[didx] = nv;
                    const double d = fabs((double)old - (double)nvT);
                    dsum += d;
                    dmax = fmax(dmax, d);
                } else {
                    Vout[didx] = ov;
                }
            }
    }
    block_partial(dsum, dmax, part_sum, part_max);
}
