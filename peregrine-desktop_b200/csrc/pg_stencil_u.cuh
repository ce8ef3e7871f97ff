// pg_stencil_u.cuh -- the plain scheme's sweep with the decisions taken
// once per solve (included inside namespace pg by pg_kernels.cu).
//
// Whether a lookahead is admissible -- the successor is finite and inside
// the velocity envelope, every swept probe lands on a free cell of the field,
// the successor's (x, y) is on the table (PeregrineSolver.jl:1106-1144 and
// the range tests of interp, 419-431) -- depends on the grid, the model and
// the occupancy, never on V.  k_stencil_mask decides it once per solve for
// every (plane, control, cell), with the reference's rounding, into one bit;
// the sweeps then only read the bit.
//
// k_stencil_u is the sweep.  With the decisions out of the way, the
// interpolation weights of a (plane, control) pair are uniform across the
// plane: the successor sits at a fixed offset (sum of the substep position
// increments) from every cell, so its x/y fractions and its 16 (h, v)
// corners and weights are one set per pair.  A thread owns a block of
// RX rows x R columns; per control it gathers an (RX+1) x (R+1) window from
// each of the 16 corner planes, shared by its RX*R cells.  FP32 arithmetic
// with FMAs; the value differs from the reference's per-cell rounding by a
// few ulp of the interpolation weights, never in a decision.

constexpr int kURX = 2;  // rows per thread
constexpr int kUR = 4;   // columns per thread

// Mask words per (plane, control, row): ceil(Ny / 32).
__host__ __device__ inline int32_t mask_words(int32_t n2) { return (n2 + 31) / 32; }

// One bit per (plane, control, x, y): control u's lookahead from the cell is
// admissible (and the cell is free).  Block = plane; threads walk (u, row,
// word) items.
template <typename T>
__global__ void __launch_bounds__(256)
    k_stencil_mask(const uint8_t* __restrict__ occ, KParams kp, const float* __restrict__ ctl,
                   uint32_t* __restrict__ mask) {
    typedef Ar<T> R_;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nctl = kp.nctl, nsub = kp.nsub, nchk = kp.nchk;
    T* sx = reinterpret_cast<T*>(smem_raw);        // [nctl][nsub] x increments
    T* sy = sx + (size_t)nctl * nsub;              // [nctl][nsub] y increments
    int32_t* sck = reinterpret_cast<int32_t*>(sy + (size_t)nctl * nsub);  // [nctl][4]
    int32_t* sok = sck + (size_t)nctl * kStencilMaxChk;                   // [nctl]
    const Layout L = make_layout(kp);
    GridT<T> g;
    load_grid(g, kp.g);
    const int64_t pl = blockIdx.x;
    int32_t i3, i4, i5, i6;
    {
        int64_t q = pl;
        i6 = (int32_t)(q % L.n[5]); q /= L.n[5];
        i5 = (int32_t)(q % L.n[4]); q /= L.n[4];
        i4 = (int32_t)(q % L.n[3]); q /= L.n[3];
        i3 = (int32_t)q;
    }
    for (int u = threadIdx.x; u < nctl; u += blockDim.x) {
        Transition<T> t;
        transition(kp, g, i3, i4, i5, i6, ctl, u, t);
        for (int k = 0; k < nsub; ++k) {
            sx[u * nsub + k] = t.incx[k];
            sy[u * nsub + k] = t.incy[k];
        }
        for (int sc = 0; sc < kStencilMaxChk; ++sc) sck[u * kStencilMaxChk + sc] = t.ck[sc];
        sok[u] = t.ok ? 1 : 0;
    }
    __syncthreads();
    const int32_t n1 = L.n[0], n2 = L.n[1], W = mask_words(n2);
    const T lo0 = g.lo[0], lo1 = g.lo[1], st0 = g.step[0], st1 = g.step[1];
    const T rs0 = (T)1 / st0, rs1 = (T)1 / st1;
    const T hx = (T)(n1 - 1), hy = (T)(n2 - 1);
    T ap[kStencilMaxChk];
    for (int sc = 0; sc < kStencilMaxChk; ++sc) ap[sc] = R_::div((T)(sc + 1), (T)(nchk > 0 ? nchk : 1));
    const uint8_t* occ_h = occ + (int64_t)i3 * n1 * n2;
    const int64_t items = (int64_t)nctl * n1 * W;
    for (int64_t it = threadIdx.x; it < items; it += blockDim.x) {
        const int u = (int)(it / ((int64_t)n1 * W));
        const int32_t rem = (int32_t)(it - (int64_t)u * n1 * W);
        const int32_t i1 = rem / W, w = rem - i1 * W;
        uint32_t bits = 0;
        if (sok[u]) {
            const T x = axisvalue(g, 0, i1);
            T xn = x;
            for (int k = 0; k < nsub; ++k) xn = R_::add(xn, sx[u * nsub + k]);
            const T dx = R_::sub(xn, x);
            bool xok = true;
            int32_t ci[kStencilMaxChk];
            for (int sc = 0; sc < kStencilMaxChk; ++sc) {
                ci[sc] = 0;
                if (sc < nchk && xok)
                    xok = probe_coord(R_::sub(R_::add(x, R_::mul(dx, ap[sc])), lo0), st0, rs0, hx,
                                      &ci[sc]);
            }
            T f1;
            if (xok) xok = succ_coord<true>(R_::sub(xn, lo0), st0, rs0, hx, &f1);
            if (xok) {
                for (int b = 0; b < 32; ++b) {
                    const int32_t j = w * 32 + b;
                    if (j >= n2) break;
                    if (occ_h[(int64_t)i1 * n2 + j]) continue;
                    const T y = axisvalue(g, 1, j);
                    T yn = y;
                    for (int k = 0; k < nsub; ++k) yn = R_::add(yn, sy[u * nsub + k]);
                    const T dy = R_::sub(yn, y);
                    bool ok = true;
                    for (int sc = 0; sc < nchk && ok; ++sc) {
                        int32_t cj = 0;
                        ok = probe_coord(R_::sub(R_::add(y, R_::mul(dy, ap[sc])), lo1), st1, rs1, hy, &cj);
                        if (ok)
                            ok = occ[((int64_t)sck[u * kStencilMaxChk + sc] * n1 + ci[sc]) * n2 + cj] == 0;
                    }
                    T f2;
                    if (ok) ok = succ_coord<true>(R_::sub(yn, lo1), st1, rs1, hy, &f2);
                    if (ok) bits |= 1u << b;
                }
            }
        }
        mask[((pl * nctl + u) * n1 + i1) * W + w] = bits;
    }
}

__host__ __device__ inline size_t stencil_mask_smem(int nctl, int nsub) {
    return (size_t)nctl * nsub * 2 * sizeof(float) + (size_t)nctl * (kStencilMaxChk + 1) * 4 + 64;
}

// Record per control for the sweep, floats then ints, 16-byte aligned:
//   float: wa[16] = w_hv*(1-tx), wb[16] = w_hv*tx, tau, ty, -, -
//   int:   plane[16], ok, ox, oy, -
constexpr int kUNT = 36;
constexpr int kUNI = 20;

__host__ __device__ inline size_t stencil_u_smem(int nctl) {
    return (size_t)nctl * (kUNT * 4 + kUNI * 4 + 4) + 64;
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

// Accumulate the 16 (h, v) corners of one control into m[a][k], the window
// row a (0..RX) x column k (0..R) combined along x.  Vector path: each
// window row is SPAN = R + VEC storage elements read with 16-byte loads from
// the aligned column c0, the window starting M elements in.
template <typename S, int RX, int R, int M>
__device__ __forceinline__ void gather_vec(const S* __restrict__ Vin, int64_t P,
                                           const int32_t* irec, const float* rec,
                                           const int32_t* roff, int32_t c0,
                                           float (&m)[RX][R + 1]) {
    constexpr int VEC = VecElem<S>::VEC;
    constexpr int NV = (R + VEC) / VEC;
#pragma unroll 1
    for (int q = 0; q < 16; q += 4) {
        const int4 pp = *reinterpret_cast<const int4*>(irec + q);
        const float4 wa4 = *reinterpret_cast<const float4*>(rec + q);
        const float4 wb4 = *reinterpret_cast<const float4*>(rec + 16 + q);
        const int32_t pq[4] = {pp.x, pp.y, pp.z, pp.w};
        const float wa[4] = {wa4.x, wa4.y, wa4.z, wa4.w};
        const float wb[4] = {wb4.x, wb4.y, wb4.z, wb4.w};
#pragma unroll 2
        for (int e = 0; e < 4; ++e) {
            const S* Vc = Vin + (int64_t)pq[e] * P + c0;
            float v[RX + 1][R + 1];
#pragma unroll
            for (int a = 0; a <= RX; ++a) {
                const uint4* src = reinterpret_cast<const uint4*>(Vc + roff[a]);
                uint4 w[NV];
#pragma unroll
                for (int t = 0; t < NV; ++t) w[t] = __ldg(src + t);
#pragma unroll
                for (int k = 0; k <= R; ++k) {
                    // k + M < SPAN by construction
                    switch (k) {
#define PG_VE(K) case K: if constexpr (K <= R) v[a][K] = VecElem<S>::template get<M + K, NV>(w); break;
                        PG_VE(0) PG_VE(1) PG_VE(2) PG_VE(3) PG_VE(4) PG_VE(5) PG_VE(6) PG_VE(7) PG_VE(8)
#undef PG_VE
                    }
                }
            }
#pragma unroll
            for (int a = 0; a < RX; ++a)
#pragma unroll
                for (int k = 0; k <= R; ++k)
                    m[a][k] = fmaf(wa[e], v[a][k], fmaf(wb[e], v[a + 1][k], m[a][k]));
        }
    }
}

// Scalar path: any columns (clamped to the row), one load per value.
template <typename S, int RX, int R>
__device__ __forceinline__ void gather_scalar(const S* __restrict__ Vin, int64_t P,
                                              const int32_t* irec, const float* rec,
                                              const int32_t* roff, const int32_t* coff,
                                              float (&m)[RX][R + 1]) {
#pragma unroll 1
    for (int q = 0; q < 16; q += 4) {
        const int4 pp = *reinterpret_cast<const int4*>(irec + q);
        const float4 wa4 = *reinterpret_cast<const float4*>(rec + q);
        const float4 wb4 = *reinterpret_cast<const float4*>(rec + 16 + q);
        const int32_t pq[4] = {pp.x, pp.y, pp.z, pp.w};
        const float wa[4] = {wa4.x, wa4.y, wa4.z, wa4.w};
        const float wb[4] = {wb4.x, wb4.y, wb4.z, wb4.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const S* Vc = Vin + (int64_t)pq[e] * P;
            float v[RX + 1][R + 1];
#pragma unroll
            for (int a = 0; a <= RX; ++a)
#pragma unroll
                for (int k = 0; k <= R; ++k) v[a][k] = (float)Conv<S>::ld(Vc + roff[a] + coff[k]);
#pragma unroll
            for (int a = 0; a < RX; ++a)
#pragma unroll
                for (int k = 0; k <= R; ++k)
                    m[a][k] = fmaf(wa[e], v[a][k], fmaf(wb[e], v[a + 1][k], m[a][k]));
        }
    }
}

template <typename S, int RX, int R>
__global__ void __launch_bounds__(256, 2)
    k_stencil_u(const S* __restrict__ Vin, S* __restrict__ Vout, const uint8_t* __restrict__ occ,
                const uint32_t* __restrict__ mask, KParams kp, const float* __restrict__ ctl,
                const int32_t* __restrict__ order, double* part_sum, double* part_max,
                int16_t* argmin) {
    constexpr int VEC = VecElem<S>::VEC;
    static_assert(R % VEC == 0, "the window width must be a multiple of the vector width");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nctl = kp.nctl;
    float* rt = reinterpret_cast<float*>(smem_raw);
    int32_t* ri = reinterpret_cast<int32_t*>(rt + (size_t)nctl * kUNT);
    int32_t* ord = ri + (size_t)nctl * kUNI;
    const Layout L = make_layout(kp);
    GridT<float> g;
    load_grid(g, kp.g);
    const float cap = kp.p.cap;
    const int64_t pl = blockIdx.x / kp.tiles_x;
    const int32_t xt = (int32_t)(blockIdx.x - pl * kp.tiles_x);
    int32_t i3, i4, i5, i6;
    {
        int64_t q = pl;
        i6 = (int32_t)(q % L.n[5]); q /= L.n[5];
        i5 = (int32_t)(q % L.n[4]); q /= L.n[4];
        i4 = (int32_t)(q % L.n[3]); q /= L.n[3];
        i3 = (int32_t)q;
    }
    const int32_t n1 = L.n[0], n2 = L.n[1], W = mask_words(n2);
    for (int u = threadIdx.x; u < nctl; u += blockDim.x) {
        ord[u] = order[u];
        Transition<float> t;
        transition(kp, g, i3, i4, i5, i6, ctl, u, t);
        float* rec = rt + (size_t)u * kUNT;
        int32_t* irec = ri + (size_t)u * kUNI;
        const float dxc = t.sumx / g.step[0], dyc = t.sumy / g.step[1];
        const float fx = floorf(dxc), fy = floorf(dyc);
        const float tx = dxc - fx, ty = dyc - fy;
        for (int c = 0; c < 16; ++c) {
            const float w = corner_weight(t, c);
            rec[c] = w * (1.0f - tx);
            rec[16 + c] = w * tx;
            irec[c] = corner_plane(g, t, c);
        }
        rec[32] = t.tau;
        rec[33] = ty;
        rec[34] = 0.0f;
        rec[35] = 0.0f;
        irec[16] = t.ok ? 1 : 0;
        irec[17] = t.ok ? (int32_t)fx : 0;
        irec[18] = t.ok ? (int32_t)fy : 0;
        irec[19] = 0;
    }
    __syncthreads();

    const int32_t x0 = xt * kp.tile_x;
    const int32_t x1 = min(x0 + kp.tile_x, n1);
    const int32_t rb_n = (x1 - x0 + RX - 1) / RX;
    const int32_t cb_n = (n2 + R - 1) / R;
    // Column blocks 1 .. cb_n-2 can take the vector path (their aligned
    // window stays inside the row for successor offsets in [-VEC, VEC-1]);
    // they are numbered first so whole warps take one path.
    const bool vec_ok = (n2 % R) == 0 && cb_n >= 3;
    const int32_t n_inner = vec_ok ? rb_n * (cb_n - 2) : 0;
    const int32_t nseg = rb_n * cb_n;
    const int64_t P = L.P;
    const S* __restrict__ Vp0 = Vin + pl * P;
    const uint8_t* occ_h = occ + (int64_t)i3 * n1 * n2;
    const uint32_t* mplane = mask + (size_t)pl * nctl * n1 * W;
    double dsum = 0.0, dmax = 0.0;

    for (int seg = threadIdx.x; seg < nseg; seg += blockDim.x) {
        int32_t rb, cb;
        bool inner;
        if (seg < n_inner) {
            rb = seg / (cb_n - 2);
            cb = 1 + (seg - rb * (cb_n - 2));
            inner = true;
        } else {
            const int32_t e = seg - n_inner;
            const int32_t ne = vec_ok ? 2 : cb_n;  // edge columns per row block
            rb = e / ne;
            const int32_t k = e - rb * ne;
            cb = vec_ok ? (k == 0 ? 0 : cb_n - 1) : k;
            inner = false;
        }
        const int32_t i1 = x0 + rb * RX;
        const int32_t j0 = cb * R;
        float old[RX][R], best[RX][R];
        int bk[RX][R];
        bool live[RX][R];
        bool any = false;
#pragma unroll
        for (int a = 0; a < RX; ++a)
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int32_t i = i1 + a, j = j0 + r;
                const bool in = i < x1 && j < n2;
                old[a][r] = in ? (float)Conv<S>::ld(Vp0 + (int64_t)i * n2 + j) : cap;
                live[a][r] = in && occ_h[(int64_t)i * n2 + j] == 0;
                any |= live[a][r];
                best[a][r] = cap;
                bk[a][r] = 0x7fffffff;
            }
        if (any) {
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
                float c[RX][R];
                if (vany) {
                    const float* rec = rt + (size_t)u * kUNT;
                    const int32_t* irec = ri + (size_t)u * kUNI;
                    const float4 tail = *reinterpret_cast<const float4*>(rec + 32);
                    const int4 itail = *reinterpret_cast<const int4*>(irec + 16);
                    const float tau = tail.x, ty = tail.y;
                    const int32_t ox = itail.y, oy = itail.z;
                    int32_t roff[RX + 1];
#pragma unroll
                    for (int a = 0; a <= RX; ++a) roff[a] = min(max(i1 + a + ox, 0), n1 - 1) * n2;
                    float m[RX][R + 1];
#pragma unroll
                    for (int a = 0; a < RX; ++a)
#pragma unroll
                        for (int k = 0; k <= R; ++k) m[a][k] = 0.0f;
                    if (inner && oy >= -VEC && oy < VEC) {
                        // warp-uniform: every lane of an inner warp has j0 % R == 0
                        const int mis = oy & (VEC - 1);
                        const int32_t c0 = j0 + oy - mis;
                        switch (mis) {
#define PG_GV(MM) case MM: if constexpr (MM < VEC) gather_vec<S, RX, R, MM>(Vin, P, irec, rec, roff, c0, m); break;
                            PG_GV(0) PG_GV(1) PG_GV(2) PG_GV(3) PG_GV(4) PG_GV(5) PG_GV(6) PG_GV(7)
#undef PG_GV
                        }
                    } else {
                        int32_t coff[R + 1];
#pragma unroll
                        for (int k = 0; k <= R; ++k) coff[k] = min(max(j0 + k + oy, 0), n2 - 1);
                        gather_scalar<S, RX, R>(Vin, P, irec, rec, roff, coff, m);
                    }
#pragma unroll
                    for (int a = 0; a < RX; ++a)
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            const float val = fmaf(ty, m[a][r + 1] - m[a][r], m[a][r]);
                            const float cv = fminf(tau + fminf(val, cap), cap);
                            c[a][r] = ((vb[a] >> r) & 1u) ? cv : cap;
                        }
                } else {
#pragma unroll
                    for (int a = 0; a < RX; ++a)
#pragma unroll
                        for (int r = 0; r < R; ++r) c[a][r] = cap;
                }
                // min over controls; equal values go to the lower table index,
                // which is what the reference's strict < in table order keeps
#pragma unroll
                for (int a = 0; a < RX; ++a)
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        if (c[a][r] < best[a][r] || (c[a][r] == best[a][r] && u < bk[a][r])) {
                            best[a][r] = c[a][r];
                            bk[a][r] = u;
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
                if (!live[a][r]) {
                    Vout[didx] = Vin[didx];
                    if (argmin) argmin[L.rowmajor(i, j, i3, i4, i5, i6)] = -1;
                    continue;
                }
                if (argmin) argmin[L.rowmajor(i, j, i3, i4, i5, i6)] = (int16_t)bk[a][r];
                if (best[a][r] < old[a][r] || (kp.relax && best[a][r] != old[a][r])) {
                    const S nv = Conv<S>::template st<float>(best[a][r]);
                    const float nvT = (float)Conv<S>::val(nv);
                    Vout[didx] = nv;
                    const double d = fabs((double)old[a][r] - (double)nvT);
                    dsum += d;
                    dmax = fmax(dmax, d);
                } else {
                    Vout[didx] = Vin[didx];
                }
            }
    }
    block_partial(dsum, dmax, part_sum, part_max);
}
