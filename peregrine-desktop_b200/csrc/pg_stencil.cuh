// pg_stencil.cuh -- the plain scheme as a position-invariant stencil
// (included by pg_kernels.cu).
//
// Nothing in the dynamics reads x or y (solver/src/Tiles.jl:94-97), so for a
// fixed (h, vx, vy, w) plane and control the successor's heading/velocity
// corners and weights, the probe heading bins and the per-substep position
// increments are shared by every (x, y) cell.  A block takes one plane (or
// an x-range of it):
//
//   phase A  one thread per control integrates the held command once and
//            stages a record in shared memory: the position increments, the
//            probe heading bins, the 16 (h, v)-corner planes and weights.
//   phase B  each thread owns R consecutive cells of one row.  Per control it
//            replays the increments (x once for the row, y per cell) so every
//            probe and envelope decision rounds exactly as the reference's
//            per-cell arithmetic (PeregrineSolver.jl:1100-1153), then gathers
//            the 64 corners through an (R+1)-wide window per corner row that
//            the R cells share.
//
// EXACT=true keeps the reference's weight products and summation order
// (bit-identical to the CPU restatement).  EXACT=false folds the x weight
// into the (h, v) weights and accumulates with FMAs.
//
// Included inside namespace pg, after the cell-form kernel's helpers.

constexpr int kStencilR = 4;  // cells per thread along y

// The quotient num/den of an axis coordinate, for the decisions only: round
// to the nearest cell and test against [0, hi] exactly as the correctly
// rounded division would, from a reciprocal multiply (|error| <= 2.4e-7
// relative) with the true division taken only within 1e-6 of a rounding
// boundary or of `hi`.  Returns false when the coordinate is off the axis.
__device__ __forceinline__ bool probe_coord(float num, float den, float rden, float hi,
                                            int32_t* cell) {
    if (num < 0.0f) return false;  // num/den < 0 exactly when num < 0 (den > 0)
    float q = __fmul_rn(num, rden);
    const float g = q * 1.0e-6f + 1.0e-30f;
    if (fabsf(q - hi) <= g || fabsf(q - floorf(q) - 0.5f) <= g) q = __fdiv_rn(num, den);
    if (q > hi) return false;
    *cell = (int32_t)rintf(q);
    return true;
}
__device__ __forceinline__ bool probe_coord(double num, double den, double, double hi,
                                            int32_t* cell) {
    const double q = __ddiv_rn(num, den);
    if (q < 0.0 || q > hi) return false;
    *cell = (int32_t)rint(q);
    return true;
}

// The successor's axis coordinate f = num/den for interpolation: the range
// test is decided exactly; the value itself is exact when EXACT, else the
// reciprocal-multiply approximation (interpolation is continuous in f).
template <bool EXACT>
__device__ __forceinline__ bool succ_coord(float num, float den, float rden, float hi, float* f) {
    if (num < 0.0f) return false;
    float q;
    if (EXACT) {
        q = __fdiv_rn(num, den);
    } else {
        q = __fmul_rn(num, rden);
        if (fabsf(q - hi) <= q * 1.0e-6f + 1.0e-30f) q = __fdiv_rn(num, den);
    }
    if (q > hi) return false;
    *f = q;
    return true;
}
template <bool EXACT>
__device__ __forceinline__ bool succ_coord(double num, double den, double, double hi, double* f) {
    const double q = __ddiv_rn(num, den);
    if (q < 0.0 || q > hi) return false;
    *f = q;
    return true;
}

// Record layout per control, in T words then int words, both padded to a
// multiple of 4 so the 16-wide blocks load as vectors:
//   T:   w[16] (fast) | w3 w3' w4 w4' w5 w5' w6 w6' + pad (exact), tau, incx[nsub], incy[nsub]
//   int: plane[16], ok, ck[nchk]
template <typename T, bool EXACT> struct RecLayout {
    int nsub, nchk, NT, NI;
    __host__ __device__ RecLayout(int ns, int nc) : nsub(ns), nchk(nc) {
        NT = ((16 + 1 + 2 * ns) + 3) & ~3;
        NI = ((16 + 1 + nc) + 3) & ~3;
    }
    static constexpr int W = 0;
    static constexpr int TAU = 16;
    __host__ __device__ int incx(int k) const { return 17 + k; }
    __host__ __device__ int incy(int k) const { return 17 + nsub + k; }
    static constexpr int PLANE = 0;
    static constexpr int OK = 16;
    __host__ __device__ int ck(int s) const { return 17 + s; }
};

template <typename T, bool EXACT>
__host__ __device__ inline size_t stencil_smem_bytes(int nctl, int nsub, int nchk) {
    RecLayout<T, EXACT> L(nsub, nchk);
    return (size_t)nctl * L.NT * sizeof(T) + (size_t)nctl * L.NI * sizeof(int32_t) +
           (size_t)nctl * sizeof(int32_t) + 64;
}

template <typename T> __device__ __forceinline__ void lds4(const T* p, T* o);
template <> __device__ __forceinline__ void lds4<float>(const float* p, float* o) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
template <> __device__ __forceinline__ void lds4<double>(const double* p, double* o) {
    const double2 a = *reinterpret_cast<const double2*>(p);
    const double2 b = *reinterpret_cast<const double2*>(p + 2);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void lds4i(const int32_t* p, int32_t* o) {
    const int4 v = *reinterpret_cast<const int4*>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}

template <typename S, typename T, bool EXACT, int NSUB>
__global__ void __launch_bounds__(256)
    k_stencil(const S* __restrict__ Vin, S* __restrict__ Vout, const uint8_t* __restrict__ occ,
              KParams kp, const float* __restrict__ ctl, const int32_t* __restrict__ order,
              double* part_sum, double* part_max, int16_t* argmin) {
    typedef Ar<T> R_;
    constexpr int R = kStencilR;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nctl = kp.nctl, nsub = kp.nsub, nchk = kp.nchk;
    const RecLayout<T, EXACT> RL(nsub, nchk);
    T* rt = reinterpret_cast<T*>(smem_raw);
    int32_t* ri = reinterpret_cast<int32_t*>(rt + (size_t)nctl * RL.NT);
    int32_t* ord = ri + (size_t)nctl * RL.NI;

    const Layout L = make_layout(kp);
    GridT<T> g;
    load_grid(g, kp.g);
    const T cap = (T)kp.p.cap;
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

    // ---- phase A: the held command integrated once per control for this plane
    for (int u = threadIdx.x; u < nctl; u += blockDim.x) {
        ord[u] = order[u];
        T* rec = rt + (size_t)u * RL.NT;
        int32_t* irec = ri + (size_t)u * RL.NI;
        Transition<T> t;
        transition(kp, g, i3, i4, i5, i6, ctl, u, t);
        for (int k = 0; k < nsub; ++k) {
            rec[RL.incx(k)] = t.incx[k];
            rec[RL.incy(k)] = t.incy[k];
        }
        rec[RL.TAU] = t.tau;
        for (int sc = 0; sc < nchk; ++sc) irec[RL.ck(sc)] = t.ck[sc];
        irec[RL.OK] = t.ok ? 1 : 0;
        for (int c = 0; c < 16; ++c) {
            irec[RL.PLANE + c] = corner_plane(g, t, c);
            if (!EXACT) rec[RL.W + c] = corner_weight(t, c);
        }
        if (EXACT) {
            for (int k = 0; k < 4; ++k) {
                rec[RL.W + 2 * k] = R_::sub((T)1, t.tt[k]);
                rec[RL.W + 2 * k + 1] = t.tt[k];
            }
            for (int k = 8; k < 16; ++k) rec[RL.W + k] = (T)0;
        }
    }
    __syncthreads();

    // ---- phase B: R consecutive cells of one row per thread.  Rows are the
    // device table's (a slab of the global table when kp.xoff > 0 or
    // kp.n1g > n1); every coordinate, range test and occupancy lookup uses
    // the global row, so a slab sweeps exactly as the whole table does.
    const int32_t n1 = L.n[0], n2 = L.n[1];
    const int32_t n1g = kp.n1g, xoff = kp.xoff;
    const int32_t x0 = xt * kp.tile_x;
    const int32_t x1 = min(x0 + kp.tile_x, n1);
    const int32_t spr = (n2 + R - 1) / R;  // segments per row
    const int32_t nseg = (x1 - x0) * spr;
    const T lo0 = g.lo[0], lo1 = g.lo[1], st0 = g.step[0], st1 = g.step[1];
    const T rs0 = (T)1 / st0, rs1 = (T)1 / st1;
    const T hx = (T)(n1g - 1), hy = (T)(n2 - 1);
    const int64_t P = L.P;
    const S* __restrict__ Vp0 = Vin + pl * P;
    // the global occupancy (Nh x n1g x n2), this plane's heading, the slab's rows
    const uint8_t* occ_h = occ + ((int64_t)i3 * n1g + xoff) * n2;
    T ap[kStencilMaxChk];
#pragma unroll
    for (int sc = 0; sc < kStencilMaxChk; ++sc) ap[sc] = R_::div((T)(sc + 1), (T)(nchk > 0 ? nchk : 1));
    double dsum = 0.0, dmax = 0.0;

    for (int seg = threadIdx.x; seg < nseg; seg += blockDim.x) {
        const int32_t i1 = x0 + seg / spr;
        const int32_t j0 = (seg - (i1 - x0) * spr) * R;
        if (i1 < kp.ux0 || i1 >= kp.ux1) {
            // a halo row of a slab: passed through unchanged
            for (int r = 0; r < R; ++r) {
                const int32_t j = j0 + r;
                if (j >= n2) break;
                const int64_t didx = pl * P + (int64_t)i1 * n2 + j;
                Vout[didx] = Vin[didx];
            }
            continue;
        }
        T old[R], y[R], best[R];
        int bk[R];
        bool live[R];  // inside the row and not blocked
        bool any = false;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int32_t j = j0 + r;
            const bool in = j < n2;
            old[r] = in ? (T)Conv<S>::ld(Vp0 + (int64_t)i1 * n2 + j) : cap;
            live[r] = in && occ_h[(int64_t)i1 * n2 + j] == 0;
            any |= live[r];
            y[r] = axisvalue(g, 1, in ? j : 0);
            best[r] = cap;
            bk[r] = 0x7fffffff;
        }
        if (any) {
            const T x = axisvalue(g, 0, xoff + i1);
            for (int uu = 0; uu < nctl; ++uu) {
                const int u = ord[uu];
                const T* rec = rt + (size_t)u * RL.NT;
                const int32_t* irec = ri + (size_t)u * RL.NI;
                T c[R];
#pragma unroll
                for (int r = 0; r < R; ++r) c[r] = cap;
                if (irec[RL.OK]) {
                    // x part, shared by the row's R cells
                    T xn = x;
                    if (NSUB > 0) {
#pragma unroll
                        for (int k = 0; k < NSUB; ++k) xn = R_::add(xn, rec[RL.incx(k)]);
                    } else {
                        for (int k = 0; k < nsub; ++k) xn = R_::add(xn, rec[RL.incx(k)]);
                    }
                    const T dx = R_::sub(xn, x);
                    bool xok = true;
                    int32_t ci[kStencilMaxChk];
#pragma unroll
                    for (int sc = 0; sc < kStencilMaxChk; ++sc) {
                        ci[sc] = 0;
                        if (sc < nchk && xok)
                            xok = probe_coord(R_::sub(R_::add(x, R_::mul(dx, ap[sc])), lo0), st0,
                                              rs0, hx, &ci[sc]);
                    }
                    T f1 = 0;
                    if (xok) xok = succ_coord<EXACT>(R_::sub(xn, lo0), st0, rs0, hx, &f1);
                    if (xok) {
                        const T b1 = R_::floor_(f1);
                        const T t1 = R_::sub(f1, b1);
                        // the successor's rows, global, then in the slab (a
                        // halo as wide as the reach keeps them inside it; the
                        // clamp only keeps a starved halo's reads in bounds)
                        const int32_t j1g = (int32_t)b1;
                        const int32_t j1 = min(max(j1g - xoff, 0), n1 - 1);
                        const int32_t j1p = min(max(min(j1g + 1, n1g - 1) - xoff, 0), n1 - 1);
                        // y part, per cell
                        T t2[R];
                        int32_t j2[R];
                        bool ok[R];
                        T incy[NSUB > 0 ? NSUB : 1];
                        if (NSUB > 0) {
#pragma unroll
                            for (int k = 0; k < NSUB; ++k) incy[k] = rec[RL.incy(k)];
                        }
                        int64_t orow[kStencilMaxChk];
#pragma unroll
                        for (int sc = 0; sc < kStencilMaxChk; ++sc)
                            orow[sc] = sc < nchk ? ((int64_t)irec[RL.ck(sc)] * n1g + ci[sc]) * n2 : 0;
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            ok[r] = live[r];
                            t2[r] = 0;
                            j2[r] = 0;
                            if (!ok[r]) continue;
                            T yn = y[r];
                            if (NSUB > 0) {
#pragma unroll
                                for (int k = 0; k < NSUB; ++k) yn = R_::add(yn, incy[k]);
                            } else {
                                for (int k = 0; k < nsub; ++k) yn = R_::add(yn, rec[RL.incy(k)]);
                            }
                            const T dy = R_::sub(yn, y[r]);
#pragma unroll
                            for (int sc = 0; sc < kStencilMaxChk; ++sc) {
                                if (sc >= nchk || !ok[r]) continue;
                                int32_t cj = 0;
                                ok[r] = probe_coord(R_::sub(R_::add(y[r], R_::mul(dy, ap[sc])), lo1),
                                                    st1, rs1, hy, &cj);
                                if (ok[r]) ok[r] = occ[orow[sc] + cj] == 0;
                            }
                            T f2 = 0;
                            if (ok[r]) ok[r] = succ_coord<EXACT>(R_::sub(yn, lo1), st1, rs1, hy, &f2);
                            if (ok[r]) {
                                const T b2 = R_::floor_(f2);
                                t2[r] = R_::sub(f2, b2);
                                j2[r] = (int32_t)b2;
                            }
                        }
                        // the window: R+1 consecutive y positions from the first
                        // live cell's corner; valid when every live cell sits at
                        // its own offset inside it
                        int32_t jbase = 0;
                        bool anyok = false, uniform = true;
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            if (!ok[r]) continue;
                            if (!anyok) { jbase = j2[r] - r; anyok = true; }
                            else uniform &= (j2[r] == jbase + r);
                        }
                        if (anyok) {
                            T acc[R];
#pragma unroll
                            for (int r = 0; r < R; ++r) acc[r] = 0;
                            int32_t wy[R + 1];
#pragma unroll
                            for (int k = 0; k <= R; ++k) wy[k] = min(max(jbase + k, 0), n2 - 1);
                            const int64_t rowa = (int64_t)j1 * n2, rowb = (int64_t)j1p * n2;
                            T w8[16];
                            int32_t pp[16];
#pragma unroll
                            for (int q = 0; q < 16; q += 4) {
                                lds4<T>(rec + RL.W + q, w8 + q);
                                lds4i(irec + RL.PLANE + q, pp + q);
                            }
                            if (uniform) {
                                if (EXACT) {
                                    const T w1[2] = {R_::sub((T)1, t1), t1};
                                    T p12[R][4];
#pragma unroll
                                    for (int r = 0; r < R; ++r) {
                                        const T w2[2] = {R_::sub((T)1, t2[r]), t2[r]};
#pragma unroll
                                        for (int q = 0; q < 4; ++q) p12[r][q] = R_::mul(w1[q & 1], w2[q >> 1]);
                                    }
#pragma unroll 2
                                    for (int hc = 0; hc < 16; ++hc) {
                                        const S* Vc = Vin + (int64_t)pp[hc] * P;
                                        T a[R + 1], b[R + 1];
#pragma unroll
                                        for (int k = 0; k <= R; ++k) {
                                            a[k] = (T)Conv<S>::ld(Vc + rowa + wy[k]);
                                            b[k] = (T)Conv<S>::ld(Vc + rowb + wy[k]);
                                        }
                                        const T w3 = w8[0 + (hc & 1)], w4 = w8[2 + ((hc >> 1) & 1)];
                                        const T w5 = w8[4 + ((hc >> 2) & 1)], w6 = w8[6 + ((hc >> 3) & 1)];
#pragma unroll
                                        for (int r = 0; r < R; ++r) {
                                            const T v[4] = {a[r], b[r], a[r + 1], b[r + 1]};
#pragma unroll
                                            for (int q = 0; q < 4; ++q) {
                                                const T wgt = R_::mul(R_::mul(R_::mul(R_::mul(p12[r][q], w3), w4), w5), w6);
                                                if (wgt != (T)0) acc[r] = R_::add(acc[r], R_::mul(wgt, v[q]));
                                            }
                                        }
                                    }
                                } else {
                                    T m[R + 1];
#pragma unroll
                                    for (int k = 0; k <= R; ++k) m[k] = 0;
#pragma unroll 4
                                    for (int hc = 0; hc < 16; ++hc) {
                                        const S* Vc = Vin + (int64_t)pp[hc] * P;
                                        const T wb = w8[hc] * t1;
                                        const T wa = w8[hc] - wb;
#pragma unroll
                                        for (int k = 0; k <= R; ++k) {
                                            const T av = (T)Conv<S>::ld(Vc + rowa + wy[k]);
                                            const T bv = (T)Conv<S>::ld(Vc + rowb + wy[k]);
                                            m[k] = fma(wa, av, fma(wb, bv, m[k]));
                                        }
                                    }
#pragma unroll
                                    for (int r = 0; r < R; ++r) acc[r] = fma(t2[r], m[r + 1] - m[r], m[r]);
                                }
                            } else {
                                // cells whose corners do not line up: each on its own
#pragma unroll
                                for (int r = 0; r < R; ++r) {
                                    if (!ok[r]) continue;
                                    const int32_t ya = j2[r], yb = min(j2[r] + 1, n2 - 1);
                                    T a0 = 0;
                                    if (EXACT) {
                                        const T w1[2] = {R_::sub((T)1, t1), t1};
                                        const T w2[2] = {R_::sub((T)1, t2[r]), t2[r]};
                                        for (int hc = 0; hc < 16; ++hc) {
                                            const S* Vc = Vin + (int64_t)pp[hc] * P;
                                            const T v[4] = {(T)Conv<S>::ld(Vc + rowa + ya), (T)Conv<S>::ld(Vc + rowb + ya),
                                                            (T)Conv<S>::ld(Vc + rowa + yb), (T)Conv<S>::ld(Vc + rowb + yb)};
                                            const T w3 = w8[0 + (hc & 1)], w4 = w8[2 + ((hc >> 1) & 1)];
                                            const T w5 = w8[4 + ((hc >> 2) & 1)], w6 = w8[6 + ((hc >> 3) & 1)];
                                            for (int q = 0; q < 4; ++q) {
                                                const T wgt = R_::mul(R_::mul(R_::mul(R_::mul(R_::mul(w1[q & 1], w2[q >> 1]), w3), w4), w5), w6);
                                                if (wgt != (T)0) a0 = R_::add(a0, R_::mul(wgt, v[q]));
                                            }
                                        }
                                    } else {
                                        for (int hc = 0; hc < 16; ++hc) {
                                            const S* Vc = Vin + (int64_t)pp[hc] * P;
                                            const T wb = w8[hc] * t1;
                                            const T wa = w8[hc] - wb;
                                            const T ma = fma(wa, (T)Conv<S>::ld(Vc + rowa + ya), wb * (T)Conv<S>::ld(Vc + rowb + ya));
                                            const T mb = fma(wa, (T)Conv<S>::ld(Vc + rowa + yb), wb * (T)Conv<S>::ld(Vc + rowb + yb));
                                            a0 += fma(t2[r], mb - ma, ma);
                                        }
                                    }
                                    acc[r] = a0;
                                }
                            }
                            const T tau = rec[RL.TAU];
#pragma unroll
                            for (int r = 0; r < R; ++r)
                                if (ok[r]) c[r] = jmin(R_::add(tau, jmin(acc[r], cap)), cap);
                        }
                    }
                }
                // min over controls; equal values go to the lower table index,
                // which is what the reference's strict < in table order keeps
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (c[r] < best[r] || (c[r] == best[r] && u < bk[r])) {
                        best[r] = c[r];
                        bk[r] = u;
                    }
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int32_t j = j0 + r;
            if (j >= n2) continue;
            const int64_t didx = pl * P + (int64_t)i1 * n2 + j;
            if (!live[r]) {
                Vout[didx] = Vin[didx];
                if (argmin) argmin[L.rowmajor(i1, j, i3, i4, i5, i6)] = -1;
                continue;
            }
            if (argmin) argmin[L.rowmajor(i1, j, i3, i4, i5, i6)] = (int16_t)bk[r];
            if (best[r] < old[r] || (kp.relax && old[r] > (T)0 && best[r] != old[r])) {
                const S nv = Conv<S>::template st<T>(best[r]);
                const T nvT = (T)Conv<S>::val(nv);
                Vout[didx] = nv;
                const double d = fabs((double)old[r] - (double)nvT);
                dsum += d;
                dmax = fmax(dmax, d);
            } else {
                Vout[didx] = Vin[didx];
            }
        }
    }
    block_partial(dsum, dmax, part_sum, part_max);
}
