// pg_stencil_d.cuh -- the FP64 precision oracle of the plain scheme's sweep
// (included inside namespace pg by pg_kernels.cu, after pg_stencil_r.cuh,
// whose successor rounding it shares).
//
// Every decision is the FP32 solver's: the admissibility bits and the
// per-(plane, control) records that k_stencil_prep writes (the swept probes,
// the range tests, the successor's (h, v) corner planes and fractions, the
// substep increments), and the per-row / per-column successor corners and
// fractions rounded in float exactly as the FP32 sweeps round them.  Only the
// value arithmetic is FP64: the (h, v) weights are formed in double from the
// record's float fractions, the 64-corner interpolation (as a blend of the 16
// corner planes over a window of rows, then the bilinear step), tau + V, the
// caps, the min and the stored table.  So FP32 against this table measures
// what storage and arithmetic precision cost, at the same model -- not the
// model differences of deciding the probes in double.
//
// Block = (plane, tile of kp.tile_x whole rows, at most 1024 cells), 256
// threads, 4 cells per thread, controls in table order; two barriers per
// control.  An oracle: written for clarity, not speed.

constexpr int kDThreads = 256;

__host__ __device__ inline size_t stencil_d_smem(int tile_x, int n2) {
    return (size_t)(tile_x + 3) * n2 * sizeof(double) + (size_t)(tile_x + n2) * sizeof(int2) +
           16 * sizeof(double) + 16 * sizeof(int32_t) + 16;
}

template <bool ARGMIN>
__global__ void __launch_bounds__(kDThreads)
    k_stencil_d(const double* __restrict__ Vin, double* __restrict__ Vout,
                const uint8_t* __restrict__ occ, const uint32_t* __restrict__ mask,
                const uint32_t* __restrict__ recs, KParams kp, double* part_sum,
                double* part_max, int16_t* argmin) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nctl = kp.nctl;
    const int32_t n1 = kp.g.n[0], n2 = kp.g.n[1], W = mask_words(n2);
    const int32_t TX = kp.tile_x;
    double* Bd = reinterpret_cast<double*>(smem_raw);            // [(TX+3) * n2]
    double* wd = Bd + (size_t)(TX + 3) * n2;                      // [16]
    int2* ent = reinterpret_cast<int2*>(wd + 16);                 // [TX + n2]
    int32_t* pc = reinterpret_cast<int32_t*>(ent + TX + n2);      // [16]
    const Layout L = make_layout(kp);
    const double cap = (double)kp.p.cap;
    const int64_t P = L.P;
    const int T = blockDim.x, tid = threadIdx.x;
    const int64_t pl = blockIdx.x / kp.tiles_x;
    const int32_t xt = (int32_t)(blockIdx.x - pl * kp.tiles_x);
    const int32_t x0 = xt * TX;
    const int32_t nr = min(TX, n1 - x0);
    const int32_t ncell = nr * n2;
    const int32_t nw = nr + 3;
    int32_t pq6[4];
    {
        int64_t pp = pl;
        pq6[3] = (int32_t)(pp % L.n[5]); pp /= L.n[5];
        pq6[2] = (int32_t)(pp % L.n[4]); pp /= L.n[4];
        pq6[1] = (int32_t)(pp % L.n[3]); pp /= L.n[3];
        pq6[0] = (int32_t)pp;
    }
    const uint8_t* occ_h = occ + ((int64_t)pq6[0] * n1 + x0) * n2;
    double best[kBCells];
    int bk[kBCells];
    uint32_t live = 0;
#pragma unroll
    for (int q = 0; q < kBCells; ++q) {
        const int32_t e = tid + q * T;
        best[q] = cap;
        bk[q] = 0x7fffffff;
        if (e < ncell && occ_h[e] == 0) live |= 1u << q;
    }
    const uint32_t* prec = recs + (size_t)pl * nctl * kURec;
    for (int u = 0; u < nctl; ++u) {
        const uint32_t* rec = prec + (size_t)u * kURec;
        if (__ldg(rec + kUNT + 18) == 0u) {
            // no cell of the plane admits this control (block-uniform)
            if constexpr (ARGMIN) {
#pragma unroll
                for (int q = 0; q < kBCells; ++q)
                    if (best[q] == cap && u < bk[q]) bk[q] = u;
            }
            continue;
        }
        const int32_t wbase = x0 + (int32_t)__ldg(rec + kUNT + 16) - 1;
        // the (h, v) weights in double from the float fractions, and planes
        if (tid < 16) {
            const int c = tid;
            double w = 1.0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double t = (double)__uint_as_float(__ldg(rec + kUTT + k));
                w *= ((c >> k) & 1) ? t : 1.0 - t;
            }
            wd[c] = w;
            pc[c] = (int32_t)__ldg(rec + kUNT + c);
        }
        // the successor's lower corner and fraction per row and per column,
        // rounded in float as the FP32 sweeps round them
        for (int32_t i = tid; i < nr + n2; i += T) {
            const bool row = i < nr;
            const float* inc = reinterpret_cast<const float*>(rec + kUInc) + (row ? 0 : kStencilMaxSub);
            int32_t li;
            float t;
            succ_li_t(kp.g, inc, kp.nsub, row, row ? x0 + i : i - nr, n1, n2, &li, &t);
            if (row)
                ent[i] = make_int2(min(max(li - wbase, 0), nw - 2), __float_as_int(t));
            else
                ent[TX + i - nr] = make_int2(min(max(li, 0), n2 - 1), __float_as_int(t));
        }
        __syncthreads();
        // blend the 16 corner planes over the window rows, in double
        for (int32_t it = tid; it < nw * n2; it += T) {
            const int32_t k = it / n2, j = it - k * n2;
            const int64_t off = (int64_t)min(max(wbase + k, 0), n1 - 1) * n2 + j;
            double acc = 0.0;
#pragma unroll 4
            for (int c = 0; c < 16; ++c) acc = fma(wd[c], __ldg(Vin + (int64_t)pc[c] * P + off), acc);
            Bd[it] = acc;
        }
        __syncthreads();
        const double tau = (double)__uint_as_float(__ldg(rec + 16));
        const uint32_t* mrow = mask + ((size_t)pl * nctl + u) * n1 * W;
#pragma unroll
        for (int q = 0; q < kBCells; ++q) {
            const int32_t e = tid + q * T;
            if (e >= ncell) break;
            const int32_t a = e / n2, j = e - a * n2;
            double cvl = cap;
            if (((live >> q) & 1u) && ((__ldg(mrow + (x0 + a) * W + (j >> 5)) >> (j & 31)) & 1u)) {
                const int2 rr = ent[a], cc = ent[TX + j];
                const double tx = (double)__int_as_float(rr.y), ty = (double)__int_as_float(cc.y);
                const int32_t ja = cc.x, jb = min(cc.x + 1, n2 - 1);
                const double* r0 = Bd + (int64_t)rr.x * n2;
                const double* r1 = r0 + n2;
                const double m0 = fma(tx, r1[ja] - r0[ja], r0[ja]);
                const double m1 = fma(tx, r1[jb] - r0[jb], r0[jb]);
                const double val = fma(ty, m1 - m0, m0);
                cvl = fmin(tau + fmin(val, cap), cap);
            }
            if (cvl < best[q] || (cvl == best[q] && u < bk[q])) {
                best[q] = cvl;
                bk[q] = u;
            }
        }
        __syncthreads();
    }
    const double* Vp0 = Vin + pl * P + (int64_t)x0 * n2;
    double* Vo0 = Vout + pl * P + (int64_t)x0 * n2;
    double dsum = 0.0, dmax = 0.0;
#pragma unroll
    for (int q = 0; q < kBCells; ++q) {
        const int32_t e = tid + q * T;
        if (e >= ncell) break;
        const double old = Vp0[e];
        const bool lv = (live >> q) & 1u;
        if constexpr (ARGMIN) {
            const int32_t a = e / n2, j = e - a * n2;
            argmin[L.rowmajor(x0 + a, j, pq6[0], pq6[1], pq6[2], pq6[3])] =
                lv ? (int16_t)bk[q] : (int16_t)-1;
        }
        if (lv && (best[q] < old || (kp.relax && old > 0.0 && best[q] != old))) {
            Vo0[e] = best[q];
            const double d = fabs(old - best[q]);
            dsum += d;
            dmax = fmax(dmax, d);
        } else {
            Vo0[e] = old;
        }
    }
    block_partial_at(dsum, dmax, part_sum, part_max, blockIdx.x);
}
