// pg_kernels.cu -- the sweep kernels of the B200 value-iteration solver.
//
// Two sweep kernels compute the same Jacobi update V' = min(V, T V):
//
//   k_cellform  one thread per cell running the reference's whole
//               cell_update (PeregrineSolver.jl:1205-1344): every scheme
//               option, the escape views, the Int8 warm-start policy.
//               Bit-identical to the CPU restatement.
//
//   k_stencil   the plain scheme (full control scan, one horizon, fixed
//               probes, 64-corner multilinear) reorganised around position
//               invariance: nothing in the dynamics reads x or y
//               (solver/src/Tiles.jl:94-97), so for a fixed (h, vx, vy, w)
//               plane and control the successor's heading/velocity corners,
//               their weights, the probe heading bins and the per-substep
//               position increments are the same for every (x, y) cell.
//               A block integrates each control ONCE for its plane, stages
//               the result in shared memory, and its threads then only
//               replay the position increments (so the probe cells and
//               envelope tests round exactly as the reference does) and
//               gather the 64 corners.  EXACT=true keeps the reference's
//               weight products and summation order (bit-identical to the
//               CPU restatement); EXACT=false lets the compiler fuse the
//               interpolation into FMAs.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "pg_device.cuh"
#include "pg_kernels.h"

namespace pg {

// 16-bit storage rounds to nearest.  A step of 0.03-0.05 s is only a few
// FP16 ulps at 16-32 s, so any directed rounding accumulates along a route
// of hundreds of steps; round-to-nearest keeps the error zero-mean, and the
// FP32 polish that follows a 16-bit solve (plain value iteration, V <- T V,
// see KParams::relax) removes it.
template <> struct Conv<__half> {
    static __device__ __forceinline__ float ld(const __half* p) { return __half2float(__ldg(p)); }
    static __device__ __forceinline__ float val(__half v) { return __half2float(v); }
    template <typename T> static __device__ __forceinline__ __half st(T v) {
        return __float2half_rn((float)v);
    }
};
template <> struct Conv<__nv_bfloat16> {
    static __device__ __forceinline__ float ld(const __nv_bfloat16* p) {
        return __bfloat162float(__ldg(p));
    }
    static __device__ __forceinline__ float val(__nv_bfloat16 v) { return __bfloat162float(v); }
    template <typename T> static __device__ __forceinline__ __nv_bfloat16 st(T v) {
        return __float2bfloat16_rn((float)v);
    }
};
// Q16: V = u * 2^-11 s, u rounded to nearest and saturated to [0, 65535]
// (0 .. 32 s, a uniform 0.49 ms quantum; the conversions are exact scalings).
template <> struct Conv<Q16> {
    static __device__ __forceinline__ float ld(const Q16* p) {
        return (float)__ldg(&p->u) * kQ16Step;
    }
    static __device__ __forceinline__ float val(Q16 v) { return (float)v.u * kQ16Step; }
    template <typename T> static __device__ __forceinline__ Q16 st(T v) {
        float f = rintf((float)v * kQ16Scale);
        f = f >= 0.0f ? fminf(f, 65535.0f) : (f < 0.0f ? 0.0f : 65535.0f);
        Q16 q;
        q.u = (uint16_t)f;
        return q;
    }
};

// ---------------------------------------------------------------------------
// small utilities
// ---------------------------------------------------------------------------
__device__ __forceinline__ Layout make_layout(const KParams& kp) {
    Layout L;
#pragma unroll
    for (int k = 0; k < 6; ++k) L.n[k] = kp.g.n[k];
    L.P = kp.P;
    L.nplanes = kp.nplanes;
    return L;
}

// Deterministic block reduction of (sum, max) into partial slot `slot`.
__device__ __forceinline__ void block_partial_at(double s, double m, double* part_sum,
                                                 double* part_max, int64_t slot) {
    __shared__ double ws[32], wm[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { ws[wid] = s; wm[wid] = m; }
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        s = lane < nw ? ws[lane] : 0.0;
        m = lane < nw ? wm[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_down_sync(0xffffffffu, s, o);
            m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
        }
        if (lane == 0) { part_sum[slot] = s; part_max[slot] = m; }
    }
}

// ... into per-block partials.
__device__ __forceinline__ void block_partial(double s, double m, double* part_sum,
                                              double* part_max) {
    block_partial_at(s, m, part_sum, part_max, blockIdx.x);
}

// One block sums the partials in a fixed order: thread t takes t, t+1024, ...
__global__ void k_reduce_parts(const double* part_sum, const double* part_max, int64_t n,
                               double* out) {
    __shared__ double ss[1024], sm[1024];
    double s = 0.0, m = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        s += part_sum[i];
        m = fmax(m, part_max[i]);
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
    if (threadIdx.x == 0) { out[0] = ss[0]; out[1] = sm[0]; }
}

template <typename S>
__global__ void k_fill(S* V, int64_t n, float v) {
    const S sv = Conv<S>::st(v);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        V[i] = sv;
}

// V[dev(tidx)] = 0 for every seed (Run.jl:1438, 1464).  tidx is row-major.
template <typename S>
__global__ void k_seed(S* V, const int64_t* tidx, int64_t nt, KParams kp) {
    const Layout L = make_layout(kp);
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nt;
         t += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = tidx[t];
        int32_t i[6];
        for (int k = 5; k >= 1; --k) { i[k] = (int32_t)(r % L.n[k]); r /= L.n[k]; }
        i[0] = (int32_t)r;
        V[L.dev(i[0], i[1], i[2], i[3], i[4], i[5])] = Conv<S>::st(0.0f);
    }
}

// Row-major float <-> device layout.
template <typename S>
__global__ void k_to_rowmajor(const S* V, float* out, KParams kp) {
    const Layout L = make_layout(kp);
    for (int64_t r0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r0 < kp.ncells;
         r0 += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = r0;
        int32_t i[6];
        for (int k = 5; k >= 1; --k) { i[k] = (int32_t)(r % L.n[k]); r /= L.n[k]; }
        i[0] = (int32_t)r;
        out[r0] = (float)Conv<S>::ld(V + L.dev(i[0], i[1], i[2], i[3], i[4], i[5]));
    }
}

template <typename S>
__global__ void k_from_rowmajor(const float* in, S* V, KParams kp) {
    const Layout L = make_layout(kp);
    for (int64_t r0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r0 < kp.ncells;
         r0 += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = r0;
        int32_t i[6];
        for (int k = 5; k >= 1; --k) { i[k] = (int32_t)(r % L.n[k]); r /= L.n[k]; }
        i[0] = (int32_t)r;
        V[L.dev(i[0], i[1], i[2], i[3], i[4], i[5])] = Conv<S>::st(in[r0]);
    }
}

// Convert between storages of the same layout (16-bit phase -> FP32 polish).
template <typename SI, typename SO>
__global__ void k_convert(const SI* in, SO* out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = Conv<SO>::st(Conv<SI>::ld(in + i));
}

// ---------------------------------------------------------------------------
// The reference's backup, one cell per thread
// ---------------------------------------------------------------------------

// V as cell_update reads it: plain, or through EscapeView
// (PeregrineSolver.jl:807-824).
template <typename T, typename S> struct VView {
    const S* V;
    const uint8_t* occ;
    Layout L;
    T cap;
    bool esc;
    bool ignore;
    __device__ __forceinline__ T get(int32_t j1, int32_t j2, int32_t j3, int32_t j4, int32_t j5,
                                     int32_t j6) const {
        if (esc && !ignore && occ[L.occ(j1, j2, j3)]) return cap;
        T v = (T)Conv<S>::ld(V + L.dev(j1, j2, j3, j4, j5, j6));
        if (!esc) return v;
        return v < (T)0 ? -v : (v < cap ? (T)0 : cap);
    }
};

// interp (PeregrineSolver.jl:399-466)
template <typename T, typename S>
__device__ T interp_ml(const VView<T, S>& vv, const GridT<T>& g, const State6<T>& s, bool nearest,
                       T cap, bool vclamp) {
    typedef Ar<T> R;
    T f1 = R::div(R::sub(s.x, g.lo[0]), g.step[0]);
    T f2 = R::div(R::sub(s.y, g.lo[1]), g.step[1]);
    T n3 = (T)g.n[2];
    T f3 = R::div(R::sub(s.h, g.lo[2]), g.step[2]);
    f3 = R::sub(f3, R::mul(R::floor_(R::div(f3, n3)), n3));
    T f4 = R::div(R::sub(s.vx, g.lo[3]), g.step[3]);
    T f5 = R::div(R::sub(s.vy, g.lo[4]), g.step[4]);
    T f6 = R::div(R::sub(s.w, g.lo[5]), g.step[5]);
    if (!(finite_(f1) && finite_(f2) && finite_(f3) && finite_(f4) && finite_(f5) && finite_(f6)))
        return cap;
    if (f1 < (T)0 || f1 > (T)(g.n[0] - 1)) return cap;
    if (f2 < (T)0 || f2 > (T)(g.n[1] - 1)) return cap;
    if (vclamp) {
        f4 = jclamp(f4, (T)0, (T)(g.n[3] - 1));
        f5 = jclamp(f5, (T)0, (T)(g.n[4] - 1));
        f6 = jclamp(f6, (T)0, (T)(g.n[5] - 1));
    } else {
        if (f4 < (T)0 || f4 > (T)(g.n[3] - 1)) return cap;
        if (f5 < (T)0 || f5 > (T)(g.n[4] - 1)) return cap;
        if (f6 < (T)0 || f6 > (T)(g.n[5] - 1)) return cap;
    }
    if (nearest) {
        int32_t i1 = (int32_t)R::rint_(f1), i2 = (int32_t)R::rint_(f2);
        int32_t i3 = ((int32_t)R::rint_(f3)) % g.n[2];
        int32_t i4 = (int32_t)R::rint_(f4), i5 = (int32_t)R::rint_(f5);
        int32_t i6 = (int32_t)R::rint_(f6);
        return vv.get(i1, i2, i3, i4, i5, i6);
    }
    T b[6] = {R::floor_(f1), R::floor_(f2), R::floor_(f3), R::floor_(f4), R::floor_(f5),
              R::floor_(f6)};
    T t[6] = {R::sub(f1, b[0]), R::sub(f2, b[1]), R::sub(f3, b[2]),
              R::sub(f4, b[3]), R::sub(f5, b[4]), R::sub(f6, b[5])};
    int32_t i[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) i[k] = (int32_t)b[k];
    T acc = (T)0;
    for (int d = 0; d < 64; ++d) {
        int c[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) c[k] = (d >> k) & 1;
        T wgt = c[0] ? t[0] : R::sub((T)1, t[0]);
#pragma unroll
        for (int k = 1; k < 6; ++k) wgt = R::mul(wgt, c[k] ? t[k] : R::sub((T)1, t[k]));
        if (wgt == (T)0) continue;
        int32_t j1 = min(i[0] + c[0], g.n[0] - 1);
        int32_t j2 = min(i[1] + c[1], g.n[1] - 1);
        int32_t j3 = (i[2] + c[2]) % g.n[2];
        int32_t j4 = min(i[3] + c[3], g.n[3] - 1);
        int32_t j5 = min(i[4] + c[4], g.n[4] - 1);
        int32_t j6 = min(i[5] + c[5], g.n[5] - 1);
        acc = R::add(acc, R::mul(wgt, vv.get(j1, j2, j3, j4, j5, j6)));
    }
    return jmin(acc, cap);
}

template <typename T>
__device__ __forceinline__ void cmpx(T& ta, int32_t& ka, T& tb, int32_t& kb) {
    if (!(ta >= tb)) {
        T t = ta; ta = tb; tb = t;
        int32_t k = ka; ka = kb; kb = k;
    }
}

// interp_kuhn (PeregrineSolver.jl:571-665): the value, and, when grad is
// given, the simplex gradient along each axis (the self-test probe reads it)
template <typename T, typename S>
__device__ T interp_kuhn(const VView<T, S>& vv, const GridT<T>& g, const State6<T>& s, T cap,
                         bool vclamp, T* grad = nullptr) {
    typedef Ar<T> R;
    T f1 = R::div(R::sub(s.x, g.lo[0]), g.step[0]);
    T f2 = R::div(R::sub(s.y, g.lo[1]), g.step[1]);
    T n3 = (T)g.n[2];
    T f3 = R::div(R::sub(s.h, g.lo[2]), g.step[2]);
    f3 = R::sub(f3, R::mul(R::floor_(R::div(f3, n3)), n3));
    T f4 = R::div(R::sub(s.vx, g.lo[3]), g.step[3]);
    T f5 = R::div(R::sub(s.vy, g.lo[4]), g.step[4]);
    T f6 = R::div(R::sub(s.w, g.lo[5]), g.step[5]);
    if (!(finite_(f1) && finite_(f2) && finite_(f3) && finite_(f4) && finite_(f5) && finite_(f6)))
        return cap;
    if (f1 < (T)0 || f1 > (T)(g.n[0] - 1)) return cap;
    if (f2 < (T)0 || f2 > (T)(g.n[1] - 1)) return cap;
    if (vclamp) {
        f4 = jclamp(f4, (T)0, (T)(g.n[3] - 1));
        f5 = jclamp(f5, (T)0, (T)(g.n[4] - 1));
        f6 = jclamp(f6, (T)0, (T)(g.n[5] - 1));
    } else {
        if (f4 < (T)0 || f4 > (T)(g.n[3] - 1)) return cap;
        if (f5 < (T)0 || f5 > (T)(g.n[4] - 1)) return cap;
        if (f6 < (T)0 || f6 > (T)(g.n[5] - 1)) return cap;
    }
    T b1 = R::floor_(f1), b2 = R::floor_(f2), b3 = R::floor_(f3);
    T b4 = R::floor_(f4), b5 = R::floor_(f5), b6 = R::floor_(f6);
    int32_t idx[6] = {(int32_t)b1, (int32_t)b2, ((int32_t)b3) % g.n[2],
                      (int32_t)b4, (int32_t)b5, (int32_t)b6};
    T t0 = R::sub(f1, b1), t1 = R::sub(f2, b2), t2 = R::sub(f3, b3);
    T t3 = R::sub(f4, b4), t4 = R::sub(f5, b5), t5 = R::sub(f6, b6);
    int32_t k0 = 1, k1 = 2, k2 = 3, k3 = 4, k4 = 5, k5 = 6;
    cmpx(t0, k0, t5, k5);
    cmpx(t1, k1, t3, k3);
    cmpx(t2, k2, t4, k4);
    cmpx(t1, k1, t2, k2);
    cmpx(t3, k3, t4, k4);
    cmpx(t0, k0, t3, k3);
    cmpx(t2, k2, t5, k5);
    cmpx(t0, k0, t1, k1);
    cmpx(t2, k2, t3, k3);
    cmpx(t4, k4, t5, k5);
    cmpx(t1, k1, t2, k2);
    cmpx(t3, k3, t4, k4);
    const T ts[6] = {t0, t1, t2, t3, t4, t5};
    const int32_t ks[6] = {k0, k1, k2, k3, k4, k5};
    T v0 = vv.get(idx[0], idx[1], idx[2], idx[3], idx[4], idx[5]);
    T acc = R::mul(R::sub((T)1, ts[0]), v0);
    T prev = v0;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const int32_t k = ks[q];
        if (k == 3) idx[2] = (idx[2] + 1) % g.n[2];
        else idx[k - 1] = min(idx[k - 1] + 1, g.n[k - 1] - 1);
        T v = vv.get(idx[0], idx[1], idx[2], idx[3], idx[4], idx[5]);
        T wq = q < 5 ? R::sub(ts[q], ts[q + 1]) : ts[5];
        acc = R::add(acc, R::mul(wq, v));
        // the edge walked along axis k: its difference over the axis step
        if (grad) grad[k - 1] = R::div(R::sub(v, prev), g.step[k - 1]);
        prev = v;
    }
    return jmin(acc, cap);
}

template <typename T, typename S>
__device__ __forceinline__ T value_at(const VView<T, S>& vv, const GridT<T>& g, const State6<T>& s,
                                      const pg_params& p) {
    if (p.simplex) return interp_kuhn(vv, g, s, (T)p.cap, p.vclamp != 0);
    return interp_ml(vv, g, s, p.nearest != 0, (T)p.cap, p.vclamp != 0);
}

// lookahead (PeregrineSolver.jl:1100-1153)
template <typename T, typename S>
__device__ T lookahead(const VView<T, S>& vv, const uint8_t* occ, bool occ_ignore,
                       const GridT<T>& g, const ModelT<T>& m, const Layout& L,
                       const State6<T>& s0, T u1, T u2, T u3, T tau, int32_t nsub,
                       const pg_params& p) {
    typedef Ar<T> R;
    const T cap = (T)p.cap;
    State6<T> ns = s0;
    if (!integrate(m, ns, u1, u2, u3, tau, nsub, p.rk2 != 0, (T*)nullptr, (T*)nullptr))
        return cap;  // NANSTATE: every difference below is non-finite
    T dx = R::sub(ns.x, s0.x), dy = R::sub(ns.y, s0.y), dh = R::sub(ns.h, s0.h);
    if (!(finite_(dx) && finite_(dy) && finite_(dh) && finite_(ns.vx) && finite_(ns.vy) &&
          finite_(ns.w)))
        return cap;
    int32_t nchk = p.checks;
    if (p.adaptive_checks) {
        T cells_pos = R::div(R::sqrt_(R::add(R::mul(dx, dx), R::mul(dy, dy))),
                             R::mul((T)0.5f, jmin(g.step[0], g.step[1])));
        T cells_rot = R::div(R::abs_(dh), R::mul((T)0.5f, g.step[2]));
        T cells = jmin(jmax(cells_pos, cells_rot), (T)1.0e4f);
        int32_t need = (int32_t)cells + 1;
        nchk = max(p.checks, min(need, 24));
    }
    const T n3f = (T)g.n[2];
    for (int32_t sc = 1; sc <= nchk; ++sc) {
        T a = R::div((T)sc, (T)nchk);
        T px = R::add(s0.x, R::mul(dx, a));
        T py = R::add(s0.y, R::mul(dy, a));
        T ph = R::add(s0.h, R::mul(dh, a));
        T gx = R::div(R::sub(px, g.lo[0]), g.step[0]);
        T gy = R::div(R::sub(py, g.lo[1]), g.step[1]);
        if (gx < (T)0 || gy < (T)0 || gx > (T)(g.n[0] - 1) || gy > (T)(g.n[1] - 1)) return cap;
        T gh = R::div(R::sub(ph, g.lo[2]), g.step[2]);
        gh = R::sub(gh, R::mul(R::floor_(R::div(gh, n3f)), n3f));
        int32_t ci = (int32_t)R::rint_(gx), cj = (int32_t)R::rint_(gy);
        int32_t ck = ((int32_t)R::rint_(gh)) % g.n[2];
        if (!occ_ignore && occ[L.occ(ci, cj, ck)]) return cap;
    }
    T snh, cnh;
    R::sincos_(ns.h, &snh, &cnh);
    State6<T> q = ns;
    q.vx = R::sub(R::mul(cnh, ns.vx), R::mul(snh, ns.vy));
    q.vy = R::add(R::mul(snh, ns.vx), R::mul(cnh, ns.vy));
    T nv = value_at(vv, g, q, p);
    return jmin(R::add(tau, nv), cap);
}

template <typename T> __device__ __forceinline__ int8_t qpol(T v) {
    typedef Ar<T> R;
    return (int8_t)(int32_t)R::rint_(R::mul(jclamp(v, (T)-1, (T)1), (T)127.0f));
}

// cell_update (PeregrineSolver.jl:1205-1344).  Returns best; b[] the command.
template <typename T, typename S>
__device__ T cell_update(const int32_t* i, const VView<T, S>& vv, const uint8_t* occ,
                         const int8_t* pol, int64_t pidx, const GridT<T>& g, const ModelT<T>& m,
                         const Layout& L, const float* ctl, int32_t nctl, const pg_params& p,
                         int32_t phase, bool esc, bool blocked, T* b) {
    typedef Ar<T> R;
    b[0] = b[1] = b[2] = (T)0;
    const bool oign = esc && blocked;
    State6<T> s;
    s.x = axisvalue(g, 0, i[0]);
    s.y = axisvalue(g, 1, i[1]);
    s.h = axisvalue(g, 2, i[2]);
    T vfx = axisvalue(g, 3, i[3]);
    T vfy = axisvalue(g, 4, i[4]);
    s.w = axisvalue(g, 5, i[5]);
    T sh0, ch0;
    R::sincos_(s.h, &sh0, &ch0);
    s.vx = R::add(R::mul(ch0, vfx), R::mul(sh0, vfy));
    s.vy = R::add(R::mul(-sh0, vfx), R::mul(ch0, vfy));
    T tau0 = cfl_tau(g, m, vfx, vfy, s.w, p);
    int32_t ns0 = substeps_for(tau0, p);

    T best = lookahead(vv, occ, oign, g, m, L, s, (T)0, (T)0, (T)0, tau0, ns0, p);
    T b1 = 0, b2 = 0, b3 = 0;
    if (pol != nullptr && !esc) {
        const T k127 = (T)(1.0f / 127.0f);
        T q1 = R::mul((T)pol[3 * pidx], k127);
        T q2 = R::mul((T)pol[3 * pidx + 1], k127);
        T q3 = R::mul((T)pol[3 * pidx + 2], k127);
        if (R::add(R::add(R::abs_(q1), R::abs_(q2)), R::abs_(q3)) > (T)1.0e-6f) {
            T c = lookahead(vv, occ, oign, g, m, L, s, q1, q2, q3, tau0, ns0, p);
            if (c < best) { best = c; b1 = q1; b2 = q2; b3 = q3; }
        }
    }
    const int32_t nnc = max(nctl - 1, 1);
    const int32_t span = p.ncoarse <= 0 ? nnc : min(p.ncoarse, nnc);
    int32_t off = p.ncoarse <= 0 ? 0 : (int32_t)(((int64_t)phase * span) % nnc);
    if (off < 0) off += nnc;
    for (int32_t j = 0; j < span; ++j) {
        int32_t k = (int32_t)(((int64_t)off + j) % nnc) + 1;
        T u1 = (T)ctl[k], u2 = (T)ctl[k + nctl], u3 = (T)ctl[k + 2 * nctl];
        T c = lookahead(vv, occ, oign, g, m, L, s, u1, u2, u3, tau0, ns0, p);
        if (c < best) { best = c; b1 = u1; b2 = u2; b3 = u3; }
    }
    T delta = (T)p.delta0;
    for (int32_t r = 0; r < p.rounds; ++r) {
        for (int32_t d = 1; d <= 6; ++d) {
            T sdl = (d % 2 == 0) ? -delta : delta;
            T e1 = d <= 2 ? sdl : (T)0;
            T e2 = (d == 3 || d == 4) ? sdl : (T)0;
            T e3 = d >= 5 ? sdl : (T)0;
            T a1 = R::add(b1, e1), a2 = R::add(b2, e2), a3 = R::add(b3, e3);
            T sm = R::add(R::add(R::abs_(a1), R::abs_(a2)), R::abs_(a3));
            T c1, c2, c3;
            if (sm < (T)1.0e-6f) { c1 = c2 = c3 = (T)0; }
            else {
                T rr = R::div((T)1, sm);
                c1 = R::mul(a1, rr); c2 = R::mul(a2, rr); c3 = R::mul(a3, rr);
            }
            if (R::add(R::add(R::abs_(c1), R::abs_(c2)), R::abs_(c3)) < (T)1.0e-6f) continue;
            T c = lookahead(vv, occ, oign, g, m, L, s, c1, c2, c3, tau0, ns0, p);
            if (c < best) { best = c; b1 = c1; b2 = c2; b3 = c3; }
        }
        delta = R::mul(delta, (T)0.5f);
    }
    if (p.ntau > 1) {
        T tau = R::mul(tau0, (T)0.5f);
        for (int32_t k = 1; k <= p.ntau; ++k) {
            if (k != 2) {
                T t = jmin(jmax(tau, (T)p.tau_min), (T)p.tau_max);
                T c = lookahead(vv, occ, oign, g, m, L, s, b1, b2, b3, t, substeps_for(t, p), p);
                if (c < best) best = c;
            }
            tau = R::mul(tau, (T)p.tau_ratio);
        }
        if (p.cfl > 0.0f) {
            T t = jmin(jmax((T)p.dt, (T)p.tau_min), (T)p.tau_max);
            T c = lookahead(vv, occ, oign, g, m, L, s, b1, b2, b3, t, substeps_for(t, p), p);
            if (c < best) best = c;
        }
    }
    b[0] = b1; b[1] = b2; b[2] = b3;
    return best;
}

__device__ __forceinline__ int16_t ctl_index(const float* ctl, int32_t nctl, float u1, float u2,
                                             float u3) {
    for (int32_t k = 0; k < nctl; ++k)
        if (ctl[k] == u1 && ctl[k + nctl] == u2 && ctl[k + 2 * nctl] == u3) return (int16_t)k;
    return (int16_t)-1;
}

// Sweep (ESC=false): gpu_sweep_kernel! (Gpu.jl:5-24) as a Jacobi update.
// Escape (ESC=true): gpu_escape_kernel! (Gpu.jl:51-67) as a Jacobi update.
template <typename S, typename T, bool ESC>
__global__ void __launch_bounds__(kCellThreads)
    k_cellform(const S* __restrict__ Vin, S* __restrict__ Vout, const uint8_t* __restrict__ occ,
               int8_t* pol, KParams kp, const float* __restrict__ ctl, double* part_sum,
               double* part_max, int16_t* argmin) {
    typedef Ar<T> R;
    const Layout L = make_layout(kp);
    GridT<T> g;
    load_grid(g, kp.g);
    ModelT<T> m;
    load_model(m, kp.m);
    const T cap = (T)kp.p.cap;
    double dsum = 0.0, dmax = 0.0;
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx < kp.ncells) {
        int64_t pl = idx / L.P;
        int32_t r = (int32_t)(idx - pl * L.P);
        int32_t i[6];
        i[0] = r / L.n[1];
        i[1] = r - i[0] * L.n[1];
        i[5] = (int32_t)(pl % L.n[5]); pl /= L.n[5];
        i[4] = (int32_t)(pl % L.n[4]); pl /= L.n[4];
        i[3] = (int32_t)(pl % L.n[3]); pl /= L.n[3];
        i[2] = (int32_t)pl;
        const bool blocked = occ[L.occ(i[0], i[1], i[2])] != 0;
        const T old = (T)Conv<S>::ld(Vin + idx);
        S outv = Vin[idx];
        VView<T, S> vv{Vin, occ, L, cap, ESC, blocked};
        if (!ESC) {
            if (blocked) {
                if (argmin) argmin[L.rowmajor(i[0], i[1], i[2], i[3], i[4], i[5])] = -1;
            } else {
                T b[3];
                T c = cell_update(i, vv, occ, pol, idx, g, m, L, ctl, kp.nctl, kp.p, kp.phase,
                                  false, false, b);
                if (argmin)
                    argmin[L.rowmajor(i[0], i[1], i[2], i[3], i[4], i[5])] =
                        ctl_index(ctl, kp.nctl, (float)b[0], (float)b[1], (float)b[2]);
                if (c < old) {
                    S nv = Conv<S>::template st<T>(c);
                    T nvT = (T)Conv<S>::val(nv);
                    outv = nv;
                    if (pol) {
                        pol[3 * idx] = qpol(b[0]);
                        pol[3 * idx + 1] = qpol(b[1]);
                        pol[3 * idx + 2] = qpol(b[2]);
                    }
                    double d = (double)old - (double)nvT;
                    dsum = d;
                    dmax = d;
                }
            }
        } else {
            // is_terminal / escape_of (PeregrineSolver.jl:860-866)
            if (!(old >= (T)0 && old < cap)) {
                const T e_old = old < (T)0 ? -old : cap;
                T b[3];
                T c = cell_update(i, vv, occ, (const int8_t*)nullptr, idx, g, m, L, ctl, kp.nctl,
                                  kp.p, kp.phase, true, blocked, b);
                if (c < e_old) {
                    outv = Conv<S>::template st<T>(-c);
                    double d = (double)e_old - (double)c;
                    dsum = d;
                    dmax = d;
                }
            }
        }
        Vout[idx] = outv;
        (void)R::add;
    }
    block_partial(dsum, dmax, part_sum, part_max);
}

#include "pg_plane.cuh"
#include "pg_stencil.cuh"
#include "pg_stencil_u.cuh"
#include "pg_stencil_b.cuh"
#include "pg_stencil_r.cuh"
#include "pg_stencil_d.cuh"
#include "pg_adjoint.cuh"

// ---------------------------------------------------------------------------
// Encoding (encode_into!, Pipeline.jl:698-780), from the device layout into
// a row-major range.
// ---------------------------------------------------------------------------
template <typename S>
__global__ void k_encode(const S* V, KParams kp, int32_t dtype, double scale, double escape_scale,
                         int64_t lo, int64_t n, uint8_t* out, unsigned long long* counts) {
    const Layout L = make_layout(kp);
    const float cap = kp.p.cap;
    const uint32_t sentinel = dtype == PG_DTYPE_U8 ? 0xffu : 0xffffu;
    const uint32_t base = dtype == PG_DTYPE_U8 ? 0xe0u : (dtype == PG_DTYPE_U16 ? 0xfc00u : 0u);
    const int64_t codes = base == 0 ? 0 : (int64_t)sentinel - (int64_t)base;
    const bool hasband = escape_scale > 0.0 && base != 0;
    const uint32_t ebase = hasband ? base : sentinel;
    const uint32_t ecodes = (uint32_t)(codes > 1 ? codes : 1);
    const double einv = escape_scale > 0.0 ? 1.0 / escape_scale : 0.0;
    unsigned long long nr = 0, ne = 0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = lo + t;
        int32_t i[6];
        for (int k = 5; k >= 1; --k) { i[k] = (int32_t)(r % L.n[k]); r /= L.n[k]; }
        i[0] = (int32_t)r;
        const float v = (float)Conv<S>::ld(V + L.dev(i[0], i[1], i[2], i[3], i[4], i[5]));
        const bool isesc = v < 0.0f && isfinite(v);
        const bool unre = v >= cap || isinf(v) || isnan(v);
        if (dtype == PG_DTYPE_F32 || dtype == PG_DTYPE_F16) {
            const bool u = !isesc && unre;
            nr += (!isesc && !u);
            ne += isesc;
            if (dtype == PG_DTYPE_F32) {
                const uint32_t bits = u ? 0x7fc00000u : __float_as_uint(v);
                reinterpret_cast<uint32_t*>(out)[t] = bits;
            } else {
                const uint16_t hb = u ? (uint16_t)0x7e00u : __half_as_ushort(__float2half_rn(v));
                reinterpret_cast<uint16_t*>(out)[t] = hb;
            }
            continue;
        }
        uint32_t code;
        if (isesc) {
            ++ne;
            const double e = -(double)v;
            const double q = __dsqrt_rn(__dmul_rn(e > 0.0 ? e : 0.0, einv));
            const uint32_t rq = (uint32_t)rint(q);
            code = ebase + (rq < ecodes - 1u ? rq : ecodes - 1u);
        } else if (unre) {
            code = sentinel;
        } else {
            ++nr;
            const uint32_t rr = (uint32_t)rint(__ddiv_rn((double)v, scale));
            code = rr >= ebase ? sentinel : rr;
        }
        if (dtype == PG_DTYPE_U8) out[t] = (uint8_t)code;
        else reinterpret_cast<uint16_t*>(out)[t] = (uint16_t)code;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nr += __shfl_down_sync(0xffffffffu, nr, o);
        ne += __shfl_down_sync(0xffffffffu, ne, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&counts[0], nr);
        atomicAdd(&counts[1], ne);
    }
}

// ---------------------------------------------------------------------------
// host-side launchers
// ---------------------------------------------------------------------------
// Kernel attributes (the dynamic shared-memory ceiling) are per device; each
// launch site sets them once per device it runs on.
static inline uint64_t device_bit() {
    int d = 0;
    cudaGetDevice(&d);
    return d >= 0 && d < 64 ? (1ull << d) : 0ull;
}

static inline int grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b > (int64_t)148 * 64) b = (int64_t)148 * 64;
    return (int)(b < 1 ? 1 : b);
}

template <typename S>
static cudaError_t fill_seed_t(void* V, const KParams& kp, const int64_t* tidx_dev, int64_t nt,
                               cudaStream_t st) {
    k_fill<S><<<grid_for(kp.ncells, 256), 256, 0, st>>>((S*)V, kp.ncells, kp.p.cap);
    if (nt > 0) k_seed<S><<<grid_for(nt, 256), 256, 0, st>>>((S*)V, tidx_dev, nt, kp);
    return cudaGetLastError();
}

cudaError_t launch_fill_seed(int storage, void* V, const KParams& kp, const int64_t* tidx_dev,
                             int64_t nt, cudaStream_t st) {
    switch (storage) {
        case PG_STORE_F32: return fill_seed_t<float>(V, kp, tidx_dev, nt, st);
        case PG_STORE_F16: return fill_seed_t<__half>(V, kp, tidx_dev, nt, st);
        case PG_STORE_BF16: return fill_seed_t<__nv_bfloat16>(V, kp, tidx_dev, nt, st);
        case PG_STORE_Q16: return fill_seed_t<Q16>(V, kp, tidx_dev, nt, st);
        case PG_STORE_F64: return fill_seed_t<double>(V, kp, tidx_dev, nt, st);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_seed_only(int storage, void* V, const KParams& kp, const int64_t* tidx_dev,
                             int64_t nt, cudaStream_t st) {
    if (nt <= 0) return cudaSuccess;
    switch (storage) {
        case PG_STORE_F32: k_seed<float><<<grid_for(nt, 256), 256, 0, st>>>((float*)V, tidx_dev, nt, kp); break;
        case PG_STORE_F16: k_seed<__half><<<grid_for(nt, 256), 256, 0, st>>>((__half*)V, tidx_dev, nt, kp); break;
        case PG_STORE_BF16: k_seed<__nv_bfloat16><<<grid_for(nt, 256), 256, 0, st>>>((__nv_bfloat16*)V, tidx_dev, nt, kp); break;
        case PG_STORE_Q16: k_seed<Q16><<<grid_for(nt, 256), 256, 0, st>>>((Q16*)V, tidx_dev, nt, kp); break;
        case PG_STORE_F64: k_seed<double><<<grid_for(nt, 256), 256, 0, st>>>((double*)V, tidx_dev, nt, kp); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_to_rowmajor(int storage, const void* V, float* out, const KParams& kp,
                               cudaStream_t st) {
    const int b = grid_for(kp.ncells, 256);
    switch (storage) {
        case PG_STORE_F32: k_to_rowmajor<float><<<b, 256, 0, st>>>((const float*)V, out, kp); break;
        case PG_STORE_F16: k_to_rowmajor<__half><<<b, 256, 0, st>>>((const __half*)V, out, kp); break;
        case PG_STORE_BF16: k_to_rowmajor<__nv_bfloat16><<<b, 256, 0, st>>>((const __nv_bfloat16*)V, out, kp); break;
        case PG_STORE_Q16: k_to_rowmajor<Q16><<<b, 256, 0, st>>>((const Q16*)V, out, kp); break;
        case PG_STORE_F64: k_to_rowmajor<double><<<b, 256, 0, st>>>((const double*)V, out, kp); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_from_rowmajor(int storage, const float* in, void* V, const KParams& kp,
                                 cudaStream_t st) {
    const int b = grid_for(kp.ncells, 256);
    switch (storage) {
        case PG_STORE_F32: k_from_rowmajor<float><<<b, 256, 0, st>>>(in, (float*)V, kp); break;
        case PG_STORE_F16: k_from_rowmajor<__half><<<b, 256, 0, st>>>(in, (__half*)V, kp); break;
        case PG_STORE_BF16: k_from_rowmajor<__nv_bfloat16><<<b, 256, 0, st>>>(in, (__nv_bfloat16*)V, kp); break;
        case PG_STORE_Q16: k_from_rowmajor<Q16><<<b, 256, 0, st>>>(in, (Q16*)V, kp); break;
        case PG_STORE_F64: k_from_rowmajor<double><<<b, 256, 0, st>>>(in, (double*)V, kp); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_convert_to_f32(int storage, const void* in, float* out, int64_t n,
                                  cudaStream_t st) {
    const int b = grid_for(n, 256);
    switch (storage) {
        case PG_STORE_F16: k_convert<__half, float><<<b, 256, 0, st>>>((const __half*)in, out, n); break;
        case PG_STORE_BF16: k_convert<__nv_bfloat16, float><<<b, 256, 0, st>>>((const __nv_bfloat16*)in, out, n); break;
        case PG_STORE_Q16: k_convert<Q16, float><<<b, 256, 0, st>>>((const Q16*)in, out, n); break;
        case PG_STORE_F32: return cudaMemcpyAsync(out, in, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename S, typename T, bool ESC>
static cudaError_t cellform_t(const void* Vin, void* Vout, const uint8_t* occ, int8_t* pol,
                              const KParams& kp, const float* ctl, const SweepBufs& sb,
                              int16_t* argmin, cudaStream_t st, int64_t* launches) {
    const int64_t blocks = (kp.ncells + kCellThreads - 1) / kCellThreads;
    if (blocks > sb.nparts) return cudaErrorInvalidValue;
    k_cellform<S, T, ESC><<<(unsigned)blocks, kCellThreads, 0, st>>>(
        (const S*)Vin, (S*)Vout, occ, pol, kp, ctl, sb.part_sum, sb.part_max, argmin);
    k_reduce_parts<<<1, 1024, 0, st>>>(sb.part_sum, sb.part_max, blocks, sb.out);
    *launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_cellform(int storage, bool esc, const void* Vin, void* Vout, const uint8_t* occ,
                            int8_t* pol, const KParams& kp, const float* ctl, const SweepBufs& sb,
                            int16_t* argmin, cudaStream_t st, int64_t* launches) {
#define PG_CF(S, T)                                                                            \
    return esc ? cellform_t<S, T, true>(Vin, Vout, occ, pol, kp, ctl, sb, argmin, st, launches)   \
               : cellform_t<S, T, false>(Vin, Vout, occ, pol, kp, ctl, sb, argmin, st, launches)
    switch (storage) {
        case PG_STORE_F32: PG_CF(float, float);
        case PG_STORE_F16: PG_CF(__half, float);
        case PG_STORE_BF16: PG_CF(__nv_bfloat16, float);
        case PG_STORE_F64: PG_CF(double, double);
    }
#undef PG_CF
    return cudaErrorInvalidValue;
}

int64_t cellform_blocks(int64_t ncells) { return (ncells + kCellThreads - 1) / kCellThreads; }
int64_t stencil_blocks(const KParams& kp) { return kp.nplanes * kp.tiles_x; }

size_t stencil_smem(int storage, bool exact, const KParams& kp) {
    const bool dbl = storage == PG_STORE_F64;
    if (dbl) return exact ? stencil_smem_bytes<double, true>(kp.nctl, kp.nsub, kp.nchk)
                          : stencil_smem_bytes<double, false>(kp.nctl, kp.nsub, kp.nchk);
    return exact ? stencil_smem_bytes<float, true>(kp.nctl, kp.nsub, kp.nchk)
                 : stencil_smem_bytes<float, false>(kp.nctl, kp.nsub, kp.nchk);
}

template <typename S, typename T, bool EXACT, int NSUB>
static cudaError_t stencil_t(const void* Vin, void* Vout, const uint8_t* occ, const KParams& kp,
                             const float* ctl, const int32_t* order, const SweepBufs& sb,
                             int16_t* argmin, cudaStream_t st, int64_t* launches) {
    const int64_t blocks = stencil_blocks(kp);
    if (blocks > sb.nparts || blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    const size_t smem = stencil_smem_bytes<T, EXACT>(kp.nctl, kp.nsub, kp.nchk);
    static std::atomic<uint64_t> attr_set{0};
    const uint64_t attr_bit = device_bit();
    if (!(attr_set.load() & attr_bit)) {
        cudaError_t e = cudaFuncSetAttribute(k_stencil<S, T, EXACT, NSUB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return e;
        attr_set.fetch_or(attr_bit);
    }
    k_stencil<S, T, EXACT, NSUB><<<(unsigned)blocks, kp.block, smem, st>>>(
        (const S*)Vin, (S*)Vout, occ, kp, ctl, order, sb.part_sum, sb.part_max, argmin);
    k_reduce_parts<<<1, 1024, 0, st>>>(sb.part_sum, sb.part_max, blocks, sb.out);
    *launches += 2;
    return cudaGetLastError();
}

template <typename S, typename T, bool EXACT>
static cudaError_t stencil_n(const void* Vin, void* Vout, const uint8_t* occ, const KParams& kp,
                             const float* ctl, const int32_t* order, const SweepBufs& sb,
                             int16_t* argmin, cudaStream_t st, int64_t* launches) {
    if (kp.nsub == 5)
        return stencil_t<S, T, EXACT, 5>(Vin, Vout, occ, kp, ctl, order, sb, argmin, st, launches);
    return stencil_t<S, T, EXACT, 0>(Vin, Vout, occ, kp, ctl, order, sb, argmin, st, launches);
}

cudaError_t launch_stencil(int storage, bool exact, const void* Vin, void* Vout, const uint8_t* occ,
                           const KParams& kp, const float* ctl, const int32_t* order,
                           const SweepBufs& sb, int16_t* argmin, cudaStream_t st,
                           int64_t* launches) {
#define PG_ST(S, T)                                                                               \
    return exact ? stencil_n<S, T, true>(Vin, Vout, occ, kp, ctl, order, sb, argmin, st, launches) \
                 : stencil_n<S, T, false>(Vin, Vout, occ, kp, ctl, order, sb, argmin, st, launches)
    switch (storage) {
        case PG_STORE_F32: PG_ST(float, float);
        case PG_STORE_F16: PG_ST(__half, float);
        case PG_STORE_BF16: PG_ST(__nv_bfloat16, float);
        case PG_STORE_F64: PG_ST(double, double);
    }
#undef PG_ST
    return cudaErrorInvalidValue;
}

cudaError_t launch_stencil_prep(const uint8_t* occ, const KParams& kp, const float* ctl,
                                uint32_t* mask, uint32_t* recs, int64_t plane0, int64_t nplanes,
                                cudaStream_t st, int64_t* launches) {
    size_t smem = stencil_prep_smem(kp.nctl, kp.nsub);
    const size_t tab = stencil_prep_tab_smem(kp.nctl, kp.g.n[1]);
    const int coltab = kp.g.n[1] <= 255 && kp.nchk <= 4 && smem + tab <= 200 * 1024;
    if (coltab) smem += tab;
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static std::atomic<uint64_t> attr_set{0};
    const uint64_t attr_bit = device_bit();
    if (!(attr_set.load() & attr_bit)) {
        cudaError_t e = cudaFuncSetAttribute(k_stencil_prep,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return e;
        attr_set.fetch_or(attr_bit);
    }
    if (plane0 < 0 || nplanes < 0 || plane0 + nplanes > kp.nplanes || nplanes > 0x7fffffffLL)
        return cudaErrorInvalidValue;
    if (nplanes == 0) return cudaSuccess;
    k_stencil_prep<<<(unsigned)nplanes, 256, smem, st>>>(occ, kp, ctl, mask, recs, coltab, plane0);
    *launches += 1;
    return cudaGetLastError();
}

// columns per thread of the masked stencil: a multiple of one 16-byte vector
template <typename S> struct UStencilR { static constexpr int R = 4; };
template <> struct UStencilR<__half> { static constexpr int R = 8; };
template <> struct UStencilR<__nv_bfloat16> { static constexpr int R = 8; };

template <typename S, bool ARGMIN>
static cudaError_t stencil_u_t(const void* Vin, void* Vout, const uint8_t* occ,
                               const uint32_t* mask, const uint32_t* recs, const KParams& kp,
                               const int32_t* order, const SweepBufs& sb, int16_t* argmin,
                               cudaStream_t st, int64_t* launches) {
    constexpr int R = UStencilR<S>::R;
    KParams ku = kp;
    ku.tile_x = kp.utile_x;
    ku.tiles_x = kp.utiles_x;
    const int64_t blocks = kp.nplanes * kp.utiles_x;
    if (blocks > sb.nparts || blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    const size_t smem = stencil_u_smem(kp.nctl);
    static std::atomic<uint64_t> attr_set{0};
    const uint64_t attr_bit = device_bit();
    if (!(attr_set.load() & attr_bit)) {
        cudaError_t e = cudaFuncSetAttribute(k_stencil_u<S, kURX, R, ARGMIN>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return e;
        attr_set.fetch_or(attr_bit);
    }
    k_stencil_u<S, kURX, R, ARGMIN><<<(unsigned)blocks, kp.ublock, smem, st>>>(
        (const S*)Vin, (S*)Vout, occ, mask, recs, ku, order, sb.part_sum, sb.part_max, argmin);
    k_reduce_parts<<<1, 1024, 0, st>>>(sb.part_sum, sb.part_max, blocks, sb.out);
    *launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_stencil_u(int storage, const void* Vin, void* Vout, const uint8_t* occ,
                             const uint32_t* mask, const uint32_t* recs, const KParams& kp,
                             const int32_t* order, const SweepBufs& sb, int16_t* argmin,
                             cudaStream_t st, int64_t* launches) {
#define PG_SU(S)                                                                                 \
    return argmin ? stencil_u_t<S, true>(Vin, Vout, occ, mask, recs, kp, order, sb, argmin, st,  \
                                         launches)                                               \
                  : stencil_u_t<S, false>(Vin, Vout, occ, mask, recs, kp, order, sb, argmin, st, \
                                          launches)
    switch (storage) {
        case PG_STORE_F32: PG_SU(float);
        case PG_STORE_F16: PG_SU(__half);
        case PG_STORE_BF16: PG_SU(__nv_bfloat16);
    }
#undef PG_SU
    return cudaErrorInvalidValue;
}

template <typename S, bool ARGMIN, bool VEC, bool OFF32>
static cudaError_t stencil_b_v(const void* Vin, void* Vout, const uint8_t* occ,
                               const uint32_t* mask, const uint32_t* recs, const KParams& kb,
                               const int32_t* order, const SweepBufs& sb, int16_t* argmin,
                               int64_t blocks, int threads, size_t smem, cudaStream_t st) {
    static std::atomic<uint64_t> attr_set{0};
    const uint64_t attr_bit = device_bit();
    if (!(attr_set.load() & attr_bit)) {
        cudaError_t e = cudaFuncSetAttribute(k_stencil_b<S, ARGMIN, VEC, OFF32>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return e;
        attr_set.fetch_or(attr_bit);
    }
    k_stencil_b<S, ARGMIN, VEC, OFF32><<<(unsigned)blocks, threads, smem, st>>>(
        (const S*)Vin, (S*)Vout, occ, mask, recs, kb, order, sb.part_sum, sb.part_max, argmin);
    return cudaSuccess;
}

template <typename S, bool ARGMIN>
static cudaError_t stencil_b_t(const void* Vin, void* Vout, const uint8_t* occ,
                               const uint32_t* mask, const uint32_t* recs, const KParams& kp,
                               const int32_t* order, const SweepBufs& sb, int16_t* argmin,
                               cudaStream_t st, int64_t* launches) {
    if (kp.btile_x <= 0 || kp.bblock <= 0 || kp.bblock > 256 || kp.nsub > kStencilMaxSub ||
        (int64_t)kp.btile_x * kp.g.n[1] > (int64_t)kp.bblock * kBCells)
        return cudaErrorInvalidValue;
    KParams kb = kp;
    kb.tile_x = kp.btile_x;
    kb.tiles_x = kp.btiles_x;
    const int64_t blocks = kp.nplanes * kp.btiles_x;
    if (blocks > sb.nparts || blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    const size_t smem = stencil_b_smem(kp.nctl, kp.btile_x, kp.g.n[1]);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    const bool vec = kp.g.n[1] % BVec<S>::N == 0;
    const bool off32 = kp.ncells <= (int64_t)0xffffffffLL;
#define PG_SBV(V, O) stencil_b_v<S, ARGMIN, V, O>(Vin, Vout, occ, mask, recs, kb, order, sb, argmin, \
                                                  blocks, kp.bblock, smem, st)
    cudaError_t e = vec ? (off32 ? PG_SBV(true, true) : PG_SBV(true, false))
                        : (off32 ? PG_SBV(false, true) : PG_SBV(false, false));
#undef PG_SBV
    if (e != cudaSuccess) return e;
    k_reduce_parts<<<1, 1024, 0, st>>>(sb.part_sum, sb.part_max, blocks, sb.out);
    *launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_stencil_b(int storage, const void* Vin, void* Vout, const uint8_t* occ,
                             const uint32_t* mask, const uint32_t* recs, const KParams& kp,
                             const int32_t* order, const SweepBufs& sb, int16_t* argmin,
                             cudaStream_t st, int64_t* launches) {
#define PG_SB(S)                                                                                 \
    return argmin ? stencil_b_t<S, true>(Vin, Vout, occ, mask, recs, kp, order, sb, argmin, st,  \
                                         launches)                                               \
                  : stencil_b_t<S, false>(Vin, Vout, occ, mask, recs, kp, order, sb, argmin, st, \
                                          launches)
    switch (storage) {
        case PG_STORE_F32: PG_SB(float);
        case PG_STORE_F16: PG_SB(__half);
        case PG_STORE_BF16: PG_SB(__nv_bfloat16);
        case PG_STORE_Q16: PG_SB(Q16);
    }
#undef PG_SB
    return cudaErrorInvalidValue;
}

cudaError_t launch_stencil_b_batch(int storage, const BatchTable* tabs, int ntab, int64_t first,
                                   int64_t count, int threads, int parity, const int32_t* done,
                                   double* part_sum, double* part_max, size_t smem, int grid,
                                   bool any_vec, bool any_scalar, bool off32, cudaStream_t st) {
#define PG_BB(S)                                                                                 \
    {                                                                                            \
        static std::atomic<uint64_t> attr_set{0};                                                            \
        const uint64_t attr_bit = device_bit();                                                  \
        if (!(attr_set.load() & attr_bit)) {                                                                         \
            cudaError_t e = cudaSuccess;                                                         \
            void (*fns[4])(const BatchTable*, int, int64_t, int64_t, int, const int32_t*,        \
                           double*, double*) = {k_stencil_b_batch<S, true, true>,                \
                                                k_stencil_b_batch<S, true, false>,               \
                                                k_stencil_b_batch<S, false, true>,               \
                                                k_stencil_b_batch<S, false, false>};             \
            for (int f = 0; f < 4 && e == cudaSuccess; ++f)                                      \
                e = cudaFuncSetAttribute(fns[f], cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                         200 * 1024);                                            \
            if (e != cudaSuccess) return e;                                                      \
            attr_set.fetch_or(attr_bit);                                                                     \
        }                                                                                        \
        if (any_vec) {                                                                           \
            if (off32)                                                                           \
                k_stencil_b_batch<S, true, true><<<grid, threads, smem, st>>>(                   \
                    tabs, ntab, first, count, parity, done, part_sum, part_max);                 \
            else                                                                                 \
                k_stencil_b_batch<S, true, false><<<grid, threads, smem, st>>>(                  \
                    tabs, ntab, first, count, parity, done, part_sum, part_max);                 \
        }                                                                                        \
        if (any_scalar) {                                                                        \
            if (off32)                                                                           \
                k_stencil_b_batch<S, false, true><<<grid, threads, smem, st>>>(                  \
                    tabs, ntab, first, count, parity, done, part_sum, part_max);                 \
            else                                                                                 \
                k_stencil_b_batch<S, false, false><<<grid, threads, smem, st>>>(                 \
                    tabs, ntab, first, count, parity, done, part_sum, part_max);                 \
        }                                                                                        \
        return cudaGetLastError();                                                               \
    }
    if (smem > 200 * 1024 || grid <= 0 || threads <= 0 || threads > 256 || threads % 32)
        return cudaErrorInvalidValue;
    switch (storage) {
        case PG_STORE_F32: PG_BB(float)
        case PG_STORE_F16: PG_BB(__half)
        case PG_STORE_BF16: PG_BB(__nv_bfloat16)
        case PG_STORE_Q16: PG_BB(Q16)
    }
#undef PG_BB
    return cudaErrorInvalidValue;
}

cudaError_t launch_reduce_batch(const BatchTable* tabs, int ntab, const double* part_sum,
                                const double* part_max, double* out, cudaStream_t st) {
    k_reduce_batch<<<ntab, 256, 0, st>>>(tabs, part_sum, part_max, out);
    return cudaGetLastError();
}

template <typename S>
static int batch_occupancy(int threads, size_t smem) {
    int nb = 0;
    cudaFuncSetAttribute(k_stencil_b_batch<S, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         200 * 1024);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_stencil_b_batch<S, true, false>,
                                                      threads, smem) != cudaSuccess)
        return 0;
    return nb;
}

int batch_blocks_per_sm(int storage, size_t smem, int threads) {
    switch (storage) {
        case PG_STORE_F32: return batch_occupancy<float>(threads, smem);
        case PG_STORE_F16: return batch_occupancy<__half>(threads, smem);
        case PG_STORE_BF16: return batch_occupancy<__nv_bfloat16>(threads, smem);
        case PG_STORE_Q16: return batch_occupancy<Q16>(threads, smem);
    }
    return 0;
}

template <typename S>
static cudaError_t r_batch_attr() {
    static std::atomic<uint64_t> attr_set{0};
    const uint64_t attr_bit = device_bit();
    if (attr_set.load() & attr_bit) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_stencil_r_batch<S, kRCellsPerThread>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kRSmemMax);
    if (e == cudaSuccess) attr_set.fetch_or(attr_bit);
    return e;
}

template <typename S>
static int r_batch_occupancy(int threads, size_t smem) {
    int nb = 0;
    if (r_batch_attr<S>() != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_stencil_r_batch<S, kRCellsPerThread>,
                                                      threads, smem) != cudaSuccess)
        return 0;
    return nb;
}

int r_batch_blocks_per_sm(int storage, size_t smem, int threads) {
    switch (storage) {
        case PG_STORE_F32: return r_batch_occupancy<float>(threads, smem);
        case PG_STORE_F16: return r_batch_occupancy<__half>(threads, smem);
        case PG_STORE_BF16: return r_batch_occupancy<__nv_bfloat16>(threads, smem);
        case PG_STORE_Q16: return r_batch_occupancy<Q16>(threads, smem);
    }
    return 0;
}

cudaError_t launch_stencil_r_batch(int storage, const BatchTable* tabs, int ntab, int64_t first,
                                   int64_t count, int threads, int parity, const int32_t* done,
                                   double* part_sum, double* part_max, size_t smem, int grid,
                                   cudaStream_t st) {
    if (threads <= 0 || threads > RShape<kRCellsPerThread>::kMaxThreads || threads % 32 != 0 ||
        grid <= 0 || smem > (size_t)kRSmemMax)
        return cudaErrorInvalidValue;
#define PG_RB(S)                                                                                 \
    {                                                                                            \
        cudaError_t e = r_batch_attr<S>();                                                       \
        if (e != cudaSuccess) return e;                                                          \
        k_stencil_r_batch<S, kRCellsPerThread><<<grid, threads, smem, st>>>(                     \
            tabs, ntab, first, count, parity, done, part_sum, part_max);                         \
        return cudaGetLastError();                                                               \
    }
    switch (storage) {
        case PG_STORE_F32: PG_RB(float);
        case PG_STORE_F16: PG_RB(__half);
        case PG_STORE_BF16: PG_RB(__nv_bfloat16);
        case PG_STORE_Q16: PG_RB(Q16);
    }
#undef PG_RB
    return cudaErrorInvalidValue;
}

cudaError_t launch_stencil_group(const uint32_t* recs, const KParams& kp, const int32_t* order,
                                 uint16_t* gord, cudaStream_t st, int64_t* launches) {
    const size_t smem = stencil_group_smem(kp.nctl);
    if (smem > 200 * 1024 || kp.nplanes > 0x7fffffffLL || kp.nctl > 0x7fff)
        return cudaErrorInvalidValue;
    static std::atomic<uint64_t> attr_set{0};
    const uint64_t attr_bit = device_bit();
    if (!(attr_set.load() & attr_bit)) {
        cudaError_t e = cudaFuncSetAttribute(k_stencil_group,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return e;
        attr_set.fetch_or(attr_bit);
    }
    k_stencil_group<<<(unsigned)kp.nplanes, 128, smem, st>>>(recs, kp, order, gord);
    *launches += 1;
    return cudaGetLastError();
}

template <typename S, bool ARGMIN, int KR>
static cudaError_t stencil_r_t(const void* Vin, void* Vout, const uint8_t* occ,
                               const uint32_t* recs, const uint32_t* tmask, const KParams& kp,
                               const uint16_t* gord, const SweepBufs& sb, int16_t* argmin,
                               cudaStream_t st, int64_t* launches) {
    if (!stencil_r_shape_ok(kp)) return cudaErrorInvalidValue;
    KParams kr = kp;
    kr.tile_x = kp.rtile_x;
    kr.tiles_x = kp.rtiles_x;
    // one block per plane sweeps all its tiles; one residual partial per tile
    const int64_t parts = kp.nplanes * kp.rtiles_x;
    if (parts > sb.nparts || kp.nplanes > 0x7fffffffLL) return cudaErrorInvalidValue;
    const size_t smem = stencil_r_smem_bytes(kp);
    if (smem > (size_t)kRSmemMax) return cudaErrorInvalidValue;
    static std::atomic<uint64_t> attr_set{0};
    const uint64_t attr_bit = device_bit();
    if (!(attr_set.load() & attr_bit)) {
        cudaError_t e = cudaFuncSetAttribute(k_stencil_r<S, ARGMIN, KR>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, kRSmemMax);
        if (e != cudaSuccess) return e;
        attr_set.fetch_or(attr_bit);
    }
    k_stencil_r<S, ARGMIN, KR><<<(unsigned)kp.nplanes, kp.rblock, smem, st>>>(
        (const S*)Vin, (S*)Vout, occ, recs, tmask, kr, gord, sb.part_sum, sb.part_max, argmin);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_reduce_parts<<<1, 1024, 0, st>>>(sb.part_sum, sb.part_max, parts, sb.out);
    *launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_stencil_r(int storage, const void* Vin, void* Vout, const uint8_t* occ,
                             const uint32_t* recs, const uint32_t* tmask, const KParams& kp,
                             const uint16_t* gord, const SweepBufs& sb, int16_t* argmin,
                             cudaStream_t st, int64_t* launches) {
#define PG_SR(S)                                                                                 \
    return argmin ? stencil_r_t<S, true, kRCellsPerThread>(Vin, Vout, occ, recs, tmask, kp,      \
                                                           gord, sb, argmin, st, launches)       \
                  : stencil_r_t<S, false, kRCellsPerThread>(Vin, Vout, occ, recs, tmask, kp,     \
                                                            gord, sb, argmin, st, launches)
    switch (storage) {
        case PG_STORE_F32: PG_SR(float);
        case PG_STORE_F16: PG_SR(__half);
        case PG_STORE_BF16: PG_SR(__nv_bfloat16);
        case PG_STORE_Q16: PG_SR(Q16);
    }
#undef PG_SR
    return cudaErrorInvalidValue;
}

template <bool ARGMIN>
static cudaError_t stencil_d_t(const void* Vin, void* Vout, const uint8_t* occ,
                               const uint32_t* mask, const uint32_t* recs, const KParams& kp,
                               const SweepBufs& sb, int16_t* argmin, cudaStream_t st,
                               int64_t* launches) {
    if (kp.btile_x <= 0 || (int64_t)kp.btile_x * kp.g.n[1] > kBCells * kDThreads ||
        kp.nsub > kStencilMaxSub)
        return cudaErrorInvalidValue;
    KParams kd = kp;
    kd.tile_x = kp.btile_x;
    kd.tiles_x = kp.btiles_x;
    const int64_t blocks = kp.nplanes * kp.btiles_x;
    if (blocks > sb.nparts || blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    const size_t smem = stencil_d_smem(kp.btile_x, kp.g.n[1]);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static std::atomic<uint64_t> attr_set{0};
    const uint64_t attr_bit = device_bit();
    if (!(attr_set.load() & attr_bit)) {
        cudaError_t e = cudaFuncSetAttribute(k_stencil_d<ARGMIN>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return e;
        attr_set.fetch_or(attr_bit);
    }
    k_stencil_d<ARGMIN><<<(unsigned)blocks, kDThreads, smem, st>>>(
        (const double*)Vin, (double*)Vout, occ, mask, recs, kd, sb.part_sum, sb.part_max, argmin);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_reduce_parts<<<1, 1024, 0, st>>>(sb.part_sum, sb.part_max, blocks, sb.out);
    *launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_stencil_d(const void* Vin, void* Vout, const uint8_t* occ,
                             const uint32_t* mask, const uint32_t* recs, const KParams& kp,
                             const SweepBufs& sb, int16_t* argmin, cudaStream_t st,
                             int64_t* launches) {
    return argmin ? stencil_d_t<true>(Vin, Vout, occ, mask, recs, kp, sb, argmin, st, launches)
                  : stencil_d_t<false>(Vin, Vout, occ, mask, recs, kp, sb, argmin, st, launches);
}

cudaError_t launch_stencil_tmask(const uint32_t* mask, const KParams& kp, int64_t plane0,
                                 int64_t nplanes, uint32_t* tmask, cudaStream_t st,
                                 int64_t* launches) {
    if (kp.rtile_x <= 0 || plane0 < 0 || nplanes < 0 || plane0 + nplanes > kp.nplanes)
        return cudaErrorInvalidValue;
    if (nplanes == 0) return cudaSuccess;
    const int32_t ts = tile_mask_stride(kp.rtile_x, kp.g.n[1]);
    const int64_t total = nplanes * kp.rtiles_x * kp.nctl * ts;
    k_stencil_tmask<<<grid_for(total, 256), 256, 0, st>>>(mask, kp, kp.rtile_x, kp.rtiles_x, ts,
                                                          plane0, nplanes, tmask);
    *launches += 1;
    return cudaGetLastError();
}

size_t stencil_tmask_bytes(const KParams& kp) {
    return (size_t)kp.nplanes * kp.rtiles_x * kp.nctl * tile_mask_stride(kp.rtile_x, kp.g.n[1]) *
           sizeof(uint32_t);
}

size_t stencil_r_smem_bytes(const KParams& kp) {
    return stencil_r_smem(kp.nctl, kp.rchunk, kp.rtile_x, kp.g.n[1], kp.rgroups, kp.nsub);
}

bool stencil_r_shape_ok(const KParams& kp) {
    const int32_t n2 = kp.g.n[1];
    return kp.rtile_x > 0 && kp.rtiles_x > 0 && kp.rblock > 0 &&
           kp.rblock <= RShape<kRCellsPerThread>::kMaxThreads && kp.rblock % 32 == 0 &&
           kp.rgroups > 0 && (int64_t)kp.rgroups * n2 <= kp.rblock &&
           kp.rtile_x + 3 <= 4 * kp.rgroups && kp.rchunk > 0 && kp.rchunk <= kp.nctl &&
           // window byte offsets fit 16 bits (the packed row entries)
           (int64_t)16 * kp.rgroups * stencil_r_row_stride(n2) <= 0xffff &&
           // the chunk's y increments fit the window buffers
           (int64_t)kp.rchunk * stencil_r_ninc(kp.nsub) <=
               (int64_t)16 * kp.rgroups * stencil_r_row_stride(n2) &&
           kp.nctl <= (int)kCtlMask && kp.nsub <= kStencilMaxSub && n2 >= 1 && n2 <= 0xffff;
}

int stencil_r_blocks_per_sm(int threads, size_t smem) {
    static std::atomic<uint64_t> attr_set{0};
    const uint64_t attr_bit = device_bit();
    if (!(attr_set.load() & attr_bit)) {
        if (cudaFuncSetAttribute(k_stencil_r<float, false, kRCellsPerThread>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, kRSmemMax) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        attr_set.fetch_or(attr_bit);
    }
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_stencil_r<float, false, kRCellsPerThread>,
                                                      threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return nb;
}

int32_t stencil_r_row_stride_host(int32_t n2) { return stencil_r_row_stride(n2); }
int32_t stencil_r_ninc_host(int nsub) { return stencil_r_ninc(nsub); }

size_t stencil_r_ctl_smem_bytes(const KParams& kp, int32_t tile_x) {
    return stencil_r_ctl_bytes(tile_x, kp.g.n[1], kp.nsub);
}

size_t stencil_b_smem_bytes(const KParams& kp) {
    return stencil_b_smem(kp.nctl, kp.btile_x, kp.g.n[1]);
}
size_t stencil_u_smem_bytes(const KParams& kp) { return stencil_u_smem(kp.nctl); }

cudaError_t launch_adj_active(const float* V, const int16_t* pol, const uint8_t* occ,
                              const uint32_t* mask, const uint32_t* recs, const KParams& kp,
                              uint8_t* active, cudaStream_t st) {
    k_adj_active<<<grid_for(kp.ncells, 256), 256, 0, st>>>(V, pol, occ, mask, recs, kp, active);
    return cudaGetLastError();
}

cudaError_t launch_adj_scatter(const double* lam_in, double* lam_out, const int16_t* pol,
                               const uint8_t* active, const uint32_t* recs, const KParams& kp,
                               cudaStream_t st) {
    k_adj_scatter<<<grid_for(kp.ncells, 256), 256, 0, st>>>(lam_in, lam_out, pol, active, recs, kp);
    return cudaGetLastError();
}

cudaError_t launch_adj_start(const float* c, double* l0, double* l1, int64_t n, const SweepBufs& sb,
                             cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(sb.nparts, 148 * 16);
    k_adj_start<<<(unsigned)blocks, 256, 0, st>>>(c, l0, l1, n, sb.part_sum, sb.part_max);
    k_reduce_parts<<<1, 1024, 0, st>>>(sb.part_sum, sb.part_max, blocks, sb.out);
    return cudaGetLastError();
}

cudaError_t launch_adj_step(const double* lout, double* lin, const float* c, int64_t n,
                            const SweepBufs& sb, cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(sb.nparts, 148 * 16);
    k_adj_step<<<(unsigned)blocks, 256, 0, st>>>(lout, lin, c, n, sb.part_sum, sb.part_max);
    k_reduce_parts<<<1, 1024, 0, st>>>(sb.part_sum, sb.part_max, blocks, sb.out);
    return cudaGetLastError();
}

cudaError_t launch_adj_count(const uint8_t* a, int64_t n, const SweepBufs& sb, cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(sb.nparts, 148 * 16);
    k_adj_count<<<(unsigned)blocks, 256, 0, st>>>(a, n, sb.part_sum, sb.part_max);
    k_reduce_parts<<<1, 1024, 0, st>>>(sb.part_sum, sb.part_max, blocks, sb.out);
    return cudaGetLastError();
}

cudaError_t launch_adj_grad(const float* V, const double* lam, const int16_t* pol,
                            const uint8_t* active, const uint32_t* recs, const KParams& kp,
                            const float* ctl, double* grad, cudaStream_t st) {
    const size_t smem = adj_grad_smem(kp.nctl);
    if (smem > 200 * 1024 || kp.nplanes > 0x7fffffffLL) return cudaErrorInvalidValue;
    static std::atomic<uint64_t> attr_set{0};
    const uint64_t attr_bit = device_bit();
    if (!(attr_set.load() & attr_bit)) {
        cudaError_t e = cudaFuncSetAttribute(k_adj_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             200 * 1024);
        if (e != cudaSuccess) return e;
        attr_set.fetch_or(attr_bit);
    }
    k_adj_grad<<<(unsigned)kp.nplanes, 128, smem, st>>>(V, lam, pol, active, recs, kp, ctl, grad);
    return cudaGetLastError();
}

size_t stencil_recs_bytes(const KParams& kp) {
    return (size_t)kp.nplanes * kp.nctl * kURec * sizeof(uint32_t);
}

size_t stencil_mask_bytes(const KParams& kp) {
    return (size_t)kp.nplanes * kp.nctl * kp.g.n[0] * mask_words(kp.g.n[1]) * sizeof(uint32_t);
}

cudaError_t launch_encode(int storage, const void* V, const KParams& kp, int32_t dtype,
                          double scale, double escape_scale, int64_t lo, int64_t n, uint8_t* out,
                          unsigned long long* counts, cudaStream_t st) {
    const int b = grid_for(n, 256);
    switch (storage) {
        case PG_STORE_F32: k_encode<float><<<b, 256, 0, st>>>((const float*)V, kp, dtype, scale, escape_scale, lo, n, out, counts); break;
        case PG_STORE_F16: k_encode<__half><<<b, 256, 0, st>>>((const __half*)V, kp, dtype, scale, escape_scale, lo, n, out, counts); break;
        case PG_STORE_BF16: k_encode<__nv_bfloat16><<<b, 256, 0, st>>>((const __nv_bfloat16*)V, kp, dtype, scale, escape_scale, lo, n, out, counts); break;
        case PG_STORE_Q16: k_encode<Q16><<<b, 256, 0, st>>>((const Q16*)V, kp, dtype, scale, escape_scale, lo, n, out, counts); break;
        case PG_STORE_F64: k_encode<double><<<b, 256, 0, st>>>((const double*)V, kp, dtype, scale, escape_scale, lo, n, out, counts); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}


// ---------------------------------------------------------------------------
// x slabs of the out-of-core driver: a slab's rows between the table's
// row-major order (the host store) and the device layout, bits unchanged
// (E = the storage's word: 4 or 2 bytes).  k_slab_in reads every row of the
// slab; k_slab_out writes the rows [r0, r1) only (row r0 first).  And the
// per-round residual: the sweep's (L1, max) folded into a running pair.
// ---------------------------------------------------------------------------
template <typename E>
__global__ void k_slab_in(const E* __restrict__ rm, E* __restrict__ V, KParams kp, int32_t row0,
                          int32_t row1) {
    const Layout L = make_layout(kp);
    const int64_t per_row = kp.ncells / L.n[0];
    const int64_t n = (int64_t)(row1 - row0) * per_row;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = k + (int64_t)row0 * per_row;
        int32_t i[6];
        for (int c = 5; c >= 1; --c) { i[c] = (int32_t)(r % L.n[c]); r /= L.n[c]; }
        i[0] = (int32_t)r;
        V[L.dev(i[0], i[1], i[2], i[3], i[4], i[5])] = rm[k];
    }
}

template <typename E>
__global__ void k_slab_out(const E* __restrict__ V, E* __restrict__ rm, KParams kp, int32_t row0,
                           int32_t row1) {
    const Layout L = make_layout(kp);
    const int64_t per_row = kp.ncells / L.n[0];
    const int64_t n = (int64_t)(row1 - row0) * per_row;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = k + (int64_t)row0 * per_row;
        int32_t i[6];
        for (int c = 5; c >= 1; --c) { i[c] = (int32_t)(r % L.n[c]); r /= L.n[c]; }
        i[0] = (int32_t)r;
        rm[k] = V[L.dev(i[0], i[1], i[2], i[3], i[4], i[5])];
    }
}

__global__ void k_accum(const double* __restrict__ red, double* __restrict__ acc) {
    acc[0] += red[0];
    acc[1] = fmax(acc[1], red[1]);
}

cudaError_t launch_slab_in(int elem_bytes, const void* rm, void* V, const KParams& kp,
                           cudaStream_t st, int32_t row0, int32_t row1) {
    if (row1 < 0) row1 = kp.g.n[0];
    if (row0 < 0 || row1 > kp.g.n[0] || row1 < row0) return cudaErrorInvalidValue;
    const int64_t n = (int64_t)(row1 - row0) * (kp.ncells / kp.g.n[0]);
    const int b = grid_for(n, 256);
    if (elem_bytes == 4)
        k_slab_in<uint32_t><<<b, 256, 0, st>>>((const uint32_t*)rm, (uint32_t*)V, kp, row0, row1);
    else if (elem_bytes == 2)
        k_slab_in<uint16_t><<<b, 256, 0, st>>>((const uint16_t*)rm, (uint16_t*)V, kp, row0, row1);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_slab_out(int elem_bytes, const void* V, void* rm, const KParams& kp,
                            int32_t row0, int32_t row1, cudaStream_t st) {
    if (row0 < 0 || row1 > kp.g.n[0] || row1 < row0) return cudaErrorInvalidValue;
    const int64_t n = (int64_t)(row1 - row0) * (kp.ncells / kp.g.n[0]);
    const int b = grid_for(n, 256);
    if (elem_bytes == 4)
        k_slab_out<uint32_t><<<b, 256, 0, st>>>((const uint32_t*)V, (uint32_t*)rm, kp, row0, row1);
    else if (elem_bytes == 2)
        k_slab_out<uint16_t><<<b, 256, 0, st>>>((const uint16_t*)V, (uint16_t*)rm, kp, row0, row1);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_accum(const double* red, double* acc, cudaStream_t st) {
    k_accum<<<1, 1, 0, st>>>(red, acc);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// The reach of one backup in x, for the halo of an x slab: the largest
// |sum of the substep x increments| over every (plane, control), in cells,
// rounded up (the successor and every swept probe lie between the cell and
// x + that sum).  One thread per (plane, control), the plain scheme's
// transition (pg_plane.cuh).
// ---------------------------------------------------------------------------
__global__ void k_reach(KParams kp, const float* __restrict__ ctl, int32_t* __restrict__ out) {
    GridT<float> g;
    load_grid(g, kp.g);
    const int64_t total = kp.nplanes * kp.nctl;
    int32_t best = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pl = i / kp.nctl;
        const int u = (int)(i - pl * kp.nctl);
        int64_t q = pl;
        const int32_t i6 = (int32_t)(q % kp.g.n[5]); q /= kp.g.n[5];
        const int32_t i5 = (int32_t)(q % kp.g.n[4]); q /= kp.g.n[4];
        const int32_t i4 = (int32_t)(q % kp.g.n[3]); q /= kp.g.n[3];
        const int32_t i3 = (int32_t)q;
        Transition<float> t;
        transition(kp, g, i3, i4, i5, i6, ctl, u, t);
        if (!t.ok) continue;
        const float c = ceilf(fabsf(t.sumx) / g.step[0]);
        best = max(best, c < 1.0e6f ? (int32_t)c : 1000000);
    }
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

cudaError_t launch_reach(const KParams& kp, const float* ctl, int32_t* out, cudaStream_t st) {
    const int64_t total = kp.nplanes * kp.nctl;
    k_reach<<<grid_for(total, 128), 128, 0, st>>>(kp, ctl, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Self-test probes: the device's own implementations of the reference's
// functions evaluated on given inputs, so the self-test can check what the
// sweeps compute (SelfTest.jl:208-258, 407-564 call the same functions).
// ---------------------------------------------------------------------------

// step_state / step_state_rk2 (PeregrineSolver.jl:203-279): one integration
// per item; a diverged state comes back as NaN in every component, as the
// reference's NANSTATE.
__global__ void k_probe_step(pg_model mdl, int32_t rk2, const float* __restrict__ states,
                             const float* __restrict__ controls, const float* __restrict__ dt,
                             const int32_t* __restrict__ nsub, int64_t n,
                             float* __restrict__ out) {
    ModelT<float> m;
    load_model(m, mdl);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float* si = states + 6 * i;
        State6<float> s{si[0], si[1], si[2], si[3], si[4], si[5]};
        const bool ok = integrate(m, s, controls[3 * i], controls[3 * i + 1], controls[3 * i + 2],
                                  dt[i], nsub[i], rk2 != 0, (float*)nullptr, (float*)nullptr);
        const float nanv = __int_as_float(0x7fc00000);
        float* o = out + 6 * i;
        o[0] = ok ? s.x : nanv; o[1] = ok ? s.y : nanv; o[2] = ok ? s.h : nanv;
        o[3] = ok ? s.vx : nanv; o[4] = ok ? s.vy : nanv; o[5] = ok ? s.w : nanv;
    }
}

// traction_gain (PeregrineSolver.jl:126-136)
__global__ void k_probe_gain(const float* __restrict__ controls, float knee, int64_t n,
                             float* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = traction_gain(controls[3 * i], controls[3 * i + 1], controls[3 * i + 2], knee);
}

// interp / interp_kuhn (PeregrineSolver.jl:399-466, 571-665) of the stored V
// at given states; grads (6 per state) for the Kuhn form when non-null.
template <typename S>
__global__ void k_probe_interp(const S* __restrict__ V, KParams kp, const float* __restrict__ states,
                               int64_t n, int32_t kuhn, int32_t nearest, int32_t vclamp, float cap,
                               float* __restrict__ out, float* __restrict__ grads) {
    GridT<float> g;
    load_grid(g, kp.g);
    VView<float, S> vv{V, nullptr, make_layout(kp), cap, false, true};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float* si = states + 6 * i;
        State6<float> s{si[0], si[1], si[2], si[3], si[4], si[5]};
        if (kuhn) {
            float gr[6] = {0, 0, 0, 0, 0, 0};
            out[i] = interp_kuhn(vv, g, s, cap, vclamp != 0, gr);
            if (grads)
                for (int k = 0; k < 6; ++k) grads[6 * i + k] = gr[k];
        } else {
            out[i] = interp_ml(vv, g, s, nearest != 0, cap, vclamp != 0);
        }
    }
}

cudaError_t launch_probe_step(const pg_model& m, int32_t rk2, const float* states,
                              const float* controls, const float* dt, const int32_t* nsub,
                              int64_t n, float* out, cudaStream_t st) {
    k_probe_step<<<grid_for(n, 128), 128, 0, st>>>(m, rk2, states, controls, dt, nsub, n, out);
    return cudaGetLastError();
}

cudaError_t launch_probe_gain(const float* controls, float knee, int64_t n, float* out,
                              cudaStream_t st) {
    k_probe_gain<<<grid_for(n, 128), 128, 0, st>>>(controls, knee, n, out);
    return cudaGetLastError();
}

cudaError_t launch_probe_interp(int storage, const void* V, const KParams& kp, const float* states,
                                int64_t n, int32_t kuhn, int32_t nearest, int32_t vclamp,
                                float cap, float* out, float* grads, cudaStream_t st) {
    const int b = grid_for(n, 128);
    switch (storage) {
        case PG_STORE_F32: k_probe_interp<float><<<b, 128, 0, st>>>((const float*)V, kp, states, n, kuhn, nearest, vclamp, cap, out, grads); break;
        case PG_STORE_F16: k_probe_interp<__half><<<b, 128, 0, st>>>((const __half*)V, kp, states, n, kuhn, nearest, vclamp, cap, out, grads); break;
        case PG_STORE_BF16: k_probe_interp<__nv_bfloat16><<<b, 128, 0, st>>>((const __nv_bfloat16*)V, kp, states, n, kuhn, nearest, vclamp, cap, out, grads); break;
        case PG_STORE_Q16: k_probe_interp<Q16><<<b, 128, 0, st>>>((const Q16*)V, kp, states, n, kuhn, nearest, vclamp, cap, out, grads); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace pg
