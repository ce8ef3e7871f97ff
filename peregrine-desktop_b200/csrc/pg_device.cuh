// pg_device.cuh -- device-side model, integrators, interpolants and the
// Bellman backup of the minimum-time value iteration, templated on the
// arithmetic type T (float for the product, double for the FP64 device
// oracle).
//
// Every operation that decides a discrete outcome (a probe cell, an envelope
// test, a corner index) goes through the explicitly rounded intrinsics in
// `Ar<T>` so nvcc cannot contract a*b+c into an FMA: the reference (Julia on
// the CPU) rounds each product and sum separately, and matching that rounding
// is what makes the cell-form kernel bit-identical to the CPU restatement.
// sin, cos and tanh are evaluated in double and rounded once, which is what
// Julia's Float32 kernels do.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pg_types.h"

namespace pg {

template <typename T> struct Ar;

template <> struct Ar<float> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float sqrt_(float a) { return __fsqrt_rn(a); }
    static __device__ __forceinline__ void sincos_(float x, float* s, float* c) {
        double sd, cd;
        ::sincos((double)x, &sd, &cd);
        *s = (float)sd;
        *c = (float)cd;
    }
    static __device__ __forceinline__ float tanh_(float x) { return (float)::tanh((double)x); }
    static __device__ __forceinline__ float floor_(float x) { return floorf(x); }
    static __device__ __forceinline__ float rint_(float x) { return rintf(x); }
    static __device__ __forceinline__ float abs_(float x) { return fabsf(x); }
};

template <> struct Ar<double> {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dadd_rn(a, -b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double sqrt_(double a) { return __dsqrt_rn(a); }
    static __device__ __forceinline__ void sincos_(double x, double* s, double* c) {
        ::sincos(x, s, c);
    }
    static __device__ __forceinline__ double tanh_(double x) { return ::tanh(x); }
    static __device__ __forceinline__ double floor_(double x) { return ::floor(x); }
    static __device__ __forceinline__ double rint_(double x) { return ::rint(x); }
    static __device__ __forceinline__ double abs_(double x) { return ::fabs(x); }
};

// Julia min / max / clamp on non-NaN values.
template <typename T> __device__ __forceinline__ T jmin(T a, T b) { return b < a ? b : a; }
template <typename T> __device__ __forceinline__ T jmax(T a, T b) { return b > a ? b : a; }
template <typename T> __device__ __forceinline__ T jclamp(T x, T lo, T hi) {
    return x > hi ? hi : (x < lo ? lo : x);
}
template <typename T> __device__ __forceinline__ bool finite_(T x) { return isfinite(x); }

// Model and grid, converted once to the arithmetic type.
template <typename T> struct ModelT {
    T B[9], A[9], q[3], S[9], D[9], c[3], eps[3], knee;
};
template <typename T> struct GridT {
    int32_t n[6];
    T lo[6], step[6];
};

template <typename T> __device__ __forceinline__ void load_model(ModelT<T>& mt, const pg_model& m) {
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        mt.B[i] = (T)m.B[i]; mt.A[i] = (T)m.A[i]; mt.S[i] = (T)m.S[i]; mt.D[i] = (T)m.D[i];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) { mt.q[i] = (T)m.q[i]; mt.c[i] = (T)m.c[i]; mt.eps[i] = (T)m.eps[i]; }
    mt.knee = (T)m.knee;
}

template <typename T> __device__ __forceinline__ void load_grid(GridT<T>& gt, const pg_grid6& g) {
#pragma unroll
    for (int k = 0; k < 6; ++k) { gt.n[k] = g.n[k]; gt.lo[k] = (T)g.lo[k]; gt.step[k] = (T)g.step[k]; }
}

// axisvalue (PeregrineSolver.jl:64)
template <typename T> __device__ __forceinline__ T axisvalue(const GridT<T>& g, int k, int32_t i) {
    typedef Ar<T> R;
    return R::add(g.lo[k], R::mul((T)i, g.step[k]));
}

// csign (PeregrineSolver.jl:117)
template <typename T> __device__ __forceinline__ T csign(T v, T e) {
    return jclamp(Ar<T>::div(v, e), (T)-1, (T)1);
}

// traction_gain (PeregrineSolver.jl:126-136)
template <typename T> __device__ __forceinline__ T traction_gain(T u1, T u2, T u3, T knee) {
    typedef Ar<T> R;
    if (isnan(knee) || knee <= (T)0) return (T)1;
    T m = R::sqrt_(R::add(R::add(R::mul(u1, u1), R::mul(u2, u2)), R::mul(u3, u3)));
    T r = R::div(m, knee);
    if (r < (T)1.0e-6f) return (T)1;
    return R::div(R::tanh_(r), r);
}

// body_accel_sat (PeregrineSolver.jl:151-163): the 14 terms of a row summed
// left to right exactly as written in the reference.
template <typename T>
__device__ __forceinline__ void body_accel_sat(const ModelT<T>& m, T u1, T u2, T u3, T vx, T vy,
                                               T w, T* a) {
    typedef Ar<T> R;
    T w2 = R::mul(w, w);
    T sx = csign(vx, m.eps[0]), sy = csign(vy, m.eps[1]), sw = csign(w, m.eps[2]);
    T dx = R::mul(R::abs_(vx), vx), dy = R::mul(R::abs_(vy), vy), dw = R::mul(R::abs_(w), w);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const int o = 3 * r;
        T s = R::mul(m.B[o], u1);
        s = R::add(s, R::mul(m.B[o + 1], u2));
        s = R::add(s, R::mul(m.B[o + 2], u3));
        s = R::add(s, R::mul(m.A[o], vx));
        s = R::add(s, R::mul(m.A[o + 1], vy));
        s = R::add(s, R::mul(m.A[o + 2], w));
        s = R::add(s, R::mul(m.q[r], w2));
        s = R::add(s, R::mul(m.S[o], sx));
        s = R::add(s, R::mul(m.S[o + 1], sy));
        s = R::add(s, R::mul(m.S[o + 2], sw));
        s = R::add(s, R::mul(m.D[o], dx));
        s = R::add(s, R::mul(m.D[o + 1], dy));
        s = R::add(s, R::mul(m.D[o + 2], dw));
        s = R::add(s, m.c[r]);
        a[r] = s;
    }
}

template <typename T> __device__ __forceinline__ bool diverged(T x, T y, T h, T vx, T vy, T w) {
    typedef Ar<T> R;
    return !finite_(R::add(R::add(R::add(R::add(R::add(x, y), h), vx), vy), w));
}

template <typename T> struct State6 { T x, y, h, vx, vy, w; };

// One integration of a held command.  When incx/incy are given, the
// per-substep position increments are recorded: the dynamics never read the
// position, so these increments are the same for every (x, y) cell and the
// stencil kernel replays them per cell to reproduce the reference's position
// rounding exactly.  Returns false on divergence (the reference's NANSTATE).
// step_state: PeregrineSolver.jl:203-223; step_state_rk2: 254-279.
template <typename T>
__device__ __forceinline__ bool integrate(const ModelT<T>& m, State6<T>& s, T u1r, T u2r, T u3r,
                                          T dt, int32_t nsub, bool rk2, T* incx, T* incy) {
    typedef Ar<T> R;
    T hs = R::div(dt, (T)nsub);
    T hh = R::mul((T)0.5f, hs);
    T gn = traction_gain(u1r, u2r, u3r, m.knee);
    T u1 = R::mul(u1r, gn), u2 = R::mul(u2r, gn), u3 = R::mul(u3r, gn);
    T x = s.x, y = s.y, h = s.h, vx = s.vx, vy = s.vy, w = s.w;
    for (int32_t k = 0; k < nsub; ++k) {
        if (diverged(x, y, h, vx, vy, w)) return false;
        if (!rk2) {
            T a[3];
            body_accel_sat(m, u1, u2, u3, vx, vy, w, a);
            T dvx = R::add(a[0], R::mul(w, vy));
            T dvy = R::sub(a[1], R::mul(w, vx));
            T sh, ch;
            R::sincos_(h, &sh, &ch);
            T ix = R::mul(R::sub(R::mul(ch, vx), R::mul(sh, vy)), hs);
            T iy = R::mul(R::add(R::mul(sh, vx), R::mul(ch, vy)), hs);
            x = R::add(x, ix);
            y = R::add(y, iy);
            if (incx) { incx[k] = ix; incy[k] = iy; }
            h = R::add(h, R::mul(w, hs));
            vx = R::add(vx, R::mul(dvx, hs));
            vy = R::add(vy, R::mul(dvy, hs));
            w = R::add(w, R::mul(a[2], hs));
        } else {
            T a[3], sh, ch;
            body_accel_sat(m, u1, u2, u3, vx, vy, w, a);
            R::sincos_(h, &sh, &ch);
            T d1x = R::sub(R::mul(ch, vx), R::mul(sh, vy));
            T d1y = R::add(R::mul(sh, vx), R::mul(ch, vy));
            T d1h = w;
            T d1vx = R::add(a[0], R::mul(w, vy));
            T d1vy = R::sub(a[1], R::mul(w, vx));
            T d1w = a[2];
            T mx = R::add(x, R::mul(d1x, hh)), my = R::add(y, R::mul(d1y, hh));
            T mh = R::add(h, R::mul(d1h, hh));
            T mvx = R::add(vx, R::mul(d1vx, hh)), mvy = R::add(vy, R::mul(d1vy, hh));
            T mw = R::add(w, R::mul(d1w, hh));
            if (diverged(mx, my, mh, mvx, mvy, mw)) return false;
            body_accel_sat(m, u1, u2, u3, mvx, mvy, mw, a);
            R::sincos_(mh, &sh, &ch);
            T d2x = R::sub(R::mul(ch, mvx), R::mul(sh, mvy));
            T d2y = R::add(R::mul(sh, mvx), R::mul(ch, mvy));
            T d2vx = R::add(a[0], R::mul(mw, mvy));
            T d2vy = R::sub(a[1], R::mul(mw, mvx));
            T ix = R::mul(d2x, hs), iy = R::mul(d2y, hs);
            x = R::add(x, ix);
            y = R::add(y, iy);
            if (incx) { incx[k] = ix; incy[k] = iy; }
            h = R::add(h, R::mul(mw, hs));
            vx = R::add(vx, R::mul(d2vx, hs));
            vy = R::add(vy, R::mul(d2vy, hs));
            w = R::add(w, R::mul(a[2], hs));
        }
    }
    s.x = x; s.y = y; s.h = h; s.vx = vx; s.vy = vy; s.w = w;
    return true;
}

// cfl_tau / substeps_for (PeregrineSolver.jl:954-989)
template <typename T>
__device__ __forceinline__ T cfl_tau(const GridT<T>& g, const ModelT<T>& m, T vfx, T vfy, T w,
                                     const pg_params& p) {
    typedef Ar<T> R;
    if (p.cfl <= 0.0f) return (T)p.dt;
    T ax = jmax(jmax(R::abs_(m.B[0]), R::abs_(m.B[1])), R::abs_(m.B[2]));
    T ay = jmax(jmax(R::abs_(m.B[3]), R::abs_(m.B[4])), R::abs_(m.B[5]));
    T aw = jmax(jmax(R::abs_(m.B[6]), R::abs_(m.B[7])), R::abs_(m.B[8]));
    T cfl = (T)p.cfl;
    T t = (T)p.tau_max;
    if (ax > (T)1.0e-6f) t = jmin(t, R::div(R::mul(cfl, g.step[3]), ax));
    if (ay > (T)1.0e-6f) t = jmin(t, R::div(R::mul(cfl, g.step[4]), ay));
    if (aw > (T)1.0e-6f) t = jmin(t, R::div(R::mul(cfl, g.step[5]), aw));
    T sp = R::sqrt_(R::add(R::mul(vfx, vfx), R::mul(vfy, vfy)));
    if (sp > (T)1.0e-3f) t = jmin(t, R::div(R::mul(cfl, jmin(g.step[0], g.step[1])), sp));
    T aw2 = R::abs_(w);
    if (aw2 > (T)1.0e-4f) t = jmin(t, R::div(R::mul(cfl, g.step[2]), aw2));
    return jclamp(t, (T)p.tau_min, (T)p.tau_max);
}

template <typename T> __device__ __forceinline__ int32_t substeps_for(T tau, const pg_params& p) {
    if (p.hmax <= 0.0f) return p.nsub;
    int32_t k = (int32_t)jmin(Ar<T>::div(tau, (T)p.hmax), (T)1.0e4f) + 1;
    return k < 1 ? 1 : (k > 64 ? 64 : k);
}

// Index arithmetic between the table's row-major order and the device
// layout.  The device stores V as planes: plane p = ((ih*Nvx+ivx)*Nvy+ivy)*Nw+iw
// holds the Nx*Ny positions, x-major, so one (h, v) slice is contiguous.
struct Layout {
    int32_t n[6];
    int64_t P;        // Nx*Ny
    int64_t nplanes;  // Nh*Nvx*Nvy*Nw
    __device__ __forceinline__ int64_t dev(int32_t i1, int32_t i2, int32_t i3, int32_t i4,
                                           int32_t i5, int32_t i6) const {
        int64_t p = (((int64_t)i3 * n[3] + i4) * n[4] + i5) * n[5] + i6;
        return p * P + (int64_t)i1 * n[1] + i2;
    }
    __device__ __forceinline__ int64_t rowmajor(int32_t i1, int32_t i2, int32_t i3, int32_t i4,
                                                int32_t i5, int32_t i6) const {
        return (((((int64_t)i1 * n[1] + i2) * n[2] + i3) * n[3] + i4) * n[4] + i5) * n[5] + i6;
    }
    __device__ __forceinline__ int32_t occ(int32_t i1, int32_t i2, int32_t i3) const {
        return ((int32_t)i3 * n[0] + i1) * n[1] + i2;
    }
};

template <typename S> struct Conv;
// Storage <-> arithmetic conversions: ld() reads global memory through the
// read-only path, val() converts a value already in registers.
template <> struct Conv<float> {
    static __device__ __forceinline__ float ld(const float* p) { return __ldg(p); }
    static __device__ __forceinline__ float val(float v) { return v; }
    template <typename T> static __device__ __forceinline__ float st(T v) { return (float)v; }
};
template <> struct Conv<double> {
    static __device__ __forceinline__ double ld(const double* p) { return __ldg(p); }
    static __device__ __forceinline__ double val(double v) { return v; }
    template <typename T> static __device__ __forceinline__ double st(T v) { return (double)v; }
};

}  // namespace pg
