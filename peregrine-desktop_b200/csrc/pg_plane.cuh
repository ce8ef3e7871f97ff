// pg_plane.cuh -- the per-(plane, control) part of a lookahead, shared by
// the stencil kernels (included inside namespace pg by pg_kernels.cu).
//
// For a plane (ih, ivx, ivy, iw) and one control, everything lookahead
// (PeregrineSolver.jl:1100-1153) computes that does not depend on the cell's
// (x, y): the integration of the held command (its per-substep position
// increments, the successor heading and velocity), the probe heading bins,
// the successor's (h, v) corner and weights.  Exact rounding as the
// reference (Ar<T> ops); this runs once per plane and control.

template <typename T> struct Transition {
    bool ok;                     // finite, inside the velocity envelope
    T tau;                       // horizon
    T incx[kStencilMaxSub];      // per-substep x increments
    T incy[kStencilMaxSub];      // per-substep y increments
    T sumx, sumy;                // their sums, left to right
    int32_t ck[kStencilMaxChk];  // probe heading bins
    int32_t jb[4];               // floor of the successor's (h, vx, vy, w) coordinate
    T tt[4];                     // and its fraction
};

template <typename T>
__device__ void transition(const KParams& kp, const GridT<T>& g, int32_t i3, int32_t i4,
                           int32_t i5, int32_t i6, const float* ctl, int u, Transition<T>& o) {
    typedef Ar<T> R_;
    const int nctl = kp.nctl, nsub = kp.nsub, nchk = kp.nchk;
    ModelT<T> m;
    load_model(m, kp.m);
    State6<T> s;
    s.x = g.lo[0];  // representative position: the dynamics never read it
    s.y = g.lo[1];
    s.h = axisvalue(g, 2, i3);
    const T vfx = axisvalue(g, 3, i4), vfy = axisvalue(g, 4, i5);
    s.w = axisvalue(g, 5, i6);
    T sh0, ch0;
    R_::sincos_(s.h, &sh0, &ch0);
    s.vx = R_::add(R_::mul(ch0, vfx), R_::mul(sh0, vfy));
    s.vy = R_::add(R_::mul(-sh0, vfx), R_::mul(ch0, vfy));
    o.tau = cfl_tau(g, m, vfx, vfy, s.w, kp.p);
    const int32_t ns = substeps_for(o.tau, kp.p);
    State6<T> e = s;
    bool ok = ns == nsub && integrate(m, e, (T)ctl[u], (T)ctl[u + nctl], (T)ctl[u + 2 * nctl],
                                      o.tau, ns, kp.p.rk2 != 0, o.incx, o.incy);
    T sx = 0, sy = 0;
    for (int k = 0; k < kStencilMaxSub; ++k) {
        if (k >= nsub || !ok) { o.incx[k] = 0; o.incy[k] = 0; }
        sx = R_::add(sx, o.incx[k]);
        sy = R_::add(sy, o.incy[k]);
    }
    o.sumx = sx;
    o.sumy = sy;
    const T dh = R_::sub(e.h, s.h);
    ok = ok && finite_(R_::sub(e.x, s.x)) && finite_(R_::sub(e.y, s.y)) && finite_(dh) &&
         finite_(e.vx) && finite_(e.vy) && finite_(e.w);
    const T n3f = (T)g.n[2];
    for (int sc = 0; sc < kStencilMaxChk; ++sc) {
        int32_t ck = 0;
        if (ok && sc < nchk) {
            const T a = R_::div((T)(sc + 1), (T)nchk);
            const T ph = R_::add(s.h, R_::mul(dh, a));
            T gh = R_::div(R_::sub(ph, g.lo[2]), g.step[2]);
            gh = R_::sub(gh, R_::mul(R_::floor_(R_::div(gh, n3f)), n3f));
            ck = ((int32_t)R_::rint_(gh)) % g.n[2];
        }
        o.ck[sc] = ck;
    }
    for (int k = 0; k < 4; ++k) { o.jb[k] = 0; o.tt[k] = 0; }
    if (ok) {
        T snh, cnh;
        R_::sincos_(e.h, &snh, &cnh);
        const T nvfx = R_::sub(R_::mul(cnh, e.vx), R_::mul(snh, e.vy));
        const T nvfy = R_::add(R_::mul(snh, e.vx), R_::mul(cnh, e.vy));
        T f3 = R_::div(R_::sub(e.h, g.lo[2]), g.step[2]);
        f3 = R_::sub(f3, R_::mul(R_::floor_(R_::div(f3, n3f)), n3f));
        T f[4] = {f3, R_::div(R_::sub(nvfx, g.lo[3]), g.step[3]),
                  R_::div(R_::sub(nvfy, g.lo[4]), g.step[4]),
                  R_::div(R_::sub(e.w, g.lo[5]), g.step[5])};
        ok = finite_(f[0]) && finite_(f[1]) && finite_(f[2]) && finite_(f[3]);
        if (ok) {
            for (int k = 1; k < 4; ++k) {
                const T hi = (T)(g.n[2 + k] - 1);
                if (kp.p.vclamp) f[k] = jclamp(f[k], (T)0, hi);
                else if (f[k] < (T)0 || f[k] > hi) ok = false;
            }
        }
        if (ok) {
            for (int k = 0; k < 4; ++k) {
                const T b = R_::floor_(f[k]);
                o.tt[k] = R_::sub(f[k], b);
                o.jb[k] = (int32_t)b;
            }
        }
    }
    o.ok = ok;
}

// Plane index of (h, v)-corner c = (c3, c4, c5, c6) bits of a transition.
template <typename T>
__device__ __forceinline__ int32_t corner_plane(const GridT<T>& g, const Transition<T>& t, int c) {
    const int c3 = c & 1, c4 = (c >> 1) & 1, c5 = (c >> 2) & 1, c6 = (c >> 3) & 1;
    const int32_t j3 = (t.jb[0] + c3) % g.n[2];
    const int32_t j4 = min(t.jb[1] + c4, g.n[3] - 1);
    const int32_t j5 = min(t.jb[2] + c5, g.n[4] - 1);
    const int32_t j6 = min(t.jb[3] + c6, g.n[5] - 1);
    return ((j3 * g.n[3] + j4) * g.n[4] + j5) * g.n[5] + j6;
}

// The (h, v)-corner weight product w3*w4*w5*w6 of corner c.
template <typename T>
__device__ __forceinline__ T corner_weight(const Transition<T>& t, int c) {
    const T w3 = (c & 1) ? t.tt[0] : (T)1 - t.tt[0];
    const T w4 = ((c >> 1) & 1) ? t.tt[1] : (T)1 - t.tt[1];
    const T w5 = ((c >> 2) & 1) ? t.tt[2] : (T)1 - t.tt[2];
    const T w6 = ((c >> 3) & 1) ? t.tt[3] : (T)1 - t.tt[3];
    return w3 * w4 * w5 * w6;
}
