/*
 * pg_oracle.c -- TEST INFRASTRUCTURE ONLY (see pg_oracle.h).
 *
 * Plain-C restatement of the reference solver's hot path.  Each function
 * names the reference lines it follows.  Compiled with -ffp-contract=off:
 * Julia does not contract a*b+c on the CPU, so neither may this.
 */
#include "pg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NAN32 (__builtin_nanf(""))

/* Julia's Float32 sin/cos/tanh evaluate in Float64 and round once. */
static inline void og_sincos(float x, float* s, float* c) {
    *s = (float)sin((double)x);
    *c = (float)cos((double)x);
}
static inline float og_tanh(float x) { return (float)tanh((double)x); }

/* Julia min/max/clamp on non-NaN Float32. */
static inline float fminj(float a, float b) { return b < a ? b : a; }
static inline float fmaxj(float a, float b) { return b > a ? b : a; }
static inline float clampj(float x, float lo, float hi) {
    return x > hi ? hi : (x < lo ? lo : x);
}
static inline int32_t imin(int32_t a, int32_t b) { return a < b ? a : b; }
static inline int32_t imax(int32_t a, int32_t b) { return a > b ? a : b; }
/* Julia round(x) = RoundNearest, ties to even */
static inline float roundj(float x) { return nearbyintf(x); }

/* ------------------------------------------------------------------ */
/* Grid (PeregrineSolver.jl:47-81)                                     */
/* ------------------------------------------------------------------ */
void og_grid_make(og_grid* g, const int32_t n[6], const double lo[6], const double hi[6]) {
    for (int k = 0; k < 6; ++k) {
        g->n[k] = n[k];
        if (k == 2) {
            g->step[k] = (float)(6.283185307179586 / (double)n[k]);
            g->lo[k] = (float)(-3.141592653589793);
        } else {
            g->step[k] = (float)((hi[k] - lo[k]) / (double)(n[k] - 1));
            g->lo[k] = (float)lo[k];
        }
    }
}

static inline float axisvalue(const og_grid* g, int k, int32_t i) {
    return g->lo[k] + (float)i * g->step[k];
}

static inline int64_t ncells(const og_grid* g) {
    int64_t c = 1;
    for (int k = 0; k < 6; ++k) c *= (int64_t)g->n[k];
    return c;
}

static inline int64_t flatten(const og_grid* g, int32_t i1, int32_t i2, int32_t i3,
                              int32_t i4, int32_t i5, int32_t i6) {
    const int32_t* n = g->n;
    return (((((int64_t)i1 * n[1] + i2) * n[2] + i3) * n[3] + i4) * n[4] + i5) * n[5] + i6;
}

static inline void unflatten(const og_grid* g, int64_t idx, int32_t* s) {
    for (int k = 5; k >= 1; --k) {
        s[k] = (int32_t)(idx % (int64_t)g->n[k]);
        idx /= (int64_t)g->n[k];
    }
    s[0] = (int32_t)idx;
}

/* ------------------------------------------------------------------ */
/* Model (PeregrineSolver.jl:117-171)                                  */
/* ------------------------------------------------------------------ */
static inline float csign(float v, float e) { return clampj(v / e, -1.0f, 1.0f); }

float og_traction_gain(float u1, float u2, float u3, float knee) {
    if (isnan(knee) || knee <= 0.0f) return 1.0f;
    float m = sqrtf(u1 * u1 + u2 * u2 + u3 * u3);
    float r = m / knee;
    if (r < 1.0e-6f) return 1.0f;
    return og_tanh(r) / r;
}

static inline void saturate(const og_model* m, float u1r, float u2r, float u3r, float* u) {
    float gn = og_traction_gain(u1r, u2r, u3r, m->knee);
    u[0] = u1r * gn;
    u[1] = u2r * gn;
    u[2] = u3r * gn;
}

static inline void body_accel_sat(const og_model* m, float u1, float u2, float u3,
                                  float vx, float vy, float w, float* a) {
    const float* B = m->B; const float* A = m->A; const float* q = m->q;
    const float* S = m->S; const float* D = m->D; const float* c = m->c;
    const float* e = m->eps;
    float w2 = w * w;
    float sx = csign(vx, e[0]), sy = csign(vy, e[1]), sw = csign(w, e[2]);
    float dx = fabsf(vx) * vx, dy = fabsf(vy) * vy, dw = fabsf(w) * w;
    for (int r = 0; r < 3; ++r) {
        const int o = 3 * r;
        float s = B[o] * u1;
        s = s + B[o + 1] * u2;
        s = s + B[o + 2] * u3;
        s = s + A[o] * vx;
        s = s + A[o + 1] * vy;
        s = s + A[o + 2] * w;
        s = s + q[r] * w2;
        s = s + S[o] * sx;
        s = s + S[o + 1] * sy;
        s = s + S[o + 2] * sw;
        s = s + D[o] * dx;
        s = s + D[o + 1] * dy;
        s = s + D[o + 2] * dw;
        s = s + c[r];
        a[r] = s;
    }
}

void og_body_accel(const og_model* m, float u1r, float u2r, float u3r, float vx,
                   float vy, float w, float out[3]) {
    float u[3];
    saturate(m, u1r, u2r, u3r, u);
    body_accel_sat(m, u[0], u[1], u[2], vx, vy, w, out);
}

/* PeregrineSolver.jl:191-192 */
static inline int diverged(float x, float y, float h, float vx, float vy, float w) {
    return !isfinite(x + y + h + vx + vy + w);
}

static const og_state NANSTATE = {NAN32, NAN32, NAN32, NAN32, NAN32, NAN32};

/* PeregrineSolver.jl:203-223 */
og_state og_step_state(const og_model* m, og_state s, float u1r, float u2r, float u3r,
                       float dt, int32_t nsub) {
    float hs = dt / (float)nsub;
    float u[3];
    saturate(m, u1r, u2r, u3r, u);
    float x = s.x, y = s.y, h = s.h, vx = s.vx, vy = s.vy, w = s.w;
    for (int32_t k = 0; k < nsub; ++k) {
        if (diverged(x, y, h, vx, vy, w)) return NANSTATE;
        float a[3];
        body_accel_sat(m, u[0], u[1], u[2], vx, vy, w, a);
        float dvx = a[0] + w * vy;
        float dvy = a[1] - w * vx;
        float sh, ch;
        og_sincos(h, &sh, &ch);
        x += (ch * vx - sh * vy) * hs;
        y += (sh * vx + ch * vy) * hs;
        h += w * hs;
        vx += dvx * hs;
        vy += dvy * hs;
        w += a[2] * hs;
    }
    og_state r = {x, y, h, vx, vy, w};
    return r;
}

/* PeregrineSolver.jl:226-235 */
static inline void state_deriv(const og_model* m, float h, float vx, float vy, float w,
                               const float* u, float* d) {
    float a[3];
    body_accel_sat(m, u[0], u[1], u[2], vx, vy, w, a);
    float sh, ch;
    og_sincos(h, &sh, &ch);
    d[0] = ch * vx - sh * vy;
    d[1] = sh * vx + ch * vy;
    d[2] = w;
    d[3] = a[0] + w * vy;
    d[4] = a[1] - w * vx;
    d[5] = a[2];
}

/* PeregrineSolver.jl:254-279 */
og_state og_step_state_rk2(const og_model* m, og_state s, float u1r, float u2r,
                           float u3r, float dt, int32_t nsub) {
    float hs = dt / (float)nsub;
    float hh = 0.5f * hs;
    float u[3];
    saturate(m, u1r, u2r, u3r, u);
    float x = s.x, y = s.y, h = s.h, vx = s.vx, vy = s.vy, w = s.w;
    for (int32_t k = 0; k < nsub; ++k) {
        if (diverged(x, y, h, vx, vy, w)) return NANSTATE;
        float d1[6], d2[6];
        state_deriv(m, h, vx, vy, w, u, d1);
        float mx = x + d1[0] * hh, my = y + d1[1] * hh, mh = h + d1[2] * hh;
        float mvx = vx + d1[3] * hh, mvy = vy + d1[4] * hh, mw = w + d1[5] * hh;
        if (diverged(mx, my, mh, mvx, mvy, mw)) return NANSTATE;
        state_deriv(m, mh, mvx, mvy, mw, u, d2);
        x += d2[0] * hs;
        y += d2[1] * hs;
        h += d2[2] * hs;
        vx += d2[3] * hs;
        vy += d2[4] * hs;
        w += d2[5] * hs;
    }
    og_state r = {x, y, h, vx, vy, w};
    return r;
}

/* ------------------------------------------------------------------ */
/* Control set (PeregrineSolver.jl:318-346)                            */
/* ------------------------------------------------------------------ */
typedef struct { float u[3]; float l1, l2; int ord; } og_ctl;

static int ctl_cmp(const void* pa, const void* pb) {
    const og_ctl* a = (const og_ctl*)pa;
    const og_ctl* b = (const og_ctl*)pb;
    if (a->l1 < b->l1) return -1;
    if (a->l1 > b->l1) return 1;
    if (a->l2 < b->l2) return -1;
    if (a->l2 > b->l2) return 1;
    return a->ord - b->ord; /* stable */
}

int og_control_set(int level, float* out, int max) {
    if (level < 1) return -1;
    int cap = 1 + 8 * (level + 1) * (level + 2) / 2;
    og_ctl* v = (og_ctl*)calloc((size_t)cap, sizeof(og_ctl));
    int n = 0;
    v[n].u[0] = v[n].u[1] = v[n].u[2] = 0.0f;
    v[n].ord = n;
    n++;
    const int sg[2] = {-1, 1};
    float L = (float)level;
    for (int a0 = 0; a0 < 2; ++a0)
        for (int b0 = 0; b0 < 2; ++b0)
            for (int c0 = 0; c0 < 2; ++c0)
                for (int i = 0; i <= level; ++i)
                    for (int j = 0; j <= level - i; ++j) {
                        int k = level - i - j;
                        float a = (float)i / L, b = (float)j / L, c = (float)k / L;
                        float p0 = a == 0.0f ? 0.0f : (float)sg[a0] * a;
                        float p1 = b == 0.0f ? 0.0f : (float)sg[b0] * b;
                        float p2 = c == 0.0f ? 0.0f : (float)sg[c0] * c;
                        int seen = 0;
                        for (int t = 0; t < n; ++t)
                            if (v[t].u[0] == p0 && v[t].u[1] == p1 && v[t].u[2] == p2) {
                                seen = 1;
                                break;
                            }
                        if (!seen) {
                            v[n].u[0] = p0; v[n].u[1] = p1; v[n].u[2] = p2;
                            v[n].ord = n;
                            n++;
                        }
                    }
    for (int t = 0; t < n; ++t) {
        float* u = v[t].u;
        v[t].l1 = fabsf(u[0]) + fabsf(u[1]) + fabsf(u[2]);
        v[t].l2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    }
    qsort(v, (size_t)n, sizeof(og_ctl), ctl_cmp);
    if (n > max) { free(v); return -n; }
    for (int t = 0; t < n; ++t) {
        out[t] = v[t].u[0];
        out[t + n] = v[t].u[1];
        out[t + 2 * n] = v[t].u[2];
    }
    free(v);
    return n;
}

/* ------------------------------------------------------------------ */
/* Escape views (PeregrineSolver.jl:807-882)                           */
/* ------------------------------------------------------------------ */
typedef struct {
    const float* V;
    const uint8_t* occ;
    int64_t blk;
    float cap;
    int esc;
    int ignore;
} vview;

static inline float vget(const vview* vv, int64_t i) {
    if (!vv->esc) return vv->V[i];
    if (!vv->ignore && vv->occ[i / vv->blk]) return vv->cap;
    float v = vv->V[i];
    return v < 0.0f ? -v : (v < vv->cap ? 0.0f : vv->cap);
}

/* ------------------------------------------------------------------ */
/* Interpolation (PeregrineSolver.jl:399-466, 571-665)                 */
/* ------------------------------------------------------------------ */
static float interp_v(const vview* vv, const og_grid* g, og_state s, int nearest,
                      float cap, int vclamp) {
    float f1 = (s.x - g->lo[0]) / g->step[0];
    float f2 = (s.y - g->lo[1]) / g->step[1];
    float n3 = (float)g->n[2];
    float f3 = (s.h - g->lo[2]) / g->step[2];
    f3 = f3 - floorf(f3 / n3) * n3;
    float f4 = (s.vx - g->lo[3]) / g->step[3];
    float f5 = (s.vy - g->lo[4]) / g->step[4];
    float f6 = (s.w - g->lo[5]) / g->step[5];
    if (!(isfinite(f1) && isfinite(f2) && isfinite(f3) && isfinite(f4) && isfinite(f5) &&
          isfinite(f6)))
        return cap;
    if (f1 < 0.0f || f1 > (float)(g->n[0] - 1)) return cap;
    if (f2 < 0.0f || f2 > (float)(g->n[1] - 1)) return cap;
    if (vclamp) {
        f4 = clampj(f4, 0.0f, (float)(g->n[3] - 1));
        f5 = clampj(f5, 0.0f, (float)(g->n[4] - 1));
        f6 = clampj(f6, 0.0f, (float)(g->n[5] - 1));
    } else {
        if (f4 < 0.0f || f4 > (float)(g->n[3] - 1)) return cap;
        if (f5 < 0.0f || f5 > (float)(g->n[4] - 1)) return cap;
        if (f6 < 0.0f || f6 > (float)(g->n[5] - 1)) return cap;
    }
    if (nearest) {
        int32_t i1 = (int32_t)roundj(f1), i2 = (int32_t)roundj(f2);
        int32_t i3 = ((int32_t)roundj(f3)) % g->n[2];
        int32_t i4 = (int32_t)roundj(f4), i5 = (int32_t)roundj(f5), i6 = (int32_t)roundj(f6);
        return vget(vv, flatten(g, i1, i2, i3, i4, i5, i6));
    }
    float b1 = floorf(f1), b2 = floorf(f2), b3 = floorf(f3);
    float b4 = floorf(f4), b5 = floorf(f5), b6 = floorf(f6);
    float t1 = f1 - b1, t2 = f2 - b2, t3 = f3 - b3, t4 = f4 - b4, t5 = f5 - b5, t6 = f6 - b6;
    int32_t i1 = (int32_t)b1, i2 = (int32_t)b2, i3 = (int32_t)b3;
    int32_t i4 = (int32_t)b4, i5 = (int32_t)b5, i6 = (int32_t)b6;
    float acc = 0.0f;
    for (int d = 0; d < 64; ++d) {
        int c1 = d & 1, c2 = (d >> 1) & 1, c3 = (d >> 2) & 1;
        int c4 = (d >> 3) & 1, c5 = (d >> 4) & 1, c6 = (d >> 5) & 1;
        float wgt = (c1 ? t1 : 1.0f - t1);
        wgt = wgt * (c2 ? t2 : 1.0f - t2);
        wgt = wgt * (c3 ? t3 : 1.0f - t3);
        wgt = wgt * (c4 ? t4 : 1.0f - t4);
        wgt = wgt * (c5 ? t5 : 1.0f - t5);
        wgt = wgt * (c6 ? t6 : 1.0f - t6);
        if (wgt == 0.0f) continue;
        int32_t j1 = imin(i1 + c1, g->n[0] - 1);
        int32_t j2 = imin(i2 + c2, g->n[1] - 1);
        int32_t j3 = (i3 + c3) % g->n[2];
        int32_t j4 = imin(i4 + c4, g->n[3] - 1);
        int32_t j5 = imin(i5 + c5, g->n[4] - 1);
        int32_t j6 = imin(i6 + c6, g->n[5] - 1);
        acc += wgt * vget(vv, flatten(g, j1, j2, j3, j4, j5, j6));
    }
    return fminj(acc, cap);
}

float og_interp(const float* V, const og_grid* g, og_state s, int nearest, float cap,
                int vclamp) {
    vview vv = {V, NULL, 1, cap, 0, 1};
    return interp_v(&vv, g, s, nearest, cap, vclamp);
}

static inline void cmpx(float* ta, int32_t* ka, float* tb, int32_t* kb) {
    if (!(*ta >= *tb)) {
        float t = *ta; *ta = *tb; *tb = t;
        int32_t k = *ka; *ka = *kb; *kb = k;
    }
}

static inline void bump(const og_grid* g, int32_t* i, int32_t k) {
    /* k is 1-based as in the reference */
    if (k == 3) i[2] = (i[2] + 1) % g->n[2];
    else i[k - 1] = imin(i[k - 1] + 1, g->n[k - 1] - 1);
}

static float interp_kuhn_v(const vview* vv, const og_grid* g, og_state s, float cap,
                           int vclamp, float* grad) {
    float f1 = (s.x - g->lo[0]) / g->step[0];
    float f2 = (s.y - g->lo[1]) / g->step[1];
    float n3 = (float)g->n[2];
    float f3 = (s.h - g->lo[2]) / g->step[2];
    f3 = f3 - floorf(f3 / n3) * n3;
    float f4 = (s.vx - g->lo[3]) / g->step[3];
    float f5 = (s.vy - g->lo[4]) / g->step[4];
    float f6 = (s.w - g->lo[5]) / g->step[5];
    if (grad) for (int k = 0; k < 6; ++k) grad[k] = 0.0f;
    if (!(isfinite(f1) && isfinite(f2) && isfinite(f3) && isfinite(f4) && isfinite(f5) &&
          isfinite(f6)))
        return cap;
    if (f1 < 0.0f || f1 > (float)(g->n[0] - 1)) return cap;
    if (f2 < 0.0f || f2 > (float)(g->n[1] - 1)) return cap;
    if (vclamp) {
        f4 = clampj(f4, 0.0f, (float)(g->n[3] - 1));
        f5 = clampj(f5, 0.0f, (float)(g->n[4] - 1));
        f6 = clampj(f6, 0.0f, (float)(g->n[5] - 1));
    } else {
        if (f4 < 0.0f || f4 > (float)(g->n[3] - 1)) return cap;
        if (f5 < 0.0f || f5 > (float)(g->n[4] - 1)) return cap;
        if (f6 < 0.0f || f6 > (float)(g->n[5] - 1)) return cap;
    }
    float b1 = floorf(f1), b2 = floorf(f2), b3 = floorf(f3);
    float b4 = floorf(f4), b5 = floorf(f5), b6 = floorf(f6);
    int32_t idx[6] = {(int32_t)b1, (int32_t)b2, ((int32_t)b3) % g->n[2],
                      (int32_t)b4, (int32_t)b5, (int32_t)b6};
    float t[6] = {f1 - b1, f2 - b2, f3 - b3, f4 - b4, f5 - b5, f6 - b6};
    int32_t k[6] = {1, 2, 3, 4, 5, 6};
    /* sort6_desc, PeregrineSolver.jl:481-497 */
    cmpx(&t[0], &k[0], &t[5], &k[5]);
    cmpx(&t[1], &k[1], &t[3], &k[3]);
    cmpx(&t[2], &k[2], &t[4], &k[4]);
    cmpx(&t[1], &k[1], &t[2], &k[2]);
    cmpx(&t[3], &k[3], &t[4], &k[4]);
    cmpx(&t[0], &k[0], &t[3], &k[3]);
    cmpx(&t[2], &k[2], &t[5], &k[5]);
    cmpx(&t[0], &k[0], &t[1], &k[1]);
    cmpx(&t[2], &k[2], &t[3], &k[3]);
    cmpx(&t[4], &k[4], &t[5], &k[5]);
    cmpx(&t[1], &k[1], &t[2], &k[2]);
    cmpx(&t[3], &k[3], &t[4], &k[4]);
    float v0 = vget(vv, flatten(g, idx[0], idx[1], idx[2], idx[3], idx[4], idx[5]));
    float acc = (1.0f - t[0]) * v0;
    float prev = v0;
    float e[6];
    for (int q = 0; q < 6; ++q) {
        bump(g, idx, k[q]);
        float v = vget(vv, flatten(g, idx[0], idx[1], idx[2], idx[3], idx[4], idx[5]));
        float wq = q < 5 ? t[q] - t[q + 1] : t[5];
        acc += wq * v;
        e[q] = (v - prev) / g->step[k[q] - 1];
        prev = v;
    }
    if (grad) {
        for (int ax = 1; ax <= 6; ++ax) {
            int q = 5;
            for (int r = 0; r < 5; ++r)
                if (k[r] == ax) { q = r; break; }
            grad[ax - 1] = e[q];
        }
    }
    return fminj(acc, cap);
}

float og_interp_kuhn(const float* V, const og_grid* g, og_state s, float cap, int vclamp,
                     float grad[6]) {
    vview vv = {V, NULL, 1, cap, 0, 1};
    return interp_kuhn_v(&vv, g, s, cap, vclamp, grad);
}

static inline float value_at(const vview* vv, const og_grid* g, og_state s,
                             const og_params* p) {
    if (p->simplex) return interp_kuhn_v(vv, g, s, p->cap, p->vclamp, NULL);
    return interp_v(vv, g, s, p->nearest, p->cap, p->vclamp);
}

/* ------------------------------------------------------------------ */
/* Horizon (PeregrineSolver.jl:954-989)                                */
/* ------------------------------------------------------------------ */
float og_cfl_tau(const og_grid* g, const og_model* m, float vfx, float vfy, float w,
                 const og_params* p) {
    if (p->cfl <= 0.0f) return p->dt;
    const float* B = m->B;
    float ax = fmaxj(fmaxj(fabsf(B[0]), fabsf(B[1])), fabsf(B[2]));
    float ay = fmaxj(fmaxj(fabsf(B[3]), fabsf(B[4])), fabsf(B[5]));
    float aw = fmaxj(fmaxj(fabsf(B[6]), fabsf(B[7])), fabsf(B[8]));
    float t = p->tau_max;
    if (ax > 1.0e-6f) t = fminj(t, p->cfl * g->step[3] / ax);
    if (ay > 1.0e-6f) t = fminj(t, p->cfl * g->step[4] / ay);
    if (aw > 1.0e-6f) t = fminj(t, p->cfl * g->step[5] / aw);
    float sp = sqrtf(vfx * vfx + vfy * vfy);
    if (sp > 1.0e-3f) t = fminj(t, p->cfl * fminj(g->step[0], g->step[1]) / sp);
    float aw2 = fabsf(w);
    if (aw2 > 1.0e-4f) t = fminj(t, p->cfl * g->step[2] / aw2);
    return clampj(t, p->tau_min, p->tau_max);
}

int32_t og_substeps_for(float tau, const og_params* p) {
    if (p->hmax <= 0.0f) return p->nsub;
    int32_t k = (int32_t)fminj(tau / p->hmax, 1.0e4f) + 1;
    return imax(1, imin(k, 64));
}

/* ------------------------------------------------------------------ */
/* lookahead (PeregrineSolver.jl:1100-1153)                            */
/* ------------------------------------------------------------------ */
static float lookahead_v(const vview* vv, const uint8_t* occ, int occ_ignore,
                         const og_grid* g, const og_model* m, og_state s, float u1,
                         float u2, float u3, float tau, int32_t nsub, const og_params* p) {
    og_state ns = p->rk2 ? og_step_state_rk2(m, s, u1, u2, u3, tau, nsub)
                         : og_step_state(m, s, u1, u2, u3, tau, nsub);
    float dx = ns.x - s.x, dy = ns.y - s.y, dh = ns.h - s.h;
    if (!(isfinite(dx) && isfinite(dy) && isfinite(dh) && isfinite(ns.vx) &&
          isfinite(ns.vy) && isfinite(ns.w)))
        return p->cap;
    int32_t nchk = p->checks;
    if (p->adaptive_checks) {
        float cells_pos = sqrtf(dx * dx + dy * dy) / (0.5f * fminj(g->step[0], g->step[1]));
        float cells_rot = fabsf(dh) / (0.5f * g->step[2]);
        float cells = fminj(fmaxj(cells_pos, cells_rot), 1.0e4f);
        int32_t need = (int32_t)cells + 1;
        nchk = imax(p->checks, imin(need, 24));
    }
    for (int32_t sc = 1; sc <= nchk; ++sc) {
        float a = (float)sc / (float)nchk;
        float px = s.x + dx * a;
        float py = s.y + dy * a;
        float ph = s.h + dh * a;
        float gx = (px - g->lo[0]) / g->step[0];
        float gy = (py - g->lo[1]) / g->step[1];
        if (gx < 0.0f || gy < 0.0f || gx > (float)(g->n[0] - 1) || gy > (float)(g->n[1] - 1))
            return p->cap;
        float n3f = (float)g->n[2];
        float gh = (ph - g->lo[2]) / g->step[2];
        gh = gh - floorf(gh / n3f) * n3f;
        int32_t ci = (int32_t)roundj(gx), cj = (int32_t)roundj(gy);
        int32_t ck = ((int32_t)roundj(gh)) % g->n[2];
        if (!occ_ignore && occ[((int64_t)ci * g->n[1] + cj) * g->n[2] + ck]) return p->cap;
    }
    float snh, cnh;
    og_sincos(ns.h, &snh, &cnh);
    og_state q = ns;
    q.vx = cnh * ns.vx - snh * ns.vy;
    q.vy = snh * ns.vx + cnh * ns.vy;
    float nv = value_at(vv, g, q, p);
    return fminj(tau + nv, p->cap);
}

float og_lookahead(const float* V, const uint8_t* occ, const og_grid* g, const og_model* m,
                   og_state s, float u1, float u2, float u3, float tau, int32_t nsub,
                   const og_params* p, int esc, int esc_blocked) {
    vview vv = {V, occ, (int64_t)g->n[3] * g->n[4] * g->n[5], p->cap, esc, esc_blocked};
    return lookahead_v(&vv, occ, esc && esc_blocked, g, m, s, u1, u2, u3, tau, nsub, p);
}

/* PeregrineSolver.jl:1165-1170 */
static inline void proj_oct(float u1, float u2, float u3, float* c) {
    float s = fabsf(u1) + fabsf(u2) + fabsf(u3);
    if (s < 1.0e-6f) { c[0] = c[1] = c[2] = 0.0f; return; }
    float r = 1.0f / s;
    c[0] = u1 * r; c[1] = u2 * r; c[2] = u3 * r;
}

/* ------------------------------------------------------------------ */
/* cell_update (PeregrineSolver.jl:1205-1344)                          */
/* ------------------------------------------------------------------ */
float og_cell_update(int64_t idx, const float* V, const uint8_t* occ, const int8_t* pol,
                     const og_grid* g, const og_model* m, const float* ctl, int32_t nctl,
                     const og_params* p, int32_t phase, int esc, float ub[3]) {
    int32_t i[6];
    unflatten(g, idx, i);
    int blocked = occ[((int64_t)i[0] * g->n[1] + i[1]) * g->n[2] + i[2]] != 0;
    vview vv = {V, occ, (int64_t)g->n[3] * g->n[4] * g->n[5], p->cap, esc, blocked};
    int oign = esc && blocked;
    ub[0] = ub[1] = ub[2] = 0.0f;
    if (!esc && blocked) return p->cap;
    og_state s;
    s.x = axisvalue(g, 0, i[0]);
    s.y = axisvalue(g, 1, i[1]);
    s.h = axisvalue(g, 2, i[2]);
    float vfx = axisvalue(g, 3, i[3]);
    float vfy = axisvalue(g, 4, i[4]);
    s.w = axisvalue(g, 5, i[5]);
    float sh0, ch0;
    og_sincos(s.h, &sh0, &ch0);
    s.vx = ch0 * vfx + sh0 * vfy;
    s.vy = (-sh0) * vfx + ch0 * vfy;
    float tau0 = og_cfl_tau(g, m, vfx, vfy, s.w, p);
    int32_t ns0 = og_substeps_for(tau0, p);

    float best = lookahead_v(&vv, occ, oign, g, m, s, 0.0f, 0.0f, 0.0f, tau0, ns0, p);
    float b1 = 0.0f, b2 = 0.0f, b3 = 0.0f;

    if (pol && !esc) {
        const float k127 = 1.0f / 127.0f;
        float q1 = (float)pol[3 * idx] * k127;
        float q2 = (float)pol[3 * idx + 1] * k127;
        float q3 = (float)pol[3 * idx + 2] * k127;
        if (fabsf(q1) + fabsf(q2) + fabsf(q3) > 1.0e-6f) {
            float c = lookahead_v(&vv, occ, oign, g, m, s, q1, q2, q3, tau0, ns0, p);
            if (c < best) { best = c; b1 = q1; b2 = q2; b3 = q3; }
        }
    }

    int32_t nnc = imax(nctl - 1, 1);
    int32_t span = p->ncoarse <= 0 ? nnc : imin(p->ncoarse, nnc);
    int32_t off = p->ncoarse <= 0 ? 0 : (int32_t)(((int64_t)phase * span) % nnc);
    if (off < 0) off += nnc;
    for (int32_t j = 0; j < span; ++j) {
        int32_t k = (int32_t)(((int64_t)off + j) % nnc) + 1;
        float u1 = ctl[k], u2 = ctl[k + nctl], u3 = ctl[k + 2 * nctl];
        float c = lookahead_v(&vv, occ, oign, g, m, s, u1, u2, u3, tau0, ns0, p);
        if (c < best) { best = c; b1 = u1; b2 = u2; b3 = u3; }
    }

    float delta = p->delta0;
    for (int32_t r = 0; r < p->rounds; ++r) {
        for (int32_t d = 1; d <= 6; ++d) {
            float sdl = (d % 2 == 0) ? -delta : delta;
            float e1 = d <= 2 ? sdl : 0.0f;
            float e2 = (d == 3 || d == 4) ? sdl : 0.0f;
            float e3 = d >= 5 ? sdl : 0.0f;
            float cc[3];
            proj_oct(b1 + e1, b2 + e2, b3 + e3, cc);
            if (fabsf(cc[0]) + fabsf(cc[1]) + fabsf(cc[2]) < 1.0e-6f) continue;
            float c = lookahead_v(&vv, occ, oign, g, m, s, cc[0], cc[1], cc[2], tau0, ns0, p);
            if (c < best) { best = c; b1 = cc[0]; b2 = cc[1]; b3 = cc[2]; }
        }
        delta *= 0.5f;
    }

    if (p->ntau > 1) {
        float tau = tau0 * 0.5f;
        for (int32_t k = 1; k <= p->ntau; ++k) {
            if (k != 2) {
                float t = fminj(fmaxj(tau, p->tau_min), p->tau_max);
                float c = lookahead_v(&vv, occ, oign, g, m, s, b1, b2, b3, t,
                                      og_substeps_for(t, p), p);
                if (c < best) best = c;
            }
            tau *= p->tau_ratio;
        }
        if (p->cfl > 0.0f) {
            float t = fminj(fmaxj(p->dt, p->tau_min), p->tau_max);
            float c = lookahead_v(&vv, occ, oign, g, m, s, b1, b2, b3, t,
                                  og_substeps_for(t, p), p);
            if (c < best) best = c;
        }
    }
    ub[0] = b1; ub[1] = b2; ub[2] = b3;
    return best;
}

/* Index of control (u1,u2,u3) in the table, or -1 (only for the argmin
 * report of the plain scheme, where the winner is always a table entry). */
static int16_t ctl_index(const float* ctl, int32_t nctl, const float* u) {
    for (int32_t k = 0; k < nctl; ++k)
        if (ctl[k] == u[0] && ctl[k + nctl] == u[1] && ctl[k + 2 * nctl] == u[2])
            return (int16_t)k;
    return -1;
}

static inline int8_t qpol(float v) {
    /* unsafe_trunc(Int8, round(clamp(v,-1,1)*127)), PeregrineSolver.jl:738 */
    return (int8_t)(int32_t)roundj(clampj(v, -1.0f, 1.0f) * 127.0f);
}

#define OG_CHUNK 4096

/* The sweep over [lo, hi); cell idx's result goes to Vout[idx - out_off]
 * (out_off = 0: a whole-table Vout; out_off = lo: a slab of hi - lo). */
static void sweep_jacobi_impl(const float* Vin, float* Vout, int64_t out_off, const uint8_t* occ,
                              int8_t* pol, const og_grid* g, const og_model* m, const float* ctl,
                              int32_t nctl, const og_params* p, int32_t phase, int64_t lo,
                              int64_t hi, int threads, double* total, double* maxd,
                              int16_t* argmin) {
    int64_t n = hi - lo;
    int64_t nchunk = (n + OG_CHUNK - 1) / OG_CHUNK;
    double* part = (double*)calloc((size_t)(nchunk > 0 ? nchunk : 1), sizeof(double));
    double* partm = (double*)calloc((size_t)(nchunk > 0 ? nchunk : 1), sizeof(double));
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#endif
    for (int64_t cidx = 0; cidx < nchunk; ++cidx) {
        int64_t a = lo + cidx * OG_CHUNK;
        int64_t b = a + OG_CHUNK < hi ? a + OG_CHUNK : hi;
        double s = 0.0, mx = 0.0;
        for (int64_t idx = a; idx < b; ++idx) {
            float ub[3];
            float c = og_cell_update(idx, Vin, occ, pol, g, m, ctl, nctl, p, phase, 0, ub);
            float old = Vin[idx];
            int32_t i3 = (int32_t)((idx / ((int64_t)g->n[3] * g->n[4] * g->n[5])) % g->n[2]);
            int64_t xy = idx / ((int64_t)g->n[2] * g->n[3] * g->n[4] * g->n[5]);
            int blocked = occ[xy * g->n[2] + i3] != 0;
            if (argmin) argmin[idx] = blocked ? (int16_t)-1 : ctl_index(ctl, nctl, ub);
            if (c < old) {
                Vout[idx - out_off] = c;
                if (pol) {
                    pol[3 * idx] = qpol(ub[0]);
                    pol[3 * idx + 1] = qpol(ub[1]);
                    pol[3 * idx + 2] = qpol(ub[2]);
                }
                double d = (double)(old - c);
                s += d;
                if (d > mx) mx = d;
            } else {
                Vout[idx - out_off] = old;
            }
        }
        part[cidx] = s;
        partm[cidx] = mx;
    }
    double t = 0.0, mx = 0.0;
    for (int64_t c = 0; c < nchunk; ++c) {
        t += part[c];
        if (partm[c] > mx) mx = partm[c];
    }
    free(part);
    free(partm);
    if (total) *total = t;
    if (maxd) *maxd = mx;
}

void og_cell_lookaheads(const float* V, const uint8_t* occ, const og_grid* g,
                        const og_model* m, const float* ctl, int32_t nctl,
                        const og_params* p, const int64_t* cells, int64_t n, int threads,
                        float* out) {
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt)
#endif
    for (int64_t c = 0; c < n; ++c) {
        int64_t idx = cells[c];
        float* o = out + c * nctl;
        int32_t i[6];
        unflatten(g, idx, i);
        if (occ[((int64_t)i[0] * g->n[1] + i[1]) * g->n[2] + i[2]]) {
            for (int32_t k = 0; k < nctl; ++k) o[k] = p->cap;
            continue;
        }
        vview vv = {V, occ, (int64_t)g->n[3] * g->n[4] * g->n[5], p->cap, 0, 0};
        og_state s;
        s.x = axisvalue(g, 0, i[0]);
        s.y = axisvalue(g, 1, i[1]);
        s.h = axisvalue(g, 2, i[2]);
        float vfx = axisvalue(g, 3, i[3]);
        float vfy = axisvalue(g, 4, i[4]);
        s.w = axisvalue(g, 5, i[5]);
        float sh0, ch0;
        og_sincos(s.h, &sh0, &ch0);
        s.vx = ch0 * vfx + sh0 * vfy;
        s.vy = (-sh0) * vfx + ch0 * vfy;
        float tau0 = og_cfl_tau(g, m, vfx, vfy, s.w, p);
        int32_t ns0 = og_substeps_for(tau0, p);
        for (int32_t k = 0; k < nctl; ++k)
            o[k] = lookahead_v(&vv, occ, 0, g, m, s, ctl[k], ctl[k + nctl], ctl[k + 2 * nctl],
                               tau0, ns0, p);
    }
}

void og_sweep_jacobi(const float* Vin, float* Vout, const uint8_t* occ, int8_t* pol,
                     const og_grid* g, const og_model* m, const float* ctl, int32_t nctl,
                     const og_params* p, int32_t phase, int64_t lo, int64_t hi, int threads,
                     double* total, double* maxd, int16_t* argmin) {
    sweep_jacobi_impl(Vin, Vout, 0, occ, pol, g, m, ctl, nctl, p, phase, lo, hi, threads, total,
                      maxd, argmin);
}

void og_sweep_jacobi_slab(const float* Vin, float* Vout_slab, const uint8_t* occ,
                          const og_grid* g, const og_model* m, const float* ctl, int32_t nctl,
                          const og_params* p, int32_t phase, int64_t lo, int64_t hi, int threads,
                          double* total, double* maxd) {
    sweep_jacobi_impl(Vin, Vout_slab, lo, occ, NULL, g, m, ctl, nctl, p, phase, lo, hi, threads,
                      total, maxd, NULL);
}

double og_sweep_inplace(float* V, const uint8_t* occ, int8_t* pol, const og_grid* g,
                        const og_model* m, const float* ctl, int32_t nctl,
                        const og_params* p, int32_t phase, int rev) {
    int64_t n = ncells(g);
    double total = 0.0;
    for (int64_t i = 1; i <= n; ++i) {
        int64_t idx = rev ? n - i : i - 1;
        float ub[3];
        float c = og_cell_update(idx, V, occ, pol, g, m, ctl, nctl, p, phase, 0, ub);
        float old = V[idx];
        if (c < old) {
            V[idx] = c;
            if (pol) {
                pol[3 * idx] = qpol(ub[0]);
                pol[3 * idx + 1] = qpol(ub[1]);
                pol[3 * idx + 2] = qpol(ub[2]);
            }
            total += (double)(old - c);
        }
    }
    return total;
}

void og_sweep_escape_jacobi(const float* Vin, float* Vout, const uint8_t* occ,
                            const og_grid* g, const og_model* m, const float* ctl,
                            int32_t nctl, const og_params* p, int32_t phase, int threads,
                            double* total) {
    int64_t n = ncells(g);
    int64_t nchunk = (n + OG_CHUNK - 1) / OG_CHUNK;
    double* part = (double*)calloc((size_t)(nchunk > 0 ? nchunk : 1), sizeof(double));
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#endif
    for (int64_t cidx = 0; cidx < nchunk; ++cidx) {
        int64_t a = cidx * OG_CHUNK;
        int64_t b = a + OG_CHUNK < n ? a + OG_CHUNK : n;
        double s = 0.0;
        for (int64_t idx = a; idx < b; ++idx) {
            float v0 = Vin[idx];
            Vout[idx] = v0;
            if (v0 >= 0.0f && v0 < p->cap) continue; /* is_terminal */
            float e_old = v0 < 0.0f ? -v0 : p->cap;   /* escape_of */
            float ub[3];
            float c = og_cell_update(idx, Vin, occ, NULL, g, m, ctl, nctl, p, phase, 1, ub);
            if (c < e_old) {
                Vout[idx] = -c;
                s += (double)(e_old - c);
            }
        }
        part[cidx] = s;
    }
    double t = 0.0;
    for (int64_t c = 0; c < nchunk; ++c) t += part[c];
    free(part);
    if (total) *total = t;
}

int og_solve_value(float* V, const uint8_t* occ, int8_t* pol, const og_grid* g,
                   const og_model* m, const int64_t* tidx, int64_t ntidx, const float* ctl,
                   int32_t nctl, const og_params* p, int32_t iters, double tol, int stop_rule,
                   int jacobi, int threads, double* last_delta, double* last_maxd) {
    int64_t n = ncells(g);
    for (int64_t i = 0; i < n; ++i) V[i] = p->cap;
    for (int64_t t = 0; t < ntidx; ++t) V[tidx[t]] = 0.0f;
    if (pol) memset(pol, 0, (size_t)(3 * n));
    int quiet_needed = 1;
    if (p->ncoarse > 0) {
        int q = (nctl - 1 + p->ncoarse - 1) / p->ncoarse;
        quiet_needed = q > 1 ? q : 1;
    }
    float* W = jacobi ? (float*)malloc((size_t)n * sizeof(float)) : NULL;
    double d = INFINITY, dm = INFINITY;
    int done = 0, quiet = 0;
    for (int it = 1; it <= iters; ++it) {
        if (jacobi) {
            og_sweep_jacobi(V, W, occ, pol, g, m, ctl, nctl, p, it - 1, 0, n, threads, &d, &dm,
                            NULL);
            memcpy(V, W, (size_t)n * sizeof(float));
        } else {
            d = og_sweep_inplace(V, occ, pol, g, m, ctl, nctl, p, it - 1, it % 2 == 1);
            dm = NAN;
        }
        for (int64_t t = 0; t < ntidx; ++t) V[tidx[t]] = 0.0f;
        done = it;
        double crit = stop_rule == 1 ? dm : d;
        quiet = crit <= tol ? quiet + 1 : 0;
        if (quiet >= quiet_needed) break;
    }
    free(W);
    if (last_delta) *last_delta = d;
    if (last_maxd) *last_maxd = dm;
    return done;
}

/* ------------------------------------------------------------------ */
/* target_cells (Pipeline.jl:504-536)                                  */
/* ------------------------------------------------------------------ */
static inline int64_t fl_i(float x) { return (int64_t)floor((double)x); }
static inline int64_t ce_i(float x) { return (int64_t)ceil((double)x); }

int64_t og_target_cells(const og_grid* g, const float s[6], const float tol[6], int64_t* out,
                        int64_t max) {
    int64_t lo[6], hi[6];
    for (int k = 0; k < 6; ++k) {
        float c = (s[k] - g->lo[k]) / g->step[k];
        if (k == 2) {
            float n3 = (float)g->n[2];
            c = c - floorf(c / n3) * n3;
        }
        float r = tol[k] / g->step[k];
        if (k == 2) {
            lo[k] = ce_i(c - r);
            hi[k] = fl_i(c + r);
        } else {
            int64_t a = ce_i(c - r), b = fl_i(c + r);
            lo[k] = a > 0 ? a : 0;
            hi[k] = b < g->n[k] - 1 ? b : g->n[k] - 1;
        }
    }
    int64_t cnt = 0;
    for (int64_t i1 = lo[0]; i1 <= hi[0]; ++i1)
        for (int64_t i2 = lo[1]; i2 <= hi[1]; ++i2)
            for (int64_t i3 = lo[2]; i3 <= hi[2]; ++i3)
                for (int64_t i4 = lo[3]; i4 <= hi[3]; ++i4)
                    for (int64_t i5 = lo[4]; i5 <= hi[4]; ++i5)
                        for (int64_t i6 = lo[5]; i6 <= hi[5]; ++i6) {
                            int64_t j3 = ((i3 % g->n[2]) + g->n[2]) % g->n[2];
                            int64_t f = flatten(g, (int32_t)i1, (int32_t)i2, (int32_t)j3,
                                                (int32_t)i4, (int32_t)i5, (int32_t)i6);
                            int dup = 0;
                            for (int64_t q = 0; q < cnt && q < max; ++q)
                                if (out[q] == f) { dup = 1; break; }
                            if (dup) continue;
                            if (cnt < max) out[cnt] = f;
                            cnt++;
                        }
    if (cnt == 0) {
        int32_t near[6];
        for (int k = 0; k < 6; ++k) {
            float c = (s[k] - g->lo[k]) / g->step[k];
            int64_t r = (int64_t)nearbyint((double)c);
            if (k == 2) near[k] = (int32_t)(((r % g->n[2]) + g->n[2]) % g->n[2]);
            else near[k] = (int32_t)(r < 0 ? 0 : (r > g->n[k] - 1 ? g->n[k] - 1 : r));
        }
        if (max > 0) out[0] = flatten(g, near[0], near[1], near[2], near[3], near[4], near[5]);
        cnt = 1;
    }
    return cnt <= max ? cnt : -cnt;
}

/* ------------------------------------------------------------------ */
/* Encoding (Pipeline.jl:620-780)                                      */
/* ------------------------------------------------------------------ */
static uint16_t f32_to_f16_bits(float f) {
    /* round to nearest even, IEEE binary16 */
    uint32_t x;
    memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t ax = x & 0x7fffffffu;
    if (ax >= 0x7f800000u) {
        if (ax > 0x7f800000u) return (uint16_t)(sign | 0x7e00u | ((ax >> 13) & 0x3ffu));
        return (uint16_t)(sign | 0x7c00u);
    }
    if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u); /* overflow to inf */
    if (ax < 0x38800000u) {                                    /* subnormal half */
        float af;
        memcpy(&af, &ax, 4);
        /* af * 2^24 rounded to nearest even gives the subnormal mantissa */
        float scaled = af * 16777216.0f;
        uint32_t mant = (uint32_t)nearbyintf(scaled);
        return (uint16_t)(sign | mant);
    }
    uint32_t mant = ax & 0x7fffffu;
    int32_t exp = (int32_t)(ax >> 23) - 127 + 15;
    uint32_t h = ((uint32_t)exp << 10) | (mant >> 13);
    uint32_t rem = mant & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1u;
    return (uint16_t)(sign | h);
}

int og_encode(const float* V, int64_t n, int dtype, double scale, float cap,
              double escape_scale, uint8_t* out, int64_t* reached, int64_t* escaped) {
    /* DTYPES: u8 (sentinel 0xff, escape_base 0xe0), u16 (0xffff, 0xfc00) */
    uint32_t sentinel = dtype == 0 ? 0xffu : 0xffffu;
    uint32_t base = dtype == 0 ? 0xe0u : (dtype == 1 ? 0xfc00u : 0u);
    int64_t codes = base == 0 ? 0 : (int64_t)sentinel - (int64_t)base;
    int hasband = escape_scale > 0.0 && base != 0;
    uint32_t ebase = hasband ? base : (dtype == 0 ? 0xffu : 0xffffu);
    uint32_t ecodes = (uint32_t)(codes > 1 ? codes : 1);
    double einv = escape_scale > 0.0 ? 1.0 / escape_scale : 0.0;
    int64_t r_ = 0, e_ = 0;
    for (int64_t i = 0; i < n; ++i) {
        float v = V[i];
        int isesc = v < 0.0f && isfinite(v);
        int unre = v >= cap || isinf(v) || isnan(v);
        if (dtype == 3 || dtype == 2) {
            int u = !isesc && unre;
            r_ += (!isesc && !u);
            e_ += isesc;
            if (dtype == 3) {
                uint32_t bits;
                if (u) bits = 0x7fc00000u;
                else memcpy(&bits, &v, 4);
                memcpy(out + 4 * i, &bits, 4);
            } else {
                uint16_t hb = u ? (uint16_t)0x7e00u : f32_to_f16_bits(v);
                memcpy(out + 2 * i, &hb, 2);
            }
            continue;
        }
        uint32_t code;
        if (isesc) {
            e_++;
            double e = -(double)v;
            double q = sqrt((e > 0.0 ? e : 0.0) * einv);
            uint32_t rq = (uint32_t)nearbyint(q);
            code = ebase + (rq < ecodes - 1u ? rq : ecodes - 1u);
        } else if (unre) {
            code = sentinel;
        } else {
            r_++;
            uint32_t r = (uint32_t)nearbyint((double)v / scale);
            code = r >= ebase ? sentinel : r;
        }
        if (dtype == 0) out[i] = (uint8_t)code;
        else {
            uint16_t c16 = (uint16_t)code;
            memcpy(out + 2 * i, &c16, 2);
        }
    }
    if (reached) *reached = r_;
    if (escaped) *escaped = e_;
    return 0;
}

/* ------------------------------------------------------------------ */
/* Occupancy (Pipeline.jl:29-399)                                      */
/* ------------------------------------------------------------------ */
static const double EPS64 = 2.220446049250313e-16;

static int inpoly(double px, double py, const double* P, int n) {
    int inside = 0;
    int j = n - 1;
    for (int i = 0; i < n; ++i) {
        double xi = P[2 * i], yi = P[2 * i + 1];
        double xj = P[2 * j], yj = P[2 * j + 1];
        if (((yi > py) != (yj > py)) && (px < (xj - xi) * (py - yi) / (yj - yi + EPS64) + xi))
            inside = !inside;
        j = i;
    }
    return inside;
}

static inline double dcross(const double* a, const double* b, const double* c) {
    return (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0]);
}

static int seg_cross(const double* p1, const double* p2, const double* p3, const double* p4) {
    double d1 = dcross(p3, p4, p1), d2 = dcross(p3, p4, p2);
    double d3 = dcross(p1, p2, p3), d4 = dcross(p1, p2, p4);
    return ((d1 > 0) != (d2 > 0)) && ((d3 > 0) != (d4 > 0));
}

static double pt_seg_dist(const double* p, const double* a, const double* b) {
    double abx = b[0] - a[0], aby = b[1] - a[1];
    double L2 = abx * abx + aby * aby;
    double t = 0.0;
    if (!(L2 <= 0)) {
        t = ((p[0] - a[0]) * abx + (p[1] - a[1]) * aby) / L2;
        t = t > 1.0 ? 1.0 : (t < 0.0 ? 0.0 : t);
    }
    double dx = p[0] - (a[0] + t * abx), dy = p[1] - (a[1] + t * aby);
    return sqrt(dx * dx + dy * dy);
}

static double seg_seg_dist(const double* a1, const double* a2, const double* b1,
                           const double* b2) {
    if (seg_cross(a1, a2, b1, b2)) return 0.0;
    double d = pt_seg_dist(a1, b1, b2);
    double e = pt_seg_dist(a2, b1, b2);
    if (e < d) d = e;
    e = pt_seg_dist(b1, a1, a2);
    if (e < d) d = e;
    e = pt_seg_dist(b2, a1, a2);
    if (e < d) d = e;
    return d;
}

static int polys_overlap(const double* A, int na, const double* B, int nb) {
    for (int i = 0; i < na; ++i)
        if (inpoly(A[2 * i], A[2 * i + 1], B, nb)) return 1;
    for (int j = 0; j < nb; ++j)
        if (inpoly(B[2 * j], B[2 * j + 1], A, na)) return 1;
    for (int i = 0; i < na; ++i)
        for (int j = 0; j < nb; ++j)
            if (seg_cross(A + 2 * i, A + 2 * ((i + 1) % na), B + 2 * j, B + 2 * ((j + 1) % nb)))
                return 1;
    return 0;
}

static int polys_too_close(const double* A, int na, const double* B, int nb, double d) {
    if (polys_overlap(A, na, B, nb)) return 1;
    if (d <= 0) return 0;
    for (int i = 0; i < na; ++i)
        for (int j = 0; j < nb; ++j)
            if (seg_seg_dist(A + 2 * i, A + 2 * ((i + 1) % na), B + 2 * j,
                             B + 2 * ((j + 1) % nb)) < d)
                return 1;
    return 0;
}

static int point_too_close(double px, double py, const double* B, int nb, double d) {
    if (inpoly(px, py, B, nb)) return 1;
    if (d <= 0) return 0;
    double p[2] = {px, py};
    for (int j = 0; j < nb; ++j)
        if (pt_seg_dist(p, B + 2 * j, B + 2 * ((j + 1) % nb)) < d) return 1;
    return 0;
}

static void footprint_reach(int nrobot, const double* robot, double th, double* r) {
    r[0] = r[1] = r[2] = r[3] = 0.0;
    if (!robot || nrobot < 3) return;
    double c = cos(th), s = sin(th);
    double xlo = -INFINITY, xhi = -INFINITY, ylo = -INFINITY, yhi = -INFINITY;
    for (int i = 0; i < nrobot; ++i) {
        double rx = c * robot[2 * i] - s * robot[2 * i + 1];
        double ry = s * robot[2 * i] + c * robot[2 * i + 1];
        if (-rx > xlo) xlo = -rx;
        if (rx > xhi) xhi = rx;
        if (-ry > ylo) ylo = -ry;
        if (ry > yhi) yhi = ry;
    }
    r[0] = xlo; r[1] = xhi; r[2] = ylo; r[3] = yhi;
}

void og_build_occupancy(const og_grid* g, int npoly, const int* nverts, const double* pts,
                        double margin_cm, int nrobot, const double* robot, int substeps,
                        double clearance_cm, const double* bounds, double wall_clearance_cm,
                        uint8_t* out) {
    int nx = g->n[0], ny = g->n[1], nh = g->n[2];
    uint8_t* occ = (uint8_t*)calloc((size_t)nx * ny * nh, 1); /* [i][j][k] */
#define OCC(i, j, k) occ[((size_t)(i) * ny + (j)) * nh + (k)]
    int point_robot = robot == NULL || nrobot < 3;
    double rad = 0.0;
    if (!point_robot)
        for (int i = 0; i < nrobot; ++i) {
            double r = sqrt(robot[2 * i] * robot[2 * i] + robot[2 * i + 1] * robot[2 * i + 1]);
            if (r > rad) rad = r;
        }
    const double tol = 1.0e-3;
    double* angles = (double*)malloc(sizeof(double) * (size_t)(substeps > 1 ? substeps : 1));
    double* Rr = (double*)malloc(sizeof(double) * 2 * (size_t)(nrobot > 0 ? nrobot : 1));
    double* body = (double*)malloc(sizeof(double) * 2 * (size_t)(nrobot > 0 ? nrobot : 1));
    for (int k = 0; k < nh; ++k) {
        double thc = (double)axisvalue(g, 2, k);
        double half = (double)g->step[2] / 2;
        int na = substeps <= 1 ? 1 : substeps;
        if (substeps <= 1) angles[0] = thc;
        else
            for (int s = 1; s <= substeps; ++s)
                angles[s - 1] = thc - half + 2 * half * (s - 1) / (substeps - 1);
        if (bounds) {
            for (int a = 0; a < na; ++a) {
                double r[4];
                footprint_reach(nrobot, robot, angles[a], r);
                double d = wall_clearance_cm;
                double bxlo = bounds[0] + d + r[0], bxhi = bounds[2] - d - r[1];
                double bylo = bounds[1] + d + r[2], byhi = bounds[3] - d - r[3];
                for (int i = 0; i < nx; ++i) {
                    double px = (double)axisvalue(g, 0, i);
                    if (!(px < bxlo - tol || px > bxhi + tol)) continue;
                    for (int j = 0; j < ny; ++j) OCC(i, j, k) = 1;
                }
                for (int j = 0; j < ny; ++j) {
                    double py = (double)axisvalue(g, 1, j);
                    if (!(py < bylo - tol || py > byhi + tol)) continue;
                    for (int i = 0; i < nx; ++i) OCC(i, j, k) = 1;
                }
            }
        }
        for (int a = 0; a < na; ++a) {
            double th = angles[a];
            if (!point_robot) {
                double c = cos(th), s = sin(th);
                for (int i = 0; i < nrobot; ++i) {
                    Rr[2 * i] = c * robot[2 * i] + (-s) * robot[2 * i + 1];
                    Rr[2 * i + 1] = s * robot[2 * i] + c * robot[2 * i + 1];
                }
            }
            const double* P = pts;
            for (int pi = 0; pi < npoly; ++pi) {
                int nv = nverts[pi];
                double pad = rad + margin_cm + clearance_cm;
                double x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY;
                for (int v = 0; v < nv; ++v) {
                    if (P[2 * v] < x0) x0 = P[2 * v];
                    if (P[2 * v] > x1) x1 = P[2 * v];
                    if (P[2 * v + 1] < y0) y0 = P[2 * v + 1];
                    if (P[2 * v + 1] > y1) y1 = P[2 * v + 1];
                }
                x0 -= pad; x1 += pad; y0 -= pad; y1 += pad;
                int64_t i0 = (int64_t)floor((x0 - (double)g->lo[0]) / (double)g->step[0]);
                int64_t i1 = (int64_t)ceil((x1 - (double)g->lo[0]) / (double)g->step[0]);
                int64_t j0 = (int64_t)floor((y0 - (double)g->lo[1]) / (double)g->step[1]);
                int64_t j1 = (int64_t)ceil((y1 - (double)g->lo[1]) / (double)g->step[1]);
                if (i0 < 0) i0 = 0;
                if (j0 < 0) j0 = 0;
                if (i1 > nx - 1) i1 = nx - 1;
                if (j1 > ny - 1) j1 = ny - 1;
                for (int64_t i = i0; i <= i1; ++i)
                    for (int64_t j = j0; j <= j1; ++j) {
                        if (OCC(i, j, k)) continue;
                        double px = (double)axisvalue(g, 0, (int32_t)i);
                        double py = (double)axisvalue(g, 1, (int32_t)j);
                        if (point_robot) {
                            OCC(i, j, k) = (uint8_t)point_too_close(px, py, P, nv, clearance_cm);
                        } else {
                            for (int v = 0; v < nrobot; ++v) {
                                body[2 * v] = Rr[2 * v] + px;
                                body[2 * v + 1] = Rr[2 * v + 1] + py;
                            }
                            OCC(i, j, k) =
                                (uint8_t)polys_too_close(body, nrobot, P, nv, clearance_cm);
                        }
                    }
                P += 2 * nv;
            }
        }
    }
    if (margin_cm > 0) {
        int64_t rx = (int64_t)ceil(margin_cm / (double)g->step[0]);
        int64_t ry = (int64_t)ceil(margin_cm / (double)g->step[1]);
        if (rx < 0) rx = 0;
        if (ry < 0) ry = 0;
        if (rx > 0 || ry > 0) {
            uint8_t* src = (uint8_t*)malloc((size_t)nx * ny * nh);
            memcpy(src, occ, (size_t)nx * ny * nh);
            for (int k = 0; k < nh; ++k)
                for (int i = 0; i < nx; ++i)
                    for (int j = 0; j < ny; ++j) {
                        if (!src[((size_t)i * ny + j) * nh + k]) continue;
                        for (int64_t di = -rx; di <= rx; ++di)
                            for (int64_t dj = -ry; dj <= ry; ++dj) {
                                int64_t ii = i + di, jj = j + dj;
                                if (ii < 0 || ii >= nx || jj < 0 || jj >= ny) continue;
                                OCC(ii, jj, k) = 1;
                            }
                    }
            free(src);
        }
    }
    memcpy(out, occ, (size_t)nx * ny * nh);
#undef OCC
    free(occ);
    free(angles);
    free(Rr);
    free(body);
}
