/*
 * pg_oracle_grad.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU FP64 reference for the gradient of a loss on the converged value
 * table with respect to the drivetrain model, built independently of the
 * CUDA adjoint: the successor's derivative comes from central differences of
 * an FP64 integration (the device uses forward-mode dual numbers), the
 * interpolation is evaluated in FP64, and the adjoint system
 * lambda = c + P^T lambda is iterated in FP64.  It takes the table and its
 * policy as given (the GPU solve's), so it checks the adjoint, not the
 * forward solve.  The reference solver never differentiates its tables;
 * the dynamics it differentiates are PeregrineSolver.jl:126-171 (traction,
 * body acceleration), 203-279 (Euler / RK2 substeps) and the interpolation
 * PeregrineSolver.jl:399-466.
 *
 * theta = (B00 B11 B22, A00 A11 A22, q0 q1 q2, S00 S11 S22, D00 D11 D22,
 * c0 c1 c2).  Arrays are row-major (omega fastest), as everywhere in the
 * oracle.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "pg_oracle.h"

#define NTH 18

typedef struct {
    double B[9], A[9], q[3], S[9], D[9], c[3], eps[3], knee;
} m64;

static double* theta_ptr(m64* m, int k) {
    const int blk = k / 3, r = k % 3;
    switch (blk) {
        case 0: return &m->B[4 * r];
        case 1: return &m->A[4 * r];
        case 2: return &m->q[r];
        case 3: return &m->S[4 * r];
        case 4: return &m->D[4 * r];
        default: return &m->c[r];
    }
}

static double csign64(double v, double e) {
    double q = v / e;
    return q > 1.0 ? 1.0 : (q < -1.0 ? -1.0 : q);
}

static void accel64(const m64* m, const double u[3], double vx, double vy, double w,
                    double a[3]) {
    const double v[3] = {vx, vy, w};
    const double sg[3] = {csign64(vx, m->eps[0]), csign64(vy, m->eps[1]), csign64(w, m->eps[2])};
    for (int r = 0; r < 3; ++r) {
        double s = 0.0;
        for (int c = 0; c < 3; ++c) s += m->B[3 * r + c] * u[c];
        for (int c = 0; c < 3; ++c) s += m->A[3 * r + c] * v[c];
        s += m->q[r] * w * w;
        for (int c = 0; c < 3; ++c) s += m->S[3 * r + c] * sg[c];
        for (int c = 0; c < 3; ++c) s += m->D[3 * r + c] * fabs(v[c]) * v[c];
        s += m->c[r];
        a[r] = s;
    }
}

/* successor in interpolation coordinates: x, y offsets, heading,
 * field-frame velocity, turn rate; 0 on divergence */
static int succ64(const m64* m, int rk2, double h0, double vfx, double vfy, double w0,
                  const double ur[3], double tau, int nsub, double out[6]) {
    double gn = 1.0;
    if (!(isnan(m->knee) || m->knee <= 0.0)) {
        const double mg = sqrt(ur[0] * ur[0] + ur[1] * ur[1] + ur[2] * ur[2]);
        const double r = mg / m->knee;
        if (r >= 1.0e-6) gn = tanh(r) / r;
    }
    const double u[3] = {ur[0] * gn, ur[1] * gn, ur[2] * gn};
    double x = 0.0, y = 0.0, h = h0, w = w0;
    double vx = cos(h0) * vfx + sin(h0) * vfy, vy = -sin(h0) * vfx + cos(h0) * vfy;
    const double hs = tau / nsub, hh = 0.5 * hs;
    for (int k = 0; k < nsub; ++k) {
        double a[3];
        accel64(m, u, vx, vy, w, a);
        const double ch = cos(h), sh = sin(h);
        const double d1x = ch * vx - sh * vy, d1y = sh * vx + ch * vy;
        const double d1vx = a[0] + w * vy, d1vy = a[1] - w * vx;
        if (!rk2) {
            x += d1x * hs; y += d1y * hs; h += w * hs;
            vx += d1vx * hs; vy += d1vy * hs; w += a[2] * hs;
        } else {
            const double mh = h + w * hh, mvx = vx + d1vx * hh, mvy = vy + d1vy * hh;
            const double mw = w + a[2] * hh;
            accel64(m, u, mvx, mvy, mw, a);
            const double c2 = cos(mh), s2 = sin(mh);
            x += (c2 * mvx - s2 * mvy) * hs;
            y += (s2 * mvx + c2 * mvy) * hs;
            h += mw * hs;
            vx += (a[0] + mw * mvy) * hs;
            vy += (a[1] - mw * mvx) * hs;
            w += a[2] * hs;
        }
        if (!isfinite(x + y + h + vx + vy + w)) return 0;
    }
    out[0] = x;
    out[1] = y;
    out[2] = h;
    out[3] = cos(h) * vx - sin(h) * vy;
    out[4] = sin(h) * vx + cos(h) * vy;
    out[5] = w;
    return 1;
}

typedef struct {
    int ok;
    double s[6];
    double d[6][NTH];
} pair64;

static double axv(const og_grid* g, int k, int i) { return (double)g->lo[k] + (double)g->step[k] * i; }

/* Per active cell: the lower corner and fractions of its successor on the
 * 6 axes; the row's 64 corners and weights are rebuilt from them in every
 * adjoint sweep (storing them would take 64 entries per cell). */
typedef struct {
    int64_t cell;
    int32_t ib[6];
    double t[6];
} row64;

static void corners(const og_grid* g, const row64* r, int d, int64_t* idx, double* w) {
    const int32_t* n = g->n;
    int32_t j[6];
    double ww = 1.0;
    for (int ax = 0; ax < 6; ++ax) {
        const int bit = (d >> ax) & 1;
        ww *= bit ? r->t[ax] : 1.0 - r->t[ax];
        if (ax == 2) j[ax] = (r->ib[ax] + bit) % n[2];
        else j[ax] = r->ib[ax] + bit < n[ax] - 1 ? r->ib[ax] + bit : n[ax] - 1;
    }
    *idx = (((((int64_t)j[0] * n[1] + j[1]) * n[2] + j[2]) * n[3] + j[3]) * n[4] + j[4]) * n[5] + j[5];
    *w = ww;
}

int og_adjoint_grad_f64(const double* V, const int16_t* pol, const uint8_t* occ, const og_grid* g,
                        const og_model* mf, const float* ctl, int32_t nctl, const og_params* p,
                        const double* c, int32_t iters, double tol, int threads, double* grad,
                        int32_t* iters_done, int64_t* nactive) {
    const int32_t* n = g->n;
    const int64_t ncells = (int64_t)n[0] * n[1] * n[2] * n[3] * n[4] * n[5];
    const int64_t nplanes = (int64_t)n[2] * n[3] * n[4] * n[5];
    const double cap = p->cap;
    const double tau = p->dt;  /* plain scheme: one horizon dt */
    m64 m0;
    for (int k = 0; k < 9; ++k) {
        m0.B[k] = mf->B[k]; m0.A[k] = mf->A[k]; m0.S[k] = mf->S[k]; m0.D[k] = mf->D[k];
    }
    for (int k = 0; k < 3; ++k) { m0.q[k] = mf->q[k]; m0.c[k] = mf->c[k]; m0.eps[k] = mf->eps[k]; }
    m0.knee = mf->knee;

    /* the (plane, control) pairs the policy uses */
    int32_t* pairmap = (int32_t*)malloc(sizeof(int32_t) * nplanes * nctl);
    if (!pairmap) return -1;
    for (int64_t k = 0; k < nplanes * nctl; ++k) pairmap[k] = -1;
    int64_t npairs = 0;
    for (int64_t e = 0; e < ncells; ++e) {
        const int u = pol[e];
        if (u < 0) continue;
        const int64_t pl = e % nplanes;  /* (h, vx, vy, w) are the fastest axes */
        if (pairmap[pl * nctl + u] < 0) pairmap[pl * nctl + u] = (int32_t)npairs++;
    }
    pair64* pairs = (pair64*)calloc((size_t)(npairs > 0 ? npairs : 1), sizeof(pair64));
    int64_t* pkey = (int64_t*)malloc(sizeof(int64_t) * (npairs > 0 ? npairs : 1));
    if (!pairs || !pkey) { free(pairmap); free(pairs); free(pkey); return -1; }
    for (int64_t k = 0; k < nplanes * nctl; ++k)
        if (pairmap[k] >= 0) pkey[pairmap[k]] = k;
    const int nsub = p->hmax > 0.0f ? og_substeps_for(p->dt, p) : p->nsub;
#pragma omp parallel for schedule(dynamic, 16) if (threads != 1)
    for (int64_t q = 0; q < npairs; ++q) {
        const int64_t pl = pkey[q] / nctl;
        const int u = (int)(pkey[q] % nctl);
        int64_t r = pl;
        const int i6 = (int)(r % n[5]); r /= n[5];
        const int i5 = (int)(r % n[4]); r /= n[4];
        const int i4 = (int)(r % n[3]); r /= n[3];
        const int i3 = (int)r;
        const double ur[3] = {ctl[u], ctl[u + nctl], ctl[u + 2 * nctl]};
        const double h0 = axv(g, 2, i3), vfx = axv(g, 3, i4), vfy = axv(g, 4, i5), w0 = axv(g, 5, i6);
        pair64* pr = &pairs[q];
        pr->ok = succ64(&m0, p->rk2, h0, vfx, vfy, w0, ur, tau, nsub, pr->s);
        for (int k = 0; k < NTH && pr->ok; ++k) {
            m64 mp = m0, mm = m0;
            const double th = *theta_ptr(&m0, k);
            const double dl = 1.0e-6 * (fabs(th) > 1.0 ? fabs(th) : 1.0);
            *theta_ptr(&mp, k) = th + dl;
            *theta_ptr(&mm, k) = th - dl;
            double sp[6], sm[6];
            if (!succ64(&mp, p->rk2, h0, vfx, vfy, w0, ur, tau, nsub, sp) ||
                !succ64(&mm, p->rk2, h0, vfx, vfy, w0, ur, tau, nsub, sm)) {
                pr->ok = 0;
                break;
            }
            for (int a = 0; a < 6; ++a) pr->d[a][k] = (sp[a] - sm[a]) / (2.0 * dl);
        }
    }

    /* active cells and their rows */
    row64* rows = (row64*)malloc(sizeof(row64) * (size_t)(ncells > 0 ? ncells : 1));
    int32_t* rowpair = (int32_t*)malloc(sizeof(int32_t) * (size_t)(ncells > 0 ? ncells : 1));
    if (!rows || !rowpair) { free(pairmap); free(pairs); free(pkey); free(rows); free(rowpair); return -1; }
    int64_t nrow = 0;
    for (int64_t e = 0; e < ncells; ++e) {
        const int u = pol[e];
        if (u < 0) continue;
        int64_t r = e;
        int32_t i[6];
        for (int k = 5; k >= 1; --k) { i[k] = (int32_t)(r % n[k]); r /= n[k]; }
        i[0] = (int32_t)r;
        if (occ[((int64_t)i[0] * n[1] + i[1]) * n[2] + i[2]]) continue;
        if (!(V[e] > 0.0 && V[e] < cap)) continue;
        const int32_t q = pairmap[(e % nplanes) * nctl + u];
        const pair64* pr = &pairs[q];
        if (!pr->ok) continue;
        double f[6];
        f[0] = (axv(g, 0, i[0]) + pr->s[0] - g->lo[0]) / g->step[0];
        f[1] = (axv(g, 1, i[1]) + pr->s[1] - g->lo[1]) / g->step[1];
        f[2] = (pr->s[2] - g->lo[2]) / g->step[2];
        f[2] -= floor(f[2] / n[2]) * n[2];
        for (int k = 3; k < 6; ++k) f[k] = (pr->s[k] - g->lo[k]) / g->step[k];
        int off = 0;
        for (int k = 0; k < 6 && !off; ++k)
            if (k != 2 && !(f[k] >= 0.0 && f[k] <= n[k] - 1)) off = 1;
        if (off) continue;
        row64 rw;
        rw.cell = e;
        for (int k = 0; k < 6; ++k) {
            const double b = floor(f[k]);
            rw.ib[k] = (int32_t)b;
            rw.t[k] = f[k] - b;
        }
        double I = 0.0;
        for (int d = 0; d < 64; ++d) {
            int64_t ci;
            double w;
            corners(g, &rw, d, &ci, &w);
            I += w * V[ci];
        }
        if (!(I < cap && tau + I < cap)) continue;
        rows[nrow] = rw;
        rowpair[nrow] = q;
        ++nrow;
    }

    /* lambda = c + P^T lambda */
    double* lam = (double*)malloc(sizeof(double) * ncells);
    double* nxt = (double*)malloc(sizeof(double) * ncells);
    if (!lam || !nxt) {
        free(pairmap); free(pairs); free(pkey); free(rows); free(rowpair); free(lam); free(nxt);
        return -1;
    }
    double cn = 0.0;
    for (int64_t e = 0; e < ncells; ++e) { lam[e] = c[e]; cn += fabs(c[e]); }
    int32_t it = 0;
    for (it = 1; it <= iters && cn > 0.0; ++it) {
        memcpy(nxt, c, sizeof(double) * ncells);
#pragma omp parallel for schedule(static) if (threads != 1)
        for (int64_t k = 0; k < nrow; ++k) {
            const double lv = lam[rows[k].cell];
            if (lv == 0.0) continue;
            for (int d = 0; d < 64; ++d) {
                int64_t ci;
                double w;
                corners(g, &rows[k], d, &ci, &w);
#pragma omp atomic
                nxt[ci] += w * lv;
            }
        }
        double r = 0.0;
        for (int64_t e = 0; e < ncells; ++e) r += fabs(nxt[e] - lam[e]);
        double* t = lam; lam = nxt; nxt = t;
        if (r <= tol * cn) break;
    }
    if (it > iters) it = iters;

    /* dL/dtheta = sum over rows of lambda(s) (grad I) . (d successor / d theta) */
    double gacc[NTH] = {0};
    for (int64_t k = 0; k < nrow; ++k) {
        const double lv = lam[rows[k].cell];
        if (lv == 0.0) continue;
        double gI[6] = {0, 0, 0, 0, 0, 0};
        for (int d = 0; d < 64; ++d) {
            int64_t ci;
            double w;
            corners(g, &rows[k], d, &ci, &w);
            for (int ax = 0; ax < 6; ++ax) {
                double pr = ((d >> ax) & 1) ? V[ci] : -V[ci];
                for (int o = 0; o < 6; ++o)
                    if (o != ax) pr *= ((d >> o) & 1) ? rows[k].t[o] : 1.0 - rows[k].t[o];
                gI[ax] += pr;
            }
        }
        const pair64* pr = &pairs[rowpair[k]];
        for (int ax = 0; ax < 6; ++ax) {
            const double ga = lv * gI[ax] / g->step[ax];
            for (int q = 0; q < NTH; ++q) gacc[q] += ga * pr->d[ax][q];
        }
    }
    for (int q = 0; q < NTH; ++q) grad[q] = gacc[q];
    if (iters_done) *iters_done = it;
    if (nactive) *nactive = nrow;
    free(pairmap); free(pairs); free(pkey); free(rows); free(rowpair); free(lam); free(nxt);
    return 0;
}
