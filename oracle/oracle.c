/*
 * oracle.c - TEST INFRASTRUCTURE ONLY: a plain-C (C99 complex + OpenMP) restatement of the reference's compiled
 * hot-path kernels (mom25d src/mom25d/core/mom25d_core.cpp), used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py as the checker. Nothing in the product links or calls this file.
 *
 * Each function cites the reference lines it restates. Arithmetic follows the reference's order so that, built
 * with the same flags (g++/gcc -O3, no FMA contraction), results agree bit for bit with the reference core.
 *
 * Layouts (all row-major, as the reference's NumPy buffers): see oracle/__init__.py.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cd;
typedef float complex cf;

typedef struct {
    int ntab, nfine, L;
    const cd *A, *Q, *cA, *cq, *cAi, *cqi;
    const double *dr, *d, *dimg;
    const int *tab, *kind;
} Tables;

typedef struct {
    int Ne, Nt;
    const int *ep, *em, *lt, *te;
    const double *ap, *am, *vp, *vm, *cent, *area, *ta, *tv;
} Mesh;

/* mom25d_core.cpp:70-78 (Tables::rest): linear interpolation at u = r / dr, clamped to nfine - 1.000001 */
static inline void rest(const Tables *tb, int t, double r, cd *ga, cd *gq)
{
    double u = r / tb->dr[t];
    const double umax = tb->nfine - 1.000001;
    if (u > umax) u = umax;
    int i = (int)u;
    double f = u - i;
    const cd *a = tb->A + (size_t)t * tb->nfine, *q = tb->Q + (size_t)t * tb->nfine;
    *ga = a[i] * (1 - f) + a[i + 1] * f;
    *gq = q[i] * (1 - f) + q[i + 1] * f;
}

/* mom25d_core.cpp:80-89 (Tables::kern): the full kernel at a centroid distance (singular parts added back) */
static inline void kern(const Tables *tb, int la, int lb, double r, cd *ga, cd *gq)
{
    int t = tb->tab[la * tb->L + lb];
    rest(tb, t, r, ga, gq);
    if (tb->kind[t] == 0) {
        if (r > 0) { *ga += tb->cA[t] / r; *gq += tb->cq[t] / r; }
        if (tb->dimg[t] > 0) {
            double ri = 1.0 / sqrt(r * r + tb->dimg[t] * tb->dimg[t]);
            *ga += tb->cAi[t] * ri; *gq += tb->cqi[t] * ri;
        }
    } else if (tb->kind[t] == 1) {
        double ri = 1.0 / sqrt(r * r + tb->d[t] * tb->d[t]);
        *ga += tb->cA[t] * ri; *gq += tb->cq[t] * ri;
    }
}

static inline double dist(const double *c, int p, int q)
{
    double dx = c[2 * p] - c[2 * q], dy = c[2 * p + 1] - c[2 * q + 1];
    return sqrt(dx * dx + dy * dy);
}

/* mom25d_core.cpp:132-173 (fill_far_t): centroid-rule Z for every edge pair, both triangles written.
 * single != 0: Z is complex64 (the value rounded on store). */
void orc_fill_far(void *Z, size_t ld, int single, const Mesh *g, const Tables *tb, double w)
{
    const cd jw = CMPLX(0, w), inv_jw = 1.0 / CMPLX(0, w);
    const int Ne = g->Ne, Nt = g->Nt;
#pragma omp parallel
    {
        cd *GA = malloc(sizeof(cd) * 2 * (size_t)Nt), *GQ = malloc(sizeof(cd) * 2 * (size_t)Nt);
#pragma omp for schedule(dynamic, 8)
        for (int m = 0; m < Ne; ++m) {
            int pm[2] = {g->ep[m], g->em[m]};
            for (int s = 0; s < 2; ++s)
                for (int q = 0; q < Nt; ++q)
                    kern(tb, g->lt[pm[s]], g->lt[q], dist(g->cent, pm[s], q), &GA[s * Nt + q], &GQ[s * Nt + q]);
            double am_[2] = {g->ap[m] * g->area[pm[0]], g->am[m] * g->area[pm[1]]};
            double dx[2], dy[2];
            dx[0] = g->cent[2 * pm[0]] - g->vp[2 * m]; dy[0] = g->cent[2 * pm[0] + 1] - g->vp[2 * m + 1];
            dx[1] = g->cent[2 * pm[1]] - g->vm[2 * m]; dy[1] = g->cent[2 * pm[1] + 1] - g->vm[2 * m + 1];
            for (int n = m; n < Ne; ++n) {
                int pn[2] = {g->ep[n], g->em[n]};
                double an[2] = {g->ap[n] * g->area[pn[0]], g->am[n] * g->area[pn[1]]};
                double ex[2], ey[2];
                ex[0] = g->cent[2 * pn[0]] - g->vp[2 * n]; ey[0] = g->cent[2 * pn[0] + 1] - g->vp[2 * n + 1];
                ex[1] = g->cent[2 * pn[1]] - g->vm[2 * n]; ey[1] = g->cent[2 * pn[1] + 1] - g->vm[2 * n + 1];
                cd v = 0;
                for (int s = 0; s < 2; ++s)
                    for (int t = 0; t < 2; ++t) {
                        size_t k = s * (size_t)Nt + pn[t];
                        double dot = dx[s] * ex[t] + dy[s] * ey[t];
                        v += am_[s] * an[t] * (jw * dot * GA[k] + 4.0 * GQ[k] * inv_jw);
                    }
                if (single) {
                    ((cf *)Z)[(size_t)m * ld + n] = (cf)v;
                    ((cf *)Z)[(size_t)n * ld + m] = (cf)v;
                } else {
                    ((cd *)Z)[(size_t)m * ld + n] = v;
                    ((cd *)Z)[(size_t)n * ld + m] = v;
                }
            }
        }
        free(GA); free(GQ);
    }
}

/* mom25d_core.cpp:176-211 (far_block): the centroid rule for row / column edge lists */
void orc_far_block(cd *out, const int *R, int nr, const int *C, int nc, const Mesh *g, const Tables *tb, double w)
{
    const cd jw = CMPLX(0, w), inv_jw = 1.0 / CMPLX(0, w);
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < nr; ++i) {
        int m = R[i];
        int pm[2] = {g->ep[m], g->em[m]};
        double am_[2] = {g->ap[m] * g->area[pm[0]], g->am[m] * g->area[pm[1]]};
        double dx[2] = {g->cent[2 * pm[0]] - g->vp[2 * m], g->cent[2 * pm[1]] - g->vm[2 * m]};
        double dy[2] = {g->cent[2 * pm[0] + 1] - g->vp[2 * m + 1], g->cent[2 * pm[1] + 1] - g->vm[2 * m + 1]};
        for (int j = 0; j < nc; ++j) {
            int n = C[j];
            int pn[2] = {g->ep[n], g->em[n]};
            double an[2] = {g->ap[n] * g->area[pn[0]], g->am[n] * g->area[pn[1]]};
            double ex[2] = {g->cent[2 * pn[0]] - g->vp[2 * n], g->cent[2 * pn[1]] - g->vm[2 * n]};
            double ey[2] = {g->cent[2 * pn[0] + 1] - g->vp[2 * n + 1], g->cent[2 * pn[1] + 1] - g->vm[2 * n + 1]};
            cd v = 0;
            for (int s = 0; s < 2; ++s)
                for (int t = 0; t < 2; ++t) {
                    cd ga, gq;
                    kern(tb, g->lt[pm[s]], g->lt[pn[t]], dist(g->cent, pm[s], pn[t]), &ga, &gq);
                    v += am_[s] * an[t] * (jw * (dx[s] * ex[t] + dy[s] * ey[t]) * ga + 4.0 * gq * inv_jw);
                }
            out[(size_t)i * nc + j] = v;
        }
    }
}

/* mom25d_core.cpp:257-314 (matvec_far_multi): Y = Z_far X for K columns, triangle-aggregated */
void orc_matvec_far_multi(cd *Y, const cd *X, int K, const Mesh *g, const Tables *tb, double w)
{
    const int Ne = g->Ne, Nt = g->Nt;
    const cd jw = CMPLX(0, w), inv_jw = 1.0 / CMPLX(0, w);
    cd *s0 = calloc((size_t)Nt * K, sizeof(cd)), *s1x = calloc((size_t)Nt * K, sizeof(cd)),
       *s1y = calloc((size_t)Nt * K, sizeof(cd));
    char *act = calloc(Nt, 1);
    for (int e = 0; e < Ne; ++e) {
        int p = g->ep[e], q = g->em[e];
        for (int c = 0; c < K; ++c) {
            cd xe = X[(size_t)e * K + c];
            cd a = g->ap[e] * g->area[p] * xe, b = g->am[e] * g->area[q] * xe;
            size_t ip = (size_t)p * K + c, iq = (size_t)q * K + c;
            s0[ip] += a; s1x[ip] += a * (g->cent[2 * p] - g->vp[2 * e]); s1y[ip] += a * (g->cent[2 * p + 1] - g->vp[2 * e + 1]);
            s0[iq] += b; s1x[iq] += b * (g->cent[2 * q] - g->vm[2 * e]); s1y[iq] += b * (g->cent[2 * q + 1] - g->vm[2 * e + 1]);
        }
        act[p] = act[q] = 1;
    }
    cd *vAx = malloc(sizeof(cd) * (size_t)Nt * K), *vAy = malloc(sizeof(cd) * (size_t)Nt * K),
       *wQ = malloc(sizeof(cd) * (size_t)Nt * K);
#pragma omp parallel
    {
        cd *ax = malloc(sizeof(cd) * K), *ay = malloc(sizeof(cd) * K), *aq = malloc(sizeof(cd) * K);
#pragma omp for schedule(dynamic, 16)
        for (int p = 0; p < Nt; ++p) {
            for (int c = 0; c < K; ++c) ax[c] = ay[c] = aq[c] = 0;
            for (int q = 0; q < Nt; ++q) {
                if (!act[q]) continue;
                cd ga, gq;
                kern(tb, g->lt[p], g->lt[q], dist(g->cent, p, q), &ga, &gq);
                const cd *S0 = &s0[(size_t)q * K], *SX = &s1x[(size_t)q * K], *SY = &s1y[(size_t)q * K];
                for (int c = 0; c < K; ++c) { ax[c] += ga * SX[c]; ay[c] += ga * SY[c]; aq[c] += gq * S0[c]; }
            }
            for (int c = 0; c < K; ++c) {
                vAx[(size_t)p * K + c] = ax[c]; vAy[(size_t)p * K + c] = ay[c]; wQ[(size_t)p * K + c] = aq[c];
            }
        }
        free(ax); free(ay); free(aq);
    }
    for (int e = 0; e < Ne; ++e) {
        int p = g->ep[e], q = g->em[e];
        double dpx = g->cent[2 * p] - g->vp[2 * e], dpy = g->cent[2 * p + 1] - g->vp[2 * e + 1];
        double dqx = g->cent[2 * q] - g->vm[2 * e], dqy = g->cent[2 * q + 1] - g->vm[2 * e + 1];
        for (int c = 0; c < K; ++c) {
            size_t ip = (size_t)p * K + c, iq = (size_t)q * K + c;
            cd yp = g->ap[e] * g->area[p] * (jw * (dpx * vAx[ip] + dpy * vAy[ip]) + 4.0 * wQ[ip] * inv_jw);
            cd ym = g->am[e] * g->area[q] * (jw * (dqx * vAx[iq] + dqy * vAy[iq]) + 4.0 * wQ[iq] * inv_jw);
            Y[(size_t)e * K + c] = yp + ym;
        }
    }
    free(s0); free(s1x); free(s1y); free(act); free(vAx); free(vAy); free(wQ);
}

/* mom25d_core.cpp:321-324 (rule_over_p) */
static inline int rule_over_p(double ap, double aq, int p, int q)
{
    const double tie = 1e-9 * (ap > aq ? ap : aq);
    return fabs(ap - aq) <= tie ? p <= q : ap < aq;
}

/* mom25d_core.cpp:331-365 (offplane_one): analytic 1/sqrt(rho^2 + d^2) over triangle V, 6-point rule outside */
void orc_offplane_one(const double *V, const double *P6, const double *W6, double d,
                      double *m0, double mro[2], double mrs[2], double *mrr)
{
    double ad = fabs(d);
    double e[3][2], L[3], tau[3][2], un[3][2];
    for (int i = 0; i < 3; ++i) {
        int j = (i + 1) % 3;
        e[i][0] = V[2 * j] - V[2 * i]; e[i][1] = V[2 * j + 1] - V[2 * i + 1];
        L[i] = sqrt(e[i][0] * e[i][0] + e[i][1] * e[i][1]);
        tau[i][0] = e[i][0] / L[i]; tau[i][1] = e[i][1] / L[i];
        un[i][0] = tau[i][1]; un[i][1] = -tau[i][0];
    }
    *m0 = 0; mro[0] = mro[1] = 0; mrs[0] = mrs[1] = 0; *mrr = 0;
    for (int k = 0; k < 6; ++k) {
        double rx = P6[2 * k], ry = P6[2 * k + 1], wq = W6[k];
        double I1 = 0, IRx = 0, IRy = 0;
        for (int i = 0; i < 3; ++i) {
            double dvx = V[2 * i] - rx, dvy = V[2 * i + 1] - ry;
            double sm = dvx * tau[i][0] + dvy * tau[i][1];
            double sp = sm + L[i];
            double t0 = dvx * un[i][0] + dvy * un[i][1];
            double R02 = t0 * t0 + d * d, R0 = sqrt(R02);
            double Rm = sqrt(R02 + sm * sm), Rp = sqrt(R02 + sp * sp);
            double lg = (R0 > 1e-14 * L[i]) ? asinh(sp / R0) - asinh(sm / R0) : 0.0;
            double beta = atan2(t0 * sp, R02 + ad * Rp) - atan2(t0 * sm, R02 + ad * Rm);
            I1 += t0 * lg - ad * beta;
            double eR = 0.5 * (R02 * lg + sp * Rp - sm * Rm);
            IRx += eR * un[i][0]; IRy += eR * un[i][1];
        }
        double Wx = IRx + rx * I1, Wy = IRy + ry * I1;
        *m0 += wq * I1;
        mro[0] += wq * rx * I1; mro[1] += wq * ry * I1;
        mrs[0] += wq * Wx; mrs[1] += wq * Wy;
        *mrr += wq * (rx * Wx + ry * Wy);
    }
}

static inline void atomic_add_cd(cd *z, cd v)
{
    double *p = (double *)z;
#pragma omp atomic
    p[0] += creal(v);
#pragma omp atomic
    p[1] += cimag(v);
}

static inline void atomic_add_cf(cf *z, cd v)
{
    float *p = (float *)z;
#pragma omp atomic
    p[0] += (float)creal(v);
#pragma omp atomic
    p[1] += (float)cimag(v);
}

/* mom25d_core.cpp:417-507 (near_core): per near triangle pair the accurate minus the centroid moments, scattered
 * to the 3 x 3 edge pairs. mode 0: added into the dense Z (single: complex64); mode 2: COO triplets (ri = -1 for
 * unused slots); mode 1: y += dZ x. stat (n x 12) keeps the analytic parts when given (stat_ready: read them). */
void orc_near(int mode, void *Z, size_t ld, int single, int *ri, int *ci, cd *vv, const cd *x, cd *y, cd *qcorr,
              double *stat, int stat_ready,
              const Mesh *g, const Tables *tb, const double *nodes, const int *tris, const double *P3,
              const double *W3, const double *P6, const double *W6, const int *P, const int *Q, int n, double w)
{
    const cd jw = CMPLX(0, w), inv_jw = 1.0 / CMPLX(0, w);
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
        const int p = P[i], q = Q[i];
        const int la = g->lt[p], lb = g->lt[q];
        const int t = tb->tab[la * tb->L + lb];
        const int same = (la == lb);
        const int np = same ? 3 : 6;
        const double *Pa = same ? P3 + 6 * (size_t)p : P6 + 12 * (size_t)p;
        const double *Pb = same ? P3 + 6 * (size_t)q : P6 + 12 * (size_t)q;
        const double *Wa = same ? W3 + 3 * (size_t)p : W6 + 6 * (size_t)p;
        const double *Wb = same ? W3 + 3 * (size_t)q : W6 + 6 * (size_t)q;
        cd M0 = 0, Mox = 0, Moy = 0, Msx = 0, Msy = 0, Mrr = 0, Mq = 0;
        for (int a = 0; a < np; ++a)
            for (int b = 0; b < np; ++b) {
                double dx = Pa[2 * a] - Pb[2 * b], dy = Pa[2 * a + 1] - Pb[2 * b + 1];
                cd ga, gq;
                rest(tb, t, sqrt(dx * dx + dy * dy), &ga, &gq);
                double wt = Wa[a] * Wb[b];
                ga *= wt; gq *= wt;
                M0 += ga; Mox += ga * Pa[2 * a]; Moy += ga * Pa[2 * a + 1];
                Msx += ga * Pb[2 * b]; Msy += ga * Pb[2 * b + 1];
                Mrr += ga * (Pa[2 * a] * Pb[2 * b] + Pa[2 * a + 1] * Pb[2 * b + 1]);
                Mq += gq;
            }
        const int keep = rule_over_p(g->area[p], g->area[q], p, q);
        const int po = keep ? p : q, qi = keep ? q : p;
        double V[6];
        for (int k = 0; k < 3; ++k) { V[2 * k] = nodes[2 * tris[3 * qi + k]]; V[2 * k + 1] = nodes[2 * tris[3 * qi + k] + 1]; }
        int nk = 0;
        double dds[2]; cd cAs[2], cqs[2];
        if (tb->kind[t] == 0) {
            dds[nk] = 0.0; cAs[nk] = tb->cA[t]; cqs[nk] = tb->cq[t]; nk++;
            if (tb->dimg[t] > 0) { dds[nk] = tb->dimg[t]; cAs[nk] = tb->cAi[t]; cqs[nk] = tb->cqi[t]; nk++; }
        } else if (tb->kind[t] == 1) {
            dds[nk] = tb->d[t]; cAs[nk] = tb->cA[t]; cqs[nk] = tb->cq[t]; nk++;
        }
        for (int k = 0; k < nk; ++k) {
            double st[6], *m = stat ? stat + 12 * (size_t)i + 6 * k : st;
            if (!(stat && stat_ready)) {
                double mro[2], mrs[2];
                orc_offplane_one(V, P6 + 12 * (size_t)po, W6 + 6 * (size_t)po, dds[k], &m[0], keep ? mro : mrs,
                                 keep ? mrs : mro, &m[5]);
                m[1] = mro[0]; m[2] = mro[1]; m[3] = mrs[0]; m[4] = mrs[1];
            }
            cd cA = cAs[k], cq = cqs[k];
            M0 += cA * m[0]; Mox += cA * m[1]; Moy += cA * m[2]; Msx += cA * m[3]; Msy += cA * m[4];
            Mrr += cA * m[5]; Mq += cq * m[0];
        }
        {
            double r = dist(g->cent, p, q);
            cd ga, gq;
            kern(tb, la, lb, r, &ga, &gq);
            double wgt = g->area[p] * g->area[q];
            double cpx = g->cent[2 * p], cpy = g->cent[2 * p + 1], cqx = g->cent[2 * q], cqy = g->cent[2 * q + 1];
            ga *= wgt; gq *= wgt;
            M0 -= ga; Mox -= ga * cpx; Moy -= ga * cpy; Msx -= ga * cqx; Msy -= ga * cqy;
            Mrr -= ga * (cpx * cqx + cpy * cqy); Mq -= gq;
        }
        if (qcorr) qcorr[i] = Mq;
        for (int s = 0; s < 3; ++s) {
            int em_ = g->te[3 * p + s];
            if (em_ < 0) continue;
            double am_ = g->ta[3 * p + s], vx = g->tv[6 * p + 2 * s], vy = g->tv[6 * p + 2 * s + 1];
            for (int u = 0; u < 3; ++u) {
                int en = g->te[3 * q + u];
                int slot = 9 * i + 3 * s + u;
                if (en < 0) { if (mode == 2) ri[slot] = -1; continue; }
                double an = g->ta[3 * q + u], wx = g->tv[6 * q + 2 * u], wy = g->tv[6 * q + 2 * u + 1];
                cd Acomb = Mrr - (wx * Mox + wy * Moy) - (vx * Msx + vy * Msy) + (vx * wx + vy * wy) * M0;
                cd val = am_ * an * (jw * Acomb + 4.0 * Mq * inv_jw);
                if (mode == 0) {
                    if (single) atomic_add_cf((cf *)Z + (size_t)em_ * ld + en, val);
                    else atomic_add_cd((cd *)Z + (size_t)em_ * ld + en, val);
                } else if (mode == 1) {
                    atomic_add_cd(y + em_, val * x[en]);
                } else {
                    ri[slot] = em_; ci[slot] = en; vv[slot] = val;
                }
            }
        }
        if (mode == 2) {
            for (int s = 0; s < 3; ++s)
                if (g->te[3 * p + s] < 0)
                    for (int u = 0; u < 3; ++u) ri[9 * i + 3 * s + u] = -1;
        }
    }
}

/* mom25d_core.cpp:1216-1263 (near_pairs): every (p, q) with rho^2 + dz^2 < (fac max(size_p, size_q))^2, sorted by
 * (p, q). Restated as the definition (all pairs tested), which yields the same set in the same order. Two passes:
 * counts (P == NULL) then the pairs. Returns the number of pairs. */
int64_t orc_near_pairs(const double *c, const double *sz, const double *zz, int Nt, double fac, int64_t *P, int64_t *Q,
                       int64_t *counts)
{
#pragma omp parallel for schedule(dynamic, 64)
    for (int p = 0; p < Nt; ++p) {
        int64_t k = 0;
        for (int q = 0; q < Nt; ++q) {
            double dx = c[2 * p] - c[2 * q], dy = c[2 * p + 1] - c[2 * q + 1], dz = zz[p] - zz[q];
            double R = fac * (sz[p] > sz[q] ? sz[p] : sz[q]);
            if (dx * dx + dy * dy + dz * dz < R * R) k++;
        }
        counts[p] = k;
    }
    int64_t total = 0;
    for (int p = 0; p < Nt; ++p) { int64_t k = counts[p]; counts[p] = total; total += k; }
    if (!P) return total;
#pragma omp parallel for schedule(dynamic, 64)
    for (int p = 0; p < Nt; ++p) {
        int64_t k = counts[p];
        for (int q = 0; q < Nt; ++q) {
            double dx = c[2 * p] - c[2 * q], dy = c[2 * p + 1] - c[2 * q + 1], dz = zz[p] - zz[q];
            double R = fac * (sz[p] > sz[q] ? sz[p] : sz[q]);
            if (dx * dx + dy * dy + dz * dz < R * R) { P[k] = p; Q[k] = q; k++; }
        }
    }
    return total;
}

/* mom25d_core.cpp:1269-1298 (radial_table_sum): out[t, v] = sum_q D(|P[t, q] - V[v]|) W[t, q] */
void orc_radial_table_sum(cd *out, const double *x, const double *y, const double *w, int64_t nt, int64_t nq,
                          const double *ax, const double *ay, int64_t nv, const cd *d, int64_t n, double dr)
{
    const double top = (double)n - 1.000001;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < nt; ++t)
        for (int64_t v = 0; v < nv; ++v) {
            cd acc = 0;
            for (int64_t q = 0; q < nq; ++q) {
                const double rx = x[t * nq + q] - ax[v], ry = y[t * nq + q] - ay[v];
                double u = hypot(rx, ry) / dr;
                if (u > top) u = top;
                const int64_t i = (int64_t)u;
                const double f = u - (double)i;
                acc += (d[i] * (1.0 - f) + d[i + 1] * f) * w[t * nq + q];
            }
            out[t * nv + v] = acc;
        }
}

/* mom25d_core.cpp:1585-1603 (fan_q): G_q x area_t x area_f between every triangle t and fan triangle F[j] */
void orc_fan_q(cd *out, const int *F, int nf, const Mesh *g, const Tables *tb)
{
#pragma omp parallel for schedule(static)
    for (int t = 0; t < g->Nt; ++t)
        for (int j = 0; j < nf; ++j) {
            cd ga, gq;
            kern(tb, g->lt[t], g->lt[F[j]], dist(g->cent, t, F[j]), &ga, &gq);
            out[(size_t)t * nf + j] = gq * (g->area[t] * g->area[F[j]]);
        }
}

/* mom25d_core.cpp:1430-1454 (hankel_real): out[s, i] = sum_k J0(rho_i kr_k) W[s, k], glibc's j0 */
void orc_hankel_real(cd *out, const double *rho, int nr, const double *kr, int nk, const cd *W, int ns)
{
#pragma omp parallel
    {
        cd *acc = malloc(sizeof(cd) * ns);
#pragma omp for schedule(static)
        for (int i = 0; i < nr; ++i) {
            for (int s = 0; s < ns; ++s) acc[s] = 0;
            for (int m = 0; m < nk; ++m) {
                double j = j0(rho[i] * kr[m]);
                for (int s = 0; s < ns; ++s) acc[s] += j * W[(size_t)s * nk + m];
            }
            for (int s = 0; s < ns; ++s) out[(size_t)s * nr + i] = acc[s];
        }
        free(acc);
    }
}

/* mom25d_core.cpp:1510-1543 (bessel_jn_complex1): J_n(z), n = 0, 1, 2: power series up to |z| = 14, Hankel's
 * asymptotic expansion (to its smallest term) beyond */
static cd jn_complex1(int n, cd z)
{
    const double PI = 3.14159265358979323846;
    const double az = cabs(z);
    if (az <= 14.0) {
        const cd h = 0.5 * z, mh2 = -h * h;
        cd term = n == 0 ? 1.0 : n == 1 ? h : 0.5 * h * h;
        cd sum = term;
        double big = cabs(term);
        for (int k = 1; k < 300; ++k) {
            term *= mh2 / ((double)k * (double)(k + n));
            sum += term;
            const double at = cabs(term);
            if (at > big) big = at;
            if (k > az && at <= 1e-18 * big) break;
        }
        return sum;
    }
    const double mu = 4.0 * n * n;
    const cd iz = 1.0 / z, chi = z - (0.5 * n + 0.25) * PI;
    cd P = 1.0, Qs = 0.0, t = 1.0;
    double prev = 1.0;
    for (int k = 1; k < 80; ++k) {
        const double m = 2.0 * k - 1.0;
        const cd nt = t * ((mu - m * m) / (8.0 * k)) * iz;
        const double at = cabs(nt);
        if (at >= prev) break;
        t = nt; prev = at;
        const double sg = ((k / 2) & 1) ? -1.0 : 1.0;
        if (k & 1) Qs += sg * t; else P += sg * t;
        if (at < 1e-17) break;
    }
    return csqrt(2.0 / (PI * z)) * (P * ccos(chi) - Qs * csin(chi));
}

void orc_bessel_jn_complex(cd *out, const cd *z, int64_t n_el, int n)
{
#pragma omp parallel for schedule(static) if (n_el > 4096)
    for (int64_t i = 0; i < n_el; ++i) out[i] = jn_complex1(n, z[i]);
}

/* mom25d_core.cpp:1563-1580 (scale_c64): Z <- diag(d) Z diag(d) in place and its complex64 copy */
void orc_scale_c64(cd *z, cf *o, const double *dd, int64_t n)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        cd *zr = z + (size_t)i * n; cf *orow = o + (size_t)i * n;
        for (int64_t j = 0; j < n; ++j) { zr[j] *= dd[i] * dd[j]; orow[j] = (cf)zr[j]; }
    }
}
