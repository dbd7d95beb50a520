/*
 * quench.c -- CPU oracle of the conjugate-gradient quench (TEST INFRASTRUCTURE).
 *
 * quench (src/quench_m.F90:100-200) minimises f = pe + press*vol over the
 * variable vector x = (x0,y0,z0 of every atom interleaved, then B0 row by
 * row) with the restarted conjugate-gradient routine VA14CD
 * (src/quench_m.F90:323-551), calling derivs (215-313) for f and g = df/dx.
 * VA14CD is Powell's restart procedure for the conjugate gradient method
 * (M.J.D. Powell, Math. Programming 12 (1977) 241-254) with the line search of
 * the Harwell VA14 routines.  This file restates its control flow label by
 * label, so that the sequence of function evaluations is the reference's;
 * the printing branches are left out (IPRINT = 0 path).
 *
 * Deviation, optional: criterion 1 replaces the acceptance test
 * gsumsq <= acc (label 210) by max_i |B0 f_i| <= fmax, the real-force bound.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_internal.h"

typedef struct {
    orc_sys *s;
    int n;           /* 3*nm + 9 */
    double *x, *g;   /* 1-based, module x(:), g(:) of quench_m */
    double *en;
    int criterion;
    double fmax;
    double last_fmax, pe;
} qctx;

/* Fortran MIN / MAX / MIN0 */
static double fmin_d(double a, double b) { return a < b ? a : b; }
static double fmax_d(double a, double b) { return a > b ? a : b; }
static int imin_i(int a, int b) { return a < b ? a : b; }

static double vol3(const double *b)
{
    return M3(b, 1, 1) * (M3(b, 2, 2) * M3(b, 3, 3) - M3(b, 2, 3) * M3(b, 3, 2)) +
           M3(b, 2, 1) * (M3(b, 3, 2) * M3(b, 1, 3) - M3(b, 1, 2) * M3(b, 3, 3)) +
           M3(b, 3, 1) * (M3(b, 1, 2) * M3(b, 2, 3) - M3(b, 2, 2) * M3(b, 1, 3));
}

/* derivs (src/quench_m.F90:215-313): f and g at x.  Returns the force status. */
static int derivs(qctx *q, double *f)
{
    orc_sys *s = q->s;
    const int nm = s->nm;
    int nm3 = 3 * nm;
    for (int i = 1; i <= 3; ++i)
        for (int j = 1; j <= 3; ++j) M3(s->b0, i, j) = q->x[++nm3];
    for (int i = 1; i <= nm; ++i) {
        s->x0[i] = q->x[3 * i - 2];
        s->y0[i] = q->x[3 * i - 1];
        s->z0[i] = q->x[3 * i];
    }
    s->vol = vol3(s->b0);
    double tg[9];
    for (int i = 1; i <= 3; ++i) {
        for (int j = 1; j <= 3; ++j) M3(tg, i, j) = 0.0;
        for (int k = 1; k <= 3; ++k)
            for (int j = 1; j <= 3; ++j) M3(tg, i, j) = M3(tg, i, j) + M3(s->b0, k, i) * M3(s->b0, k, j);
    }
    int st = orc_force(s);
    if (st) return st;
    orc_energy_calc(s, q->en + 1);
    for (int i = 1; i <= q->n; ++i) q->g[i] = 0.0;
    double pe = 0.0;
    for (int i = 1; i <= nm; ++i) pe = pe + q->en[i];
    q->pe = pe;
    for (int i = 1; i <= nm; ++i) {
        q->g[3 * i - 2] = (-M3(tg, 1, 1) * s->fx[i] - M3(tg, 1, 2) * s->fy[i] - M3(tg, 1, 3) * s->fz[i]);
        q->g[3 * i - 1] = (-M3(tg, 2, 1) * s->fx[i] - M3(tg, 2, 2) * s->fy[i] - M3(tg, 2, 3) * s->fz[i]);
        q->g[3 * i] = (-M3(tg, 3, 1) * s->fx[i] - M3(tg, 3, 2) * s->fy[i] - M3(tg, 3, 3) * s->fz[i]);
    }
    *f = pe + s->press * s->vol;
    nm3 = 3 * nm;
    if (s->ivol < 1 || s->ivol == 4) {
        for (int i = 1; i <= 3; ++i)
            for (int j = 1; j <= 3; ++j) {
                ++nm3;
                if (s->ivol == 4 && i * j != 9) continue;
                q->g[nm3] = -M3(s->tp, i, j) + s->press * M3(s->tc, i, j);
            }
    }
    /* largest real force |B0 f| (for criterion 1 and reporting) */
    double fm = 0.0;
    for (int i = 1; i <= nm; ++i) {
        double fx = s->fx[i], fy = s->fy[i], fz = s->fz[i];
        double rx = M3(s->b0, 1, 1) * fx + M3(s->b0, 1, 2) * fy + M3(s->b0, 1, 3) * fz;
        double ry = M3(s->b0, 2, 1) * fx + M3(s->b0, 2, 2) * fy + M3(s->b0, 2, 3) * fz;
        double rz = M3(s->b0, 3, 1) * fx + M3(s->b0, 3, 2) * fy + M3(s->b0, 3, 3) * fz;
        double a = sqrt(rx * rx + ry * ry + rz * rz);
        if (a > fm) fm = a;
    }
    q->last_fmax = fm;
    return 0;
}

static int accepted(const qctx *q, double gsumsq, double acc)
{
    if (q->criterion == 1) return q->last_fmax <= q->fmax;
    return !(gsumsq > acc);
}

/*
 * VA14CD(FUNCT, N, F, DFN, ACC) of src/quench_m.F90:323-551 with maxfn = nsteps.
 * out[0] f, out[1] pe, out[2] gsumsq, out[3] max real force, out[4] function
 * evaluations, out[5] iterations, out[6] iflag (0 converged, 1 maxfn, 2 CG error),
 * out[7] force status.
 */
int orc_quench(orc_sys *s, int maxfn, int criterion, double fmax, double *out)
{
    const int nm = s->nm;
    const int n = 3 * nm + 9;
    qctx q;
    q.s = s; q.n = n; q.criterion = criterion; q.fmax = fmax; q.last_fmax = 0.0; q.pe = 0.0;
    q.x = (double *)calloc((size_t)n + 1, sizeof(double));
    q.g = (double *)calloc((size_t)n + 1, sizeof(double));
    q.en = (double *)calloc((size_t)nm + 1, sizeof(double));
    double *dr = (double *)calloc((size_t)n + 1, sizeof(double));
    double *dgr = (double *)calloc((size_t)n + 1, sizeof(double));
    double *d = (double *)calloc((size_t)n + 1, sizeof(double));
    double *gs = (double *)calloc((size_t)n + 1, sizeof(double));
    double *xx = (double *)calloc((size_t)n + 1, sizeof(double));
    double *gg = (double *)calloc((size_t)n + 1, sizeof(double));
    double *x = q.x, *g = q.g;

    /* quench: pack x (src/quench_m.F90:108-124) */
    for (int i = 1; i <= nm; ++i) {
        x[3 * i - 2] = s->x0[i];
        x[3 * i - 1] = s->y0[i];
        x[3 * i] = s->z0[i];
    }
    int nm3 = 3 * nm;
    for (int i = 1; i <= 3; ++i)
        for (int j = 1; j <= 3; ++j) x[++nm3] = M3(s->b0, i, j);
    const double dfn = 0.1;
    const double acc = 5.0e-7 * nm;

    double f = 0.0;
    double xnew = 0.0, dgstep = 0.0, fmin = 0.0, dginit = 0.0, xmin = 0.0, finit = 0.0;
    double gsinit = 0.0, gmin = 0.0, gm = 0.0, xbound = 0.0, clt = 0.0, gnew = 0.0;
    double ggstar = 0.0, beta = 0.0, gamden = 0.0, gsumsq = 0.0, c, dtest, gamma, toplin, xold;
    int itcrs = 0, maxfnk = 0, noerr = 0, iflag = 0, iretry = -2, iterc = 0, maxfnc = 1;
    int fstat = 0;

    goto L190;
L10:
    xnew = fabs(dfn + dfn) / gsumsq;
    dgstep = -gsumsq;
L20:
    itcrs = n + 1;
L30:
    if (maxfnk >= maxfnc) goto L50;
    f = fmin;
    for (int i = 1; i <= n; ++i) {
        x[i] = xx[i];
        g[i] = gg[i];
    }
L50:
    if (iflag > 0) goto L230;
    if (itcrs <= n) goto L70;
    for (int i = 1; i <= n; ++i) d[i] = -g[i];
L70:
    /* printing branches omitted (IPRINT = 0) */
    iterc = iterc + 1;
    dginit = 0.0;
    for (int i = 1; i <= n; ++i) {
        gs[i] = g[i];
        dginit = dginit + d[i] * g[i];
    }
    if (dginit >= 0.0) goto L320;
    xmin = 0.0;
    fmin = f;
    finit = f;
    gsinit = gsumsq;
    gmin = dginit;
    gm = dginit;
    xbound = -1.0;
    xnew = xnew * fmin_d(1.0, dgstep / dginit);
    dgstep = dginit;
L170:
    c = xnew - xmin;
    dtest = 0.0;
    for (int i = 1; i <= n; ++i) {
        x[i] = xx[i] + c * d[i];
        dtest = dtest + fabs(x[i] - xx[i]);
    }
    if (dtest <= 0.0) clt = 0.7;
    if (dtest <= 0.0) goto L300;
    if (fmax_d(xbound, xmin - c) < 0.0) clt = 0.1;
    maxfnc = maxfnc + 1;
L190:
    fstat = derivs(&q, &f);
    if (fstat) { iflag = 3; goto L240; }
    if (maxfnc <= 1) goto L210;
    gnew = 0.0;
    for (int i = 1; i <= n; ++i) gnew = gnew + d[i] * g[i];
    if (f < fmin) goto L210;
    if (f > fmin) goto L250;
    if (fabs(gnew) > fabs(gmin)) goto L250;
L210:
    maxfnk = maxfnc;
    gsumsq = 0.0;
    for (int i = 1; i <= n; ++i) gsumsq = gsumsq + g[i] * g[i];
    if (!accepted(&q, gsumsq, acc)) goto L250;
L230:
    goto L240;
L240:
    goto done;
L250:
    if (maxfnc != maxfn) goto L270;
    iflag = 1;
    goto L30;
L270:
    if (maxfnk < maxfnc) goto L300;
    for (int i = 1; i <= n; ++i) {
        xx[i] = x[i];
        gg[i] = g[i];
    }
    if (maxfnc <= 1) goto L10;
    gm = gnew;
    if (gm <= dginit) goto L310;
    ggstar = 0.0;
    for (int i = 1; i <= n; ++i) ggstar = ggstar + gs[i] * g[i];
    beta = (gsumsq - ggstar) / (gm - dginit);
L300:
    if (fabs(gm) > clt * fabs(dginit)) goto L310;
    if (fabs(gm * beta) <= clt * gsumsq) goto L380;
L310:
    clt = clt + 0.3;
    if (clt <= 0.8) goto L340;
L320:
    iretry = -iretry;
    if (imin_i(iretry, maxfnk) >= 2) goto L20;
    noerr = noerr + 1;
    if (noerr < 5) goto L20;
    iflag = 2;
    goto L30;
L340:
    xold = xnew;
    xnew = 0.5 * (xmin + xold);
    if (maxfnk < maxfnc) goto L350;
    if (gmin * gnew <= 0.0) goto L350;
    xnew = 10.0 * xold;
    if (xbound >= 0.0) xnew = 0.5 * (xold + xbound);
L350:
    toplin = (3.0 * gnew + gmin - 4.0 * (f - fmin) / (xold - xmin));
    c = gnew - toplin * (xold - xnew) / (xold - xmin);
    if (maxfnk < maxfnc) goto L360;
    if (gmin * gnew <= 0.0) xbound = xmin;
    xmin = xold;
    fmin = f;
    gmin = gnew;
    goto L370;
L360:
    xbound = xold;
L370:
    if (c * gmin >= 0.0) goto L170;
    xnew = (xmin * c - xnew * gmin) / (c - gmin);
    goto L170;
L380:
    if (fmin_d(f, fmin) < finit) goto L390;
    if (gsumsq >= gsinit) goto L320;
L390:
    if (itcrs >= n) goto L420;
    if (fabs(ggstar) >= 0.2 * gsumsq) goto L420;
    gamma = 0.0;
    c = 0.0;
    for (int i = 1; i <= n; ++i) {
        gamma = gamma + gg[i] * dgr[i];
        c = c + gg[i] * dr[i];
    }
    gamma = gamma / gamden;
    if (fabs(beta * gm + gamma * c) >= 0.2 * gsumsq) goto L420;
    for (int i = 1; i <= n; ++i) d[i] = -gg[i] + beta * d[i] + gamma * dr[i];
    itcrs = itcrs + 1;
    goto L30;
L420:
    itcrs = 2;
    gamden = gm - dginit;
    for (int i = 1; i <= n; ++i) {
        dr[i] = d[i];
        dgr[i] = gg[i] - gs[i];
        d[i] = -gg[i] + beta * d[i];
    }
    goto L30;

done:
    /* quench: unpack x into the positions and the box (src/quench_m.F90:138-160) */
    for (int i = 1; i <= nm; ++i) {
        s->x0[i] = x[3 * i - 2];
        s->y0[i] = x[3 * i - 1];
        s->z0[i] = x[3 * i];
    }
    nm3 = 3 * nm;
    for (int i = 1; i <= 3; ++i)
        for (int j = 1; j <= 3; ++j) M3(s->b0, i, j) = x[++nm3];
    s->vol = vol3(s->b0);
    if (out) {
        out[0] = f;
        out[1] = q.pe;
        out[2] = gsumsq;
        out[3] = q.last_fmax;
        out[4] = (double)maxfnc;
        out[5] = (double)iterc;
        out[6] = (double)iflag;
        out[7] = (double)fstat;
    }
    free(q.x); free(q.g); free(q.en);
    free(dr); free(dgr); free(d); free(gs); free(xx); free(gg);
    return fstat;
}
