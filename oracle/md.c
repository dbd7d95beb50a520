/*
 * md.c -- oracle restatement of the MOLDY MD hot path.  TEST INFRASTRUCTURE
 * ONLY (see moldy_oracle.h).  Each routine names the reference routine and
 * lines it restates; loop order, OpenMP structure (per-link-cell locks) and
 * floating-point expression order follow the Fortran.  Run with one thread
 * for bit-reproducible results; more threads only for timing.
 */
#include "oracle_internal.h"

#include <math.h>
#include <string.h>

/* src/linkcell_m.F90:66 */
#define HMEPS 0.4999999999

/* src/constants_m.F90:87-93 */
#define BOLTZMANN 1.3806504e-23
#define ELECTRON_C 1.602176487e-19
#define BK (BOLTZMANN / ELECTRON_C)

static double *dalloc(int n) { return (double *)calloc((size_t)n + 1, sizeof(double)); }
static int *ialloc(int n) { return (int *)calloc((size_t)n + 1, sizeof(int)); }

void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_get_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

orc_sys *orc_create(int nm, int nnbrs, int ivol, int ntcm, int atomstress,
                    double rnear, double deltat, double press, double bdel2)
{
    if (nm < 1 || nnbrs < 1) return NULL;
    orc_sys *s = (orc_sys *)calloc(1, sizeof(orc_sys));
    s->nm = nm; s->nnbrs = nnbrs; s->ivol = ivol; s->ntcm = ntcm;
    s->atomstress = atomstress; s->rnear = rnear; s->deltat = deltat;
    s->press = press; s->bdel2 = bdel2; s->ntc = 0;
    s->nlcx = s->nlcy = s->nlcz = 3;
    double **d[] = {&s->x0, &s->y0, &s->z0, &s->x1, &s->y1, &s->z1, &s->x2, &s->y2, &s->z2,
                    &s->x1dt2, &s->y1dt2, &s->z1dt2, &s->fx, &s->fy, &s->fz, &s->rho,
                    &s->afrho, &s->dafrho, &s->stx, &s->sty, &s->stz, &s->atomic_mass, &s->del2};
    for (size_t k = 0; k < sizeof(d) / sizeof(d[0]); ++k) *d[k] = dalloc(nm);
    s->atomic_number = ialloc(nm);
    s->link = ialloc(nm);
    s->ic = ialloc(nm);
    s->numn = ialloc(nm);
    s->nlist = (int *)calloc((size_t)nnbrs * (size_t)nm, sizeof(int));
    return s;
}

static void free_cells(orc_sys *s)
{
#ifdef _OPENMP
    if (s->locks) {
        for (int i = 0; i <= s->nlocks; ++i) omp_destroy_lock(&s->locks[i]);
        free(s->locks);
        s->locks = NULL;
    }
#endif
    free(s->l0);
    s->l0 = NULL;
}

void orc_destroy(orc_sys *s)
{
    if (!s) return;
    double *d[] = {s->x0, s->y0, s->z0, s->x1, s->y1, s->z1, s->x2, s->y2, s->z2,
                   s->x1dt2, s->y1dt2, s->z1dt2, s->fx, s->fy, s->fz, s->rho,
                   s->afrho, s->dafrho, s->stx, s->sty, s->stz, s->atomic_mass, s->del2};
    for (size_t k = 0; k < sizeof(d) / sizeof(d[0]); ++k) free(d[k]);
    free(s->atomic_number); free(s->link); free(s->ic); free(s->numn); free(s->nlist);
    free_cells(s);
    orc_free_tables(s);
    free(s);
}

/* ------------------------------------------------------------------ state */
void orc_set_state(orc_sys *s, const double *x0, const double *y0, const double *z0,
                   const double *x1, const double *y1, const double *z1,
                   const double *x2, const double *y2, const double *z2,
                   const double *b0, const double *b1, const double *b2,
                   const int *atomic_number, const double *atomic_mass,
                   const double *del2, const double *tgid)
{
    size_t n = (size_t)s->nm * sizeof(double);
    if (x0) memcpy(s->x0 + 1, x0, n);
    if (y0) memcpy(s->y0 + 1, y0, n);
    if (z0) memcpy(s->z0 + 1, z0, n);
    if (x1) memcpy(s->x1 + 1, x1, n);
    if (y1) memcpy(s->y1 + 1, y1, n);
    if (z1) memcpy(s->z1 + 1, z1, n);
    if (x2) memcpy(s->x2 + 1, x2, n);
    if (y2) memcpy(s->y2 + 1, y2, n);
    if (z2) memcpy(s->z2 + 1, z2, n);
    if (b0) memcpy(s->b0, b0, 9 * sizeof(double));
    if (b1) memcpy(s->b1, b1, 9 * sizeof(double));
    if (b2) memcpy(s->b2, b2, 9 * sizeof(double));
    if (atomic_number) memcpy(s->atomic_number + 1, atomic_number, (size_t)s->nm * sizeof(int));
    if (atomic_mass) memcpy(s->atomic_mass + 1, atomic_mass, n);
    if (del2) memcpy(s->del2 + 1, del2, n);
    if (tgid) memcpy(s->tgid, tgid, 9 * sizeof(double));
}

void orc_get_state(const orc_sys *s, double *x0, double *y0, double *z0,
                   double *x1, double *y1, double *z1,
                   double *x2, double *y2, double *z2,
                   double *b0, double *b1, double *b2, double *tgid)
{
    size_t n = (size_t)s->nm * sizeof(double);
    if (x0) memcpy(x0, s->x0 + 1, n);
    if (y0) memcpy(y0, s->y0 + 1, n);
    if (z0) memcpy(z0, s->z0 + 1, n);
    if (x1) memcpy(x1, s->x1 + 1, n);
    if (y1) memcpy(y1, s->y1 + 1, n);
    if (z1) memcpy(z1, s->z1 + 1, n);
    if (x2) memcpy(x2, s->x2 + 1, n);
    if (y2) memcpy(y2, s->y2 + 1, n);
    if (z2) memcpy(z2, s->z2 + 1, n);
    if (b0) memcpy(b0, s->b0, 9 * sizeof(double));
    if (b1) memcpy(b1, s->b1, 9 * sizeof(double));
    if (b2) memcpy(b2, s->b2, 9 * sizeof(double));
    if (tgid) memcpy(tgid, s->tgid, 9 * sizeof(double));
}

void orc_get_forces(const orc_sys *s, double *fx, double *fy, double *fz)
{
    size_t n = (size_t)s->nm * sizeof(double);
    memcpy(fx, s->fx + 1, n); memcpy(fy, s->fy + 1, n); memcpy(fz, s->fz + 1, n);
}

void orc_get_density(const orc_sys *s, double *rho, double *afrho, double *dafrho)
{
    size_t n = (size_t)s->nm * sizeof(double);
    if (rho) memcpy(rho, s->rho + 1, n);
    if (afrho) memcpy(afrho, s->afrho + 1, n);
    if (dafrho) memcpy(dafrho, s->dafrho + 1, n);
}

void orc_get_atomstress(const orc_sys *s, double *sx, double *sy, double *sz)
{
    size_t n = (size_t)s->nm * sizeof(double);
    memcpy(sx, s->stx + 1, n); memcpy(sy, s->sty + 1, n); memcpy(sz, s->stz + 1, n);
}

void orc_get_force_out(const orc_sys *s, double *o)
{
    o[0] = s->pe; o[1] = s->vol;
    const double *m[] = {s->tp, s->tk, s->tc, s->tg, s->tgdot, s->tgid, s->fb};
    for (int k = 0; k < 7; ++k) memcpy(o + 2 + 9 * k, m[k], 9 * sizeof(double));
}

void orc_set_ntc(orc_sys *s, int ntc) { s->ntc = ntc; }
int orc_get_ntc(const orc_sys *s) { return s->ntc; }

/* ------------------------------------------------------------- geometry */
/* src/parrinellorahman_m.F90:149-173 (pr_get_realsep_from_dx) */
static inline double realsep(const orc_sys *s, double *dx, double *dy, double *dz)
{
    int iv = s->ivol;
    if (iv == 0 || iv == 1 || iv == 4) {
        *dx = *dx - round(*dx); *dy = *dy - round(*dy); *dz = *dz - round(*dz);
    } else if (iv == 2) {
        *dx = *dx - round(*dx); *dy = *dy - round(*dy);
    } else if (iv == 5) {
        *dz = *dz - round(*dz);
    }
    const double *b = s->b0;
    double rx = M3(b, 1, 1) * *dx + M3(b, 1, 2) * *dy + M3(b, 1, 3) * *dz;
    double ry = M3(b, 2, 1) * *dx + M3(b, 2, 2) * *dy + M3(b, 2, 3) * *dz;
    double rz = M3(b, 3, 1) * *dx + M3(b, 3, 2) * *dy + M3(b, 3, 3) * *dz;
    return sqrt(rx * rx + ry * ry + rz * rz);
}

/* src/parrinellorahman_m.F90:223-227 (pr_get_metric_tensor: volume) */
static double box_volume(const double *b)
{
    return M3(b, 1, 1) * (M3(b, 2, 2) * M3(b, 3, 3) - M3(b, 2, 3) * M3(b, 3, 2)) +
           M3(b, 2, 1) * (M3(b, 3, 2) * M3(b, 1, 3) - M3(b, 1, 2) * M3(b, 3, 3)) +
           M3(b, 3, 1) * (M3(b, 1, 2) * M3(b, 2, 3) - M3(b, 2, 2) * M3(b, 1, 3));
}

/* src/matrix_m.F90:60-79 */
static void matrix_multiply3(const double *a, const double *b, double *c)
{
    for (int i = 1; i <= 3; ++i) {
        for (int j = 1; j <= 3; ++j) M3(c, i, j) = 0.0;
        for (int k = 1; k <= 3; ++k)
            for (int j = 1; j <= 3; ++j) M3(c, i, j) = M3(c, i, j) + M3(a, i, k) * M3(b, k, j);
    }
}

/* src/matrix_m.F90:89-119; returns 1 when the determinant is zero */
static int matrix_invert3(const double *a, double *b)
{
    double deta = M3(a, 1, 1) * (M3(a, 2, 2) * M3(a, 3, 3) - M3(a, 2, 3) * M3(a, 3, 2));
    deta = deta + M3(a, 2, 1) * (M3(a, 3, 2) * M3(a, 1, 3) - M3(a, 1, 2) * M3(a, 3, 3));
    deta = deta + M3(a, 3, 1) * (M3(a, 1, 2) * M3(a, 2, 3) - M3(a, 1, 3) * M3(a, 2, 2));
    M3(b, 1, 1) = M3(a, 2, 2) * M3(a, 3, 3) - M3(a, 2, 3) * M3(a, 3, 2);
    M3(b, 1, 2) = M3(a, 3, 1) * M3(a, 2, 3) - M3(a, 2, 1) * M3(a, 3, 3);
    M3(b, 1, 3) = M3(a, 2, 1) * M3(a, 3, 2) - M3(a, 3, 1) * M3(a, 2, 2);
    M3(b, 2, 1) = M3(a, 3, 2) * M3(a, 1, 3) - M3(a, 1, 2) * M3(a, 3, 3);
    M3(b, 2, 2) = M3(a, 1, 1) * M3(a, 3, 3) - M3(a, 1, 3) * M3(a, 3, 1);
    M3(b, 2, 3) = M3(a, 3, 1) * M3(a, 1, 2) - M3(a, 1, 1) * M3(a, 3, 2);
    M3(b, 3, 1) = M3(a, 1, 2) * M3(a, 2, 3) - M3(a, 1, 3) * M3(a, 2, 2);
    M3(b, 3, 2) = M3(a, 2, 1) * M3(a, 1, 3) - M3(a, 2, 3) * M3(a, 1, 1);
    M3(b, 3, 3) = M3(a, 1, 1) * M3(a, 2, 2) - M3(a, 1, 2) * M3(a, 2, 1);
    if (fabs(deta) == 0.0) return 1;
    for (int k = 0; k < 9; ++k) b[k] = b[k] / deta;
    return 0;
}

/* ----------------------------------------------------------- link cells */
void orc_set_nlc(orc_sys *s, int nlcx, int nlcy, int nlcz)
{
    free_cells(s);
    s->nlcx = nlcx; s->nlcy = nlcy; s->nlcz = nlcz;
    s->ncell = nlcx * nlcy * nlcz;
    s->l0 = ialloc(s->ncell);
#ifdef _OPENMP
    s->nlocks = s->ncell;
    s->locks = (omp_lock_t *)malloc(((size_t)s->ncell + 1) * sizeof(omp_lock_t));
    for (int i = 0; i <= s->ncell; ++i) omp_init_lock(&s->locks[i]);
#endif
}

void orc_get_nlc(const orc_sys *s, int *n3) { n3[0] = s->nlcx; n3[1] = s->nlcy; n3[2] = s->nlcz; }

static inline int cell_of(const orc_sys *s, int i)
{
    int ix = (int)((s->x0[i] - round(s->x0[i]) + HMEPS) * (double)s->nlcx);
    int iy = (int)((s->y0[i] - round(s->y0[i]) + HMEPS) * (double)s->nlcy);
    int iz = (int)((s->z0[i] - round(s->z0[i]) + HMEPS) * (double)s->nlcz);
    return ix + s->nlcx * iy + s->nlcx * s->nlcy * iz + 1;
}

/* src/linkcell_m.F90:122-198 (linkup) */
void orc_linkup(orc_sys *s)
{
    int *l1 = ialloc(s->ncell);
    for (int ip = 1; ip <= s->ncell; ++ip) s->l0[ip] = 0;
    for (int i = 1; i <= s->nm; ++i) {
        int ip = cell_of(s, i);
        s->ic[i] = ip;
        int me = l1[ip];
        if (me != 0) { s->link[me] = i; l1[ip] = i; }
        else { s->l0[ip] = i; l1[ip] = i; }
    }
    for (int ip = 1; ip <= s->ncell; ++ip) {
        int me = l1[ip];
        if (me == 0) continue;
        s->link[me] = s->l0[ip];
    }
    free(l1);
}

/* src/linkcell_m.F90:215-274 (relink) */
void orc_relink(orc_sys *s)
{
    for (int i = 1; i <= s->nm; ++i) {
        int ip = cell_of(s, i);
        if (ip == s->ic[i]) continue;
        int me = s->ic[i];
        int j = s->l0[me];
        while (s->link[j] != i) j = s->link[j];
        s->link[j] = s->link[i];
        s->l0[me] = s->link[j];
        if (i == j) s->l0[me] = 0;
        j = s->l0[ip];
        if (s->l0[ip] == 0) j = i;
        s->link[i] = s->link[j];
        s->link[j] = i;
        s->ic[i] = ip;
        s->l0[ip] = i;
    }
}

void orc_get_linkcells(const orc_sys *s, int *l0, int *link, int *ic)
{
    if (l0) memcpy(l0, s->l0 + 1, (size_t)s->ncell * sizeof(int));
    if (link) memcpy(link, s->link + 1, (size_t)s->nm * sizeof(int));
    if (ic) memcpy(ic, s->ic + 1, (size_t)s->nm * sizeof(int));
}

/* src/neighbourlist_m.F90:103-276 (update_neighbourlist): half list over the
 * 14-cell half stencil, j after i inside the home cell, r < rnear. */
int orc_update_neighbourlist(orc_sys *s)
{
    const int nx = s->nlcx, ny = s->nlcy, nz = s->nlcz, nn = s->nnbrs;
    int overflow = 0;
    for (int i = 1; i <= s->nm; ++i) s->numn[i] = 0;
    const int *l0 = s->l0, *link = s->link;
#pragma omp parallel for schedule(static) reduction(| : overflow)
    for (int ip = 1; ip <= s->ncell; ++ip) {
        int ix = (ip - 1) % nx + 1;
        int iy = ((ip - 1) / nx) % ny + 1;
        int iz = ((ip - 1) / (nx * ny)) % nz + 1;
        int i = l0[ip];
        if (l0[ip] == 0) continue;
        for (int kz = 2; kz <= 3; ++kz) {
            int jz = iz + kz - 2;
            if (jz - nz - 1 == 0) jz = 1;
            int kk = (kz == 3) ? 1 : 2;
            int jzn = (jz - 1) * nx * ny;
            for (int ky = kk; ky <= 3; ++ky) {
                int jy = iy + ky - 2;
                if (jy == 0) jy = ny;
                if (jy - ny - 1 == 0) jy = 1;
                int kl = (kz == 2 && ky == 2) ? 2 : 1;
                int jyzn = jzn + (jy - 1) * nx;
                for (int kx = kl; kx <= 3; ++kx) {
                    int jx = ix + kx - 2;
                    if (jx == 0) jx = nx;
                    if (jx - nx - 1 == 0) jx = 1;
                    int jp = jx + jyzn;
                    for (;;) { /* linkloop */
                        int j;
                        if (ip == jp) {
                            j = link[i];
                            if (j == l0[ip]) { i = l0[ip]; break; }
                        } else {
                            j = l0[jp];
                            if (j == 0) break;
                        }
                        for (;;) { /* testcandidates */
                            double dx = s->x0[i] - s->x0[j];
                            double dy = s->y0[i] - s->y0[j];
                            double dz = s->z0[i] - s->z0[j];
                            double r = realsep(s, &dx, &dy, &dz);
                            if (r < s->rnear) {
                                s->numn[i] = s->numn[i] + 1;
                                if (s->numn[i] > nn) overflow = 1;
                                else s->nlist[(size_t)(s->numn[i] - 1) + (size_t)nn * (size_t)(i - 1)] = j;
                            }
                            j = link[j];
                            if (j == l0[jp]) break;
                        }
                        i = link[i];
                        if (i == l0[ip]) break;
                    }
                }
            }
        }
    }
    return overflow;
}

void orc_get_nlist(const orc_sys *s, int *nlist, int *numn)
{
    if (nlist) memcpy(nlist, s->nlist, (size_t)s->nnbrs * (size_t)s->nm * sizeof(int));
    if (numn) memcpy(numn, s->numn + 1, (size_t)s->nm * sizeof(int));
}

#ifdef _OPENMP
#define LOCK_SWITCH(cell)                                         \
    do {                                                          \
        if ((cell) != neighlc) {                                  \
            if (neighlc > 0) omp_unset_lock(&s->locks[neighlc]);  \
            neighlc = (cell);                                     \
            omp_set_lock(&s->locks[neighlc]);                     \
        }                                                         \
    } while (0)
#define LOCK_RELEASE()                                            \
    do { if (neighlc > 0) omp_unset_lock(&s->locks[neighlc]); } while (0)
#else
#define LOCK_SWITCH(cell) do { (void)(cell); } while (0)
#define LOCK_RELEASE() do { } while (0)
#endif

/* src/dynamics_m.F90:497-579 (rhoset) */
static void rhoset(orc_sys *s)
{
    const int nn = s->nnbrs;
    for (int i = 1; i <= s->nm; ++i) s->rho[i] = 0.0;
#pragma omp parallel
    {
        int neighlc = 0;
#pragma omp for schedule(static) nowait
        for (int i = 1; i <= s->nm; ++i) {
            double rho_tmp = 0.0;
            for (int k = 1; k <= s->numn[i]; ++k) {
                int j = s->nlist[(size_t)(k - 1) + (size_t)nn * (size_t)(i - 1)];
                double dx = s->x0[i] - s->x0[j];
                double dy = s->y0[i] - s->y0[j];
                double dz = s->z0[i] - s->z0[j];
                double r = realsep(s, &dx, &dy, &dz);
                LOCK_SWITCH(s->ic[j]);
                s->rho[j] = s->rho[j] + orc_phi(s, r);
                rho_tmp = rho_tmp + orc_phi(s, r);
            }
            LOCK_SWITCH(s->ic[i]);
            s->rho[i] = s->rho[i] + rho_tmp;
        }
        LOCK_RELEASE();
    }
}

/* src/potential_m.F90:148-169 (embed): rho <= 1e-40 keeps stale values */
static double embed(orc_sys *s)
{
    double pexx = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : pexx)
    for (int i = 1; i <= s->nm; ++i) {
        if (s->rho[i] <= 1e-40) continue;
        s->afrho[i] = orc_emb(s, s->rho[i]);
        pexx = pexx + s->afrho[i];
        s->dafrho[i] = orc_demb(s, s->rho[i]);
    }
    return pexx;
}

/* src/thermostat_m.F90:127-177 (kinten) */
static void kinten(orc_sys *s)
{
    double *tk = s->tk, *b0 = s->b0, *b1 = s->b1;
    for (int k = 0; k < 9; ++k) tk[k] = 0.0;
    for (int i = 1; i <= s->nm; ++i) {
        if (s->atomic_number[i] == 0) continue;
        double m = s->atomic_mass[i], x1 = s->x1[i], y1 = s->y1[i], z1 = s->z1[i];
        double mvx = (M3(b0, 1, 1) * x1 + M3(b0, 1, 2) * y1 + M3(b0, 1, 3) * z1) * m;
        double mvy = (M3(b0, 2, 1) * x1 + M3(b0, 2, 2) * y1 + M3(b0, 2, 3) * z1) * m;
        double mvz = (M3(b0, 3, 1) * x1 + M3(b0, 3, 2) * y1 + M3(b0, 3, 3) * z1) * m;
        M3(tk, 1, 1) = M3(tk, 1, 1) + x1 * mvx;
        M3(tk, 2, 1) = M3(tk, 2, 1) + x1 * mvy;
        M3(tk, 3, 1) = M3(tk, 3, 1) + x1 * mvz;
        M3(tk, 1, 2) = M3(tk, 1, 2) + y1 * mvx;
        M3(tk, 2, 2) = M3(tk, 2, 2) + y1 * mvy;
        M3(tk, 3, 2) = M3(tk, 3, 2) + y1 * mvz;
        M3(tk, 1, 3) = M3(tk, 1, 3) + z1 * mvx;
        M3(tk, 2, 3) = M3(tk, 2, 3) + z1 * mvy;
        M3(tk, 3, 3) = M3(tk, 3, 3) + z1 * mvz;
    }
    for (int i = 1; i <= 3; ++i)
        for (int j = 1; j <= 3; ++j) M3(tk, i, j) = M3(tk, i, j) / (s->deltat * s->deltat);
    double *tgd = s->tgdot;
    for (int k = 0; k < 9; ++k) tgd[k] = 0.0;
    for (int i = 1; i <= 3; ++i)
        for (int k = 1; k <= 3; ++k)
            for (int j = 1; j <= 3; ++j)
                M3(tgd, i, j) = M3(tgd, i, j) + M3(b0, k, i) * M3(b1, k, j) + M3(b1, k, i) * M3(b0, k, j);
}

/* src/dynamics_m.F90:135-401 (force) */
int orc_force(orc_sys *s)
{
    const int nn = s->nnbrs;
    int status = 0;
    for (int k = 0; k < 9; ++k) { s->tp[k] = 0.0; s->tg[k] = 0.0; }
    s->ke = 0.0;
    for (int i = 1; i <= s->nm; ++i) {
        s->stx[i] = 0.0; s->sty[i] = 0.0; s->stz[i] = 0.0;
        s->fx[i] = 0.0; s->fy[i] = 0.0; s->fz[i] = 0.0;
    }
    s->vol = box_volume(s->b0);
    s->ntc = s->ntc + 1;
    if (s->ntc == 1) status = orc_update_neighbourlist(s);
    if (s->ntc == s->ntcm) s->ntc = 0;
    if (status) return status;

    rhoset(s);
    s->pe = embed(s);

    double *b0 = s->b0;
    for (int i = 1; i <= 3; ++i)
        for (int k = 1; k <= 3; ++k)
            for (int j = 1; j <= 3; ++j) M3(s->tg, i, j) = M3(s->tg, i, j) + M3(b0, k, i) * M3(b0, k, j);

    double pe = s->pe;
    double tp11 = 0, tp21 = 0, tp31 = 0, tp12 = 0, tp22 = 0, tp32 = 0, tp13 = 0, tp23 = 0, tp33 = 0;
#pragma omp parallel reduction(+ : pe, tp11, tp21, tp31, tp12, tp22, tp32, tp13, tp23, tp33)
    {
        int neighlc = 0;
#pragma omp for schedule(static) nowait
        for (int i = 1; i <= s->nm; ++i) {
            double fxi = 0.0, fyi = 0.0, fzi = 0.0;
            for (int k = 1; k <= s->numn[i]; ++k) {
                int j = s->nlist[(size_t)(k - 1) + (size_t)nn * (size_t)(i - 1)];
                double dx = s->x0[i] - s->x0[j];
                double dy = s->y0[i] - s->y0[j];
                double dz = s->z0[i] - s->z0[j];
                double r = realsep(s, &dx, &dy, &dz);
                double r_recip = 1.0 / r;
                double pp = orc_vee(s, r);
                double fpp = -orc_dvee(s, r) * r_recip;
                pe = pe + pp;
                double fcp = -(1.0 * (orc_dphi(s, r) * s->dafrho[i] + orc_dphi(s, r) * s->dafrho[j])) * r_recip;
                double fp = fpp + fcp;
                double rx = M3(b0, 1, 1) * dx + M3(b0, 1, 2) * dy + M3(b0, 1, 3) * dz;
                double ry = M3(b0, 2, 1) * dx + M3(b0, 2, 2) * dy + M3(b0, 2, 3) * dz;
                double rz = M3(b0, 3, 1) * dx + M3(b0, 3, 2) * dy + M3(b0, 3, 3) * dz;
                if (s->atomstress) {
                    s->stx[i] = s->stx[i] + rx * fp;
                    s->sty[i] = s->sty[i] + ry * fp;
                    s->stz[i] = s->stz[i] + rz * fp;
                }
                if ((s->atomic_mass[i] + s->atomic_mass[j]) > 0.1) {
                    tp11 = tp11 + dx * rx * fp;
                    tp21 = tp21 + dx * ry * fp;
                    tp31 = tp31 + dx * rz * fp;
                    tp12 = tp12 + dy * rx * fp;
                    tp22 = tp22 + dy * ry * fp;
                    tp32 = tp32 + dy * rz * fp;
                    tp13 = tp13 + dz * rx * fp;
                    tp23 = tp23 + dz * ry * fp;
                    tp33 = tp33 + dz * rz * fp;
                }
                double ddfx = -(dx * fp), ddfy = -(dy * fp), ddfz = -(dz * fp);
                LOCK_SWITCH(s->ic[j]);
                s->fx[j] = s->fx[j] + ddfx;
                s->fy[j] = s->fy[j] + ddfy;
                s->fz[j] = s->fz[j] + ddfz;
                fxi = fxi + ddfx;
                fyi = fyi + ddfy;
                fzi = fzi + ddfz;
            }
            LOCK_SWITCH(s->ic[i]);
            s->fx[i] = s->fx[i] - fxi;
            s->fy[i] = s->fy[i] - fyi;
            s->fz[i] = s->fz[i] - fzi;
        }
        LOCK_RELEASE();
    }
    s->pe = pe;
    double *tp = s->tp;
    M3(tp, 1, 1) = tp11; M3(tp, 2, 1) = tp21; M3(tp, 3, 1) = tp31;
    M3(tp, 1, 2) = tp12; M3(tp, 2, 2) = tp22; M3(tp, 3, 2) = tp32;
    M3(tp, 1, 3) = tp13; M3(tp, 2, 3) = tp23; M3(tp, 3, 3) = tp33;

    double *tc = s->tc;
    M3(tc, 1, 1) = M3(b0, 2, 2) * M3(b0, 3, 3) - M3(b0, 2, 3) * M3(b0, 3, 2);
    M3(tc, 2, 1) = M3(b0, 3, 2) * M3(b0, 1, 3) - M3(b0, 1, 2) * M3(b0, 3, 3);
    M3(tc, 3, 1) = M3(b0, 1, 2) * M3(b0, 2, 3) - M3(b0, 2, 2) * M3(b0, 1, 3);
    M3(tc, 1, 2) = M3(b0, 2, 3) * M3(b0, 3, 1) - M3(b0, 3, 3) * M3(b0, 2, 1);
    M3(tc, 2, 2) = M3(b0, 3, 3) * M3(b0, 1, 1) - M3(b0, 1, 3) * M3(b0, 3, 1);
    M3(tc, 3, 2) = M3(b0, 1, 3) * M3(b0, 2, 1) - M3(b0, 1, 1) * M3(b0, 2, 3);
    M3(tc, 1, 3) = M3(b0, 2, 1) * M3(b0, 3, 2) - M3(b0, 3, 1) * M3(b0, 2, 2);
    M3(tc, 2, 3) = M3(b0, 3, 1) * M3(b0, 1, 2) - M3(b0, 1, 1) * M3(b0, 3, 2);
    M3(tc, 3, 3) = M3(b0, 1, 1) * M3(b0, 2, 2) - M3(b0, 2, 1) * M3(b0, 1, 2);
    kinten(s);
    for (int i = 1; i <= 3; ++i)
        for (int j = 1; j <= 3; ++j)
            M3(s->fb, i, j) = M3(s->tk, i, j) + M3(s->tp, i, j) - s->press * M3(s->tc, i, j);
    return 0;
}

/* src/quench_m.F90:562-624 (velocityverlet) */
int orc_velocityverlet(orc_sys *s)
{
    double sxi = 0.0, syi = 0.0, szi = 0.0;
    int n = s->nm;
    for (int i = 1; i <= n; ++i) {
        s->x1dt2[i] = s->x1[i] + s->x2[i];
        s->y1dt2[i] = s->y1[i] + s->y2[i];
        s->z1dt2[i] = s->z1[i] + s->z2[i];
    }
    for (int i = 1; i <= n; ++i) {
        s->x0[i] = s->x0[i] + s->x1dt2[i];
        s->y0[i] = s->y0[i] + s->y1dt2[i];
        s->z0[i] = s->z0[i] + s->z1dt2[i];
    }
    if (s->ivol == 4) {
        M3(s->b1, 3, 3) = M3(s->b1, 3, 3) + M3(s->b2, 3, 3);
        M3(s->b0, 3, 3) = M3(s->b0, 3, 3) + M3(s->b1, 3, 3);
    }
    if (s->ivol < 1) {
        for (int k = 0; k < 9; ++k) s->b1[k] = s->b1[k] + s->b2[k];
        for (int k = 0; k < 9; ++k) s->b0[k] = s->b0[k] + s->b1[k];
    }
    int st = orc_force(s);
    if (st) return st;
    double *tgid = s->tgid;
    if (s->ivol < 1) {
        for (int k = 0; k < 9; ++k) s->b2[k] = s->bdel2 * s->fb[k];
        for (int k = 0; k < 9; ++k) s->b1[k] = s->b1[k] + s->b2[k];
    }
    if (s->ivol == 4) {
        M3(s->b2, 3, 3) = s->bdel2 * M3(s->fb, 3, 3);
        for (int k = 0; k < 9; ++k) s->b1[k] = s->b1[k] + s->b2[k];
    }
    for (int i = 1; i <= n; ++i) {
        if (s->atomic_number[i] == 0 || s->atomic_mass[i] < 0.1) continue;
        double x1 = s->x1[i], y1 = s->y1[i], z1 = s->z1[i];
        if (s->ivol == 0) {
            sxi = M3(tgid, 1, 1) * x1 + M3(tgid, 1, 2) * y1 + M3(tgid, 1, 3) * z1;
            syi = M3(tgid, 2, 1) * x1 + M3(tgid, 2, 2) * y1 + M3(tgid, 2, 3) * z1;
            szi = M3(tgid, 3, 1) * x1 + M3(tgid, 3, 2) * y1 + M3(tgid, 3, 3) * z1;
        }
        if (s->ivol == 4) szi = M3(tgid, 3, 3) * z1;
        s->x2[i] = s->del2[i] * s->fx[i] - 0.5 * sxi;
        s->y2[i] = s->del2[i] * s->fy[i] - 0.5 * syi;
        s->z2[i] = s->del2[i] * s->fz[i] - 0.5 * szi;
    }
    for (int i = 1; i <= n; ++i) {
        s->x1[i] = s->x1dt2[i] + s->x2[i];
        s->y1[i] = s->y1dt2[i] + s->y2[i];
        s->z1[i] = s->z1dt2[i] + s->z2[i];
    }
    return 0;
}

/* src/dynamics_m.F90:649-734 (update_therm_avs); s123 = s1, s2, s3 */
void orc_update_therm_avs(orc_sys *s, double *s123)
{
    double s1 = 0.0, s2 = 0.0, s3 = 0.0;
    double *b0 = s->b0, *b1 = s->b1, *tg = s->tg, *tgd = s->tgdot, *tgid = s->tgid;
    for (int k = 0; k < 9; ++k) { tg[k] = 0.0; tgd[k] = 0.0; }
    for (int i = 1; i <= 3; ++i)
        for (int k = 1; k <= 3; ++k)
            for (int j = 1; j <= 3; ++j) {
                M3(tg, i, j) = M3(tg, i, j) + M3(b0, k, i) * M3(b0, k, j);
                if (s->ivol != 1)
                    M3(tgd, i, j) = M3(tgd, i, j) + M3(b1, k, i) * M3(b0, k, j) + M3(b0, k, i) * M3(b1, k, j);
            }
    /* pr_get_tgid (src/parrinellorahman_m.F90:254-261) */
    matrix_invert3(tg, s->tginv);
    matrix_multiply3(s->tginv, tgd, tgid);
    s->vol = box_volume(b0);
    double vol = s->vol;
    double bxx = (M3(b0, 2, 2) * M3(b0, 3, 3) - M3(b0, 2, 3) * M3(b0, 3, 2)) / vol;
    double bxy = (M3(b0, 2, 3) * M3(b0, 3, 1) - M3(b0, 3, 3) * M3(b0, 2, 1)) / vol;
    double bxz = (M3(b0, 2, 1) * M3(b0, 3, 2) - M3(b0, 3, 1) * M3(b0, 2, 2)) / vol;
    double byx = (M3(b0, 3, 2) * M3(b0, 1, 3) - M3(b0, 1, 2) * M3(b0, 3, 3)) / vol;
    double byy = (M3(b0, 1, 1) * M3(b0, 3, 3) - M3(b0, 1, 3) * M3(b0, 3, 1)) / vol;
    double byz = (M3(b0, 3, 1) * M3(b0, 1, 2) - M3(b0, 1, 1) * M3(b0, 3, 2)) / vol;
    double bzx = (M3(b0, 1, 2) * M3(b0, 2, 3) - M3(b0, 2, 2) * M3(b0, 1, 3)) / vol;
    double bzy = (M3(b0, 1, 3) * M3(b0, 2, 1) - M3(b0, 1, 1) * M3(b0, 2, 3)) / vol;
    double bzz = (M3(b0, 1, 1) * M3(b0, 2, 2) - M3(b0, 1, 2) * M3(b0, 2, 1)) / vol;
    for (int i = 1; i <= s->nm; ++i) {
        if (s->atomic_number[i] == 0) continue;
        double x1 = s->x1[i], y1 = s->y1[i], z1 = s->z1[i];
        double sxi = M3(tgid, 1, 1) * x1 + M3(tgid, 1, 2) * y1 + M3(tgid, 1, 3) * z1;
        double syi = M3(tgid, 2, 1) * x1 + M3(tgid, 2, 2) * y1 + M3(tgid, 2, 3) * z1;
        double szi = M3(tgid, 3, 1) * x1 + M3(tgid, 3, 2) * y1 + M3(tgid, 3, 3) * z1;
        double fxip = 2.0 * s->x2[i] + sxi;
        double fyip = 2.0 * s->y2[i] + syi;
        double fzip = 2.0 * s->z2[i] + szi;
        double fxi = bxx * fxip + bxy * fyip + bxz * fzip;
        double fyi = byx * fxip + byy * fyip + byz * fzip;
        double fzi = bzx * fxip + bzy * fyip + bzz * fzip;
        double f2 = fxi * fxi + fyi * fyi + fzi * fzi;
        s1 = s1 + f2;
        s2 = s2 + f2 * f2;
        double rxi = M3(b0, 1, 1) * x1 + M3(b0, 1, 2) * y1 + M3(b0, 1, 3) * z1;
        double ryi = M3(b0, 2, 1) * x1 + M3(b0, 2, 2) * y1 + M3(b0, 2, 3) * z1;
        double rzi = M3(b0, 3, 1) * x1 + M3(b0, 3, 2) * y1 + M3(b0, 3, 3) * z1;
        s3 = s3 + s->atomic_mass[i] * (rxi * rxi + ryi * ryi + rzi * rzi);
    }
    s123[0] = s1; s123[1] = s2; s123[2] = s3;
}

/* src/dynamics_m.F90:412-483 (energy_calc): always the exact pair function */
void orc_energy_calc(orc_sys *s, double *en_atom)
{
    const int nn = s->nnbrs;
    double *en = (double *)malloc(((size_t)s->nm + 1) * sizeof(double));
    for (int i = 1; i <= s->nm; ++i) en[i] = s->afrho[i];
    for (int i = 1; i <= s->nm; ++i) {
        for (int k = 1; k <= s->numn[i]; ++k) {
            int j = s->nlist[(size_t)(k - 1) + (size_t)nn * (size_t)(i - 1)];
            double dx = s->x0[i] - s->x0[j];
            double dy = s->y0[i] - s->y0[j];
            double dz = s->z0[i] - s->z0[j];
            double r = realsep(s, &dx, &dy, &dz);
            double pp = orc_vee_src(s, r);
            en[i] = en[i] + pp / 2.0;
            en[j] = en[j] + pp / 2.0;
        }
    }
    memcpy(en_atom, en + 1, (size_t)s->nm * sizeof(double));
    free(en);
}

/* src/moldin.F90:445-477: force, tgid = tg^-1 tgdot, initial x2 and b2 */
int orc_md_init(orc_sys *s)
{
    int st = orc_force(s);
    if (st) return st;
    if (matrix_invert3(s->tg, s->tginv)) return 4;
    matrix_multiply3(s->tginv, s->tgdot, s->tgid);
    double *t = s->tgid;
    for (int i = 1; i <= s->nm; ++i) {
        double x1 = s->x1[i], y1 = s->y1[i], z1 = s->z1[i];
        double a1 = M3(t, 1, 1) * x1 + M3(t, 1, 2) * y1 + M3(t, 1, 3) * z1;
        double a2 = M3(t, 2, 1) * x1 + M3(t, 2, 2) * y1 + M3(t, 2, 3) * z1;
        double a3 = M3(t, 3, 1) * x1 + M3(t, 3, 2) * y1 + M3(t, 3, 3) * z1;
        s->x2[i] = s->del2[i] * s->fx[i] - 0.5 * a1;
        s->y2[i] = s->del2[i] * s->fy[i] - 0.5 * a2;
        s->z2[i] = s->del2[i] * s->fz[i] - 0.5 * a3;
    }
    for (int k = 0; k < 9; ++k) s->b2[k] = s->bdel2 * s->fb[k];
    return 0;
}

/* scalev (src/thermostat_m.F90:317-395): Nose-Hoover Euler thermostat */
void orc_scalev(orc_sys *s)
{
    if (!(s->nose > 0.0)) return;
    double sx = 0.0, sy = 0.0, sz = 0.0, s3 = 0.0;
    for (int i = 1; i <= s->nm; ++i) {
        sx = sx + s->x1[i];
        sy = sy + s->y1[i];
        sz = sz + s->z1[i];
    }
    const double fnm = (double)(float)s->nm; /* float(simparam%nm) */
    sx = sx / fnm;
    sy = sy / fnm;
    sz = sz / fnm;
    const double *b0 = s->b0;
    for (int i = 1; i <= s->nm; ++i) {
        if (s->atomic_number[i] == 0 || s->atomic_mass[i] < 0.1) continue;
        s->x1[i] = s->x1[i] - sx;
        s->y1[i] = s->y1[i] - sy;
        s->z1[i] = s->z1[i] - sz;
        double rx = M3(b0, 1, 1) * s->x1[i] + M3(b0, 1, 2) * s->y1[i] + M3(b0, 1, 3) * s->z1[i];
        double ry = M3(b0, 2, 1) * s->x1[i] + M3(b0, 2, 2) * s->y1[i] + M3(b0, 2, 3) * s->z1[i];
        double rz = M3(b0, 3, 1) * s->x1[i] + M3(b0, 3, 2) * s->y1[i] + M3(b0, 3, 3) * s->z1[i];
        s3 = s3 + s->atomic_mass[i] * (rx * rx + ry * ry + rz * rz);
    }
    double ke = s3 / (s->deltat * s->deltat) / 2.0;
    if (ke > 0.0) s->snhf = (ke - s->rqke) / (s->nose * (double)s->nm);
    s->snhv = s->snhv - s->snhf;
    for (int i = 1; i <= s->nm; ++i) {
        if (s->atomic_number[i] == 0 || s->atomic_mass[i] < 0.1) continue;
        s->x1[i] = s->x1[i] * (1.0 + s->snhv);
        s->y1[i] = s->y1[i] * (1.0 + s->snhv);
        s->z1[i] = s->z1[i] * (1.0 + s->snhv);
    }
}

void orc_set_thermostat(orc_sys *s, double nose, double rqke)
{
    s->nose = nose;
    s->rqke = rqke;
}

void orc_get_thermostat(const orc_sys *s, double *out4)
{
    out4[0] = s->nose; out4[1] = s->rqke; out4[2] = s->snhv; out4[3] = s->thermotimer;
}

/* src/moldin.F90:752-835: one mdloop iteration without output; scalev once
 * per femtosecond (fs = 0.098227 model units, src/moldin.F90:132) */
int orc_md_step(orc_sys *s, double *o)
{
    int st = orc_velocityverlet(s);
    if (st) return st;
    double s123[3];
    orc_update_therm_avs(s, s123);
    double ke = s123[2] / (s->deltat * s->deltat) / 2.0;
    double temp = ke / (1.5 * BK * (double)s->nm);
    double boxke = 0.0;
    for (int i = 1; i <= 3; ++i)
        for (int j = 1; j <= 3; ++j) boxke = boxke + (M3(s->b1, i, j) * M3(s->b1, i, j)) / s->bdel2;
    double te = ke + s->pe;
    double h = te + s->press * s->vol;
    double th = h + boxke;
    if (s->ntc == 0) orc_relink(s);
    s->thermotimer = s->thermotimer + s->deltat;
    if (s->thermotimer >= 0.098227) {
        s->thermotimer = s->thermotimer - 0.098227;
        if (s->nose != 0.0) orc_scalev(s);
    }
    if (o) {
        o[0] = ke; o[1] = s->pe; o[2] = te; o[3] = h; o[4] = th; o[5] = s->vol;
        o[6] = s123[0]; o[7] = s123[1]; o[8] = s123[2]; o[9] = temp; o[10] = boxke;
        o[11] = (double)s->ntc;
    }
    return 0;
}
