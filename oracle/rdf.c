/*
 * rdf.c -- radial distribution function and Ackland-Jones local structure
 * (src/analysis_m.F90:497-760), restated for the CPU oracle (TEST
 * INFRASTRUCTURE).
 *
 * Histogram (analysis_m.F90:580-608), two pair sets:
 *   mode 0  the half neighbour list as it stands, pairs with
 *           rsq <= (maxbin/binsperangstrom)**2 (integer division, as written);
 *   mode 1  every pair j < i, the older form of the routine that wrote the
 *           reference's shipped tests/reference/bcc_iron/rdf.dat (its counts
 *           reach bin maxbin, i.e. r up to (maxbin+1)/binsperangstrom).
 * In both, ibin = int(r * binsperangstrom), pairs with ibin > maxbin are
 * dropped and vacancies (atomic number 0) are skipped.  ibin = 0 (the
 * reference would write nbin(0,...) out of bounds) is kept in bin 0.
 *
 * Fourth-neighbour radius (analysis_m.F90:619-637) and the Ackland-Jones
 * bond-angle classification (analysis_m.F90:644-757): the default-REAL
 * literals (1.45, the ctheta bounds, the score constants) are single
 * precision, and the scores are computed in single precision, as gfortran
 * evaluates them.  rnatoms is set for isp <= jsp only; the restatement uses
 * rn(isp,jsp) for both orders.
 */
#include <math.h>
#include <string.h>

#include "oracle_internal.h"

/* pr_get_realsep2_from_dx (src/parrinellorahman_m.F90:184-212) */
static double realsep2(const orc_sys *s, double dx, double dy, double dz)
{
    int iv = s->ivol;
    if (iv == 0 || iv == 1 || iv == 4) {
        dx = dx - round(dx); dy = dy - round(dy); dz = dz - round(dz);
    } else if (iv == 2) {
        dx = dx - round(dx); dy = dy - round(dy);
    } else if (iv == 5) {
        dz = dz - round(dz);
    }
    const double *b = s->b0;
    double rx = M3(b, 1, 1) * dx + M3(b, 1, 2) * dy + M3(b, 1, 3) * dz;
    double ry = M3(b, 2, 1) * dx + M3(b, 2, 2) * dy + M3(b, 2, 3) * dz;
    double rz = M3(b, 3, 1) * dx + M3(b, 3, 2) * dy + M3(b, 3, 3) * dz;
    return rx * rx + ry * ry + rz * rz;
}

static double sep2(const orc_sys *s, int i, int j)
{
    return realsep2(s, s->x0[i] - s->x0[j], s->y0[i] - s->y0[j], s->z0[i] - s->z0[j]);
}

/* hist[(ibin * nspec + si) * nspec + sj], ibin 0..maxbin; spec[] is 0-based
 * over atoms (species index of atom i+1); natoms[nspec] counts the
 * non-vacancy atoms of the particle loop; nclose counts pairs with r <= 2 A
 * (the routine's "too close" warning). */
void orc_rdf(const orc_sys *s, int mode, int maxbin, int bpa, const int *spec, int nspec, long long *hist,
             long long *natoms, long long *nclose)
{
    const int nm = s->nm, nn = s->nnbrs;
    const size_t nh = (size_t)(maxbin + 1) * nspec * nspec;
    memset(hist, 0, nh * sizeof(long long));
    for (int k = 0; k < nspec; ++k) natoms[k] = 0;
    long long close = 0;
    const int q = maxbin / bpa;
    const double rsqmax = (double)(q * q);
    const double minrad = 2.0;
    for (int i = 1; i <= nm; ++i)
        if (s->atomic_number[i] != 0) natoms[spec[i - 1]] += 1;
#pragma omp parallel reduction(+ : close)
    {
        long long *h = (long long *)calloc(nh, sizeof(long long));
#pragma omp for schedule(dynamic, 64)
        for (int i = 1; i <= nm; ++i) {
            if (s->atomic_number[i] == 0) continue;
            const int kmax = mode == 0 ? s->numn[i] : i - 1;
            for (int k = 1; k <= kmax; ++k) {
                const int j = mode == 0 ? s->nlist[(size_t)(k - 1) + (size_t)nn * (size_t)(i - 1)] : k;
                if (s->atomic_number[j] == 0) continue;
                const double rsq = sep2(s, i, j);
                if (mode == 0 && rsq > rsqmax) continue;
                const double r = sqrt(rsq);
                const int ibin = (int)(r * (double)bpa);
                if (r <= minrad) close += 1;
                if (ibin > maxbin) continue;
                h[((size_t)ibin * nspec + spec[i - 1]) * nspec + spec[j - 1]] += 1;
            }
        }
#pragma omp critical
        for (size_t k = 0; k < nh; ++k) hist[k] += h[k];
        free(h);
    }
    *nclose = close;
}

/* rnatoms(isp,jsp), isp <= jsp, from the histogram (analysis_m.F90:619-637):
 * the radius of the bin where the cumulative pair count first reaches
 * 4 min(natoms); rneighbour carries over between species pairs when the test
 * never passes.  rn[si * nspec + sj] and rn[sj * nspec + si] both receive it. */
void orc_rdf_rneighbour(const long long *hist, const long long *natoms, int maxbin, int bpa, int nspec, double *rn)
{
    double rneighbour = 0.0;
    for (int isp = 0; isp < nspec; ++isp)
        for (int jsp = isp; jsp < nspec; ++jsp) {
            long long icount = 0;
            const long long lim = 4 * (natoms[isp] < natoms[jsp] ? natoms[isp] : natoms[jsp]);
            for (int ibin = 1; ibin <= maxbin; ++ibin) {
                long long irdf = hist[((size_t)ibin * nspec + isp) * nspec + jsp];
                if (isp != jsp) irdf += hist[((size_t)ibin * nspec + jsp) * nspec + isp];
                if (icount < lim) {
                    icount = icount + irdf;
                    rneighbour = (double)((float)ibin / (float)bpa);
                }
            }
            rn[isp * nspec + jsp] = rneighbour;
            rn[jsp * nspec + isp] = rneighbour;
        }
}

/* The eight ctheta windows (analysis_m.F90:695-714); -1 for the unused band */
static int chi_bin(double ct)
{
    if (ct < (double)-0.945f) return 0;
    if (ct < (double)-0.915f) return 1;
    if (ct < (double)-0.755f) return 2;
    if (ct < (double)-0.705f) return 3;
    if (ct < (double)-0.195f) return -1;
    if (ct < (double)0.195f) return 4;
    if (ct < (double)0.245f) return 5;
    if (ct < (double)0.795f) return 6;
    if (ct < (double)1.0f) return 7;
    return -1;
}

/* Ackland-Jones assignment from chi and nn (analysis_m.F90:724-751):
 * 0 unknown, 1 bcc, 2 fcc, 3 hcp, 4 icosahedral */
static int aj_assign(const int *chi, int nn)
{
    float bccscore = 0.35f * (float)chi[4];
    bccscore = bccscore / (float)(chi[5] + chi[6] + chi[7] - chi[4]);
    float fcchcp = fabsf(24.0f - (float)chi[6]) / 24.0f;
    int t = chi[0] + chi[1] - 6;
    float fccscore = 0.61f * (float)((t < 0 ? -t : t) + chi[2]);
    fccscore = fccscore / 6.0f;
    float hcpscore = (fabsf((float)chi[0] - 3.0f) + fabsf((float)(chi[0] + chi[1] + chi[2] + chi[3]) - 9.0f)) / 12.0f;
    double icoscore = (double)chi[4];
    if (nn > 11) {
        if (chi[0] == 7) bccscore = 0.0f;
        if (chi[0] == 6) fccscore = 0.0f;
        if (chi[0] == 3) hcpscore = 0.0f;
    }
    int aj;
    if (chi[7] > 0) {
        aj = 0;
    } else if (icoscore < 3.0) {
        aj = 4;
        if (nn != 12) aj = 0;
    } else if ((double)bccscore <= (double)fcchcp) {
        aj = 1;
        if (nn < 11) aj = 0;
    } else if (nn != 12) {
        aj = 0;
    } else if ((double)fccscore < (double)hcpscore) {
        aj = 2;
    } else {
        aj = 3;
    }
    return aj;
}

/* Per atom: aj[nm], nn[nm] and chi[8 nm] (may be NULL).  mode 0 takes the
 * full list from the half list (analysis_m.F90:562-578), mode 1 every other
 * atom.  rn as written by orc_rdf_rneighbour. */
void orc_ackland_jones(const orc_sys *s, int mode, const int *spec, int nspec, const double *rn, int *aj, int *nnout,
                       int *chiout)
{
    const int nm = s->nm, nn = s->nnbrs;
    int *numfull = NULL, *nfull = NULL, cap = 0;
    if (mode == 0) {
        numfull = (int *)calloc((size_t)nm + 1, sizeof(int));
        for (int i = 1; i <= nm; ++i) numfull[i] = s->numn[i];
        for (int i = 1; i <= nm; ++i)
            for (int k = 1; k <= s->numn[i]; ++k) {
                int j = s->nlist[(size_t)(k - 1) + (size_t)nn * (size_t)(i - 1)];
                numfull[j] += 1;
            }
        for (int i = 1; i <= nm; ++i) cap = numfull[i] > cap ? numfull[i] : cap;
        nfull = (int *)calloc((size_t)cap * (size_t)nm + 1, sizeof(int));
        int *fill = (int *)calloc((size_t)nm + 1, sizeof(int));
        for (int i = 1; i <= nm; ++i)
            for (int k = 1; k <= s->numn[i]; ++k) {
                nfull[(size_t)(i - 1) * cap + fill[i]++] = s->nlist[(size_t)(k - 1) + (size_t)nn * (size_t)(i - 1)];
            }
        for (int i = 1; i <= nm; ++i)
            for (int k = 1; k <= s->numn[i]; ++k) {
                int j = s->nlist[(size_t)(k - 1) + (size_t)nn * (size_t)(i - 1)];
                nfull[(size_t)(j - 1) * cap + fill[j]++] = i;
            }
        free(fill);
    }
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 1; i <= nm; ++i) {
        int chi[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int count = 0;
        const int nfi = mode == 0 ? numfull[i] : nm;
        for (int jn = 0; jn < nfi; ++jn) {
            const int j = mode == 0 ? nfull[(size_t)(i - 1) * cap + jn] : jn + 1;
            if (j == i) continue;
            const double rsqj = sep2(s, i, j);
            const double rj = rn[spec[i - 1] * nspec + spec[j - 1]];
            if (rsqj > (double)1.45f * (rj * rj)) continue;
            count = count + 1;
            for (int kn = jn + 1; kn < nfi; ++kn) {
                const int k = mode == 0 ? nfull[(size_t)(i - 1) * cap + kn] : kn + 1;
                if (k == i) continue;
                const double rsqk = sep2(s, i, k);
                const double rk = rn[spec[i - 1] * nspec + spec[k - 1]];
                if (rsqk > (double)1.45f * (rk * rk)) continue;
                const double rsq = sep2(s, k, j);
                const double ct = (rsqj + rsqk - rsq) / 2.0 / sqrt(rsqj * rsqk);
                const int b = chi_bin(ct);
                if (b >= 0) chi[b] += 1;
            }
        }
        aj[i - 1] = aj_assign(chi, count);
        nnout[i - 1] = count;
        if (chiout)
            for (int b = 0; b < 8; ++b) chiout[8 * (size_t)(i - 1) + b] = chi[b];
    }
    free(numfull);
    free(nfull);
}
