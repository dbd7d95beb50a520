/*
 * fetm.c -- oracle restatement of the FETRANSMETAL Fe-Fe potential and of the
 * lookup_m tables.  TEST INFRASTRUCTURE ONLY (see moldy_oracle.h).
 *
 * Arithmetic follows the Fortran expression order term by term, including the
 * places where the reference writes default-REAL (single precision) literals
 * inside double-precision expressions (for example bier_cut1 = 0.9 and the
 * Biersack screening length), because those promotions change table bits.
 * Compile with -ffp-contract=off so that no multiply-add is fused.
 */
#include "oracle_internal.h"

#include <math.h>
#include <string.h>

/* src/constants_m.F90:88-89 */
#define ELECTRON 1.602176487e-19
#define ANGSTROM 1.0e-10

/* src/fetransmetal.F90:569-579 (xH0) */
static double heaviside0(double x) { return (x < 0.0) ? 0.0 : 1.0; }

/* src/fetransmetal.F90:414-431 (biersack) */
static double biersack(double r, int na1, int na2)
{
    double zed = (double)(na1 * na2) * 8.98755178e9 * ELECTRON / ANGSTROM;
    /* a = (0.8854*0.529)/(na1**0.666666667+na2**0.666666667)**0.5, all REAL*4 */
    float pa = powf((float)na1, 0.666666667f);
    float pb = powf((float)na2, 0.666666667f);
    float af = (0.8854f * 0.529f) / powf(pa + pb, 0.5f);
    double a = (double)af;
    double x = r / a;
    double phib = (double)0.1818f * exp(-((double)3.2f * x));
    phib = phib + (double)0.5099f * exp(-((double)0.9423f * x));
    phib = phib + (double)0.2802f * exp(-((double)0.4029f * x));
    phib = phib + (double)0.02817f * exp(-((double)0.2016f * x));
    return zed * phib / r;
}

/* src/fetransmetal.F90:434-454 (dvee_biersack) */
static double dvee_biersack(double r, int na1, int na2)
{
    double zed = (double)(na1 * na2) * 8.98755178e9 * ELECTRON / ANGSTROM;
    float pa = powf((float)na1, 0.666666667f);
    float pb = powf((float)na2, 0.666666667f);
    float af = (0.8854f * 0.529f) / powf(pa + pb, 0.5f);
    double a = (double)af;
    double x = r / a;
    double s = (1.0 / r + 3.2 / a) * 0.1818 * exp(-(3.2 * x));
    s = s + (1.0 / r + 0.9423 / a) * 0.5099 * exp(-(0.9423 * x));
    s = s + (1.0 / r + 0.4029 / a) * 0.2802 * exp(-(0.4029 * x));
    s = s + (1.0 / r + 0.2016 / a) * 0.02817 * exp(-(0.2016 * x));
    return -((zed / r) * s);
}

/* src/fetransmetal.F90:511-528 (expjoin): cubic Hermite join in log space */
static double expjoin(double a1, double x1, double v1, double a2, double x2,
                      double v2, double r)
{
    double vv1 = v1 / x1, xx1 = log(x1), vv2 = v2 / x2, xx2 = log(x2);
    double t = (r - a1) / (a2 - a1);
    double h00 = (((2.0 * t) * t) * t - (3.0 * t) * t) + 1.0;
    double h10 = ((t * t) * t - (2.0 * t) * t) + t;
    double h01 = -(((2.0 * t) * t) * t) + (3.0 * t) * t;
    double h11 = (t * t) * t - t * t;
    double sp = h00 * xx1 + h10 * vv1 * (a2 - a1);
    sp = sp + h01 * xx2;
    sp = sp + h11 * vv2 * (a2 - a1);
    return exp(sp);
}

/* src/fetransmetal.F90:530-551 (dexpjoin) */
static double dexpjoin(double a1, double x1, double v1, double a2, double x2,
                       double v2, double r)
{
    double vv1 = v1 / x1, xx1 = log(x1), vv2 = v2 / x2, xx2 = log(x2);
    double t = (r - a1) / (a2 - a1);
    double d00 = (6.0 * t) * t - 6.0 * t;
    double d10 = ((3.0 * t) * t - 4.0 * t) + 1.0;
    double d01 = -((6.0 * t) * t) + 6.0 * t;
    double d11 = (3.0 * t) * t - 2.0 * t;
    double ds = d00 * xx1 + d10 * vv1 * (a2 - a1);
    ds = ds + d01 * xx2;
    ds = ds + d11 * vv2 * (a2 - a1);
    ds = ds / (a2 - a1);
    double h00 = (((2.0 * t) * t) * t - (3.0 * t) * t) + 1.0;
    double h10 = ((t * t) * t - (2.0 * t) * t) + t;
    double h01 = -(((2.0 * t) * t) * t) + (3.0 * t) * t;
    double h11 = (t * t) * t - t * t;
    double sp = h00 * xx1 + h10 * vv1 * (a2 - a1);
    sp = sp + h01 * xx2;
    sp = sp + h11 * vv2 * (a2 - a1);
    return ds * exp(sp);
}

/* src/fetransmetal.F90:100-159 (vee_src), Fe-Fe branch */
static double fetm_vee_src(const orc_sys *s, double r)
{
    double ans = 0.0;
    if (r > s->bier_cut2) {
        for (int i = 0; i < s->nv; ++i) {
            double d = s->rv[i] - r * s->p1;
            ans = ans + s->av[i] * ((d * d) * d) * heaviside0(d);
        }
        ans = ans * s->dp2;
    } else if (r > s->bier_cut1) {
        ans = expjoin(s->bier_cut1, s->sc[0], s->sc[1], s->bier_cut2, s->sc[2], s->sc[3], r);
    } else if (r < s->bier_cut1) {
        ans = biersack(r, 26, 26);
    }
    return ans;
}

/* src/fetransmetal.F90:167-219 (dvee_src) */
static double fetm_dvee_src(const orc_sys *s, double r)
{
    double ans = 0.0;
    if (r > s->bier_cut2) {
        for (int i = 0; i < s->nv; ++i) {
            double d = s->rv[i] - r * s->p1;
            ans = ans - s->p1 * 3.0 * s->av[i] * (d * d) * heaviside0(d);
        }
        ans = ans * s->dp2;
    } else if (r > s->bier_cut1) {
        ans = dexpjoin(s->bier_cut1, s->sc[0], s->sc[1], s->bier_cut2, s->sc[2], s->sc[3], r);
    } else if (r < s->bier_cut1) {
        ans = dvee_biersack(r, 26, 26);
    }
    return ans;
}

/* polynomial part of phi_src / dphi_src, used with and without the flat core */
static double phi_poly(const orc_sys *s, double r)
{
    double ans = 0.0;
    for (int i = 0; i < s->np; ++i) {
        double d = s->rp[i] - r * s->p3;
        ans = ans + s->ap[i] * ((d * d) * d) * heaviside0(d);
    }
    return ans * s->dp4;
}

static double dphi_poly(const orc_sys *s, double r)
{
    double ans = 0.0;
    for (int i = 0; i < s->np; ++i) {
        double d = s->rp[i] - r * s->p3;
        ans = ans - 3.0 * s->p3 * s->ap[i] * (d * d) * heaviside0(d);
    }
    return ans * s->dp4;
}

/* src/fetransmetal.F90:227-285 (phi_src): flat below the maximum of phi */
static double fetm_phi_src(const orc_sys *s, double r)
{
    if (r < s->phi_cut1) return s->phi_cut2;
    return phi_poly(s, r);
}

/* src/fetransmetal.F90:293-366 (dphi_src) */
static double fetm_dphi_src(const orc_sys *s, double r)
{
    if (r < s->phi_cut1) return 0.0;
    return dphi_poly(s, r);
}

/* src/fetransmetal.F90:375-385 (emb_src) */
static double fetm_emb_src(double rho) { return -(1.0 * sqrt(rho > 0.0 ? rho : 0.0)); }

/* src/fetransmetal.F90:394-404 (demb_src) */
static double fetm_demb_src(double rho)
{
    double d = 0.0;
    if (rho > 0.0) d = -(0.5 / sqrt(rho));
    return d;
}

/* the material module in use: FETRANSMETAL (potential 0) or the Fe-Fe
 * functions of IRON_CARBON (potential 1, ironcarbon.c) */
double orc_vee_src(const orc_sys *s, double r) { return s->potential == 1 ? orc_ic_vee(r) : fetm_vee_src(s, r); }
double orc_dvee_src(const orc_sys *s, double r) { return s->potential == 1 ? orc_ic_dvee(r) : fetm_dvee_src(s, r); }
double orc_phi_src(const orc_sys *s, double r) { return s->potential == 1 ? orc_ic_phi(r) : fetm_phi_src(s, r); }
double orc_dphi_src(const orc_sys *s, double r) { return s->potential == 1 ? orc_ic_dphi(r) : fetm_dphi_src(s, r); }
double orc_emb_src(const orc_sys *s, double rho) { return s->potential == 1 ? orc_ic_emb(rho) : fetm_emb_src(rho); }
double orc_demb_src(const orc_sys *s, double rho) { return s->potential == 1 ? orc_ic_demb(rho) : fetm_demb_src(rho); }

int orc_set_iron_carbon(orc_sys *s)
{
    s->potential = 1;
    s->fetm_set = 1;
    return 0;
}

/* src/fetransmetal.F90:896-926 (phi_turn): bisection for the maximum of phi,
 * evaluated while phi_cut for this pair is still zero (module storage). */
static double phi_turn(const orc_sys *s)
{
    double lo = 0.0, hi = 3.0;
    if (dphi_poly(s, lo) < 0.0) return -1.0;
    if (dphi_poly(s, hi) >= 0.0) return -1.0;
    for (int i = 0; i < 500; ++i) {
        double mid = (hi + lo) / 2.0;
        double g = dphi_poly(s, mid);
        if (g > 0.0) lo = mid; else hi = mid;
    }
    return (hi + lo) / 2.0;
}

int orc_set_fetm(orc_sys *s, int nv, const double *av, const double *rv,
                 int np, const double *ap, const double *rp)
{
    if (nv < 1 || nv > ORC_MAXCOEF || np < 1 || np > ORC_MAXCOEF) return 2;
    s->potential = 0;
    s->nv = nv;
    s->np = np;
    for (int i = 0; i < nv; ++i) { s->av[i] = av[i]; s->rv[i] = rv[i]; }
    for (int i = 0; i < np; ++i) { s->ap[i] = ap[i]; s->rp[i] = rp[i]; }
    /* Fe-Fe scalings SolSol_(:,5) = 1, then columns 1 and 3 inverted
     * (src/fetransmetal.F90:826-862, find_coeff 931-954) */
    s->p1 = 1.0 / 1.0; s->dp2 = 1.0; s->p3 = 1.0 / 1.0; s->dp4 = 1.0;
    /* src/fetransmetal.F90:732-733: REAL*4 literals stored in REAL*8 */
    s->bier_cut1 = (double)0.9f;
    s->bier_cut2 = (double)1.9f;
    /* spline join data, src/fetransmetal.F90:866-876 */
    s->phi_cut1 = 0.0;
    s->phi_cut2 = 0.0;
    double eps = (double)0.000000000001f;
    s->sc[0] = biersack(s->bier_cut1 - eps, 26, 26);
    s->sc[1] = dvee_biersack(s->bier_cut1 - eps, 26, 26);
    s->sc[2] = orc_vee_src(s, s->bier_cut2 + eps);
    s->sc[3] = orc_dvee_src(s, s->bier_cut2 + eps);
    /* src/fetransmetal.F90:881-889 */
    double pc = phi_turn(s);
    if (pc < 0.0) return 3;
    s->phi_cut1 = pc;
    s->phi_cut2 = orc_phi_src(s, pc);
    s->fetm_set = 1;
    s->potential = 0;
    return 0;
}

void orc_get_fetm_derived(const orc_sys *s, double *out8)
{
    out8[0] = s->bier_cut1; out8[1] = s->bier_cut2;
    out8[2] = s->sc[0]; out8[3] = s->sc[1]; out8[4] = s->sc[2]; out8[5] = s->sc[3];
    out8[6] = s->phi_cut1; out8[7] = s->phi_cut2;
}

/* src/lookup_m.F90:161-203 and 213-251, driven by
 * src/potential_m.F90:181-228 (rmin=0, rmax=6, rhomin=0, rhomax=10000) */
int orc_set_lookup(orc_sys *s, int uselookup, int nlookup)
{
    if (!s->fetm_set) return 1;
    s->uselookup = uselookup;
    if (!uselookup) return 0;
    if (nlookup < 2) return 2;
    s->nlookup = nlookup;
    orc_free_tables(s);
    size_t n = (size_t)nlookup + 1;
    for (int k = 0; k < 6; ++k) s->tab[k] = (double *)calloc(n, sizeof(double));

    /* get_supported_potential_range: FETRANSMETAL 0..6, IRON_CARBON 0..5.4 (src/iron_carbon.F90:91-92) */
    s->vp_rmin = 0.0; s->vp_rmax = s->potential == 1 ? 5.4 : 6.0;
    s->vp_range = s->vp_rmax - s->vp_rmin;
    s->vp_reciprange = 1.0 / s->vp_range;
    s->vp_recipnlkp = 1.0 / (double)nlookup;
    s->vp_recipstep = (double)nlookup / s->vp_range;
    for (int i = 0; i <= nlookup; ++i) {
        double r = s->vp_rmin + (double)i * s->vp_range * s->vp_recipnlkp;
        s->tab[0][i] = orc_vee_src(s, r);
        s->tab[1][i] = orc_dvee_src(s, r);
        s->tab[2][i] = orc_phi_src(s, r);
        s->tab[3][i] = orc_dphi_src(s, r);
    }
    s->e_rmin = 0.0; s->e_rmax = 10000.0;
    s->e_range = s->e_rmax - s->e_rmin;
    s->e_reciprange = 1.0 / s->e_range;
    s->e_recipnlkp = 1.0 / (double)nlookup;
    s->e_recipstep = (double)nlookup / s->e_range;
    for (int i = 0; i <= nlookup; ++i) {
        double r = s->e_rmin + (double)i * s->e_range * s->e_recipnlkp;
        s->tab[4][i] = orc_emb_src(s, r);
        s->tab[5][i] = orc_demb_src(s, r);
    }
    return 0;
}

/* Tables handed over by a caller in the lookup_m layout (src/lookup_m.F90:64-78):
 * nlookup intervals over [rmin, rmax] for vee, dvee, phi, dphi and over
 * [rhomin, rhomax] for emb, demb; the reciprocal ranges are formed as
 * calculate_lookup_table_* does (src/lookup_m.F90:161-251). */
int orc_set_tables(orc_sys *s, int nlookup, double rmin, double rmax, double rhomin, double rhomax,
                   const double *vee, const double *dvee, const double *phi, const double *dphi,
                   const double *emb, const double *demb)
{
    if (nlookup < 2) return 2;
    if (!(rmax > rmin) || !(rhomax > rhomin)) return 3;
    orc_free_tables(s);
    size_t n = (size_t)nlookup + 1;
    const double *src[6] = {vee, dvee, phi, dphi, emb, demb};
    for (int k = 0; k < 6; ++k) {
        s->tab[k] = (double *)malloc(n * sizeof(double));
        memcpy(s->tab[k], src[k], n * sizeof(double));
    }
    s->uselookup = 1;
    s->nlookup = nlookup;
    s->vp_rmin = rmin; s->vp_rmax = rmax;
    s->vp_range = rmax - rmin;
    s->vp_reciprange = 1.0 / s->vp_range;
    s->vp_recipnlkp = 1.0 / (double)nlookup;
    s->vp_recipstep = (double)nlookup / s->vp_range;
    s->e_rmin = rhomin; s->e_rmax = rhomax;
    s->e_range = rhomax - rhomin;
    s->e_reciprange = 1.0 / s->e_range;
    s->e_recipnlkp = 1.0 / (double)nlookup;
    s->e_recipstep = (double)nlookup / s->e_range;
    return 0;
}

void orc_free_tables(orc_sys *s)
{
    for (int k = 0; k < 6; ++k) { free(s->tab[k]); s->tab[k] = NULL; }
}

void orc_get_tables(const orc_sys *s, double *vee, double *dvee, double *phi,
                    double *dphi, double *emb, double *demb)
{
    size_t n = (size_t)s->nlookup + 1;
    double *dst[6] = {vee, dvee, phi, dphi, emb, demb};
    for (int k = 0; k < 6; ++k)
        if (dst[k] && s->tab[k]) memcpy(dst[k], s->tab[k], n * sizeof(double));
}

/* src/lookup_m.F90:307-346 (get_value_from_lookup_veephi) */
double orc_lookup_r(const orc_sys *s, const double *t, double r)
{
    if (r >= s->vp_rmax) return t[s->nlookup];
    int idx = (int)((double)s->nlookup * (r - s->vp_rmin) * s->vp_reciprange);
    double rlow = s->vp_rmin + s->vp_range * (double)idx * s->vp_recipnlkp;
    double dr = (r - rlow) * s->vp_recipstep;
    return t[idx] * (1.0 - dr) + t[idx + 1] * dr;
}

/* src/lookup_m.F90:356-394 (get_value_from_lookup_emb) */
double orc_lookup_rho(const orc_sys *s, const double *t, double rho)
{
    if (rho >= s->e_rmax) return t[s->nlookup];
    int idx = (int)((double)s->nlookup * (rho - s->e_rmin) * s->e_reciprange);
    double rlow = s->e_rmin + s->e_range * (double)idx * s->e_recipnlkp;
    double dr = (rho - rlow) * s->e_recipstep;
    return t[idx] * (1.0 - dr) + t[idx + 1] * dr;
}

double orc_src(const orc_sys *s, int which, double r)
{
    switch (which) {
    case 0: return orc_vee_src(s, r);
    case 1: return orc_dvee_src(s, r);
    case 2: return orc_phi_src(s, r);
    case 3: return orc_dphi_src(s, r);
    case 4: return orc_emb_src(s, r);
    case 5: return orc_demb_src(s, r);
    }
    return 0.0;
}

double orc_lookup(const orc_sys *s, int which, double r)
{
    if (which < 4) return orc_lookup_r(s, s->tab[which], r);
    return orc_lookup_rho(s, s->tab[which], r);
}

/* potential_m dispatch (src/potential_m.F90:288-417) */
double orc_vee(const orc_sys *s, double r) { return s->uselookup ? orc_lookup_r(s, s->tab[0], r) : orc_vee_src(s, r); }
double orc_dvee(const orc_sys *s, double r) { return s->uselookup ? orc_lookup_r(s, s->tab[1], r) : orc_dvee_src(s, r); }
double orc_phi(const orc_sys *s, double r) { return s->uselookup ? orc_lookup_r(s, s->tab[2], r) : orc_phi_src(s, r); }
double orc_dphi(const orc_sys *s, double r) { return s->uselookup ? orc_lookup_r(s, s->tab[3], r) : orc_dphi_src(s, r); }
double orc_emb(const orc_sys *s, double rho) { return s->uselookup ? orc_lookup_rho(s, s->tab[4], rho) : orc_emb_src(s, rho); }
double orc_demb(const orc_sys *s, double rho) { return s->uselookup ? orc_lookup_rho(s, s->tab[5], rho) : orc_demb_src(s, rho); }
