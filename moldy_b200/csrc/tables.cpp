// tables.cpp -- FETRANSMETAL Fe-Fe set-up and the lookup_m tables, built once
// on the host and uploaded (the reference also builds them on the host,
// src/potential_m.F90:181-228).
//
// The Fe-Fe functions (src/fetransmetal.F90):
//   V(r)   = sum_k a_k (r_k - r)^3 H(r_k - r)                 r > bier_cut2
//          = exp(cubic Hermite in log V) joining Biersack to V  bier_cut1 < r < bier_cut2
//          = Biersack-Ziegler screened Coulomb                  r < bier_cut1
//   phi(r) = sum_k A_k (R_k - r)^3 H(R_k - r), held flat below its maximum
//   F(rho) = -sqrt(rho)
// The reference writes several constants as default-REAL (single precision)
// literals inside double expressions; those promotions are kept because they
// change table bits (bier_cut1 = 0.9 is 0.89999997615814209 in double).
// Host code is compiled without floating-point contraction.
#include <cmath>

#include "engine.h"

namespace moldy {
namespace {

struct FeFe {
    int nv, np;
    const double *av, *rv, *ap, *rp;
    double cut1, cut2, join[4], phi_top_r, phi_top_v;
    double a_screen, zed;

    static double step(double x) { return x < 0.0 ? 0.0 : 1.0; }

    // Biersack-Ziegler (src/fetransmetal.F90:414-454) for Z1 = Z2 = 26
    void screening() {
        const double electron = 1.602176487e-19, angstrom = 1.0e-10;
        zed = (double)(26 * 26) * 8.98755178e9 * electron / angstrom;
        float p = powf(26.0f, 0.666666667f);
        float a = (0.8854f * 0.529f) / powf(p + p, 0.5f);
        a_screen = (double)a;
    }
    double biersack(double r) const {
        double x = r / a_screen;
        double s = (double)0.1818f * std::exp(-((double)3.2f * x));
        s = s + (double)0.5099f * std::exp(-((double)0.9423f * x));
        s = s + (double)0.2802f * std::exp(-((double)0.4029f * x));
        s = s + (double)0.02817f * std::exp(-((double)0.2016f * x));
        return zed * s / r;
    }
    double dbiersack(double r) const {
        double a = a_screen, x = r / a;
        double s = (1.0 / r + 3.2 / a) * 0.1818 * std::exp(-(3.2 * x));
        s = s + (1.0 / r + 0.9423 / a) * 0.5099 * std::exp(-(0.9423 * x));
        s = s + (1.0 / r + 0.4029 / a) * 0.2802 * std::exp(-(0.4029 * x));
        s = s + (1.0 / r + 0.2016 / a) * 0.02817 * std::exp(-(0.2016 * x));
        return -((zed / r) * s);
    }
    // log-space cubic Hermite join, value (src/fetransmetal.F90:511-528) and
    // derivative (530-551); t is the reduced coordinate on [cut1, cut2]
    void join_eval(double r, double *v, double *dv) const {
        double a1 = cut1, a2 = cut2, h = a2 - a1;
        double s1 = join[1] / join[0], l1 = std::log(join[0]);
        double s2 = join[3] / join[2], l2 = std::log(join[2]);
        double t = (r - a1) / h;
        double e = (((2.0 * t) * t) * t - (3.0 * t) * t + 1.0) * l1 +
                   ((t * t) * t - (2.0 * t) * t + t) * s1 * h;
        e = e + (-(((2.0 * t) * t) * t) + (3.0 * t) * t) * l2;
        e = e + ((t * t) * t - t * t) * s2 * h;
        if (v) *v = std::exp(e);
        if (dv) {
            double d = ((6.0 * t) * t - 6.0 * t) * l1 + ((3.0 * t) * t - 4.0 * t + 1.0) * s1 * h;
            d = d + (-((6.0 * t) * t) + 6.0 * t) * l2;
            d = d + ((3.0 * t) * t - 2.0 * t) * s2 * h;
            d = d / h;
            *dv = d * std::exp(e);
        }
    }
    double pair_poly(double r) const {
        double s = 0.0;
        for (int i = 0; i < nv; ++i) {
            double d = rv[i] - r;
            s = s + av[i] * ((d * d) * d) * step(d);
        }
        return s;
    }
    double dpair_poly(double r) const {
        double s = 0.0;
        for (int i = 0; i < nv; ++i) {
            double d = rv[i] - r;
            s = s - 1.0 * 3.0 * av[i] * (d * d) * step(d);
        }
        return s;
    }
    double dens_poly(double r) const {
        double s = 0.0;
        for (int i = 0; i < np; ++i) {
            double d = rp[i] - r;
            s = s + ap[i] * ((d * d) * d) * step(d);
        }
        return s;
    }
    double ddens_poly(double r) const {
        double s = 0.0;
        for (int i = 0; i < np; ++i) {
            double d = rp[i] - r;
            s = s - 3.0 * 1.0 * ap[i] * (d * d) * step(d);
        }
        return s;
    }
    double vee(double r) const {
        if (r > cut2) return pair_poly(r);
        if (r > cut1) { double v; join_eval(r, &v, nullptr); return v; }
        if (r < cut1) return biersack(r);
        return 0.0;
    }
    double dvee(double r) const {
        if (r > cut2) return dpair_poly(r);
        if (r > cut1) { double d; join_eval(r, nullptr, &d); return d; }
        if (r < cut1) return dbiersack(r);
        return 0.0;
    }
    double phi(double r) const { return r < phi_top_r ? phi_top_v : dens_poly(r); }
    double dphi(double r) const { return r < phi_top_r ? 0.0 : ddens_poly(r); }

    // set_up_m (src/fetransmetal.F90:768-926) for the Fe-Fe pair
    bool set_up() {
        cut1 = (double)0.9f;
        cut2 = (double)1.9f;
        screening();
        const double eps = (double)0.000000000001f;
        join[0] = biersack(cut1 - eps);
        join[1] = dbiersack(cut1 - eps);
        join[2] = pair_poly(cut2 + eps);
        join[3] = dpair_poly(cut2 + eps);
        // maximum of phi by 500 bisection steps on its slope over [0, 3]
        double lo = 0.0, hi = 3.0;
        if (ddens_poly(lo) < 0.0 || ddens_poly(hi) >= 0.0) return false;
        for (int i = 0; i < 500; ++i) {
            double mid = (hi + lo) / 2.0;
            if (ddens_poly(mid) > 0.0) lo = mid; else hi = mid;
        }
        phi_top_r = (hi + lo) / 2.0;
        phi_top_v = dens_poly(phi_top_r);
        return true;
    }
};

}  // namespace

// Builds ht from the Fe-Fe knots; returns MOLDY_OK or an error code.
int build_fetm_tables(HostTables &ht, int nv, const double *av, const double *rv, int np,
                      const double *ap, const double *rp, int uselookup, int nlookup) {
    if (nv < 1 || nv > 8 || np < 1 || np > 8) return MOLDY_ERR_INVALID;
    FeFe f{nv, np, av, rv, ap, rp};
    if (!f.set_up()) return MOLDY_ERR_INVALID;
    ht.fetm = true;
    ht.exact = (uselookup == 0);
    ht.nv = nv; ht.np = np;
    for (int i = 0; i < nv; ++i) { ht.av[i] = av[i]; ht.rv[i] = rv[i]; }
    for (int i = 0; i < np; ++i) { ht.ap[i] = ap[i]; ht.rp[i] = rp[i]; }
    ht.bier_cut1 = f.cut1; ht.bier_cut2 = f.cut2;
    for (int k = 0; k < 4; ++k) ht.sc[k] = f.join[k];
    ht.phi_cut1 = f.phi_top_r; ht.phi_cut2 = f.phi_top_v;
    ht.bier_a = f.a_screen; ht.bier_zed = f.zed;
    // tables are built in both modes (exact mode uses them for nothing but
    // moldy_gpu_get_tables)
    if (nlookup < 2) nlookup = 5000;
    ht.nlookup = nlookup;
    ht.rmin = 0.0; ht.rmax = 6.0; ht.rhomin = 0.0; ht.rhomax = 10000.0;
    size_t n = (size_t)nlookup + 1;
    ht.vee.assign(n, 0.0); ht.dvee.assign(n, 0.0); ht.phi.assign(n, 0.0); ht.dphi.assign(n, 0.0);
    ht.emb.assign(n, 0.0); ht.demb.assign(n, 0.0);
    // calculate_lookup_table_veephi / _emb (src/lookup_m.F90:161-251)
    double range = ht.rmax - ht.rmin, recipn = 1.0 / (double)nlookup;
    for (int i = 0; i <= nlookup; ++i) {
        double r = ht.rmin + (double)i * range * recipn;
        ht.vee[i] = f.vee(r);
        ht.dvee[i] = f.dvee(r);
        ht.phi[i] = f.phi(r);
        ht.dphi[i] = f.dphi(r);
    }
    double erange = ht.rhomax - ht.rhomin;
    for (int i = 0; i <= nlookup; ++i) {
        double rho = ht.rhomin + (double)i * erange * recipn;
        ht.emb[i] = -(1.0 * std::sqrt(rho > 0.0 ? rho : 0.0));
        ht.demb[i] = rho > 0.0 ? -(0.5 / std::sqrt(rho)) : 0.0;
    }
    ht.set = true;
    return MOLDY_OK;
}

// Contracts table gradients g[6] (vee, dvee, phi, dphi, emb, demb; nlookup+1
// each) with d(table)/d(knot) of the functions above: dL/da_k, dL/dr_k of the
// pair sum, dL/dA_k, dL/dR_k of the density sum.  Below bier_cut1 the pair
// function is Biersack alone and has no knot dependence; between the cuts it
// depends on the knots through the join's end values V(c), V'(c) at
// c = bier_cut2 + 1e-12; phi below its maximum r_top is the value at r_top,
// whose knot derivative is the partial one (phi' vanishes at r_top).  The emb
// tables of F = -sqrt(rho) carry no knot parameters.
int fetm_knot_vjp(const HostTables &ht, const double *const g[6], double *g_av, double *g_rv,
                  double *g_ap, double *g_rp) {
    if (!ht.fetm || ht.nlookup < 2) return MOLDY_ERR_UNSUPPORTED;
    const int nv = ht.nv, np = ht.np, n = ht.nlookup;
    const double *av = ht.av, *rv = ht.rv, *ap = ht.ap, *rp = ht.rp;
    double gav[8] = {0}, grv[8] = {0}, gap[8] = {0}, grp[8] = {0};
    const double cut1 = ht.bier_cut1, cut2 = ht.bier_cut2, top = ht.phi_cut1;
    const double c = cut2 + (double)0.000000000001f;
    const double j0 = ht.sc[0], j1 = ht.sc[1], j2 = ht.sc[2], j3 = ht.sc[3];
    const double h = cut2 - cut1, l1 = std::log(j0), s1 = j1 / j0, l2 = std::log(j2), s2 = j3 / j2;
    double gj2 = 0.0, gj3 = 0.0;   // dL/dV(c), dL/dV'(c)
    // phi below r_top: partial derivatives at r_top
    double dtop_a[8], dtop_r[8];
    for (int k = 0; k < np; ++k) {
        double d = rp[k] - top, H = d < 0.0 ? 0.0 : 1.0;
        dtop_a[k] = d * d * d * H;
        dtop_r[k] = 3.0 * ap[k] * d * d * H;
    }
    const double range = ht.rmax - ht.rmin, recipn = 1.0 / (double)n;
    for (int i = 0; i <= n; ++i) {
        const double r = ht.rmin + (double)i * range * recipn;
        const double gv = g[0] ? g[0][i] : 0.0, gd = g[1] ? g[1][i] : 0.0;
        const double gp = g[2] ? g[2][i] : 0.0, gdp = g[3] ? g[3][i] : 0.0;
        if (gv != 0.0 || gd != 0.0) {
            if (r > cut2) {
                for (int k = 0; k < nv; ++k) {
                    double d = rv[k] - r;
                    if (d < 0.0) continue;
                    gav[k] += gv * d * d * d - gd * 3.0 * d * d;
                    grv[k] += gv * 3.0 * av[k] * d * d - gd * 6.0 * av[k] * d;
                }
            } else if (r > cut1) {
                double t = (r - cut1) / h;
                double h00 = 2 * t * t * t - 3 * t * t + 1, h10 = t * t * t - 2 * t * t + t;
                double h01 = -2 * t * t * t + 3 * t * t, h11 = t * t * t - t * t;
                double d00 = 6 * t * t - 6 * t, d10 = 3 * t * t - 4 * t + 1;
                double d01 = -6 * t * t + 6 * t, d11 = 3 * t * t - 2 * t;
                double e = h00 * l1 + h10 * s1 * h + h01 * l2 + h11 * s2 * h;
                double dl = (d00 * l1 + d10 * s1 * h + d01 * l2 + d11 * s2 * h) / h;
                double V = std::exp(e);
                double de2 = h01 / j2 - h11 * h * j3 / (j2 * j2), de3 = h11 * h / j2;
                double dd2 = (d01 / j2 - d11 * h * j3 / (j2 * j2)) / h, dd3 = d11 / j2;
                // V = exp(e), D = dl V
                gj2 += gv * V * de2 + gd * (dd2 * V + dl * V * de2);
                gj3 += gv * V * de3 + gd * (dd3 * V + dl * V * de3);
            }
        }
        if (gp != 0.0 || gdp != 0.0) {
            if (r < top) {
                for (int k = 0; k < np; ++k) { gap[k] += gp * dtop_a[k]; grp[k] += gp * dtop_r[k]; }
            } else {
                for (int k = 0; k < np; ++k) {
                    double d = rp[k] - r;
                    if (d < 0.0) continue;
                    gap[k] += gp * d * d * d - gdp * 3.0 * d * d;
                    grp[k] += gp * 3.0 * ap[k] * d * d - gdp * 6.0 * ap[k] * d;
                }
            }
        }
    }
    // V(c) = sum a_k (r_k - c)^3, V'(c) = -3 sum a_k (r_k - c)^2 (terms with r_k >= c)
    for (int k = 0; k < nv; ++k) {
        double d = rv[k] - c;
        if (d < 0.0) continue;
        gav[k] += gj2 * d * d * d - gj3 * 3.0 * d * d;
        grv[k] += gj2 * 3.0 * av[k] * d * d - gj3 * 6.0 * av[k] * d;
    }
    for (int k = 0; k < nv; ++k) {
        if (g_av) g_av[k] = gav[k];
        if (g_rv) g_rv[k] = grv[k];
    }
    for (int k = 0; k < np; ++k) {
        if (g_ap) g_ap[k] = gap[k];
        if (g_rp) g_rp[k] = grp[k];
    }
    return MOLDY_OK;
}

// ------------------------------------------------------- IRON_CARBON Fe-Fe --
// The Fe-Fe functions of the IRON_CARBON material module (Hepburn-Ackland,
// src/iron_carbon.F90): Biersack-Ziegler below 1 A, exp(cubic) join up to
// 2.05 A (a default-REAL literal, as written), 13 cubic knots beyond
// (118-266); phi a sum of 3 cubic knots (431-591); F(rho) = -sqrt(rho)
// - 6.7314115586063e-4 rho^2 + 7.6514905604792e-8 rho^4, constant beyond
// rho = 257 (599-696).  Tables over r in [0, 5.4] (pot_rmax, line 92).
namespace {

struct IronCarbonFe {
    static constexpr double bierFe = 9734.159682000001;
    static constexpr double b1 = 0.1818, x1 = -28.616172142695042, b2 = 0.5099, x2 = -8.42656844064423;
    static constexpr double b3 = 0.2802, x3 = -3.6029549238411973, b4 = 0.02817, x4 = -1.8028188449897875;
    static constexpr double j1 = 7.411957380630116, j2 = -0.6409989885339922;
    static constexpr double j3 = -2.6049191728604733, j4 = 0.6263733940718166;
    static constexpr double p1 = 4.2, p2 = 3.2, p3 = 2.4;
    static constexpr double q1 = 0.47193527075943, q2 = 0.01471074009883, q3 = 11.68685940797;
    static constexpr double rhocap = 257.0;
    const double knot[13] = {5.3, 4.7, 4.2, 3.7, 3.3, 3.0, 2.8, 2.7, 2.6, 2.5, 2.4, 2.3, 2.2};
    const double amp[13] = {-0.0030458824556234, -0.058531821042271, 0.35018615891957, -1.0260416933564,
                            2.657740612828,      -2.3194358924605,   0.80656414937789, -0.77361294129713,
                            4.2099676494795,     -2.4989799053251,   2.2077118733936,  15.738054058489,
                            -27.444805994228};

    static double step(double x) { return x < 0.0 ? 0.0 : 1.0; }
    static bool spline(double r) { return r > (double)2.05f; }
    static double joinexp(double r) { return std::exp(j1 + j2 * r + j3 * r * r + j4 * r * r * r); }

    double vee(double r) const {
        if (r < 1.0)
            return (bierFe / r) * (b1 * std::exp(x1 * r) + b2 * std::exp(x2 * r) + b3 * std::exp(x3 * r) +
                                   b4 * std::exp(x4 * r));
        if (spline(r)) {
            double v = 0.0;
            for (int k = 0; k < 13; ++k) {
                double d = knot[k] - r;
                v = v + (step(d) * amp[k] * ((d * d) * d));
            }
            return v;
        }
        return joinexp(r);
    }
    double dvee(double r) const {
        if (r < 1.0)
            return -(bierFe / r) * ((1.0 / r - x1) * b1 * std::exp(x1 * r) + (1.0 / r - x2) * b2 * std::exp(x2 * r) +
                                    (1.0 / r - x3) * b3 * std::exp(x3 * r) + (1.0 / r - x4) * b4 * std::exp(x4 * r));
        if (spline(r)) {
            double v = 0.0;
            for (int k = 0; k < 13; ++k) {
                double d = knot[k] - r;
                v = v + (3.0 * step(d) * amp[k] * (d * d));
            }
            return -v;
        }
        return (j2 + 2.0 * j3 * r + 3.0 * j4 * r * r) * joinexp(r);
    }
    static double phi(double r) {
        double d1 = p1 - r, d2 = p2 - r, d3 = p3 - r;
        return step(d1) * q1 * ((d1 * d1) * d1) - step(d2) * q2 * ((d2 * d2) * d2) + step(d3) * q3 * ((d3 * d3) * d3);
    }
    static double dphi(double r) {
        double d1 = p1 - r, d2 = p2 - r, d3 = p3 - r;
        return -(3.0 * step(d1) * q1 * (d1 * d1) - 3.0 * step(d2) * q2 * (d2 * d2) + 3.0 * step(d3) * q3 * (d3 * d3));
    }
    static double embcore(double x) {
        return (-1.0) * std::pow(x, 0.5) - (6.7314115586063e-4) * (x * x) + (7.6514905604792e-8) * ((x * x) * (x * x));
    }
    // the high-pressure correction of the reference has a zero amplitude
    static double emb(double x) { return x > rhocap ? embcore(rhocap) : embcore(x); }
    static double demb(double x) {
        if (x <= 0.0 || x > rhocap) return 0.0;
        return 0.5 * (-1.0) * std::pow(x, -0.5) - 2.0 * (6.7314115586063e-4) * x + 4.0 * (7.6514905604792e-8) * ((x * x) * x);
    }
};

}  // namespace

int build_iron_carbon_tables(HostTables &ht, int nlookup) {
    if (nlookup < 2) nlookup = 5000;
    IronCarbonFe f;
    ht = HostTables();
    ht.fetm = false;
    ht.exact = false;
    ht.nlookup = nlookup;
    ht.rmin = 0.0; ht.rmax = 5.4; ht.rhomin = 0.0; ht.rhomax = 10000.0;
    size_t n = (size_t)nlookup + 1;
    ht.vee.assign(n, 0.0); ht.dvee.assign(n, 0.0); ht.phi.assign(n, 0.0); ht.dphi.assign(n, 0.0);
    ht.emb.assign(n, 0.0); ht.demb.assign(n, 0.0);
    double range = ht.rmax - ht.rmin, recipn = 1.0 / (double)nlookup;
    for (int i = 0; i <= nlookup; ++i) {
        double r = ht.rmin + (double)i * range * recipn;
        ht.vee[i] = f.vee(r);
        ht.dvee[i] = f.dvee(r);
        ht.phi[i] = f.phi(r);
        ht.dphi[i] = f.dphi(r);
    }
    double erange = ht.rhomax - ht.rhomin;
    for (int i = 0; i <= nlookup; ++i) {
        double rho = ht.rhomin + (double)i * erange * recipn;
        ht.emb[i] = f.emb(rho);
        ht.demb[i] = f.demb(rho);
    }
    ht.set = true;
    return MOLDY_OK;
}

}  // namespace moldy
