/*
 * ironcarbon.c -- Fe-Fe functions of the IRON_CARBON material module
 * (Hepburn-Ackland Fe-C, src/iron_carbon.F90), restated for the CPU oracle
 * (TEST INFRASTRUCTURE).  Only the Fe-Fe pair (Z = 26) is restated: it is the
 * potential of the reference's shipped bcc-iron golden run
 * (tests/reference/bcc_iron).
 *
 *   V(r)   Biersack-Ziegler for r < 1, exp(cubic) join for 1 <= r <= 2.05,
 *          13 cubic knots for r > 2.05              (src/iron_carbon.F90:118-266)
 *   phi(r) 3 cubic knots                            (431-507, 515-591)
 *   F(rho) -sqrt(rho) - 6.7314115586063e-4 rho^2 + 7.6514905604792e-8 rho^4,
 *          held at its value at rho = 257 beyond it (599-696)
 *
 * The single-precision literal 2.05 of the branch test is kept as the
 * reference writes it.  Tables span r in [0, 5.4] (pot_rmax, line 92).
 */
#include <math.h>

#include "oracle_internal.h"

static const double bierFe = 9734.159682000001;
static const double bier1 = 0.1818, bierx1 = -28.616172142695042;
static const double bier2 = 0.5099, bierx2 = -8.42656844064423;
static const double bier3 = 0.2802, bierx3 = -3.6029549238411973;
static const double bier4 = 0.02817, bierx4 = -1.8028188449897875;
static const double vcut[13] = {5.3, 4.7, 4.2, 3.7, 3.3, 3.0, 2.8, 2.7, 2.6, 2.5, 2.4, 2.3, 2.2};
static const double vpar[13] = {-0.0030458824556234, -0.058531821042271, 0.35018615891957, -1.0260416933564,
                                2.657740612828,      -2.3194358924605,   0.80656414937789, -0.77361294129713,
                                4.2099676494795,     -2.4989799053251,   2.2077118733936,  15.738054058489,
                                -27.444805994228};
static const double join1 = 7.411957380630116, join2 = -0.6409989885339922;
static const double join3 = -2.6049191728604733, join4 = 0.6263733940718166;
static const double pcut1 = 4.2, pcut2 = 3.2, pcut3 = 2.4;
static const double ppar1 = 0.47193527075943, ppar2 = 0.01471074009883, ppar3 = 11.68685940797;
static const double acludge = 0.0, rcludge = 28.5, rx = 257.0;

static double xh0(double x) { return x < 0.0 ? 0.0 : 1.0; }

/* r.gt.2.05 with a default-REAL literal */
static int spline_branch(double r) { return r > (double)2.05f; }

double orc_ic_vee(double r)
{
    if (r < 1.0)
        return (bierFe / r) * (bier1 * exp(bierx1 * r) + bier2 * exp(bierx2 * r) + bier3 * exp(bierx3 * r) +
                               bier4 * exp(bierx4 * r));
    if (spline_branch(r)) {
        double v = 0.0;
        for (int k = 0; k < 13; ++k) {
            double d = vcut[k] - r;
            v = v + (xh0(d) * vpar[k] * ((d * d) * d));
        }
        return v;
    }
    return exp(join1 + join2 * r + join3 * r * r + join4 * r * r * r);
}

double orc_ic_dvee(double r)
{
    if (r < 1.0)
        return -(bierFe / r) * ((1.0 / r - bierx1) * bier1 * exp(bierx1 * r) +
                                (1.0 / r - bierx2) * bier2 * exp(bierx2 * r) +
                                (1.0 / r - bierx3) * bier3 * exp(bierx3 * r) +
                                (1.0 / r - bierx4) * bier4 * exp(bierx4 * r));
    if (spline_branch(r)) {
        double v = 0.0;
        for (int k = 0; k < 13; ++k) {
            double d = vcut[k] - r;
            v = v + (3.0 * xh0(d) * vpar[k] * (d * d));
        }
        return -v;
    }
    return (join2 + 2.0 * join3 * r + 3.0 * join4 * r * r) * exp(join1 + join2 * r + join3 * r * r + join4 * r * r * r);
}

double orc_ic_phi(double r)
{
    double d1 = pcut1 - r, d2 = pcut2 - r, d3 = pcut3 - r;
    return xh0(d1) * ppar1 * ((d1 * d1) * d1) - xh0(d2) * ppar2 * ((d2 * d2) * d2) +
           xh0(d3) * ppar3 * ((d3 * d3) * d3);
}

double orc_ic_dphi(double r)
{
    double d1 = pcut1 - r, d2 = pcut2 - r, d3 = pcut3 - r;
    return -(3.0 * xh0(d1) * ppar1 * (d1 * d1) - 3.0 * xh0(d2) * ppar2 * (d2 * d2) +
             3.0 * xh0(d3) * ppar3 * (d3 * d3));
}

static double emb_core(double r)
{
    return (-1.0) * pow(r, 0.5) - (6.7314115586063e-4) * (r * r) + (7.6514905604792e-8) * ((r * r) * (r * r));
}

double orc_ic_emb(double rho)
{
    double e = emb_core(rho);
    if (rho > rcludge) e = e + acludge * ((rho - rcludge) * (rho - rcludge) * (rho - rcludge));
    if (rho > rx) e = emb_core(rx) + acludge * ((rx - rcludge) * (rx - rcludge) * (rx - rcludge));
    return e;
}

double orc_ic_demb(double rho)
{
    if (rho <= 0.0 || rho > rx) return 0.0;
    double d = 0.5 * (-1.0) * pow(rho, -0.5) - 2.0 * (6.7314115586063e-4) * rho +
               4.0 * (7.6514905604792e-8) * ((rho * rho) * rho);
    if (rho > rcludge) d = d + 3.0 * acludge * ((rho - rcludge) * (rho - rcludge));
    return d;
}
