/*
 * oracle_internal.h -- private state of the CPU oracle (TEST INFRASTRUCTURE).
 * The struct mirrors the reference's module globals (particles_m, dynamics_m,
 * parrinellorahman_m, linkcell_m, neighbourlist_m, potential_m, lookup_m).
 */
#ifndef MOLDY_ORACLE_INTERNAL_H
#define MOLDY_ORACLE_INTERNAL_H

#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "moldy_oracle.h"

#define ORC_MAXCOEF 16

/* Fortran-style 1-based access to a column-major 3x3 matrix */
#define M3(a, i, j) ((a)[((i) - 1) + 3 * ((j) - 1)])

struct orc_sys {
    /* simparameters subset (src/params_m.F90:44-162) */
    int nm, nnbrs, ivol, ntcm, ntc, atomstress;
    int nlcx, nlcy, nlcz, ncell;
    double rnear, deltat, press, bdel2;

    /* FETRANSMETAL Fe-Fe data (src/fetransmetal.F90:70-90) */
    int nv, np, fetm_set;
    int potential;   /* 0 FETRANSMETAL, 1 IRON_CARBON Fe-Fe */
    double av[ORC_MAXCOEF], rv[ORC_MAXCOEF], ap[ORC_MAXCOEF], rp[ORC_MAXCOEF];
    double p1, dp2, p3, dp4;
    double bier_cut1, bier_cut2, sc[4], phi_cut1, phi_cut2;

    /* lookup tables (src/lookup_m.F90:64-78) */
    int uselookup, nlookup;
    double *tab[6];
    double vp_rmin, vp_rmax, vp_range, vp_reciprange, vp_recipnlkp, vp_recipstep;
    double e_rmin, e_rmax, e_range, e_reciprange, e_recipnlkp, e_recipstep;

    /* per-atom arrays, 1-based (index 0 unused) */
    double *x0, *y0, *z0, *x1, *y1, *z1, *x2, *y2, *z2;
    double *x1dt2, *y1dt2, *z1dt2;
    double *fx, *fy, *fz, *rho, *afrho, *dafrho, *stx, *sty, *stz;
    int *atomic_number;
    double *atomic_mass, *del2;

    /* box tensors (src/parrinellorahman_m.F90:102-115) */
    double b0[9], b1[9], b2[9], tk[9], tc[9], tg[9], tp[9];
    double tginv[9], tgdot[9], tgid[9], fb[9];
    double vol, pe, ke;

    /* thermostat_m (src/thermostat_m.F90:54-57) and the mdloop's thermotimer */
    double nose, rqke, snhv, snhf, thermotimer;

    /* link cells and neighbour list */
    int *l0, *link, *ic;
    int *nlist, *numn;
#ifdef _OPENMP
    omp_lock_t *locks;
#endif
    int nlocks;
};

void orc_free_tables(orc_sys *s);
double orc_vee_src(const orc_sys *s, double r);
double orc_dvee_src(const orc_sys *s, double r);
double orc_phi_src(const orc_sys *s, double r);
double orc_dphi_src(const orc_sys *s, double r);
double orc_emb_src(const orc_sys *s, double rho);
double orc_demb_src(const orc_sys *s, double rho);
double orc_ic_vee(double r);
double orc_ic_dvee(double r);
double orc_ic_phi(double r);
double orc_ic_dphi(double r);
double orc_ic_emb(double rho);
double orc_ic_demb(double rho);
double orc_lookup_r(const orc_sys *s, const double *t, double r);
double orc_lookup_rho(const orc_sys *s, const double *t, double rho);
double orc_vee(const orc_sys *s, double r);
double orc_dvee(const orc_sys *s, double r);
double orc_phi(const orc_sys *s, double r);
double orc_dphi(const orc_sys *s, double r);
double orc_emb(const orc_sys *s, double rho);
double orc_demb(const orc_sys *s, double rho);

#endif
