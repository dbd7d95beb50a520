/*
 * moldy_oracle.h -- CPU oracle for the MOLDY EAM force hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, FP64 restatement of the
 * reference Fortran (gjackland/moldy, FETRANSMETAL build) used as the parity
 * checker for the CUDA library and as the timed CPU baseline.  It is never
 * linked into, called by, or shipped with the product library.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 *
 * Parity status: the reference cannot be compiled here (no Fortran compiler),
 * and the reference's shipped golden outputs were produced with a different
 * material module (IRON_CARBON).  The restatement is therefore pinned by
 * known-answer properties computed from the reference's own coefficient file
 * (perfect-lattice energy/density, zero forces, force = -dE/dx), not by
 * reference-produced vectors.
 *
 * Conventions follow the reference exactly: atom and link-cell indices are
 * 1-based with 0 meaning "none"; 3x3 matrices are column-major like Fortran
 * B0(3,3); positions are fractional, x1 = v*dt and x2 = a*dt^2/2 fractional.
 */
#ifndef MOLDY_ORACLE_H
#define MOLDY_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sys orc_sys;

/* lifecycle ---------------------------------------------------------------*/
orc_sys *orc_create(int nm, int nnbrs, int ivol, int ntcm, int atomstress,
                    double rnear, double deltat, double press, double bdel2);
void orc_destroy(orc_sys *s);
void orc_set_threads(int nthreads);
int orc_get_max_threads(void);

/* potential: FETRANSMETAL Fe-Fe (src/fetransmetal.F90) -----------------------*/
/* coefficients as read from pot_026_026.in; runs set_up_m (spline joins,
 * phi maximum by bisection).  Returns 0 on success. */
int orc_set_fetm(orc_sys *s, int nv, const double *av, const double *rv,
                 int np, const double *ap, const double *rp);
/* uselookup=1: build the six lookup_m tables with nlookup intervals
 * (r in [0,6], rho in [0,10000]); uselookup=0: exact *_src evaluation. */
int orc_set_lookup(orc_sys *s, int uselookup, int nlookup);
/* a caller's own lookup_m tables (nlookup + 1 nodes each, r in [rmin, rmax],
 * rho in [rhomin, rhomax]); switches to lookup mode.  Returns 0 on success. */
int orc_set_tables(orc_sys *s, int nlookup, double rmin, double rmax, double rhomin, double rhomax,
                   const double *vee, const double *dvee, const double *phi, const double *dphi,
                   const double *emb, const double *demb);
/* the Fe-Fe functions of the IRON_CARBON module (src/iron_carbon.F90) in place of FETRANSMETAL */
int orc_set_iron_carbon(orc_sys *s);
void orc_get_tables(const orc_sys *s, double *vee, double *dvee, double *phi,
                    double *dphi, double *emb, double *demb);
void orc_get_fetm_derived(const orc_sys *s, double *out8);
double orc_src(const orc_sys *s, int which, double r);    /* 0..5: vee dvee phi dphi emb demb */
double orc_lookup(const orc_sys *s, int which, double r); /* table interpolation */

/* state -------------------------------------------------------------------*/
void orc_set_state(orc_sys *s, const double *x0, const double *y0, const double *z0,
                   const double *x1, const double *y1, const double *z1,
                   const double *x2, const double *y2, const double *z2,
                   const double *b0, const double *b1, const double *b2,
                   const int *atomic_number, const double *atomic_mass,
                   const double *del2, const double *tgid);
void orc_get_state(const orc_sys *s, double *x0, double *y0, double *z0,
                   double *x1, double *y1, double *z1,
                   double *x2, double *y2, double *z2,
                   double *b0, double *b1, double *b2, double *tgid);
void orc_get_forces(const orc_sys *s, double *fx, double *fy, double *fz);
void orc_get_density(const orc_sys *s, double *rho, double *afrho, double *dafrho);
void orc_get_atomstress(const orc_sys *s, double *sx, double *sy, double *sz);
/* pe, vol, then tp tk tc tg tgdot tgid fb (9 each, column-major): 65 doubles */
void orc_get_force_out(const orc_sys *s, double *out65);
void orc_set_ntc(orc_sys *s, int ntc);
int orc_get_ntc(const orc_sys *s);

/* link cells / neighbour list (src/linkcell_m.F90, src/neighbourlist_m.F90) */
void orc_set_nlc(orc_sys *s, int nlcx, int nlcy, int nlcz);
void orc_get_nlc(const orc_sys *s, int *nlc3);
void orc_linkup(orc_sys *s);
void orc_relink(orc_sys *s);
void orc_get_linkcells(const orc_sys *s, int *l0, int *link, int *ic);
int orc_update_neighbourlist(orc_sys *s);          /* 0 ok, 1 overflow */
void orc_get_nlist(const orc_sys *s, int *nlist, int *numn); /* nlist(nnbrs,nm) */

/* the hot path ------------------------------------------------------------*/
int orc_force(orc_sys *s);                            /* dynamics_m::force */
int orc_velocityverlet(orc_sys *s);                   /* quench_m::velocityverlet */
void orc_update_therm_avs(orc_sys *s, double *s123);  /* dynamics_m::update_therm_avs */
void orc_energy_calc(orc_sys *s, double *en_atom);    /* dynamics_m::energy_calc */
/* moldin strain-loop preparation: force, tgid, initial x2 and b2 */
int orc_md_init(orc_sys *s);
/* thermostat_m::scalev (src/thermostat_m.F90:317-395); nose = 0 is off */
void orc_set_thermostat(orc_sys *s, double nose, double rqke);
void orc_get_thermostat(const orc_sys *s, double *out4); /* nose, rqke, snhv, thermotimer */
void orc_scalev(orc_sys *s);
/* quench_m::quench with VA14CD and derivs (src/quench_m.F90:100-551); maxfn is
 * NSTEPS; criterion 0: gsumsq <= 5e-7 nm, 1: max real force <= fmax.
 * out8: f, pe, gsumsq, max |B0 f|, evaluations, iterations, iflag, status
 * (pe and max |B0 f| are those of the last evaluation). */
int orc_quench(orc_sys *s, int maxfn, int criterion, double fmax, double *out8);
/* one mdloop iteration: velocityverlet, update_therm_avs, thermo, relink.
 * out12 = ke, pe, te, h, th, vol, s1, s2, s3, temperature, boxke, ntc */
int orc_md_step(orc_sys *s, double *out12);
/* analysis_m::rdf (src/analysis_m.F90:497-760).  mode 0: half-list pairs;
 * mode 1: every pair j < i.  spec[nm]: 0-based species index per atom.
 * hist[((ibin * nspec) + si) * nspec + sj], ibin 0..maxbin. */
void orc_rdf(const orc_sys *s, int mode, int maxbin, int bpa, const int *spec, int nspec, long long *hist,
             long long *natoms, long long *nclose);
void orc_rdf_rneighbour(const long long *hist, const long long *natoms, int maxbin, int bpa, int nspec, double *rn);
void orc_ackland_jones(const orc_sys *s, int mode, const int *spec, int nspec, const double *rn, int *aj, int *nn,
                       int *chi);

#ifdef __cplusplus
}
#endif
#endif
