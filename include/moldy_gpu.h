/*
 * moldy_gpu.h -- C ABI of the B200 (sm_100a) MOLDY EAM hot-path library.
 *
 * libmoldy_gpu.so replaces the bodies of the reference's hot-path Fortran
 * subroutines (gjackland/moldy).  The reference has no argument-passing API:
 * its routines act on module globals.  Each entry point below names the
 * routine it replaces; a Fortran ISO_C_BINDING shim keeps the original
 * names and copies the module globals in and out of these calls.
 *
 * Conventions (identical to the reference):
 *  - FP64 everywhere at the boundary; int32 integers;
 *  - positions x0,y0,z0 are fractional, x1 = B0^-1 v dt, x2 = B0^-1 a dt^2/2;
 *  - 3x3 matrices are column-major, exactly Fortran's B0(3,3);
 *  - atom and link-cell indices exported to the caller are 1-based;
 *  - nlist is Fortran NLIST(nnbrs, nm): column i holds atom i's neighbours.
 * Every call returns an int status (MOLDY_OK = 0); the message of the last
 * failure on the calling thread is returned by moldy_gpu_last_error().
 * A handle is not re-entrant: call it from one host thread at a time.
 */
#ifndef MOLDY_GPU_H
#define MOLDY_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes ----------------------------------------------------------*/
#define MOLDY_OK 0
#define MOLDY_ERR_INVALID 1            /* bad argument */
#define MOLDY_ERR_NEIGHBOUR_OVERFLOW 2 /* numn(i) > nnbrs: src/neighbourlist_m.F90:222-229 "stop" */
#define MOLDY_ERR_SINGULAR_BOX 3       /* det(tg) == 0: src/matrix_m.F90:110-113 "stop" */
#define MOLDY_ERR_CUDA 4               /* CUDA runtime failure (message has the CUDA error) */
#define MOLDY_ERR_ORDER 5              /* call order, e.g. force before the potential is set
                                          (src/fetransmetal.F90:110-113 exits here) */
#define MOLDY_ERR_CAPACITY 6           /* an internal capacity was exceeded (message says which) */
#define MOLDY_ERR_UNSUPPORTED 7        /* option not provided by this build */
#define MOLDY_ERR_NO_DEVICE 8          /* no CUDA device, or the kernels were not built for it */

/* precision of the pair arithmetic */
#define MOLDY_PREC_FP64 0   /* all arithmetic in FP64 */
#define MOLDY_PREC_MIXED 1  /* FP32 geometry/tables/pair forces, FP64 accumulation and state */

/* Run parameters: the subset of simparameters (src/params_m.F90:44-162) the
 * hot path reads, already in model units (src/params_m.F90:207-208,412,454). */
typedef struct moldy_params {
    double rnear;     /* neighbour radius rcut + rpad (src/moldin.F90:248) */
    double deltat;    /* time step, model units */
    double press;     /* external pressure, model units */
    double bdel2;     /* deltat^2 / (2 * bmass * nm) (src/params_m.F90:207-208) */
    int32_t nm;       /* number of atoms */
    int32_t nnbrs;    /* neighbour-list capacity per atom (default 150) */
    int32_t ivol;     /* 0 NPT, 1 NVE, 2 free z, 3 cluster, 4 z-only box, 5 pillar */
    int32_t ntcm;     /* neighbour-list rebuild interval ("nbrupdate") */
    int32_t ntc;      /* steps since the last rebuild (normally 0 at start) */
    int32_t nlcx, nlcy, nlcz; /* link cells; 0 = derive as moldin does (src/moldin.F90:252-257) */
    int32_t atomstress;       /* accumulate per-atom stress (src/dynamics_m.F90:279-283) */
    int32_t precision;        /* MOLDY_PREC_FP64 or MOLDY_PREC_MIXED */
    int32_t device;           /* CUDA device ordinal */
    int32_t reserved;
} moldy_params;

/* Results of one force evaluation: the module globals force() sets. */
typedef struct moldy_force_out {
    double pe;        /* potential energy (eV) */
    double vol;       /* box volume (A^3) */
    double tp[9];     /* configurational virial (src/dynamics_m.F90:288-296) */
    double tk[9];     /* kinetic stress (src/thermostat_m.F90:127-164) */
    double tc[9];     /* cofactors of B0 (src/dynamics_m.F90:365-373) */
    double tg[9];     /* B0^T B0 */
    double tgdot[9];  /* B0^T B1 + B1^T B0 */
    double tgid[9];   /* tg^-1 tgdot used by the integrator */
    double fb[9];     /* box force tk + tp - P tc (src/dynamics_m.F90:390-394) */
    int32_t ntc;      /* rebuild counter after the call */
    int32_t rebuilt;  /* 1 when this call rebuilt the neighbour list */
} moldy_force_out;

/* One mdloop iteration's thermodynamics (src/moldin.F90:760-791). */
typedef struct moldy_thermo {
    double ke, pe, te, h, th, vol;  /* eV, eV, eV, eV, eV, A^3 */
    double s1, s2, s3;              /* update_therm_avs sums (src/dynamics_m.F90:649-734) */
    double temp, boxke;             /* K, eV */
    int32_t ntc, rebuilt;
} moldy_thermo;

typedef struct moldy_gpu moldy_gpu;

/* lifecycle ---------------------------------------------------------------*/
/* Allocates the device state for p->nm atoms (init_particles_m,
 * init_neighbourlist_m, init_linkcell_m, init_dynamics_m). */
int moldy_gpu_create(const moldy_params *p, moldy_gpu **out);
int moldy_gpu_destroy(moldy_gpu *h);
/* Message for the last failing call on this thread ("" if none). */
const char *moldy_gpu_last_error(void);
/* Library version string. */
const char *moldy_gpu_version(void);

/* potential ---------------------------------------------------------------*/
/* FETRANSMETAL Fe-Fe from the pot_026_026.in coefficients: runs set_up_m
 * (src/fetransmetal.F90:768-926) and, for uselookup != 0, builds the lookup_m
 * tables with nlookup intervals (src/potential_m.F90:181-228,
 * src/lookup_m.F90:161-251); uselookup == 0 evaluates the *_src functions
 * exactly (src/potential_m.F90:272-280). */
int moldy_gpu_set_fetm_fe(moldy_gpu *h, int32_t nv, const double *av, const double *rv,
                          int32_t np, const double *ap, const double *rp,
                          int32_t uselookup, int32_t nlookup);
/* Caller-built lookup tables for one species pair (potential_set_lookup
 * output): vee, dvee, phi, dphi on r in [rmin, rmax], emb, demb on rho in
 * [rhomin, rhomax], each with nlookup+1 entries (0:nlookup). */
int moldy_gpu_set_tables(moldy_gpu *h, int32_t nlookup, double rmin, double rmax,
                         double rhomin, double rhomax, const double *vee,
                         const double *dvee, const double *phi, const double *dphi,
                         const double *emb, const double *demb);
/* The Fe-Fe functions of the IRON_CARBON material module (src/iron_carbon.F90:
 * Hepburn-Ackland Fe-C), tabulated as potential_set_lookup does over r in
 * [0, 5.4] A and rho in [0, 10000] (lookup mode only; energy_calc and the knot
 * gradients need the FETRANSMETAL forms and return MOLDY_ERR_UNSUPPORTED).
 * moldy_ic_build_tables (no device needed) returns the same six tables. */
int moldy_gpu_set_iron_carbon_fe(moldy_gpu *h, int32_t nlookup);
int moldy_ic_build_tables(int32_t nlookup, double *vee, double *dvee, double *phi, double *dphi,
                          double *emb, double *demb);
/* Copies the six tables back (any pointer may be NULL). */
int moldy_gpu_get_tables(moldy_gpu *h, double *vee, double *dvee, double *phi,
                         double *dphi, double *emb, double *demb);

/* state (particles_m / parrinellorahman_m globals) ------------------------*/
/* Any pointer may be NULL to leave that array unchanged. */
int moldy_gpu_set_state(moldy_gpu *h, const double *x0, const double *y0, const double *z0,
                        const double *x1, const double *y1, const double *z1,
                        const double *x2, const double *y2, const double *z2,
                        const double *b0, const double *b1, const double *b2,
                        const int32_t *atomic_number, const double *atomic_mass,
                        const double *del2, const double *tgid);
int moldy_gpu_get_state(moldy_gpu *h, double *x0, double *y0, double *z0,
                        double *x1, double *y1, double *z1,
                        double *x2, double *y2, double *z2,
                        double *b0, double *b1, double *b2, double *tgid);
/* fx, fy, fz of dynamics_m (fractional forces; real force is B0 f) */
int moldy_gpu_get_forces(moldy_gpu *h, double *fx, double *fy, double *fz);
/* rho, afrho = F(rho), dafrho = F'(rho) of particles_m */
int moldy_gpu_get_density(moldy_gpu *h, double *rho, double *afrho, double *dafrho);
/* stressx/y/z of particles_m (only accumulated when atomstress != 0) */
int moldy_gpu_get_atomstress(moldy_gpu *h, double *sx, double *sy, double *sz);
int moldy_gpu_set_ntc(moldy_gpu *h, int32_t ntc);

/* link cells and neighbour list ---------------------------------------------*/
int moldy_gpu_linkup(moldy_gpu *h);   /* src/linkcell_m.F90:122-198 */
int moldy_gpu_relink(moldy_gpu *h);   /* src/linkcell_m.F90:215-274 */
/* l0(ncell), link(nm), ic(nm) exactly as linkcell_m holds them (1-based). */
int moldy_gpu_get_linkcells(moldy_gpu *h, int32_t *l0, int32_t *link, int32_t *ic);
/* src/neighbourlist_m.F90:103-276 */
int moldy_gpu_update_neighbourlist(moldy_gpu *h);
/* NLIST(nnbrs, nm) and NUMN(nm), entries 1-based, same order as the reference. */
int moldy_gpu_get_neighbourlist(moldy_gpu *h, int32_t *nlist, int32_t *numn);
/* The transpose of that list, as the same build writes it: row i holds the
 * atoms j with i in NLIST(:, j) -- i's own link cell before i, then the 13
 * cells of the mirror half stencil (offsets negated, in reverse order), each
 * cell in chain order.  Same layout as moldy_gpu_get_neighbourlist.  No
 * reference counterpart: the reference walks only the half list. */
int moldy_gpu_get_reverse_list(moldy_gpu *h, int32_t *rlist, int32_t *numr);

/* the hot path --------------------------------------------------------------*/
/* dynamics_m::force (src/dynamics_m.F90:135-401): rebuild schedule (ntc),
 * rhoset, embed, pair and embedding forces, virial, tc, kinten, fb.
 * out may be NULL; forces stay on the device (moldy_gpu_get_forces). */
int moldy_gpu_force(moldy_gpu *h, moldy_force_out *out);
/* quench_m::velocityverlet (src/quench_m.F90:562-624), one step. */
int moldy_gpu_velocityverlet(moldy_gpu *h, moldy_force_out *out);
/* dynamics_m::update_therm_avs (src/dynamics_m.F90:649-734): s123 = s1, s2, s3 */
int moldy_gpu_update_therm_avs(moldy_gpu *h, double *s123);
/* moldin strain-loop preparation (src/moldin.F90:445-477): force, then
 * tgid = tg^-1 tgdot, x2 = del2 f - tgid x1 / 2, b2 = bdel2 fb. */
int moldy_gpu_md_init(moldy_gpu *h, moldy_force_out *out);
/* nsteps mdloop iterations (src/moldin.F90:752-791): velocityverlet,
 * update_therm_avs, thermodynamics, relink when ntc wraps.  thermo (may be
 * NULL) receives nsteps records. */
int moldy_gpu_md_steps(moldy_gpu *h, int32_t nsteps, moldy_thermo *thermo);
/* dynamics_m::energy_calc (src/dynamics_m.F90:412-483): per-atom energy with
 * the exact pair function. */
int moldy_gpu_energy_calc(moldy_gpu *h, double *en_atom);
/* thermostat_m::scalev (src/thermostat_m.F90:317-395), the Nose-Hoover Euler
 * thermostat.  moldy_gpu_set_thermostat sets simparam%nose and simparam%rqke
 * (nose = 0: off, the default).  With nose > 0, moldy_gpu_md_steps calls
 * scalev once per femtosecond of simulated time as the mdloop does
 * (src/moldin.F90:828-835: a timer advanced by deltat against the constant
 * 0.098227).  moldy_gpu_scalev calls it once now.  out4: nose, rqke, snhv
 * (the accumulated scaling), the timer. */
int moldy_gpu_set_thermostat(moldy_gpu *h, double nose, double rqke);
int moldy_gpu_get_thermostat(moldy_gpu *h, double *out4);
int moldy_gpu_scalev(moldy_gpu *h);
/* Waits for all work queued on the handle's stream. */
int moldy_gpu_synchronize(moldy_gpu *h);

/* instrumentation (no counterpart in the reference) --------------------------*/
/* The cudaStream_t all of the handle's work is queued on. */
int moldy_gpu_get_stream(moldy_gpu *h, void **stream);
/* Per-kernel-family timing with CUDA events on that stream (off by default);
 * launch counts are always kept. */
int moldy_gpu_set_profiling(moldy_gpu *h, int32_t enable);
int moldy_gpu_reset_kernel_stats(moldy_gpu *h);
/* Accumulated device time (ms, when profiling) and kernel launches of one
 * family since the last reset; kernel ids are 0 .. MOLDY_KERNEL_FAMILIES-1. */
int moldy_gpu_kernel_stats(moldy_gpu *h, int32_t kernel, double *total_ms, int64_t *launches);
const char *moldy_gpu_kernel_name(int32_t kernel);
#define MOLDY_KERNEL_FAMILIES 16

/* kernel variants (no counterpart in the reference) -------------------------*/
/* The screening-density pass and the force pass are compiled in
 * MOLDY_TUNE_VARIANTS variants each: how many list entries a thread gathers
 * before using them, with or without L2 prefetches of the next atom's data,
 * and two or three resident blocks per SM (registers per thread).
 * moldy_gpu_autotune times every variant on the current configuration with
 * nreps force evaluations (positions, velocities, the rebuild counter and the
 * neighbour list are left unchanged) and keeps the fastest of each pass.
 * times_ms (3*MOLDY_TUNE_VARIANTS, may be NULL) receives the mean time per
 * launch: screening-density, then zeros (the density pass is fused into it),
 * then forces; chosen (3, may be NULL) the selected variants in that order.
 * moldy_gpu_set_variants takes the same three numbers (the second is unused). */
#define MOLDY_TUNE_VARIANTS 8
/* Skin of the intermediate list (A, default 0.3): it holds the half-list pairs
 * within min(rnear, table cut + skin) and is rebuilt on the device whenever
 * the displacements since its build could bring an unlisted pair inside the
 * cut.  It is filtered from the outer list, the half-list pairs within
 * min(rnear, table cut + max(outer skin, skin + 0.4)) (outer skin default
 * 1.0 A), which is rebuilt from the half list whenever the displacements since
 * its own build could bring an unlisted pair within the intermediate radius.
 * Results depend on neither skin; only the time per step does. */
int moldy_gpu_set_mid_skin(moldy_gpu *h, double skin);
int moldy_gpu_set_outer_skin(moldy_gpu *h, double skin);
/* builds of the outer list so far */
int moldy_gpu_get_outer_builds(moldy_gpu *h, int32_t *builds);
int moldy_gpu_autotune(moldy_gpu *h, int32_t nreps, double *times_ms, int32_t *chosen);
int moldy_gpu_set_variants(moldy_gpu *h, int32_t screen, int32_t density, int32_t forces);
/* out3[0]: directed interacting pairs (inside the table range) of the last
 * force evaluation, twice the contributing half-list pairs; out3[1]: how many
 * times the intermediate list (half-list pairs within the table cut + skin)
 * has been built; out3[2]: list entries the screening pass reads per step
 * (the intermediate rows). */
int moldy_gpu_get_list_stats(moldy_gpu *h, double *out3);

/* adjoint (no counterpart in the reference) ---------------------------------*/
/* Gradients of a scalar loss L(E, F, sigma) with respect to the potential, for
 * force-matching fits.  E is pe, F the real forces B0 f (what
 * write_energy_forces_stress prints, src/dynamics_m.F90:588-619) and
 * sigma(i,j) = -sum_k b0(j,k) tp(i,k) / vol, all as the last moldy_gpu_force
 * (or velocityverlet / md_init / md_steps) computed them at the current state
 * and tables; otherwise MOLDY_ERR_ORDER.  Inputs: g_energy = dL/dE, g_force =
 * dL/dF (3*nm host doubles, x|y|z; NULL = 0), g_stress = dL/dsigma (9 host
 * doubles, column-major; NULL = 0).  Lookup mode only (else
 * MOLDY_ERR_UNSUPPORTED); the gradient is exact for the linearly interpolated
 * tables and computed in FP64 whatever the handle's precision, with rho
 * recomputed on the device.
 * moldy_gpu_table_gradients: dL/d(table node), nlookup+1 doubles per table
 * (any pointer may be NULL).
 * moldy_gpu_knot_gradients: dL/d(knot parameters) of the FETRANSMETAL Fe-Fe
 * functions set by moldy_gpu_set_fetm_fe (src/fetransmetal.F90:74-77): nv
 * values each for av and rv, np each for ap and rp (F = -sqrt(rho) has none). */
int moldy_gpu_table_gradients(moldy_gpu *h, double g_energy, const double *g_force,
                              const double *g_stress, double *g_vee, double *g_dvee,
                              double *g_phi, double *g_dphi, double *g_emb, double *g_demb);
int moldy_gpu_knot_gradients(moldy_gpu *h, double g_energy, const double *g_force,
                             const double *g_stress, double *g_av, double *g_rv,
                             double *g_ap, double *g_rp);
/* Host-only helpers (no device needed).  moldy_fetm_build_tables builds the six
 * lookup tables (nlookup+1 each) of the Fe-Fe knots as potential_set_lookup
 * does (src/potential_m.F90:181-228).  moldy_fetm_knot_vjp contracts table
 * gradients g_vee..g_demb (nlookup+1 each, any may be NULL) with the
 * derivative of those tables in the knots, as moldy_gpu_knot_gradients does. */
int moldy_fetm_build_tables(int32_t nv, const double *av, const double *rv, int32_t np,
                            const double *ap, const double *rp, int32_t nlookup,
                            double *vee, double *dvee, double *phi, double *dphi,
                            double *emb, double *demb);
int moldy_fetm_knot_vjp(int32_t nv, const double *av, const double *rv, int32_t np,
                        const double *ap, const double *rp, int32_t nlookup,
                        const double *g_vee, const double *g_dvee, const double *g_phi,
                        const double *g_dphi, const double *g_emb, const double *g_demb,
                        double *g_av, double *g_rv, double *g_ap, double *g_rp);

/* analysis_m::rdf (src/analysis_m.F90:497-760) at the current device state.
 *
 * moldy_gpu_rdf: pair-distance histogram hist[(ibin * nspec + si) * nspec + sj]
 * for ibin = int(r * binsperangstrom) in 0..maxbin (bin 0 holds the pairs the
 * reference would write out of bounds).  mode 0 bins the half neighbour list
 * as it stands, pairs with rsq <= (maxbin/binsperangstrom)**2 in integer
 * division (analysis_m.F90:580-608); mode 1 bins every pair of atoms, the
 * older form of the routine that wrote the reference's shipped rdf.dat
 * (every box width must exceed 2 (maxbin+1)/binsperangstrom).  species[nm]
 * holds each atom's 0-based species index (atomic_index - 1), NULL for one
 * species; atoms with atomic number 0 are vacancies and are skipped.
 * natoms[nspec] counts the non-vacancy atoms, *nclose the pairs closer than
 * 2 A (the routine's warning); either may be NULL.
 *
 * moldy_gpu_ackland_jones: per-atom class aj (0 unknown, 1 bcc, 2 fcc, 3 hcp,
 * 4 icosahedral), coordination nn and, unless NULL, the eight bond-angle
 * counts chi[8 i + k] (analysis_m.F90:644-757), for neighbours within
 * rsq <= 1.45 rn[si * nspec + sj]^2 (rn: the fourth-neighbour radii the
 * routine estimates from the histogram, analysis_m.F90:619-637).  mode 0
 * takes the full list from the half list, mode 1 every atom.  Fails with
 * MOLDY_ERR_CAPACITY when an atom has more than 32 such neighbours. */
int moldy_gpu_rdf(moldy_gpu *h, int32_t mode, int32_t maxbin, int32_t binsperangstrom, const int32_t *species,
                  int32_t nspec, uint64_t *hist, int64_t *natoms, int64_t *nclose);
int moldy_gpu_ackland_jones(moldy_gpu *h, int32_t mode, const int32_t *species, int32_t nspec, const double *rn,
                            int32_t *aj, int32_t *nn, int32_t *chi);

/* batched supercells (no counterpart in the reference's API) ----------------*/
/* Many independent systems of uneven size (strained or perturbed replicas)
 * evaluated together: each launch covers every system.  Atoms of all systems
 * are concatenated, each system's in the reference's order.  Per system the
 * results are those of force() + energy_calc() (src/dynamics_m.F90:135-483)
 * in lookup mode, and the quench is quench_m::quench with VA14CD and derivs
 * (src/quench_m.F90:100-551) at a fixed box (ivol = 1).  Each system keeps
 * its own list of the pairs within rcut + skin, found by neighbour-cell tiles
 * and rebuilt on the device once one of its atoms has moved half the skin
 * (moldy_gpu_batch_set_skin); the passes keep the pairs inside the table cut,
 * and beyond it every pair contributes zero, so the sums are those of a
 * complete list.  Each box must be wider than twice the interaction range in
 * every direction (MOLDY_ERR_INVALID otherwise). */
typedef struct moldy_batch moldy_batch;
int moldy_gpu_batch_create(int32_t nsys, const int32_t *natoms, double press, int32_t device,
                           moldy_batch **out);
int moldy_gpu_batch_destroy(moldy_batch *h);
/* FETRANSMETAL Fe-Fe knots, lookup tables of nlookup intervals (as
 * moldy_gpu_set_fetm_fe with uselookup = 1); energy_calc uses the exact pair function. */
int moldy_gpu_batch_set_fetm_fe(moldy_batch *h, int32_t nv, const double *av, const double *rv,
                                int32_t np, const double *ap, const double *rp, int32_t nlookup);
/* x0, y0, z0: concatenated fractional positions; b0: 9 doubles per system
 * (column-major); mass: per atom, NULL keeps the current (55.845 by default).
 * Any pointer may be NULL to keep that part; b0 fixes the cell grids. */
int moldy_gpu_batch_set_state(moldy_batch *h, const double *x0, const double *y0,
                              const double *z0, const double *b0, const double *mass);
int moldy_gpu_batch_get_state(moldy_batch *h, double *x0, double *y0, double *z0);
/* One evaluation of every system.  out13 (13 doubles per system, may be NULL):
 * pe of energy_calc (F + exact pair function), pe of force (F + tabulated pair
 * function), largest real force |B0 f| (eV/A), vol, tp (column-major, the
 * virial of force(), pairs with m_i + m_j > 0.1). */
int moldy_gpu_batch_force(moldy_batch *h, double *out13);
/* fractional forces, per-atom energies (energy_calc; force routine), rho/F/F' */
int moldy_gpu_batch_get_forces(moldy_batch *h, double *fx, double *fy, double *fz);
/* Interleaved forms: xyz[3i..3i+2] are atom i's fractional position or
 * fractional force (the layout of quench_m's x vector), one copy each way. */
int moldy_gpu_batch_set_positions(moldy_batch *h, const double *xyz);
int moldy_gpu_batch_get_forces_xyz(moldy_batch *h, double *fxyz);
int moldy_gpu_batch_get_energies(moldy_batch *h, double *en_calc, double *en_force);
int moldy_gpu_batch_get_density(moldy_batch *h, double *rho, double *afrho, double *dafrho);
/* Conjugate-gradient quench of every system with at most maxfn function values
 * each (VA14CD's MAXFN = NSTEPS).  criterion 0: the reference's acceptance,
 * sum of squared gradient <= 5e-7 nm; 1: largest real force <= fmax (eV/A).
 * out8 (8 doubles per system, may be NULL): f = pe + press vol at the returned
 * point, pe and largest real force of the last evaluation, sum of squared
 * gradient, function values, iterations, iflag (0 converged, 1 maxfn reached,
 * 2 VA14CD's conjugate-gradient error return), 0.  The positions are left at
 * the returned points (moldy_gpu_batch_get_state). */
int moldy_gpu_batch_quench(moldy_batch *h, int32_t maxfn, int32_t criterion, double fmax,
                           double *out8);
/* Tile shape of the list builds: lanes per home atom (4, 8, 16 or 32; default
 * 8) and how many candidates a warp stages in shared memory (0..256, default
 * 256; the rest are read from global memory). */
int moldy_gpu_batch_set_tiles(moldy_batch *h, int32_t lanes, int32_t staged);
/* Chooses, on the live configuration, the lanes per home atom of the tile
 * screen (4, 8, 16, 32; timed on evaluations that rebuild every list), the
 * row entries gathered at a time by the per-atom passes (1, 2, 4; timed with
 * current lists) and, where the persistent evaluation applies, its lanes per
 * atom (1, 2, 4; timed with current lists), nreps evaluations each in the
 * current precision, and keeps the fastest.  times_ms (10 doubles, may be
 * NULL) receives the mean times in that order (the last three 0 where the
 * persistent evaluation does not apply), chosen (3 int32, may be NULL) the
 * tile lanes, the entries and the lanes per atom (0: not tuned).  Results do
 * not depend on the tile lanes or the entries; the lanes per atom change the
 * order of each atom's FP64 sums.  Positions and boxes are unchanged. */
int moldy_gpu_batch_autotune(moldy_batch *h, int32_t nreps, double *times_ms, int32_t *chosen);
/* One evaluation of every system (as moldy_gpu_batch_force) with its four
 * launches timed by CUDA events on the batch's stream: the list check, the
 * tile screen, the density pass and the force pass, into ms4 (ms);
 * rebuild = 1 rebuilds every list first. */
int moldy_gpu_batch_kernel_times(moldy_batch *h, int32_t rebuild, double *ms4);
/* The persistent evaluation: moldy_gpu_batch_force evaluates every system in
 * one launch (k_batch_eval) when the precision is mixed, energy_calc is off,
 * every atom is heavier than 0.05 and the largest system's records (16 bytes
 * per atom) fit in one block's shared memory.  A resident grid of blocks
 * takes the systems in descending size from a device queue; per system the
 * block checks (and rebuilds) the list, stages the atoms in shared memory as
 * fixed-point records and runs the density and force passes with `lanes`
 * lanes per atom, then the per-system sums.  The launch (with the kernel that
 * marks every system active) is captured once in a CUDA graph and replayed;
 * it is captured again when the tile or lane choices or a buffer change.
 * enable = 0 keeps the per-pass launches (default 1). */
int moldy_gpu_batch_set_persistent(moldy_batch *h, int32_t enable);
/* Lanes per atom in the persistent evaluation's passes: 1, 2 or 4 (default 2;
 * moldy_gpu_batch_autotune chooses). */
int moldy_gpu_batch_set_atom_lanes(moldy_batch *h, int32_t lanes);
/* *applies = 1 when moldy_gpu_batch_force runs the persistent evaluation. */
int moldy_gpu_batch_persistent_applies(moldy_batch *h, int32_t *applies);
/* Device times (ms) of the persistent evaluation: ms2[0] with every list
 * current, ms2[1] with every list rebuilt in the same launch.
 * MOLDY_ERR_UNSUPPORTED where it does not apply. */
int moldy_gpu_batch_eval_times(moldy_batch *h, double *ms2);
/* Precision of the per-atom density and force passes of moldy_gpu_batch_force:
 * 0 all FP64 (default); 1 mixed: separations, distances, table interpolation
 * and pair forces in FP32 from FP64 position differences, every sum in FP64,
 * and energy_calc's exact pair energy at the FP64 distance.  The quench always
 * evaluates in FP64: its line search compares energies that differ in the
 * seventh digit, below what FP32 distances resolve. */
int moldy_gpu_batch_set_precision(moldy_batch *h, int32_t mixed);
/* Whether moldy_gpu_batch_force also forms energy_calc's per-atom energies
 * (src/dynamics_m.F90:412-483, the exact pair function at every pair inside
 * the cut): 1 (default) yes; 0 no, and the energy_calc sums and
 * moldy_gpu_batch_get_energies' en_calc read zero.  The force routine's
 * energy, the forces and the virial do not depend on it; the quench always
 * forms them, since derivs (src/quench_m.F90:215-323) takes its energy from
 * energy_calc. */
int moldy_gpu_batch_set_energy_calc(moldy_batch *h, int32_t enable);
/* Force matching over all systems of a batch (no counterpart in the
 * reference; it differentiates what write_energy_forces_stress prints,
 * src/dynamics_m.F90:588-619).  set_references takes the reference real
 * forces (3 * ntot doubles, interleaved x, y, z per atom, atom order) and
 * stresses (9 doubles per system, sigma(i,j) at i + 3 j, in the model units
 * of moldy_gpu_batch_force's tp: sigma(i,j) = -sum_k b0(j,k) tp(i,k) / vol).  force_matching then runs one FP64 evaluation of
 * every system, writes each system's loss
 *   L_s = w_force sum_i |F_i - F_i^ref|^2 + w_stress |sigma_s - sigma_s^ref|^2
 * into loss[nsys], and dL/d(table) of sum_s L_s into table_grads[6 * (nlookup
 * + 1)] (vee, dvee, phi, dphi, emb, demb; vee and emb get none, the loss holds
 * no energy).  Pairs inside the table cut enter, which carries every node
 * below the cut and every knot derivative (moldy_fetm_knot_vjp contracts the
 * table gradients to the knots). */
int moldy_gpu_batch_set_references(moldy_batch *h, const double *fref_xyz, const double *sref);
int moldy_gpu_batch_force_matching(moldy_batch *h, double w_force, double w_stress, double *loss,
                                   double *table_grads);
/* Row entries one thread gathers before it evaluates them in the per-atom
 * passes: 1, 2 or 4 (default 4).  Results do not depend on it. */
int moldy_gpu_batch_set_gather(moldy_batch *h, int32_t entries);
/* Verlet skin of the per-system lists (default 0.3 A): a system's list holds
 * the pairs within rcut + skin (less where its box is narrower than twice
 * that) and is rebuilt once one of its atoms has moved more than half the
 * skin since the last build, or after its box changed.  0 rebuilds at every
 * evaluation in which an atom moved. */
int moldy_gpu_batch_set_skin(moldy_batch *h, double skin);
/* out2[0]: system list builds so far; out2[1]: system evaluations so far. */
int moldy_gpu_batch_list_stats(moldy_batch *h, int64_t *out2);
/* Entries of the compact rows (the pairs within each system's list radius,
 * both directions) summed over all atoms, as the last evaluation left them. */
int moldy_gpu_batch_row_entries(moldy_batch *h, int64_t *total);
/* Kernel launches queued so far by this handle; its cudaStream_t. */
int moldy_gpu_batch_launches(moldy_batch *h, int64_t *launches);
int moldy_gpu_batch_get_stream(moldy_batch *h, void **stream);

/* force evaluation without device allocation -----------------------------*/
/* No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (device memory owned by another allocator, or code that must not allocate
 * while it runs): one EAM force evaluation (rhoset, embed and the pair loop
 * of src/dynamics_m.F90:135-401) on buffers the caller owns, with its
 * intermediates in a fixed __device__ array inside this library, so the call
 * allocates nothing.  Limit: nm <= MOLDY_NOALLOC_MAX_ATOMS, else
 * MOLDY_ERR_CAPACITY.  Device pointers: x0,y0,z0 (fractional), mass (may be
 * NULL: every pair enters the virial), nlist/numn (NLIST(nnbrs,nm) with
 * 1-based entries, NUMN(nm)), the six tables (nlookup+1 entries each),
 * fx,fy,fz (fractional forces, overwritten) and energy_virial (10 doubles:
 * pe, then tp column-major).  b0 is a host array (column-major 3x3).  Work
 * is queued on `stream` (a cudaStream_t, NULL = legacy default stream) and
 * the call returns after it finishes.  The first call on each device looks
 * up the array's device address; make that first call before any stream
 * capture; the cached address belongs to the device's primary context, so a
 * device reset or a caller-made context between calls is not supported.
 * Every call shares the array: calls that overlap on the GPU race and give
 * wrong results.  Unlike embed (src/potential_m.F90:162), an atom with
 * rho <= 1e-40 gets F = F' = 0 (the array may hold another system's F').
 * A NUMN count outside 0..nnbrs or an NLIST entry outside 1..nm returns
 * MOLDY_ERR_INVALID (the row is clamped, the entry skipped). */
#define MOLDY_NOALLOC_MAX_ATOMS 262144
int moldy_gpu_force_noalloc(int32_t nm, int32_t nnbrs, int32_t ivol,
                            const double *x0, const double *y0, const double *z0,
                            const double *mass, const double *b0,
                            const int32_t *nlist, const int32_t *numn, int32_t nlookup,
                            double rmin, double rmax, double rhomin, double rhomax,
                            const double *vee, const double *dvee, const double *phi,
                            const double *dphi, const double *emb, const double *demb,
                            double *fx, double *fy, double *fz, double *energy_virial,
                            void *stream);

#ifdef __cplusplus
}
#endif
#endif /* MOLDY_GPU_H */
