// engine.h -- host-side state of one MOLDY system on one GPU.
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/moldy_gpu.h"
#include "common.cuh"

namespace moldy {

// Device buffers of one system.  Atom arrays are in the reference's atom
// order; the link-cell structure is a CSR over cells whose segments list each
// cell's atoms in the reference's chain (traversal) order.
struct DeviceState {
    // particles_m
    double4 *pos = nullptr;       // (x0, y0, z0, -)
    double *x1 = nullptr;         // 3*nm, SoA x|y|z
    double *x2 = nullptr;         // 3*nm
    double *f = nullptr;          // 3*nm fx|fy|fz
    double *rho = nullptr, *afrho = nullptr, *dafrho = nullptr;
    double *stress = nullptr;     // 3*nm
    double *mass = nullptr, *del2 = nullptr;
    int32_t *znum = nullptr;
    double *en_atom = nullptr;
    // link cells (linkcell_m)
    int32_t *ic = nullptr;        // cell of each atom, 0-based
    int32_t *cell_start = nullptr, *cell_atoms = nullptr, *cell_pos = nullptr;
    int32_t *cell_count = nullptr;
    // relink scratch
    int32_t *ic_new = nullptr, *arr_count = nullptr, *arr_start = nullptr, *arr_list = nullptr;
    int32_t *work = nullptr, *new_count = nullptr, *new_start = nullptr, *cell_atoms2 = nullptr;
    // neighbour list (neighbourlist_m) as the reference holds NLIST(nnbrs, nm):
    // entry k of atom i at nlist[i*nnbrs + k], 0-based atom ids; rlist/numr
    // hold each atom's reverse half row (the atoms j with i in row(j)),
    // written by the same build, entry-major: entry k of atom j at
    // rlist[k*nm + j]
    int32_t *nlist = nullptr, *numn = nullptr;
    int32_t *rlist = nullptr, *numr = nullptr;
    // scratch of the structure analysis (rdf.cu), grown on demand
    void *rdf = nullptr;
    size_t rdf_bytes = 0;
    // fixed-point fractional positions (2^32 units per box length; written with
    // pos) for the mixed screening pass; posq2 adds F'(rho) as a float in w for
    // the mixed force pass
    int4 *posq = nullptr, *posq2 = nullptr;
    // positions with F'(rho) in w, written by the density pass for the FP64 force pass
    double4 *pos2 = nullptr;
    // compact full list of the pairs inside the table cut, entry-major:
    // entry e of atom i at alist[e * nm + i] (e < pair_cap), bit 31 set when
    // j is in i's own half-list row; pair_cnt[i] entries
    int32_t *alist = nullptr, *pair_cnt = nullptr;
    // outer FULL list: the half-list pairs within r_out = r_cut + outer skin
    // when built, entered in both rows (bit 31 on the owner's copy),
    // entry-major; row of atom i: its own entries (half-list order), then its
    // reverse entries (reverse-row order), out_cnt[i] in all; xout holds the
    // positions at build time
    int32_t *olist = nullptr, *out_cnt = nullptr;
    int4 *xout = nullptr;                  // fixed-point (posq) snapshot
    int4 *xhalf = nullptr;                 // fixed-point snapshot at the last half-list build
    // intermediate FULL list: the outer-list pairs within r_mid = r_cut + skin
    // when built, entry-major, mid_cnt[i] entries from slot 0 (bit 31 kept);
    // xbuild holds the positions at build time
    int32_t *mlist = nullptr, *mid_cnt = nullptr;
    int4 *xbuild = nullptr;                // fixed-point (posq) snapshot
    // tables
    double4 *tab_r4 = nullptr;
    double2 *tab_e2 = nullptr;
    float4 *tab_r4f = nullptr;
    float2 *tab_e2f = nullptr;
    void *tab_aux = nullptr;               // phi2 / phi2f node-pair tables
    // per-step thermo records of an md_steps call (kThermoRec doubles each), grown on demand
    double *thermo_rec = nullptr;
    int thermo_cap = 0;
    // reductions, flags and box state
    double *partials = nullptr;
    int32_t *flags = nullptr;     // [0] neighbour overflow, [1] relink inconsistency,
                                  // [2] overflow atom, [3] active-list overflow, [4] its count,
                                  // [5] intermediate-row overflow, [6] its count,
                                  // [8] outer-row overflow, [9] its count,
                                  // [10] reverse half-row overflow, [11] its count,
                                  // [12] a link cell too full for the reverse-row masks
    // per (cell rank r of the half stencil, round of 32 home atoms, atom j):
    // the home atoms of j's source cell whose half-list rows hold j (one bit
    // per home atom of the round), written by the half-list build
    uint32_t *revmask = nullptr;
    BoxState *box = nullptr;
    int32_t *scan_tmp = nullptr;
    // adjoint (allocated on first use): full tables and their gradients
    // (6 * (nlookup+1) each), then rho, F', mu, nu and dL/dF (7 * nm)
    double *adj = nullptr;
    size_t adj_cap = 0;
};

// Arguments of the table adjoint: the full tables (device) and dL/dE, dL/dsigma.
struct AdjointArgs {
    int nm, ivol, n, nnbrs;   // nnbrs: the half list's row stride
    const double *vee, *dvee, *phi, *dphi, *emb, *demb;
    double rmin, rmax, r_reciprange, r_recipstep;
    double emin, emax, e_reciprange, e_recipstep;
    double recipn;
    double gs[9], gE;
};

constexpr double kMidSkin = 0.3;       // default r_mid - table cut (A); r_mid is at most rnear
constexpr double kOutSkin = 1.0;       // default r_out - table cut (A); r_out is at most rnear

// Host-side table data (potential_m / lookup_m).
struct HostTables {
    bool set = false;
    int nlookup = 0;
    std::vector<double> vee, dvee, phi, dphi, emb, demb;
    double rmin = 0, rmax = 6, rhomin = 0, rhomax = 10000;
    bool fetm = false;      // FETRANSMETAL analytic data available
    bool exact = false;     // evaluate analytically
    int nv = 0, np = 0;
    double av[8] = {0}, rv[8] = {0}, ap[8] = {0}, rp[8] = {0};
    double bier_cut1 = 0, bier_cut2 = 0, sc[4] = {0, 0, 0, 0};
    double phi_cut1 = 0, phi_cut2 = 0, bier_a = 0, bier_zed = 0;
};

// Kernel families timed by the optional per-kernel CUDA-event profiler.
enum KernelId {
    K_DRIFT = 0, K_LINKUP, K_RELINK, K_NLIST, K_DENSITY, K_SCREEN, K_PAIR, K_FINALIZE,
    K_MID, K_THERM, K_THERM_FIN, K_ENERGY, K_MDINIT, K_ADJOINT, K_SCALEV, K_RDF, K_COUNT
};
extern const char *const kKernelNames[K_COUNT];

// Counts launches per kernel family; when enabled, brackets each launch with
// CUDA events on the engine's stream and accumulates the elapsed times.
struct Profiler {
    bool on = false;
    long long launches[K_COUNT] = {0};
    double total_ms[K_COUNT] = {0};
    std::vector<cudaEvent_t> pool;
    struct Pending { int id; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    int open_id = -1;
    cudaEvent_t open_ev = nullptr;
    cudaEvent_t get();
    void begin(int id, cudaStream_t s);
    void end(int id, cudaStream_t s);
    void harvest();          // after a stream synchronisation
    void reset();
    ~Profiler();
};

class Engine {
  public:
    explicit Engine(const moldy_params &p);
    ~Engine();

    int set_fetm(int nv, const double *av, const double *rv, int np, const double *ap,
                 const double *rp, int uselookup, int nlookup);
    int set_iron_carbon(int nlookup);
    int set_tables(int nlookup, double rmin, double rmax, double rhomin, double rhomax,
                   const double *vee, const double *dvee, const double *phi, const double *dphi,
                   const double *emb, const double *demb);
    int get_tables(double *vee, double *dvee, double *phi, double *dphi, double *emb, double *demb);
    int set_state(const double *x0, const double *y0, const double *z0, const double *x1,
                  const double *y1, const double *z1, const double *x2, const double *y2,
                  const double *z2, const double *b0, const double *b1, const double *b2,
                  const int32_t *zn, const double *mass, const double *del2, const double *tgid);
    int get_state(double *x0, double *y0, double *z0, double *x1, double *y1, double *z1,
                  double *x2, double *y2, double *z2, double *b0, double *b1, double *b2,
                  double *tgid);
    int get_array3(const double *dev, double *a, double *b, double *c);
    int get_density(double *rho, double *afrho, double *dafrho);
    int linkup();
    int relink();
    int get_linkcells(int32_t *l0, int32_t *link, int32_t *ic);
    int update_neighbourlist();
    int get_neighbourlist(int32_t *nlist, int32_t *numn, bool reverse = false);
    int force(moldy_force_out *out);
    int velocityverlet(moldy_force_out *out);
    int update_therm_avs(double *s123);
    int md_init(moldy_force_out *out);
    int md_steps(int nsteps, moldy_thermo *thermo);
    int energy_calc(double *en_atom);
    int synchronize();
    int table_gradients(double gE, const double *gF, const double *gS, double *const g[6]);
    // thermostat (thermostat_m): nose = 0 switches scalev off
    int set_thermostat(double nose, double rqke);
    int get_thermostat(double *out4);
    int scalev();
    // analysis_m::rdf (src/analysis_m.F90:497-760): pair histogram, then the
    // Ackland-Jones classification with the fourth-neighbour radii rn
    int rdf(int mode, int maxbin, int bpa, const int32_t *species, int nspec, uint64_t *hist, int64_t *natoms,
            int64_t *nclose);
    int ackland_jones(int mode, const int32_t *species, int nspec, const double *rn, int32_t *aj, int32_t *nn,
                      int32_t *chi);
    int knot_gradients(double gE, const double *gF, const double *gS, double *g_av, double *g_rv,
                       double *g_ap, double *g_rp);
    void set_ntc(int ntc) { ntc_ = ntc; }
    cudaStream_t &stream_ref() { return stream_; }
    Profiler prof;
    int device() const { return device_; }
    int precision() const { return precision_; }
    // kernel variant per tunable family (K_SCREEN, K_DENSITY, K_PAIR)
    int variant[K_COUNT] = {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};
    int autotune(int nsteps, double *times_ms);
    // sizes the compact, intermediate and outer rows for the pairs inside
    // rcut, r_mid and r_out at the current atom density (at least min_pair /
    // min_mid / min_out entries)
    int ensure_active_capacity(int min_pair, int min_mid = 0, int min_out = 0);
    double rmid = 0.0, rcut = 0.0;   // intermediate-list radius and table cut (A)
    double rout = 0.0;                // outer-list radius (A)
    double mid_skin = kMidSkin;       // r_mid = min(rnear, rcut + mid_skin)
    double out_skin = kOutSkin;       // r_out = min(rnear, rcut + max(out_skin, mid_skin + 0.4))
    int set_mid_skin(double skin);
    int set_out_skin(double skin);
    void set_list_radii();

    DeviceState d;
    Params prm;
    HostTables ht;
    Tables tab;

  private:
    int check_ready();
    int upload_tables();
    int force_device(bool *rebuilt);     // queue force on the stream
    int fetch_force_out(moldy_force_out *out);
    int check_flags();

    cudaStream_t stream_ = nullptr;
    int device_ = 0;
    int ntcm_ = 1, ntc_ = 0;
    int precision_ = MOLDY_PREC_FP64;
    bool state_set_ = false, cells_ready_ = false, list_ready_ = false;
    bool potential_set_ = false;
    bool forces_current_ = false;   // force outputs match the state and tables
    double host_vol_ = 0.0;         // last box volume seen on the host
    double nose_ = 0.0, rqke_ = 0.0; // scalev parameters (simparam%nose, simparam%rqke)
    double thermotimer_ = 0.0;      // time since the last scalev (the mdloop's thermotimer)
    int active_overflow_ = 0;       // largest compact row of an overflowing evaluation
    int mid_overflow_ = 0;          // largest intermediate row of an overflowing build
    int out_overflow_ = 0;          // largest outer row of an overflowing build
  public:
    int kin_blocks = 0;             // blocks whose kinetic-moment partials the last drift wrote
    bool skip_rho = false;          // the next evaluation need not store rho (an inner md_steps step)
    int therm_blocks = 0;           // > 0: the last drift took update_therm_avs, for k_mid_decide to finish
    double *therm_rec = nullptr;    // device slot for that step's thermo record (or none)
    int rec_indexed = 0;            // therm_rec is the first record; the box holds the index
  private:
    bool mid_dirty_ = true;         // the intermediate list must be rebuilt before use
  public:
    bool mid_dirty() const { return mid_dirty_; }
    void clear_mid_dirty() { mid_dirty_ = false; }
  private:
    double *part_embed_ = nullptr, *part_force_ = nullptr;   // slices of d.partials
    BoxState *host_box_ = nullptr;                            // pinned staging
    int host_box_cap_ = 0;
    double *host_rec_ = nullptr;                              // pinned thermo records
    int host_rec_cap_ = 0;
};

constexpr int kAtomThreads = 256;
constexpr int kMaxBlocks = 148 * 8;    // grid-stride kernels: 8 blocks per SM
constexpr int kPairCapMin = 24;        // least compact-row entries per atom
constexpr int kMidCapMin = 32;         // least intermediate-row entries per atom
constexpr int kOutCapMin = 48;         // least outer-row entries per atom
constexpr double kFemtosecond = 0.098227;   // the mdloop's "fs" (src/moldin.F90:132), model time units

// Grid of the streaming per-atom kernels that leave block partials (drift,
// kinetic moment, thermo sums): 4 blocks of 256 per SM, one resident wave, so
// the one-block reductions that follow read few partials.  The same for all
// of them, so the fused and the separate thermo sums agree to the bit.
int stream_blocks(int nm);

inline int grid_blocks(long long work, int threads) {
    long long nb = (work + threads - 1) / threads;
    if (nb < 1) nb = 1;
    return (int)(nb < kMaxBlocks ? nb : kMaxBlocks);
}

// Launches a step kernel with programmatic stream serialization: the GPU may
// start scheduling its blocks while the previous kernel on the stream drains
// (the kernel calls grid_dep_wait before touching any data), which hides the
// launch gap between the kernels of a step.
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), int grid, int block, cudaStream_t s, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// kernel launchers (defined in the .cu files)
void launch_linkup(DeviceState &d, const Params &p, cudaStream_t s);
void launch_relink(DeviceState &d, const Params &p, cudaStream_t s);
// scratch: ceil(n / 2048) ints for the multi-block scan (null: one block)
void launch_exclusive_scan(const int32_t *in, int32_t *out, int n, cudaStream_t s, int32_t *scratch = nullptr);
void launch_export_linkcells(const DeviceState &d, const Params &p, int32_t *l0, int32_t *link,
                             cudaStream_t s);
void launch_build_nlist(DeviceState &d, const Params &p, cudaStream_t s);
// rows (atom-major as NLIST itself, or entry-major; counts cnt) as
// NLIST(nnbrs, nm), 1-based, unused slots zero
void launch_export_nlist(const int32_t *rows, const int32_t *cnt, bool atom_major, const Params &p, int32_t *out,
                         cudaStream_t s);
constexpr int kVariants = 8;           // compiled variants per tunable pass
// store_rho false: rho is not written (no caller reads it before the next
// evaluation overwrites it: the inner steps of an md_steps call)
int launch_screen_density(DeviceState &d, const Params &p, const Tables &t, bool mixed, int variant,
                          double *partials, cudaStream_t s, bool store_rho = true);
int launch_forces(DeviceState &d, const Params &p, const Tables &t, bool mixed, int mode,
                  int variant, double *partials, cudaStream_t s);
void launch_finalize_force(DeviceState &d, const Params &p, const double *part_embed, int nblk_embed,
                           const double *part_force, int nblk_force, const double *part_kin, int nblk_kin,
                           int mode, cudaStream_t s);
// therm: also take the update_therm_avs of the step that ended with the last
// force evaluation (x1 and x2 unchanged since)
int launch_drift(DeviceState &d, const Params &p, double *kin_partials, bool therm, cudaStream_t s);
int launch_kinetic(DeviceState &d, const Params &p, double *partials, cudaStream_t s);
// therm_nblk > 0: finish the drift kernel's deferred update_therm_avs first
// rec_indexed: rec is the first thermo record and the box's rec_step says
// which one this launch writes (then advances it), for replayed steps
// half_build: the half list is rebuilt this step (the outer and intermediate
// lists are kept when the outer list provably needs nothing new from it)
void launch_mid_decide(DeviceState &d, const Params &p, double rmid, double rcut, double rout, int force,
                       int half_build, int apply_box, int therm_nblk, double *rec, cudaStream_t s,
                       int rec_indexed = 0);
void launch_set_rec_step(DeviceState &d, int step, cudaStream_t s);
// the outer list from the half list when k_mid_decide asked for it, then the
// intermediate list from the outer list when it asked for that
void launch_mid_build(DeviceState &d, const Params &p, double rmid, double rout, cudaStream_t s);
void launch_md_init_x2(DeviceState &d, const Params &p, cudaStream_t s);
// update_therm_avs with the thermo finalization in its last block; prep
// when the call does not directly follow a force evaluation
// rec: where the step's thermo record goes (kThermoRec doubles, device; may be null)
int launch_therm(DeviceState &d, const Params &p, bool prep, double *rec, cudaStream_t s);
constexpr int kThermoRec = 11;
constexpr int kRevRounds = 3;                  // rounds of 32 home atoms the reverse-row masks cover
constexpr int kRevPlanes = 14 * kRevRounds;
void launch_energy_calc(DeviceState &d, const Params &p, const Tables &t, cudaStream_t s);
void launch_scalev(DeviceState &d, const Params &p, double nose, double rqke, cudaStream_t s);
void launch_count_screened(const DeviceState &d, const Params &p, unsigned long long *out, cudaStream_t s);
size_t adjoint_smem_bytes(int nlookup);
void launch_table_adjoint(const DeviceState &d, const AdjointArgs &a, double *grads, double *scr,
                          const double *gF, cudaStream_t s);
int upload_device_tables(const HostTables &h, double4 **r4d, float4 **r4fd, double2 **e2d, float2 **e2fd,
                         void **auxd,
                         Tables &t, double *rcull_out);
int build_fetm_tables(HostTables &ht, int nv, const double *av, const double *rv, int np,
                      const double *ap, const double *rp, int uselookup, int nlookup);
int set_last_error(int code, const std::string &msg);
int build_iron_carbon_tables(HostTables &ht, int nlookup);
int fetm_knot_vjp(const HostTables &ht, const double *const g[6], double *g_av, double *g_rv,
                  double *g_ap, double *g_rp);

}  // namespace moldy
