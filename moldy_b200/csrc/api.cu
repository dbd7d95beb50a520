// api.cu -- the Engine (host orchestration of one system on one GPU) and the
// extern "C" entry points declared in include/moldy_gpu.h.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "engine.h"

namespace moldy {

int build_fetm_tables(HostTables &ht, int nv, const double *av, const double *rv, int np,
                      const double *ap, const double *rp, int uselookup, int nlookup);

namespace {
thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    return fail(MOLDY_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
int dev_alloc(T **p, size_t n, const char *what) {
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(MOLDY_ERR_CUDA, std::string("cudaMalloc ") + what + " (" +
                                        std::to_string(n * sizeof(T)) + " bytes): " +
                                        cudaGetErrorString(e));
    }
    return MOLDY_OK;
}

#define CHECK(call)                                                       \
    do {                                                                  \
        int rc_ = (call);                                                 \
        if (rc_ != MOLDY_OK) return rc_;                                  \
    } while (0)

#define CUDA_CHECK(call, what)                                            \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) return cuda_fail(e_, what);                \
    } while (0)

__global__ void k_pack_pos(int nm, const double *__restrict__ x, const double *__restrict__ y,
                           const double *__restrict__ z, int mask, double4 *__restrict__ pos,
                           int4 *__restrict__ posq) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nm) return;
    double4 p = pos[a];
    if (mask & 1) p.x = x[a];
    if (mask & 2) p.y = y[a];
    if (mask & 4) p.z = z[a];
    pos[a] = p;
    posq[a] = make_int4(fix32(p.x), fix32(p.y), fix32(p.z), 0);
}

__global__ void k_unpack_pos(int nm, const double4 *__restrict__ pos, double *__restrict__ xyz) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nm) return;
    double4 p = pos[a];
    xyz[a] = p.x;
    xyz[nm + a] = p.y;
    xyz[2 * nm + a] = p.z;
}

}  // namespace

// ---------------------------------------------------------------- Profiler --
const char *const kKernelNames[K_COUNT] = {
    "drift", "linkup", "relink", "build_nlist", "density", "screen_density", "forces",
    "finalize_force", "mid_list", "therm", "finalize_therm", "energy_calc", "md_init_x2", "adjoint", "scalev", "rdf"};

cudaEvent_t Profiler::get() {
    if (!pool.empty()) {
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void Profiler::begin(int id, cudaStream_t s) {
    if (!on) return;
    open_id = id;
    open_ev = get();
    cudaEventRecord(open_ev, s);
}

void Profiler::end(int id, cudaStream_t s) {
    if (!on || open_id != id || !open_ev) return;
    cudaEvent_t b = get();
    cudaEventRecord(b, s);
    pending.push_back({id, open_ev, b});
    open_id = -1;
    open_ev = nullptr;
}

void Profiler::harvest() {
    for (auto &p : pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) total_ms[p.id] += ms;
        pool.push_back(p.a);
        pool.push_back(p.b);
    }
    pending.clear();
    cudaGetLastError();
}

void Profiler::reset() {
    harvest();
    for (int k = 0; k < K_COUNT; ++k) { launches[k] = 0; total_ms[k] = 0.0; }
}

Profiler::~Profiler() {
    for (auto &p : pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    for (auto e : pool) cudaEventDestroy(e);
}

// one launcher call = nk kernels of family id
#define LAUNCH(E, id, nk, s, call)          \
    do {                                    \
        (E).prof.begin((id), (s));          \
        call;                               \
        (E).prof.end((id), (s));            \
        (E).prof.launches[(id)] += (nk);    \
    } while (0)

// ------------------------------------------------------------------ Engine --
Engine::Engine(const moldy_params &p) {
    prm.rnear = p.rnear;
    prm.deltat = p.deltat;
    prm.press = p.press;
    prm.bdel2 = p.bdel2;
    prm.nm = p.nm;
    prm.nnbrs = p.nnbrs;
    prm.ivol = p.ivol;
    prm.atomstress = p.atomstress;
    prm.nlcx = p.nlcx;
    prm.nlcy = p.nlcy;
    prm.nlcz = p.nlcz;
    prm.ncell = 0;
    prm.pair_cap = kPairCapMin;
    prm.mid_cap = kMidCapMin;
    prm.out_cap = kOutCapMin;
    ntcm_ = p.ntcm;
    ntc_ = p.ntc;
    precision_ = p.precision;
    device_ = p.device;
    std::memset(&tab, 0, sizeof(tab));
}

Engine::~Engine() {
    if (device_ >= 0) cudaSetDevice(device_);
    void *bufs[] = {d.pos, d.x1, d.x2, d.f, d.rho, d.afrho, d.dafrho, d.stress, d.mass, d.del2,
                    d.znum, d.en_atom, d.ic, d.cell_start, d.cell_atoms, d.cell_pos, d.cell_count,
                    d.ic_new, d.arr_count, d.arr_start, d.arr_list, d.work, d.new_count,
                    d.new_start, d.cell_atoms2, d.nlist, d.numn, d.posq, d.posq2, d.pos2, d.alist,
                    d.pair_cnt, d.olist, d.out_cnt, d.rlist, d.numr, d.xout, d.xhalf, d.mlist, d.mid_cnt, d.xbuild, d.tab_r4, d.tab_e2,
                    d.tab_r4f, d.tab_e2f, d.tab_aux, d.partials, d.flags, d.revmask, d.box, d.scan_tmp, d.adj, d.rdf};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (host_box_) cudaFreeHost(host_box_);
    if (host_rec_) cudaFreeHost(host_rec_);
    if (d.thermo_rec) cudaFree(d.thermo_rec);
    if (stream_) cudaStreamDestroy(stream_);
}

static int alloc_cells(Engine &E) {
    Params &p = E.prm;
    DeviceState &d = E.d;
    p.ncell = p.nlcx * p.nlcy * p.nlcz;
    int nc = p.ncell;
    CHECK(dev_alloc(&d.cell_start, nc + 1, "cell_start"));
    CHECK(dev_alloc(&d.cell_count, nc, "cell_count"));
    CHECK(dev_alloc(&d.arr_count, nc, "arr_count"));
    CHECK(dev_alloc(&d.arr_start, nc + 1, "arr_start"));
    CHECK(dev_alloc(&d.new_count, nc, "new_count"));
    CHECK(dev_alloc(&d.new_start, nc + 1, "new_start"));
    if (d.scan_tmp) cudaFree(d.scan_tmp);
    d.scan_tmp = nullptr;
    CHECK(dev_alloc(&d.scan_tmp, nc / 2048 + 2, "scan blocks"));
    return MOLDY_OK;
}

static int init_engine(Engine &E, int device) {
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(MOLDY_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    if (device < 0 || device >= ndev) return fail(MOLDY_ERR_INVALID, "device ordinal out of range");
    CUDA_CHECK(cudaSetDevice(device), "cudaSetDevice");
    cudaDeviceProp prop;
    CUDA_CHECK(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    if (prop.major != 10) return fail(MOLDY_ERR_NO_DEVICE, "kernels are built for sm_100a only; device is sm_" +
                                                              std::to_string(prop.major * 10 + prop.minor));
    const Params &p = E.prm;
    DeviceState &d = E.d;
    size_t nm = (size_t)p.nm;
    CHECK(dev_alloc(&d.pos, nm, "pos"));
    CHECK(dev_alloc(&d.x1, 3 * nm, "x1"));
    CHECK(dev_alloc(&d.x2, 3 * nm, "x2"));
    CHECK(dev_alloc(&d.f, 3 * nm, "f"));
    CHECK(dev_alloc(&d.rho, nm, "rho"));
    CHECK(dev_alloc(&d.afrho, nm, "afrho"));
    CHECK(dev_alloc(&d.dafrho, nm, "dafrho"));
    CHECK(dev_alloc(&d.stress, 3 * nm, "stress"));
    CHECK(dev_alloc(&d.mass, nm, "mass"));
    CHECK(dev_alloc(&d.del2, nm, "del2"));
    CHECK(dev_alloc(&d.znum, nm, "atomic_number"));
    CHECK(dev_alloc(&d.en_atom, 3 * nm, "en_atom/staging"));
    CHECK(dev_alloc(&d.ic, nm, "ic"));
    CHECK(dev_alloc(&d.cell_atoms, nm, "cell_atoms"));
    CHECK(dev_alloc(&d.cell_pos, nm, "cell_pos"));
    CHECK(dev_alloc(&d.ic_new, nm, "ic_new"));
    CHECK(dev_alloc(&d.arr_list, nm, "arr_list"));
    CHECK(dev_alloc(&d.work, 2 * nm, "relink work"));
    CHECK(dev_alloc(&d.cell_atoms2, nm, "cell_atoms2"));
    CHECK(dev_alloc(&d.nlist, nm * (size_t)p.nnbrs, "nlist"));
    CHECK(dev_alloc(&d.numn, nm, "numn"));
    CHECK(dev_alloc(&d.posq, nm, "posq"));
    CHECK(dev_alloc(&d.posq2, nm, "posq2"));
    CHECK(dev_alloc(&d.pos2, nm, "pos2"));
    CHECK(dev_alloc(&d.alist, nm * (size_t)p.pair_cap, "compact list"));
    CHECK(dev_alloc(&d.pair_cnt, nm, "pair_cnt"));
    CHECK(dev_alloc(&d.olist, nm * (size_t)p.out_cap, "outer list"));
    CHECK(dev_alloc(&d.out_cnt, nm, "out_cnt"));
    CHECK(dev_alloc(&d.rlist, nm * (size_t)p.nnbrs, "reverse half rows"));
    CHECK(dev_alloc(&d.numr, nm, "numr"));
    CHECK(dev_alloc(&d.xout, nm, "xout"));
    CHECK(dev_alloc(&d.xhalf, nm, "xhalf"));
    CHECK(dev_alloc(&d.mlist, nm * (size_t)p.mid_cap, "intermediate list"));
    CHECK(dev_alloc(&d.mid_cnt, nm, "mid_cnt"));
    CHECK(dev_alloc(&d.xbuild, nm, "xbuild"));
    CHECK(dev_alloc(&d.partials, 3 * (size_t)kMaxBlocks * kPartials, "partials"));
    CHECK(dev_alloc(&d.flags, 16, "flags"));
    CHECK(dev_alloc(&d.revmask, (size_t)kRevPlanes * nm, "reverse-row masks"));
    CHECK(dev_alloc(&d.box, 1, "box"));
    CUDA_CHECK(cudaMemset(d.pos, 0, nm * sizeof(double4)), "memset pos");
    CUDA_CHECK(cudaMemset(d.x1, 0, 3 * nm * sizeof(double)), "memset x1");
    CUDA_CHECK(cudaMemset(d.x2, 0, 3 * nm * sizeof(double)), "memset x2");
    CUDA_CHECK(cudaMemset(d.f, 0, 3 * nm * sizeof(double)), "memset f");
    CUDA_CHECK(cudaMemset(d.rho, 0, nm * sizeof(double)), "memset rho");
    CUDA_CHECK(cudaMemset(d.afrho, 0, nm * sizeof(double)), "memset afrho");
    CUDA_CHECK(cudaMemset(d.dafrho, 0, nm * sizeof(double)), "memset dafrho");
    CUDA_CHECK(cudaMemset(d.stress, 0, 3 * nm * sizeof(double)), "memset stress");
    CUDA_CHECK(cudaMemset(d.numn, 0, nm * sizeof(int32_t)), "memset numn");
    CUDA_CHECK(cudaMemset(d.posq, 0, nm * sizeof(int4)), "memset posq");
    CUDA_CHECK(cudaMemset(d.posq2, 0, nm * sizeof(int4)), "memset posq2");
    CUDA_CHECK(cudaMemset(d.pos2, 0, nm * sizeof(double4)), "memset pos2");
    CUDA_CHECK(cudaMemset(d.pair_cnt, 0, nm * sizeof(int32_t)), "memset pair_cnt");
    CUDA_CHECK(cudaMemset(d.out_cnt, 0, nm * sizeof(int32_t)), "memset out_cnt");
    CUDA_CHECK(cudaMemset(d.numr, 0, nm * sizeof(int32_t)), "memset numr");
    CUDA_CHECK(cudaMemset(d.mid_cnt, 0, nm * sizeof(int32_t)), "memset mid_cnt");
    CUDA_CHECK(cudaMemset(d.xbuild, 0, nm * sizeof(int4)), "memset xbuild");
    CUDA_CHECK(cudaMemset(d.xout, 0, nm * sizeof(int4)), "memset xout");
    CUDA_CHECK(cudaMemset(d.xhalf, 0, nm * sizeof(int4)), "memset xhalf");
    CUDA_CHECK(cudaMemset(d.flags, 0, 16 * sizeof(int32_t)), "memset flags");
    CUDA_CHECK(cudaMemset(d.box, 0, sizeof(BoxState)), "memset box");
    if (p.nlcx > 0 && p.nlcy > 0 && p.nlcz > 0) CHECK(alloc_cells(E));
    return MOLDY_OK;
}

int Engine::check_ready() {
    if (!potential_set_) return fail(MOLDY_ERR_ORDER, "the potential must be set (set_up) before force evaluation");
    if (!state_set_) return fail(MOLDY_ERR_ORDER, "moldy_gpu_set_state must be called first");
    if (prm.ncell == 0) return fail(MOLDY_ERR_ORDER, "link cells undefined: give nlcx/nlcy/nlcz or B0");
    return MOLDY_OK;
}

// Device copies of the host tables (lookup_m layout): double4 r nodes up to
// the first node from which vee, dvee, phi and dphi are all zero, double2 rho
// nodes, FP32 copies of both, and the Tables descriptor.  rcull is the radius
// at and beyond which every pair contributes exactly zero (exact mode: the
// largest knot), times 1 + 1e-12; 1e150 when the tables never reach zero.
int upload_device_tables(const HostTables &h, double4 **r4d, float4 **r4fd, double2 **e2d, float2 **e2fd,
                         void **auxd,
                         Tables &t, double *rcull_out) {
    int n = h.nlookup;
    int cut = n + 1;
    for (int i = n; i >= 0; --i) {
        if (h.vee[i] != 0.0 || h.dvee[i] != 0.0 || h.phi[i] != 0.0 || h.dphi[i] != 0.0) break;
        cut = i;
    }
    int nr = (cut <= n - 1) ? cut + 2 : n + 1;
    std::vector<double4> r4(nr);
    // FP32 nodes in pairs (node k, node k+1 - node k) so that one 32-byte load
    // brings an interval and its interpolation is one fused multiply-add per
    // value (the difference is the FP32 subtraction the device would do); the
    // density table keeps (phi_k, phi_k+1 - phi_k) side by side
    std::vector<float4> r4f(2 * (size_t)nr, make_float4(0.f, 0.f, 0.f, 0.f));
    std::vector<double2> phi2(nr, make_double2(0.0, 0.0));
    std::vector<float2> phi2f(nr, make_float2(0.f, 0.f));
    for (int i = 0; i < nr; ++i) {
        r4[i] = make_double4(h.vee[i], h.dvee[i], h.phi[i], h.dphi[i]);
        const float4 q = make_float4((float)h.vee[i], (float)h.dvee[i], (float)h.phi[i], (float)h.dphi[i]);
        r4f[2 * (size_t)i] = q;
        phi2[i].x = h.phi[i];
        phi2f[i].x = (float)h.phi[i];
        if (i > 0) phi2[i - 1].y = h.phi[i];
    }
    for (int i = 0; i + 1 < nr; ++i) {
        const float4 a = r4f[2 * (size_t)i], b = r4f[2 * (size_t)i + 2];
        r4f[2 * (size_t)i + 1] = make_float4(b.x - a.x, b.y - a.y, b.z - a.z, b.w - a.w);
        phi2f[i].y = phi2f[i + 1].x - phi2f[i].x;
    }
    std::vector<double2> e2(n + 1);
    std::vector<float2> e2f(n + 1);
    for (int i = 0; i <= n; ++i) {
        e2[i] = make_double2(h.emb[i], h.demb[i]);
        e2f[i] = make_float2((float)h.emb[i], (float)h.demb[i]);
    }
    void *old[] = {*r4d, *e2d, *r4fd, *e2fd, *auxd};
    for (void *b : old)
        if (b) cudaFree(b);
    *r4d = nullptr; *e2d = nullptr; *r4fd = nullptr; *e2fd = nullptr; *auxd = nullptr;
    CHECK(dev_alloc(r4d, nr, "tables"));
    CHECK(dev_alloc(r4fd, 2 * (size_t)nr, "tables"));
    // phi2 (nr double2), then phi2f (nr float2)
    unsigned char *aux = nullptr;
    CHECK(dev_alloc(&aux, (size_t)nr * (sizeof(double2) + sizeof(float2)), "tables"));
    *auxd = aux;
    CHECK(dev_alloc(e2d, n + 1, "tables"));
    CHECK(dev_alloc(e2fd, n + 1, "tables"));
    CUDA_CHECK(cudaMemcpy(*r4d, r4.data(), nr * sizeof(double4), cudaMemcpyHostToDevice), "tables");
    CUDA_CHECK(cudaMemcpy(*r4fd, r4f.data(), 2 * (size_t)nr * sizeof(float4), cudaMemcpyHostToDevice), "tables");
    CUDA_CHECK(cudaMemcpy(aux, phi2.data(), nr * sizeof(double2), cudaMemcpyHostToDevice), "tables");
    CUDA_CHECK(cudaMemcpy(aux + nr * sizeof(double2), phi2f.data(), nr * sizeof(float2), cudaMemcpyHostToDevice),
               "tables");
    CUDA_CHECK(cudaMemcpy(*e2d, e2.data(), (n + 1) * sizeof(double2), cudaMemcpyHostToDevice), "tables");
    CUDA_CHECK(cudaMemcpy(*e2fd, e2f.data(), (n + 1) * sizeof(float2), cudaMemcpyHostToDevice), "tables");

    t.r4 = *r4d; t.e2 = *e2d; t.r4f = *r4fd; t.e2f = *e2fd;
    t.phi2 = reinterpret_cast<const double2 *>(aux);
    t.phi2f = reinterpret_cast<const float2 *>(aux + nr * sizeof(double2));
    t.nlookup = n;
    t.nr = nr;
    t.idx_cut = cut;
    t.exact = h.exact ? 1 : 0;
    t.vp_rmin = h.rmin; t.vp_rmax = h.rmax;
    t.vp_range = h.rmax - h.rmin;
    t.vp_reciprange = 1.0 / t.vp_range;
    t.vp_recipnlkp = 1.0 / (double)n;
    t.vp_recipstep = (double)n / t.vp_range;
    t.e_rmin = h.rhomin; t.e_rmax = h.rhomax;
    t.e_range = h.rhomax - h.rhomin;
    t.e_reciprange = 1.0 / t.e_range;
    t.e_recipnlkp = 1.0 / (double)n;
    t.e_recipstep = (double)n / t.e_range;
    double rcull;
    if (h.exact) {
        rcull = 0.0;
        for (int i = 0; i < h.nv; ++i) rcull = std::max(rcull, h.rv[i]);
        for (int i = 0; i < h.np; ++i) rcull = std::max(rcull, h.rp[i]);
    } else if (cut <= n - 1) {
        rcull = h.rmin + (double)cut * t.vp_range * t.vp_recipnlkp;
    } else {
        rcull = 1.0e300;
    }
    double rc = rcull < 1e150 ? rcull * (1.0 + 1.0e-12) : 1.0e150;
    t.rcull2 = rc * rc;
    t.rcull2f = (float)(rc * rc * (1.0 + 1.0e-6));
    t.recipstep_f = (float)t.vp_recipstep;
    t.xoff_f = (float)(-h.rmin * t.vp_recipstep);
    t.tail_f = r4f[2 * (size_t)(nr - 1)];
    t.nv = h.nv; t.np = h.np;
    for (int i = 0; i < 8; ++i) { t.av[i] = h.av[i]; t.rv[i] = h.rv[i]; t.ap[i] = h.ap[i]; t.rp[i] = h.rp[i]; }
    t.bier_cut1 = h.bier_cut1; t.bier_cut2 = h.bier_cut2;
    for (int k = 0; k < 4; ++k) t.sc[k] = h.sc[k];
    t.phi_cut1 = h.phi_cut1; t.phi_cut2 = h.phi_cut2;
    t.bier_a = h.bier_a; t.bier_zed = h.bier_zed;
    *rcull_out = rc;
    return MOLDY_OK;
}

int set_last_error(int code, const std::string &msg) { return fail(code, msg); }

int Engine::upload_tables() {
    double rc = 0.0;
    CHECK(upload_device_tables(ht, &d.tab_r4, &d.tab_r4f, &d.tab_e2, &d.tab_e2f, &d.tab_aux, tab, &rc));
    rcut = rc < 1e150 ? rc : prm.rnear;
    set_list_radii();
    potential_set_ = true;
    forces_current_ = false;
    return MOLDY_OK;
}

int Engine::set_fetm(int nv, const double *av, const double *rv, int np, const double *ap,
                     const double *rp, int uselookup, int nlookup) {
    if (!av || !rv || !ap || !rp) return fail(MOLDY_ERR_INVALID, "null coefficient pointer");
    int rc = build_fetm_tables(ht, nv, av, rv, np, ap, rp, uselookup, nlookup);
    if (rc != MOLDY_OK) return fail(rc, "FETRANSMETAL set-up failed (coefficient counts 1..8, phi must have a maximum in [0,3])");
    return upload_tables();
}

int Engine::set_iron_carbon(int nlookup) {
    build_iron_carbon_tables(ht, nlookup);
    return upload_tables();
}

int Engine::set_tables(int nlookup, double rmin, double rmax, double rhomin, double rhomax,
                       const double *vee, const double *dvee, const double *phi, const double *dphi,
                       const double *emb, const double *demb) {
    if (nlookup < 2) return fail(MOLDY_ERR_INVALID, "nlookup must be >= 2");
    if (!vee || !dvee || !phi || !dphi || !emb || !demb) return fail(MOLDY_ERR_INVALID, "null table pointer");
    if (!(rmax > rmin) || !(rhomax > rhomin)) return fail(MOLDY_ERR_INVALID, "empty table range");
    size_t n = (size_t)nlookup + 1;
    ht = HostTables();
    ht.nlookup = nlookup;
    ht.rmin = rmin; ht.rmax = rmax; ht.rhomin = rhomin; ht.rhomax = rhomax;
    ht.vee.assign(vee, vee + n); ht.dvee.assign(dvee, dvee + n);
    ht.phi.assign(phi, phi + n); ht.dphi.assign(dphi, dphi + n);
    ht.emb.assign(emb, emb + n); ht.demb.assign(demb, demb + n);
    ht.set = true;
    return upload_tables();
}

int Engine::get_tables(double *vee, double *dvee, double *phi, double *dphi, double *emb, double *demb) {
    if (!ht.set) return fail(MOLDY_ERR_ORDER, "no tables");
    size_t n = (size_t)ht.nlookup + 1;
    const std::vector<double> *src[] = {&ht.vee, &ht.dvee, &ht.phi, &ht.dphi, &ht.emb, &ht.demb};
    double *dst[] = {vee, dvee, phi, dphi, emb, demb};
    for (int k = 0; k < 6; ++k)
        if (dst[k]) std::memcpy(dst[k], src[k]->data(), n * sizeof(double));
    return MOLDY_OK;
}

int Engine::set_state(const double *x0, const double *y0, const double *z0, const double *x1,
                      const double *y1, const double *z1, const double *x2, const double *y2,
                      const double *z2, const double *b0, const double *b1, const double *b2,
                      const int32_t *zn, const double *mass, const double *del2, const double *tgid) {
    size_t nm = (size_t)prm.nm, nb = nm * sizeof(double);
    cudaStream_t s = stream_;
    if (x0 || y0 || z0) {
        double *tmp = d.en_atom;   // 3*nm staging
        if (x0) CUDA_CHECK(cudaMemcpyAsync(tmp, x0, nb, cudaMemcpyHostToDevice, s), "set x0");
        if (y0) CUDA_CHECK(cudaMemcpyAsync(tmp + nm, y0, nb, cudaMemcpyHostToDevice, s), "set y0");
        if (z0) CUDA_CHECK(cudaMemcpyAsync(tmp + 2 * nm, z0, nb, cudaMemcpyHostToDevice, s), "set z0");
        int mask = (x0 ? 1 : 0) | (y0 ? 2 : 0) | (z0 ? 4 : 0);
        k_pack_pos<<<(prm.nm + 255) / 256, 256, 0, s>>>(prm.nm, tmp, tmp + nm, tmp + 2 * nm, mask, d.pos,
                                                         d.posq);
    }
    const double *v1[3] = {x1, y1, z1}, *v2[3] = {x2, y2, z2};
    for (int k = 0; k < 3; ++k) {
        if (v1[k]) CUDA_CHECK(cudaMemcpyAsync(d.x1 + k * nm, v1[k], nb, cudaMemcpyHostToDevice, s), "set x1");
        if (v2[k]) CUDA_CHECK(cudaMemcpyAsync(d.x2 + k * nm, v2[k], nb, cudaMemcpyHostToDevice, s), "set x2");
    }
    if (b0) CUDA_CHECK(cudaMemcpyAsync(d.box->b0, b0, 9 * sizeof(double), cudaMemcpyHostToDevice, s), "set b0");
    if (b1) CUDA_CHECK(cudaMemcpyAsync(d.box->b1, b1, 9 * sizeof(double), cudaMemcpyHostToDevice, s), "set b1");
    if (b2) CUDA_CHECK(cudaMemcpyAsync(d.box->b2, b2, 9 * sizeof(double), cudaMemcpyHostToDevice, s), "set b2");
    if (tgid) CUDA_CHECK(cudaMemcpyAsync(d.box->tgid, tgid, 9 * sizeof(double), cudaMemcpyHostToDevice, s), "set tgid");
    if (zn) CUDA_CHECK(cudaMemcpyAsync(d.znum, zn, nm * sizeof(int32_t), cudaMemcpyHostToDevice, s), "set atomic_number");
    if (mass) CUDA_CHECK(cudaMemcpyAsync(d.mass, mass, nb, cudaMemcpyHostToDevice, s), "set atomic_mass");
    if (del2) CUDA_CHECK(cudaMemcpyAsync(d.del2, del2, nb, cudaMemcpyHostToDevice, s), "set del2");
    if (b0 && prm.ncell == 0) {
        // src/moldin.F90:252-257: diagonal elements only, at least 3 cells
        int n3[3];
        for (int k = 0; k < 3; ++k) {
            int v = (int)(b0[4 * k] / prm.rnear);
            n3[k] = v < 3 ? 3 : v;
        }
        prm.nlcx = n3[0]; prm.nlcy = n3[1]; prm.nlcz = n3[2];
        CHECK(alloc_cells(*this));
    }
    if (b0) host_vol_ = std::fabs(b0[0] * (b0[4] * b0[8] - b0[7] * b0[5]) + b0[1] * (b0[5] * b0[6] - b0[3] * b0[8]) +
                                  b0[2] * (b0[3] * b0[7] - b0[4] * b0[6]));
    if (x0 && zn && mass && del2 && b0) state_set_ = true;
    if (x0 || y0 || z0 || b0 || mass) forces_current_ = false;
    CUDA_CHECK(cudaStreamSynchronize(s), "set_state");
    return MOLDY_OK;
}

int Engine::get_state(double *x0, double *y0, double *z0, double *x1, double *y1, double *z1,
                      double *x2, double *y2, double *z2, double *b0, double *b1, double *b2,
                      double *tgid) {
    size_t nm = (size_t)prm.nm, nb = nm * sizeof(double);
    cudaStream_t s = stream_;
    if (x0 || y0 || z0) {
        double *tmp = d.en_atom;
        k_unpack_pos<<<(prm.nm + 255) / 256, 256, 0, s>>>(prm.nm, d.pos, tmp);
        if (x0) CUDA_CHECK(cudaMemcpyAsync(x0, tmp, nb, cudaMemcpyDeviceToHost, s), "get x0");
        if (y0) CUDA_CHECK(cudaMemcpyAsync(y0, tmp + nm, nb, cudaMemcpyDeviceToHost, s), "get y0");
        if (z0) CUDA_CHECK(cudaMemcpyAsync(z0, tmp + 2 * nm, nb, cudaMemcpyDeviceToHost, s), "get z0");
    }
    double *v1[3] = {x1, y1, z1}, *v2[3] = {x2, y2, z2};
    for (int k = 0; k < 3; ++k) {
        if (v1[k]) CUDA_CHECK(cudaMemcpyAsync(v1[k], d.x1 + k * nm, nb, cudaMemcpyDeviceToHost, s), "get x1");
        if (v2[k]) CUDA_CHECK(cudaMemcpyAsync(v2[k], d.x2 + k * nm, nb, cudaMemcpyDeviceToHost, s), "get x2");
    }
    if (b0) CUDA_CHECK(cudaMemcpyAsync(b0, d.box->b0, 9 * sizeof(double), cudaMemcpyDeviceToHost, s), "get b0");
    if (b1) CUDA_CHECK(cudaMemcpyAsync(b1, d.box->b1, 9 * sizeof(double), cudaMemcpyDeviceToHost, s), "get b1");
    if (b2) CUDA_CHECK(cudaMemcpyAsync(b2, d.box->b2, 9 * sizeof(double), cudaMemcpyDeviceToHost, s), "get b2");
    if (tgid) CUDA_CHECK(cudaMemcpyAsync(tgid, d.box->tgid, 9 * sizeof(double), cudaMemcpyDeviceToHost, s), "get tgid");
    CUDA_CHECK(cudaStreamSynchronize(s), "get_state");
    return MOLDY_OK;
}

int Engine::get_array3(const double *dev, double *a, double *b, double *c) {
    size_t nm = (size_t)prm.nm, nb = nm * sizeof(double);
    double *o[3] = {a, b, c};
    for (int k = 0; k < 3; ++k)
        if (o[k]) CUDA_CHECK(cudaMemcpyAsync(o[k], dev + k * nm, nb, cudaMemcpyDeviceToHost, stream_), "get array");
    CUDA_CHECK(cudaStreamSynchronize(stream_), "get array");
    return MOLDY_OK;
}

int Engine::get_density(double *rho, double *afrho, double *dafrho) {
    size_t nb = (size_t)prm.nm * sizeof(double);
    if (rho) CUDA_CHECK(cudaMemcpyAsync(rho, d.rho, nb, cudaMemcpyDeviceToHost, stream_), "get rho");
    if (afrho) CUDA_CHECK(cudaMemcpyAsync(afrho, d.afrho, nb, cudaMemcpyDeviceToHost, stream_), "get afrho");
    if (dafrho) CUDA_CHECK(cudaMemcpyAsync(dafrho, d.dafrho, nb, cudaMemcpyDeviceToHost, stream_), "get dafrho");
    CUDA_CHECK(cudaStreamSynchronize(stream_), "get density");
    return MOLDY_OK;
}

int Engine::linkup() {
    if (!state_set_) return fail(MOLDY_ERR_ORDER, "linkup before set_state");
    if (prm.ncell == 0) return fail(MOLDY_ERR_ORDER, "link cells undefined");
    LAUNCH(*this, K_LINKUP, 4, stream_, launch_linkup(d, prm, stream_));
    cells_ready_ = true;
    CUDA_CHECK(cudaGetLastError(), "linkup");
    return MOLDY_OK;
}

int Engine::relink() {
    if (!cells_ready_) return linkup();
    LAUNCH(*this, K_RELINK, 6, stream_, launch_relink(d, prm, stream_));
    CUDA_CHECK(cudaGetLastError(), "relink");
    return MOLDY_OK;
}

int Engine::get_linkcells(int32_t *l0, int32_t *link, int32_t *ic) {
    if (!cells_ready_) return fail(MOLDY_ERR_ORDER, "link cells not built");
    int32_t *dl0 = nullptr, *dlink = nullptr;
    CHECK(dev_alloc(&dl0, prm.ncell, "export"));
    int rc = dev_alloc(&dlink, prm.nm, "export");
    if (rc != MOLDY_OK) { cudaFree(dl0); return rc; }
    launch_export_linkcells(d, prm, dl0, dlink, stream_);
    std::vector<int32_t> icv(prm.nm);
    cudaMemcpyAsync(icv.data(), d.ic, prm.nm * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_);
    if (l0) cudaMemcpyAsync(l0, dl0, prm.ncell * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_);
    if (link) cudaMemcpyAsync(link, dlink, prm.nm * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_);
    cudaError_t e = cudaStreamSynchronize(stream_);
    cudaFree(dl0);
    cudaFree(dlink);
    if (e != cudaSuccess) return cuda_fail(e, "get_linkcells");
    if (ic)
        for (int a = 0; a < prm.nm; ++a) ic[a] = icv[a] + 1;
    return MOLDY_OK;
}

int Engine::check_flags() {
    int32_t f[12];
    CUDA_CHECK(cudaMemcpyAsync(f, d.flags, sizeof(f), cudaMemcpyDeviceToHost, stream_), "flags");
    int32_t st = 0;
    CUDA_CHECK(cudaMemcpyAsync(&st, &d.box->status, sizeof(st), cudaMemcpyDeviceToHost, stream_), "flags");
    CUDA_CHECK(cudaStreamSynchronize(stream_), "synchronize");
    prof.harvest();
    if (f[0]) {
        cudaMemsetAsync(d.flags, 0, sizeof(f), stream_);
        char msg[200];
        std::snprintf(msg, sizeof msg,
                      "attempt to list more than %d neighbours of atom %d: increase nnbrs "
                      "(src/neighbourlist_m.F90:222-229)", prm.nnbrs, f[2]);
        return fail(MOLDY_ERR_NEIGHBOUR_OVERFLOW, msg);
    }
    if (f[1]) {
        cudaMemsetAsync(d.flags, 0, sizeof(f), stream_);
        return fail(MOLDY_ERR_CAPACITY, "link-cell relink produced inconsistent cell counts");
    }
    if (f[10]) {
        cudaMemsetAsync(d.flags, 0, sizeof(f), stream_);
        return fail(MOLDY_ERR_NEIGHBOUR_OVERFLOW, "an atom appears in the half-list rows of " +
                                                      std::to_string(f[11]) + " atoms, more than nnbrs (" +
                                                      std::to_string(prm.nnbrs) + "): increase nnbrs");
    }
    if (f[3] || f[5] || f[8]) {
        cudaMemsetAsync(d.flags, 0, sizeof(f), stream_);
        active_overflow_ = f[3] ? f[4] : 0;
        mid_overflow_ = f[5] ? f[6] : 0;
        out_overflow_ = f[8] ? f[9] : 0;
        if (f[5] || f[8]) mid_dirty_ = true;
        if (f[8] && !f[3] && !f[5])
            return fail(MOLDY_ERR_CAPACITY, "an atom has " + std::to_string(f[9]) +
                                                " neighbours within r_out, more than the outer row holds (" +
                                                std::to_string(prm.out_cap) + ")");
        if (f[3])
            return fail(MOLDY_ERR_CAPACITY, "an atom has " + std::to_string(f[4]) +
                                                " interacting neighbours, more than the compact row holds (" +
                                                std::to_string(prm.pair_cap) + ")");
        return fail(MOLDY_ERR_CAPACITY, "an atom has " + std::to_string(f[6]) +
                                            " neighbours within r_mid, more than the intermediate row holds (" +
                                            std::to_string(prm.mid_cap) + ")");
    }
    if (st) {
        cudaMemsetAsync(&d.box->status, 0, sizeof(int32_t), stream_);
        return fail(MOLDY_ERR_SINGULAR_BOX, "matrix_invert: determinant is zero (src/matrix_m.F90:110-113)");
    }
    return MOLDY_OK;
}

int Engine::update_neighbourlist() {
    CHECK(check_ready());
    if (!cells_ready_) CHECK(linkup());
    LAUNCH(*this, K_NLIST, 1, stream_, launch_build_nlist(d, prm, stream_));
    list_ready_ = true;
    CUDA_CHECK(cudaGetLastError(), "update_neighbourlist");
    return check_flags();
}

int Engine::get_neighbourlist(int32_t *nlist, int32_t *numn, bool reverse) {
    if (!list_ready_) return fail(MOLDY_ERR_ORDER, "neighbour list not built");
    const int32_t *rows = reverse ? d.rlist : d.nlist, *cnt = reverse ? d.numr : d.numn;
    size_t ne = (size_t)prm.nm * prm.nnbrs;
    if (nlist) {
        int32_t *tmp = nullptr;
        CHECK(dev_alloc(&tmp, ne, "nlist export"));
        launch_export_nlist(rows, cnt, !reverse, prm, tmp, stream_);
        cudaError_t e = cudaMemcpyAsync(nlist, tmp, ne * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
        cudaFree(tmp);
        if (e != cudaSuccess) return cuda_fail(e, "get_neighbourlist");
    }
    if (numn) {
        CUDA_CHECK(cudaMemcpyAsync(numn, cnt, prm.nm * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_), "numn");
        CUDA_CHECK(cudaStreamSynchronize(stream_), "numn");
    }
    return MOLDY_OK;
}

// Queues dynamics_m::force; mode 0 force, 1 velocity Verlet, 2 md_init.
static int queue_force(Engine &E, int mode, int &ntc, int ntcm, bool &cells_ready, bool &list_ready,
                       bool *rebuilt, cudaStream_t s) {
    DeviceState &d = E.d;
    CHECK(E.ensure_active_capacity(0));
    const Params &p = E.prm;
    ntc = ntc + 1;
    const bool rb = (ntc == 1 || !list_ready);
    // mode 1 (velocity Verlet) advances the box here, after the drift kernel;
    // force calls outside velocity Verlet, and a first or invalidated half
    // list, always rebuild the outer and intermediate lists; a scheduled
    // half-list rebuild in velocity Verlet lets k_mid_decide keep them when
    // they need nothing from it
    const int force_mid = (mode == 1 && list_ready && !E.mid_dirty()) ? 0 : 1;
    E.clear_mid_dirty();
    LAUNCH(E, K_MID, 1, s,
           launch_mid_decide(d, p, E.rmid, E.rcut, E.rout, force_mid, rb ? 1 : 0, mode == 1 ? 1 : 0,
                             E.therm_blocks, E.therm_rec, s, E.rec_indexed));
    E.therm_blocks = 0;
    E.therm_rec = nullptr;
    if (rb) {
        if (!cells_ready) { LAUNCH(E, K_LINKUP, 4, s, launch_linkup(d, p, s)); cells_ready = true; }
        LAUNCH(E, K_NLIST, 1, s, launch_build_nlist(d, p, s));
        list_ready = true;
    }
    if (ntc == ntcm) ntc = 0;
    LAUNCH(E, K_MID, 1, s, launch_mid_build(d, p, E.rmid, E.rout, s));   // outer and intermediate builds
    const bool mixed = E.precision() == MOLDY_PREC_MIXED;
    double *pe = d.partials, *pf = d.partials + (size_t)kMaxBlocks * kPartials;
    double *pk = d.partials + 2 * (size_t)kMaxBlocks * kPartials;
    int nbe = 0, nbf = 0;
    // kinten's moment: taken by the drift kernel in velocity Verlet
    if (mode != 1) LAUNCH(E, K_DRIFT, 1, s, E.kin_blocks = launch_kinetic(d, p, pk, s));
    LAUNCH(E, K_SCREEN, 1, s,
           nbe = launch_screen_density(d, p, E.tab, mixed, E.variant[K_SCREEN], pe, s, !E.skip_rho));
    E.skip_rho = false;
    LAUNCH(E, K_PAIR, 1, s,
           nbf = launch_forces(d, p, E.tab, mixed, mode == 1 ? 1 : 0, E.variant[K_PAIR], pf, s));
    LAUNCH(E, K_FINALIZE, 1, s, launch_finalize_force(d, p, pe, nbe, pf, nbf, pk, E.kin_blocks, mode, s));
    if (rebuilt) *rebuilt = rb;
    return MOLDY_OK;
}

int Engine::force_device(bool *rebuilt) {
    return queue_force(*this, 0, ntc_, ntcm_, cells_ready_, list_ready_, rebuilt, stream_);
}

int Engine::fetch_force_out(moldy_force_out *out) {
    if (!host_box_) {
        CUDA_CHECK(cudaMallocHost((void **)&host_box_, sizeof(BoxState) * 4), "pinned staging");
        host_box_cap_ = 4;
    }
    CUDA_CHECK(cudaMemcpyAsync(host_box_, d.box, sizeof(BoxState), cudaMemcpyDeviceToHost, stream_), "box");
    CHECK(check_flags());
    CUDA_CHECK(cudaGetLastError(), "force");
    if (out) {
        const BoxState &B = host_box_[0];
        host_vol_ = B.vol;
        out->pe = B.pe;
        out->vol = B.vol;
        std::memcpy(out->tp, B.tp, sizeof(out->tp));
        std::memcpy(out->tk, B.tk, sizeof(out->tk));
        std::memcpy(out->tc, B.tc, sizeof(out->tc));
        std::memcpy(out->tg, B.tg, sizeof(out->tg));
        std::memcpy(out->tgdot, B.tgdot, sizeof(out->tgdot));
        std::memcpy(out->tgid, B.tgid, sizeof(out->tgid));
        std::memcpy(out->fb, B.fb, sizeof(out->fb));
        out->ntc = ntc_;
    }
    return MOLDY_OK;
}

int Engine::force(moldy_force_out *out) {
    CHECK(check_ready());
    const int ntc0 = ntc_;
    for (int attempt = 0;; ++attempt) {
        bool rb = false;
        active_overflow_ = 0;
        mid_overflow_ = 0;
        out_overflow_ = 0;
        CHECK(force_device(&rb));
        int rc = fetch_force_out(out);
        if (rc == MOLDY_ERR_CAPACITY && (active_overflow_ > 0 || mid_overflow_ > 0 || out_overflow_ > 0) &&
            attempt < 3) {
            // a force evaluation changes nothing but the rebuild counter and
            // the lists: grow the overflowing rows and evaluate again
            CHECK(ensure_active_capacity(active_overflow_ > 0 ? active_overflow_ + 8 : 0,
                                         mid_overflow_ > 0 ? mid_overflow_ + 16 : 0,
                                         out_overflow_ > 0 ? out_overflow_ + 16 : 0));
            ntc_ = ntc0;
            continue;
        }
        CHECK(rc);
        if (out) out->rebuilt = rb ? 1 : 0;
        forces_current_ = true;
        return MOLDY_OK;
    }
}

int Engine::ensure_active_capacity(int min_pair, int min_mid, int min_out) {
    // pairs inside a radius: (4 pi / 3) r^3 n/V, with margin for fluctuations
    auto expected = [&](double r) {
        return (4.0 * M_PI / 3.0) * r * r * r * (double)prm.nm / host_vol_;
    };
    int need_pair = std::max(kPairCapMin, min_pair), need_mid = std::max(kMidCapMin, min_mid);
    int need_out = std::max(kOutCapMin, min_out);
    if (host_vol_ > 0.0 && rcut > 0.0 && rcut < prm.rnear * 2.0) {
        need_pair = std::max(need_pair, (int)std::ceil(1.25 * expected(rcut) + 8.0));
        need_mid = std::max(need_mid, (int)std::ceil(1.25 * expected(rmid) + 16.0));
        need_out = std::max(need_out, (int)std::ceil(1.25 * expected(rout) + 16.0));
    }
    need_pair = std::min(need_pair, std::max(2 * prm.nnbrs, kPairCapMin));
    need_mid = std::min(need_mid, std::max(2 * prm.nnbrs, kMidCapMin));
    need_out = std::min(need_out, std::max(2 * prm.nnbrs, kOutCapMin));
    if (need_out > prm.out_cap) {
        if (d.olist) cudaFree(d.olist);
        d.olist = nullptr;
        CHECK(dev_alloc(&d.olist, (size_t)prm.nm * (size_t)need_out, "outer list"));
        prm.out_cap = need_out;
        mid_dirty_ = true;
    }
    if (need_pair > prm.pair_cap) {
        if (d.alist) cudaFree(d.alist);
        d.alist = nullptr;
        CHECK(dev_alloc(&d.alist, (size_t)prm.nm * (size_t)need_pair, "compact list"));
        prm.pair_cap = need_pair;
    }
    if (need_mid > prm.mid_cap) {
        if (d.mlist) cudaFree(d.mlist);
        d.mlist = nullptr;
        CHECK(dev_alloc(&d.mlist, (size_t)prm.nm * (size_t)need_mid, "intermediate list"));
        prm.mid_cap = need_mid;
        mid_dirty_ = true;
    }
    return MOLDY_OK;
}

int Engine::velocityverlet(moldy_force_out *out) {
    CHECK(check_ready());
    bool rb = false;
    LAUNCH(*this, K_DRIFT, 1, stream_,
               kin_blocks = launch_drift(d, prm, d.partials + 2 * (size_t)kMaxBlocks * kPartials, false, stream_));
    CHECK(queue_force(*this, 1, ntc_, ntcm_, cells_ready_, list_ready_, &rb, stream_));
    CHECK(fetch_force_out(out));
    if (out) out->rebuilt = rb ? 1 : 0;
    forces_current_ = true;
    return MOLDY_OK;
}

int Engine::update_therm_avs(double *s123) {
    CHECK(check_ready());
    LAUNCH(*this, K_THERM, 3, stream_, launch_therm(d, prm, true, nullptr, stream_));   // prep, sums, finish
    if (!host_box_) {
        CUDA_CHECK(cudaMallocHost((void **)&host_box_, sizeof(BoxState) * 4), "pinned staging");
        host_box_cap_ = 4;
    }
    CUDA_CHECK(cudaMemcpyAsync(host_box_, d.box, sizeof(BoxState), cudaMemcpyDeviceToHost, stream_), "box");
    CHECK(check_flags());
    if (s123) { s123[0] = host_box_[0].s1; s123[1] = host_box_[0].s2; s123[2] = host_box_[0].s3; }
    return MOLDY_OK;
}

int Engine::md_init(moldy_force_out *out) {
    CHECK(check_ready());
    bool rb = false;
    CHECK(queue_force(*this, 2, ntc_, ntcm_, cells_ready_, list_ready_, &rb, stream_));
    LAUNCH(*this, K_MDINIT, 1, stream_, launch_md_init_x2(d, prm, stream_));
    CHECK(fetch_force_out(out));
    if (out) out->rebuilt = rb ? 1 : 0;
    forces_current_ = true;
    return MOLDY_OK;
}

int Engine::md_steps(int nsteps, moldy_thermo *thermo) {
    CHECK(check_ready());
    if (nsteps < 0) return fail(MOLDY_ERR_INVALID, "nsteps < 0");
    // per-step thermo records are written on the device and copied back once
    if (thermo && d.thermo_cap < nsteps) {
        if (d.thermo_rec) cudaFree(d.thermo_rec);
        d.thermo_rec = nullptr;
        d.thermo_cap = 0;
        CHECK(dev_alloc(&d.thermo_rec, (size_t)kThermoRec * nsteps, "thermo records"));
        d.thermo_cap = nsteps;
    }
    if (thermo && host_rec_cap_ < nsteps) {
        if (host_rec_) cudaFreeHost(host_rec_);
        host_rec_ = nullptr;
        host_rec_cap_ = 0;
        CUDA_CHECK(cudaMallocHost((void **)&host_rec_, sizeof(double) * kThermoRec * nsteps), "pinned staging");
        host_rec_cap_ = nsteps;
    }
    std::vector<int> ntcs(nsteps), rbs(nsteps);
    // update_therm_avs of step k reads x1 and x2 as step k's force evaluation
    // left them.  Unless scalev changes x1 first, or k is the last step, it is
    // deferred into the drift kernel of step k + 1, which reads both anyway,
    // and finished by the k_mid_decide that follows it.
    bool therm_pending = false;
    // An ordinary step (the thermo sums of the step before deferred into its
    // drift, no half-list build or relink, no scalev, not the last step) makes
    // the same launches with the same arguments throughout a call: it is
    // captured once into a CUDA graph and replayed.  Its k_mid_decide takes the
    // thermo record index from the box, which a one-thread kernel sets before
    // the first replay after any other step.  Not while profiling (the
    // per-launch events).
    cudaGraphExec_t step_graph = nullptr;
    bool graph_failed = prof.on || nsteps < 8, rec_synced = false;
    long long per_replay[K_COUNT] = {};
    for (int k = 0; k < nsteps; ++k) {
        bool rb = false;
        {
            // this step's scalev decision, as made below
            double tt = thermotimer_ + prm.deltat;
            bool sv = false;
            if (tt >= kFemtosecond) {
                tt = tt - kFemtosecond;
                sv = nose_ > 0.0;
            }
            const bool ordinary = therm_pending && k < nsteps - 1 && !sv && list_ready_ && cells_ready_ &&
                                  ntc_ != 0 && ntc_ + 1 != ntcm_ && !mid_dirty_;
            if (ordinary && !graph_failed && !step_graph) {
                // capture one ordinary step; the host-side state it changes is
                // put back, and advanced below for every replay
                CHECK(ensure_active_capacity(0));
                const int ntc0 = ntc_, kin0 = kin_blocks, tb0 = therm_blocks;
                double *tr0 = therm_rec;
                const bool skip0 = skip_rho, dirty0 = mid_dirty_;
                long long l0[K_COUNT];
                for (int q = 0; q < K_COUNT; ++q) l0[q] = prof.launches[q];
                cudaGraph_t g = nullptr;
                cudaError_t e = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal);
                int rc = MOLDY_OK;
                if (e == cudaSuccess) {
                    LAUNCH(*this, K_DRIFT, 1, stream_,
                           kin_blocks = launch_drift(d, prm, d.partials + 2 * (size_t)kMaxBlocks * kPartials, true,
                                                     stream_));
                    therm_blocks = kin_blocks;
                    therm_rec = thermo ? d.thermo_rec : nullptr;
                    rec_indexed = 1;
                    skip_rho = true;
                    bool rbc = false;
                    int ntc_c = ntc_;
                    bool cr = cells_ready_, lr = list_ready_;
                    rc = queue_force(*this, 1, ntc_c, ntcm_, cr, lr, &rbc, stream_);
                    e = cudaStreamEndCapture(stream_, &g);
                }
                rec_indexed = 0;
                for (int q = 0; q < K_COUNT; ++q) {
                    per_replay[q] = prof.launches[q] - l0[q];
                    prof.launches[q] = l0[q];
                }
                ntc_ = ntc0; kin_blocks = kin0; therm_blocks = tb0; therm_rec = tr0; skip_rho = skip0;
                mid_dirty_ = dirty0;
                if (rc == MOLDY_OK && e == cudaSuccess && g) e = cudaGraphInstantiate(&step_graph, g, 0);
                if (g) cudaGraphDestroy(g);
                if (rc != MOLDY_OK || e != cudaSuccess || !step_graph) {
                    cudaGetLastError();
                    if (step_graph) cudaGraphExecDestroy(step_graph);
                    step_graph = nullptr;
                    graph_failed = true;
                }
            }
            if (ordinary && step_graph) {
                if (!rec_synced) {
                    launch_set_rec_step(d, k - 1, stream_);
                    rec_synced = true;
                }
                cudaError_t e = cudaGraphLaunch(step_graph, stream_);
                if (e != cudaSuccess) {
                    cudaGraphExecDestroy(step_graph);
                    return cuda_fail(e, "md_steps graph launch");
                }
                for (int q = 0; q < K_COUNT; ++q) prof.launches[q] += per_replay[q];
                // the host-side state of the replayed step
                thermotimer_ = tt;
                ntc_ = ntc_ + 1;
                mid_dirty_ = false;
                therm_blocks = 0;
                therm_rec = nullptr;
                skip_rho = false;
                ntcs[k] = ntc_;
                rbs[k] = 0;
                therm_pending = true;
                continue;
            }
            rec_synced = false;
        }
        LAUNCH(*this, K_DRIFT, 1, stream_,
               kin_blocks = launch_drift(d, prm, d.partials + 2 * (size_t)kMaxBlocks * kPartials, therm_pending,
                                         stream_));
        if (therm_pending) {
            therm_blocks = kin_blocks;
            therm_rec = thermo ? d.thermo_rec + (size_t)kThermoRec * (k - 1) : nullptr;
        }
        // src/moldin.F90:828-835: scalev once per femtosecond of simulated time,
        // with the mdloop's own constant for one femtosecond
        thermotimer_ = thermotimer_ + prm.deltat;
        bool scalev = false;
        if (thermotimer_ >= kFemtosecond) {
            thermotimer_ = thermotimer_ - kFemtosecond;
            scalev = nose_ > 0.0;
        }
        skip_rho = k < nsteps - 1;   // rho is read only after the last step
        CHECK(queue_force(*this, 1, ntc_, ntcm_, cells_ready_, list_ready_, &rb, stream_));
        ntcs[k] = ntc_;
        rbs[k] = rb ? 1 : 0;
        therm_pending = !(scalev || k == nsteps - 1);
        if (!therm_pending)
            LAUNCH(*this, K_THERM, 2, stream_,
                   launch_therm(d, prm, false, thermo ? d.thermo_rec + (size_t)kThermoRec * k : nullptr, stream_));
        if (ntc_ == 0) LAUNCH(*this, K_RELINK, 6, stream_, launch_relink(d, prm, stream_));
        if (scalev) LAUNCH(*this, K_SCALEV, 4, stream_, launch_scalev(d, prm, nose_, rqke_, stream_));
    }
    if (step_graph) cudaGraphExecDestroy(step_graph);
    CUDA_CHECK(cudaGetLastError(), "md_steps launch");
    if (thermo && nsteps > 0)
        CUDA_CHECK(cudaMemcpyAsync(host_rec_, d.thermo_rec, sizeof(double) * kThermoRec * nsteps,
                                   cudaMemcpyDeviceToHost, stream_), "thermo");
    CHECK(check_flags());
    if (thermo) {
        for (int k = 0; k < nsteps; ++k) {
            const double *r = host_rec_ + (size_t)kThermoRec * k;
            moldy_thermo &t = thermo[k];
            t.ke = r[0]; t.pe = r[1]; t.te = r[2]; t.h = r[3]; t.th = r[4]; t.vol = r[5];
            t.s1 = r[6]; t.s2 = r[7]; t.s3 = r[8]; t.temp = r[9]; t.boxke = r[10];
            t.ntc = ntcs[k]; t.rebuilt = rbs[k];
        }
    }
    forces_current_ = true;
    return MOLDY_OK;
}

int Engine::energy_calc(double *en_atom) {
    CHECK(check_ready());
    if (!ht.fetm) return fail(MOLDY_ERR_UNSUPPORTED, "energy_calc needs the analytic pair function (FETRANSMETAL set-up)");
    if (!list_ready_) return fail(MOLDY_ERR_ORDER, "energy_calc before any force evaluation");
    LAUNCH(*this, K_ENERGY, 1, stream_, launch_energy_calc(d, prm, tab, stream_));
    if (en_atom) CUDA_CHECK(cudaMemcpyAsync(en_atom, d.en_atom, prm.nm * sizeof(double), cudaMemcpyDeviceToHost, stream_), "en_atom");
    CUDA_CHECK(cudaStreamSynchronize(stream_), "energy_calc");
    CUDA_CHECK(cudaGetLastError(), "energy_calc");
    return MOLDY_OK;
}

// Times every compiled variant of the screening, density and force passes on
// the current configuration (force passes only: positions, velocities, the
// rebuild counter and the neighbour list are left as they are) and keeps the
// fastest variant of each.  times_ms[3*kVariants] receives the mean time per
// launch of (family, variant).
int Engine::autotune(int nreps, double *times_ms) {
    CHECK(check_ready());
    if (nreps < 1) nreps = 1;
    if (!list_ready_) {
        if (!cells_ready_) CHECK(linkup());
        LAUNCH(*this, K_NLIST, 1, stream_, launch_build_nlist(d, prm, stream_));
        list_ready_ = true;
    }
    const bool mixed = precision_ == MOLDY_PREC_MIXED;
    const int fams[2] = {K_SCREEN, K_PAIR};   // density is fused into the screening pass
    LAUNCH(*this, K_MID, 1, stream_, launch_mid_decide(d, prm, rmid, rcut, rout, 1, 0, 0, 0, nullptr, stream_));
    LAUNCH(*this, K_MID, 1, stream_, launch_mid_build(d, prm, rmid, rout, stream_));
    double *pe = d.partials, *pf = d.partials + (size_t)kMaxBlocks * kPartials;
    auto passes = [&]() {
        LAUNCH(*this, K_SCREEN, 1, stream_,
               launch_screen_density(d, prm, tab, mixed, variant[K_SCREEN], pe, stream_));
        LAUNCH(*this, K_PAIR, 1, stream_,
               launch_forces(d, prm, tab, mixed, 0, variant[K_PAIR], pf, stream_));
    };
    bool was_on = prof.on;
    CUDA_CHECK(cudaStreamSynchronize(stream_), "autotune");
    prof.harvest();
    prof.on = true;
    if (times_ms)
        for (int v = 0; v < kVariants; ++v) times_ms[kVariants + v] = 0.0;
    for (int fi = 0; fi < 2; ++fi) {
        int fam = fams[fi], best = variant[fam];
        double best_ms = 1e300;
        for (int v = 0; v < kVariants; ++v) {
            variant[fam] = v;
            passes();                                  // warm-up with this variant
            CUDA_CHECK(cudaStreamSynchronize(stream_), "autotune");
            prof.harvest();
            double t0 = prof.total_ms[fam];
            for (int r = 0; r < nreps; ++r) passes();
            CUDA_CHECK(cudaStreamSynchronize(stream_), "autotune");
            prof.harvest();
            double ms = (prof.total_ms[fam] - t0) / nreps;
            if (times_ms) times_ms[(fi == 0 ? 0 : 2) * kVariants + v] = ms;
            if (ms < best_ms) { best_ms = ms; best = v; }
        }
        variant[fam] = best;
    }
    prof.on = was_on;
    CUDA_CHECK(cudaGetLastError(), "autotune");
    return check_flags();
}

// dL/d(table) for L with dL/dE = gE, dL/dF = gF (real forces, 3*nm host,
// x|y|z) and dL/dsigma = gS (column-major 3x3 host, may be NULL), at the
// state and neighbour list of the last force evaluation.
int Engine::table_gradients(double gE, const double *gF, const double *gS, double *const g[6]) {
    CHECK(check_ready());
    if (!forces_current_ || !list_ready_)
        return fail(MOLDY_ERR_ORDER, "table gradients need a force evaluation at the current state and tables");
    if (ht.exact) return fail(MOLDY_ERR_UNSUPPORTED, "table gradients need lookup mode (uselookup = 1)");
    const int n = ht.nlookup, nb = n + 1;
    const size_t smem = adjoint_smem_bytes(n);
    if (smem > 200 * 1024) return fail(MOLDY_ERR_CAPACITY, "nlookup above 12799 does not fit the shared-memory histograms");
    const size_t nm = (size_t)prm.nm, need = 12 * (size_t)nb + 7 * nm;
    if (d.adj_cap < need) {
        if (d.adj) cudaFree(d.adj);
        d.adj = nullptr;
        d.adj_cap = 0;
        CHECK(dev_alloc(&d.adj, need, "adjoint scratch"));
        d.adj_cap = need;
    }
    double *tabs = d.adj, *grads = tabs + 6 * (size_t)nb, *scr = grads + 6 * (size_t)nb, *dgF = scr + 4 * nm;
    const std::vector<double> *src[6] = {&ht.vee, &ht.dvee, &ht.phi, &ht.dphi, &ht.emb, &ht.demb};
    for (int k = 0; k < 6; ++k)
        CUDA_CHECK(cudaMemcpyAsync(tabs + k * nb, src[k]->data(), nb * sizeof(double), cudaMemcpyHostToDevice,
                                   stream_), "adjoint tables");
    if (gF) CUDA_CHECK(cudaMemcpyAsync(dgF, gF, 3 * nm * sizeof(double), cudaMemcpyHostToDevice, stream_), "dL/dF");
    else CUDA_CHECK(cudaMemsetAsync(dgF, 0, 3 * nm * sizeof(double), stream_), "dL/dF");
    AdjointArgs a;
    a.nm = prm.nm; a.ivol = prm.ivol; a.n = n; a.nnbrs = prm.nnbrs;
    a.vee = tabs; a.dvee = tabs + nb; a.phi = tabs + 2 * nb; a.dphi = tabs + 3 * nb;
    a.emb = tabs + 4 * nb; a.demb = tabs + 5 * nb;
    a.rmin = tab.vp_rmin; a.rmax = tab.vp_rmax;
    a.r_reciprange = tab.vp_reciprange; a.r_recipstep = tab.vp_recipstep;
    a.emin = tab.e_rmin; a.emax = tab.e_rmax;
    a.e_reciprange = tab.e_reciprange; a.e_recipstep = tab.e_recipstep;
    a.recipn = tab.vp_recipnlkp;
    for (int k = 0; k < 9; ++k) a.gs[k] = gS ? gS[k] : 0.0;
    a.gE = gE;
    LAUNCH(*this, K_ADJOINT, 5, stream_, launch_table_adjoint(d, a, grads, scr, dgF, stream_));
    for (int k = 0; k < 6; ++k)
        if (g[k]) CUDA_CHECK(cudaMemcpyAsync(g[k], grads + k * nb, nb * sizeof(double), cudaMemcpyDeviceToHost,
                                             stream_), "table gradients");
    CUDA_CHECK(cudaStreamSynchronize(stream_), "table gradients");
    CUDA_CHECK(cudaGetLastError(), "table gradients");
    prof.harvest();
    return MOLDY_OK;
}

// dL/d(knots) of the FETRANSMETAL Fe-Fe functions: the table gradients
// contracted with the derivative of the tables in the knot parameters.
int Engine::knot_gradients(double gE, const double *gF, const double *gS, double *g_av, double *g_rv,
                           double *g_ap, double *g_rp) {
    if (!ht.fetm) return fail(MOLDY_ERR_UNSUPPORTED, "knot gradients need the FETRANSMETAL set-up");
    const size_t nb = (size_t)ht.nlookup + 1;
    std::vector<double> buf(6 * nb);
    double *g[6];
    for (int k = 0; k < 6; ++k) g[k] = buf.data() + k * nb;
    CHECK(table_gradients(gE, gF, gS, g));
    const double *cg[6] = {g[0], g[1], g[2], g[3], g[4], g[5]};
    int rc = fetm_knot_vjp(ht, cg, g_av, g_rv, g_ap, g_rp);
    if (rc != MOLDY_OK) return fail(rc, "knot gradient contraction failed");
    return MOLDY_OK;
}

// A thinner skin shortens the intermediate rows the screening pass walks every
// step and makes their rebuilds (decided on the device) more frequent.
int Engine::set_mid_skin(double skin) {
    if (!(skin > 0.0) || !(skin <= 3.0)) return fail(MOLDY_ERR_INVALID, "skin must be in (0, 3] A");
    mid_skin = skin;
    set_list_radii();
    mid_dirty_ = true;
    return MOLDY_OK;
}

// The outer list is filtered into the intermediate list at each of its
// rebuilds and is itself rebuilt from the half list only when the
// displacements since its build could bring an unlisted pair within r_mid:
// a thicker outer skin makes those rebuilds rarer and its rows longer.
int Engine::set_out_skin(double skin) {
    if (!(skin > 0.0) || !(skin <= 3.0)) return fail(MOLDY_ERR_INVALID, "skin must be in (0, 3] A");
    out_skin = skin;
    set_list_radii();
    mid_dirty_ = true;
    return MOLDY_OK;
}

void Engine::set_list_radii() {
    if (!(rcut > 0.0)) return;
    rmid = std::min(prm.rnear, rcut + mid_skin);
    rout = std::min(prm.rnear, rcut + std::max(out_skin, mid_skin + 0.4));
}

int Engine::set_thermostat(double nose, double rqke) {
    if (!(nose >= 0.0)) return fail(MOLDY_ERR_INVALID, "nose must be >= 0");
    nose_ = nose;
    rqke_ = rqke;
    return MOLDY_OK;
}

int Engine::get_thermostat(double *out4) {
    double v[2] = {0.0, 0.0};
    CUDA_CHECK(cudaMemcpyAsync(&v[0], &d.box->snhv, sizeof(double), cudaMemcpyDeviceToHost, stream_), "snhv");
    CUDA_CHECK(cudaMemcpyAsync(&v[1], &d.box->scalev_ke, sizeof(double), cudaMemcpyDeviceToHost, stream_), "ke");
    CUDA_CHECK(cudaStreamSynchronize(stream_), "thermostat");
    out4[0] = nose_; out4[1] = rqke_; out4[2] = v[0]; out4[3] = thermotimer_;
    return MOLDY_OK;
}

// one scalev call (src/thermostat_m.F90:317-395), whatever the timer
int Engine::scalev() {
    CHECK(check_ready());
    if (nose_ > 0.0) LAUNCH(*this, K_SCALEV, 4, stream_, launch_scalev(d, prm, nose_, rqke_, stream_));
    CUDA_CHECK(cudaStreamSynchronize(stream_), "scalev");
    CUDA_CHECK(cudaGetLastError(), "scalev");
    return MOLDY_OK;
}

int Engine::synchronize() {
    CUDA_CHECK(cudaStreamSynchronize(stream_), "synchronize");
    prof.harvest();
    return MOLDY_OK;
}

}  // namespace moldy

// ================================================================ C ABI ====
using moldy::Engine;
using moldy::fail;

struct moldy_gpu {
    Engine *e;
};

#define GUARD(h)                                                                   \
    do {                                                                           \
        if (!(h) || !(h)->e) return fail(MOLDY_ERR_INVALID, "null handle");        \
        cudaSetDevice((h)->e->device());                                          \
    } while (0)

#define TRY(expr)                                                                  \
    try {                                                                          \
        return (expr);                                                             \
    } catch (const std::bad_alloc &) {                                             \
        return fail(MOLDY_ERR_CAPACITY, "host allocation failed");                 \
    } catch (...) {                                                                \
        return fail(MOLDY_ERR_INVALID, "unexpected exception");                    \
    }

namespace moldy {
int engine_create(const moldy_params *p, Engine **out);
int force_noalloc(int nm, int nnbrs, int ivol, const double *x0, const double *y0, const double *z0,
                  const double *mass, const double *b0, const int32_t *nlist, const int32_t *numn,
                  int nlookup, double rmin, double rmax, double rhomin, double rhomax,
                  const double *vee, const double *dvee, const double *phi, const double *dphi,
                  const double *emb, const double *demb, double *fx, double *fy, double *fz,
                  double *energy_virial, cudaStream_t s, std::string &err);
}

extern "C" {

const char *moldy_gpu_last_error(void) { return moldy::g_last_error.c_str(); }

const char *moldy_gpu_version(void) { return "moldy_b200 0.1 (sm_100a)"; }

int moldy_gpu_create(const moldy_params *p, moldy_gpu **out) {
    if (!p || !out) return fail(MOLDY_ERR_INVALID, "null argument");
    *out = nullptr;
    if (p->nm < 1) return fail(MOLDY_ERR_INVALID, "nm must be >= 1");
    if (p->nnbrs < 1) return fail(MOLDY_ERR_INVALID, "nnbrs must be >= 1");
    if (p->ivol < 0 || p->ivol > 5) return fail(MOLDY_ERR_INVALID, "ivol must be 0..5");
    if (p->ntcm < 1) return fail(MOLDY_ERR_INVALID, "ntcm (nbrupdate) must be >= 1");
    if (!(p->rnear > 0.0)) return fail(MOLDY_ERR_INVALID, "rnear must be > 0");
    if (!(p->deltat > 0.0)) return fail(MOLDY_ERR_INVALID, "deltat must be > 0");
    if ((p->nlcx || p->nlcy || p->nlcz) && (p->nlcx < 3 || p->nlcy < 3 || p->nlcz < 3))
        return fail(MOLDY_ERR_INVALID, "link cells must be >= 3 per direction (src/moldin.F90:255-257)");
    if (p->precision != MOLDY_PREC_FP64 && p->precision != MOLDY_PREC_MIXED)
        return fail(MOLDY_ERR_INVALID, "precision must be MOLDY_PREC_FP64 or MOLDY_PREC_MIXED");
    if ((long long)p->nm * (long long)p->nnbrs > (1LL << 40)) return fail(MOLDY_ERR_INVALID, "nm*nnbrs too large");
    Engine *e = nullptr;
    int rc;
    try {
        rc = moldy::engine_create(p, &e);
    } catch (const std::bad_alloc &) {
        return fail(MOLDY_ERR_CAPACITY, "host allocation failed");
    }
    if (rc != MOLDY_OK) return rc;
    moldy_gpu *h = new (std::nothrow) moldy_gpu;
    if (!h) { delete e; return fail(MOLDY_ERR_CAPACITY, "host allocation failed"); }
    h->e = e;
    *out = h;
    return MOLDY_OK;
}

int moldy_gpu_destroy(moldy_gpu *h) {
    if (!h) return MOLDY_OK;
    delete h->e;
    delete h;
    return MOLDY_OK;
}

int moldy_gpu_set_fetm_fe(moldy_gpu *h, int32_t nv, const double *av, const double *rv, int32_t np,
                          const double *ap, const double *rp, int32_t uselookup, int32_t nlookup) {
    GUARD(h);
    TRY(h->e->set_fetm(nv, av, rv, np, ap, rp, uselookup, nlookup));
}

int moldy_gpu_set_tables(moldy_gpu *h, int32_t nlookup, double rmin, double rmax, double rhomin,
                         double rhomax, const double *vee, const double *dvee, const double *phi,
                         const double *dphi, const double *emb, const double *demb) {
    GUARD(h);
    TRY(h->e->set_tables(nlookup, rmin, rmax, rhomin, rhomax, vee, dvee, phi, dphi, emb, demb));
}

int moldy_gpu_get_tables(moldy_gpu *h, double *vee, double *dvee, double *phi, double *dphi,
                         double *emb, double *demb) {
    GUARD(h);
    TRY(h->e->get_tables(vee, dvee, phi, dphi, emb, demb));
}

int moldy_gpu_set_state(moldy_gpu *h, const double *x0, const double *y0, const double *z0,
                        const double *x1, const double *y1, const double *z1, const double *x2,
                        const double *y2, const double *z2, const double *b0, const double *b1,
                        const double *b2, const int32_t *atomic_number, const double *atomic_mass,
                        const double *del2, const double *tgid) {
    GUARD(h);
    TRY(h->e->set_state(x0, y0, z0, x1, y1, z1, x2, y2, z2, b0, b1, b2, atomic_number, atomic_mass,
                        del2, tgid));
}

int moldy_gpu_get_state(moldy_gpu *h, double *x0, double *y0, double *z0, double *x1, double *y1,
                        double *z1, double *x2, double *y2, double *z2, double *b0, double *b1,
                        double *b2, double *tgid) {
    GUARD(h);
    TRY(h->e->get_state(x0, y0, z0, x1, y1, z1, x2, y2, z2, b0, b1, b2, tgid));
}

int moldy_gpu_get_forces(moldy_gpu *h, double *fx, double *fy, double *fz) {
    GUARD(h);
    TRY(h->e->get_array3(h->e->d.f, fx, fy, fz));
}

int moldy_gpu_get_density(moldy_gpu *h, double *rho, double *afrho, double *dafrho) {
    GUARD(h);
    TRY(h->e->get_density(rho, afrho, dafrho));
}

int moldy_gpu_get_atomstress(moldy_gpu *h, double *sx, double *sy, double *sz) {
    GUARD(h);
    TRY(h->e->get_array3(h->e->d.stress, sx, sy, sz));
}

int moldy_gpu_set_ntc(moldy_gpu *h, int32_t ntc) {
    GUARD(h);
    if (ntc < 0) return fail(MOLDY_ERR_INVALID, "ntc < 0");
    h->e->set_ntc(ntc);
    return MOLDY_OK;
}

int moldy_gpu_linkup(moldy_gpu *h) { GUARD(h); TRY(h->e->linkup()); }
int moldy_gpu_relink(moldy_gpu *h) { GUARD(h); TRY(h->e->relink()); }

int moldy_gpu_get_linkcells(moldy_gpu *h, int32_t *l0, int32_t *link, int32_t *ic) {
    GUARD(h);
    TRY(h->e->get_linkcells(l0, link, ic));
}

int moldy_gpu_update_neighbourlist(moldy_gpu *h) { GUARD(h); TRY(h->e->update_neighbourlist()); }

int moldy_gpu_get_neighbourlist(moldy_gpu *h, int32_t *nlist, int32_t *numn) {
    GUARD(h);
    TRY(h->e->get_neighbourlist(nlist, numn));
}

int moldy_gpu_get_reverse_list(moldy_gpu *h, int32_t *rlist, int32_t *numr) {
    GUARD(h);
    TRY(h->e->get_neighbourlist(rlist, numr, true));
}

int moldy_gpu_force(moldy_gpu *h, moldy_force_out *out) { GUARD(h); TRY(h->e->force(out)); }

int moldy_gpu_velocityverlet(moldy_gpu *h, moldy_force_out *out) { GUARD(h); TRY(h->e->velocityverlet(out)); }

int moldy_gpu_update_therm_avs(moldy_gpu *h, double *s123) { GUARD(h); TRY(h->e->update_therm_avs(s123)); }

int moldy_gpu_md_init(moldy_gpu *h, moldy_force_out *out) { GUARD(h); TRY(h->e->md_init(out)); }

int moldy_gpu_md_steps(moldy_gpu *h, int32_t nsteps, moldy_thermo *thermo) {
    GUARD(h);
    TRY(h->e->md_steps(nsteps, thermo));
}

int moldy_gpu_energy_calc(moldy_gpu *h, double *en_atom) { GUARD(h); TRY(h->e->energy_calc(en_atom)); }

int moldy_gpu_synchronize(moldy_gpu *h) { GUARD(h); TRY(h->e->synchronize()); }

int moldy_gpu_rdf(moldy_gpu *h, int32_t mode, int32_t maxbin, int32_t binsperangstrom, const int32_t *species,
                  int32_t nspec, uint64_t *hist, int64_t *natoms, int64_t *nclose) {
    GUARD(h);
    TRY(h->e->rdf(mode, maxbin, binsperangstrom, species, nspec, hist, natoms, nclose));
}

int moldy_gpu_ackland_jones(moldy_gpu *h, int32_t mode, const int32_t *species, int32_t nspec, const double *rn,
                            int32_t *aj, int32_t *nn, int32_t *chi) {
    GUARD(h);
    TRY(h->e->ackland_jones(mode, species, nspec, rn, aj, nn, chi));
}

int moldy_gpu_get_stream(moldy_gpu *h, void **stream) {
    GUARD(h);
    if (!stream) return fail(MOLDY_ERR_INVALID, "null argument");
    *stream = (void *)h->e->stream_ref();
    return MOLDY_OK;
}

int moldy_gpu_set_profiling(moldy_gpu *h, int32_t enable) {
    GUARD(h);
    h->e->prof.harvest();
    h->e->prof.on = enable != 0;
    return MOLDY_OK;
}

int moldy_gpu_reset_kernel_stats(moldy_gpu *h) {
    GUARD(h);
    cudaStreamSynchronize(h->e->stream_ref());
    h->e->prof.reset();
    return MOLDY_OK;
}

int moldy_gpu_kernel_stats(moldy_gpu *h, int32_t kernel, double *total_ms, int64_t *launches) {
    GUARD(h);
    if (kernel < 0 || kernel >= moldy::K_COUNT) return fail(MOLDY_ERR_INVALID, "kernel id out of range");
    cudaStreamSynchronize(h->e->stream_ref());
    h->e->prof.harvest();
    if (total_ms) *total_ms = h->e->prof.total_ms[kernel];
    if (launches) *launches = h->e->prof.launches[kernel];
    return MOLDY_OK;
}

int moldy_gpu_force_noalloc(int32_t nm, int32_t nnbrs, int32_t ivol, const double *x0,
                            const double *y0, const double *z0, const double *mass, const double *b0,
                            const int32_t *nlist, const int32_t *numn, int32_t nlookup, double rmin,
                            double rmax, double rhomin, double rhomax, const double *vee,
                            const double *dvee, const double *phi, const double *dphi,
                            const double *emb, const double *demb, double *fx, double *fy,
                            double *fz, double *energy_virial, void *stream) {
    std::string err;
    int rc = moldy::force_noalloc(nm, nnbrs, ivol, x0, y0, z0, mass, b0, nlist, numn, nlookup, rmin,
                                  rmax, rhomin, rhomax, vee, dvee, phi, dphi, emb, demb, fx, fy, fz,
                                  energy_virial, (cudaStream_t)stream, err);
    if (rc != MOLDY_OK) return fail(rc, err);
    return MOLDY_OK;
}

int moldy_gpu_autotune(moldy_gpu *h, int32_t nreps, double *times_ms, int32_t *chosen) {
    GUARD(h);
    int rc;
    try {
        rc = h->e->autotune(nreps, times_ms);
    } catch (const std::bad_alloc &) {
        return fail(MOLDY_ERR_CAPACITY, "host allocation failed");
    }
    if (rc == MOLDY_OK && chosen) {
        chosen[0] = h->e->variant[moldy::K_SCREEN];
        chosen[1] = h->e->variant[moldy::K_DENSITY];
        chosen[2] = h->e->variant[moldy::K_PAIR];
    }
    return rc;
}

int moldy_gpu_get_list_stats(moldy_gpu *h, double *out3) {
    GUARD(h);
    if (!out3) return fail(MOLDY_ERR_INVALID, "null argument");
    moldy::Engine &E = *h->e;
    double np = 0.0;
    int32_t nb = 0;
    unsigned long long ns = 0;
    cudaStream_t st = E.stream_ref();
    // the reduction scratch is idle between calls
    unsigned long long *cnt = reinterpret_cast<unsigned long long *>(E.d.partials);
    cudaError_t e = cudaMemcpyAsync(&np, &E.d.box->npairs, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&nb, &E.d.box->mid_builds, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && nb > 0) {
        moldy::launch_count_screened(E.d, E.prm, cnt, st);
        e = cudaMemcpyAsync(&ns, cnt, sizeof(ns), cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return moldy::cuda_fail(e, "get_list_stats");
    out3[0] = np;
    out3[1] = (double)nb;
    out3[2] = (double)ns;
    return MOLDY_OK;
}

int moldy_gpu_set_variants(moldy_gpu *h, int32_t screen, int32_t density, int32_t forces) {
    GUARD(h);
    int v[3] = {screen, density, forces};
    for (int k = 0; k < 3; ++k)
        if (v[k] < 0 || v[k] >= moldy::kVariants) return fail(MOLDY_ERR_INVALID, "variant out of range");
    h->e->variant[moldy::K_SCREEN] = screen;
    h->e->variant[moldy::K_DENSITY] = density;
    h->e->variant[moldy::K_PAIR] = forces;
    return MOLDY_OK;
}

int moldy_gpu_table_gradients(moldy_gpu *h, double g_energy, const double *g_force, const double *g_stress,
                              double *g_vee, double *g_dvee, double *g_phi, double *g_dphi, double *g_emb,
                              double *g_demb) {
    GUARD(h);
    double *const g[6] = {g_vee, g_dvee, g_phi, g_dphi, g_emb, g_demb};
    TRY(h->e->table_gradients(g_energy, g_force, g_stress, g));
}

int moldy_gpu_knot_gradients(moldy_gpu *h, double g_energy, const double *g_force, const double *g_stress,
                             double *g_av, double *g_rv, double *g_ap, double *g_rp) {
    GUARD(h);
    TRY(h->e->knot_gradients(g_energy, g_force, g_stress, g_av, g_rv, g_ap, g_rp));
}

int moldy_gpu_set_iron_carbon_fe(moldy_gpu *h, int32_t nlookup) {
    GUARD(h);
    TRY(h->e->set_iron_carbon(nlookup));
}

int moldy_ic_build_tables(int32_t nlookup, double *vee, double *dvee, double *phi, double *dphi, double *emb,
                          double *demb) {
    try {
        if (nlookup < 2) return fail(MOLDY_ERR_INVALID, "nlookup < 2");
        moldy::HostTables ht;
        moldy::build_iron_carbon_tables(ht, nlookup);
        double *out[6] = {vee, dvee, phi, dphi, emb, demb};
        const std::vector<double> *src[6] = {&ht.vee, &ht.dvee, &ht.phi, &ht.dphi, &ht.emb, &ht.demb};
        for (int k = 0; k < 6; ++k)
            if (out[k]) std::memcpy(out[k], src[k]->data(), src[k]->size() * sizeof(double));
        return MOLDY_OK;
    } catch (...) {
        return fail(MOLDY_ERR_CAPACITY, "host allocation failed");
    }
}

int moldy_gpu_set_mid_skin(moldy_gpu *h, double skin) {
    GUARD(h);
    TRY(h->e->set_mid_skin(skin));
}

int moldy_gpu_set_outer_skin(moldy_gpu *h, double skin) {
    GUARD(h);
    TRY(h->e->set_out_skin(skin));
}

int moldy_gpu_get_outer_builds(moldy_gpu *h, int32_t *builds) {
    GUARD(h);
    if (!builds) return fail(MOLDY_ERR_INVALID, "null argument");
    moldy::Engine &E = *h->e;
    cudaStream_t st = E.stream_ref();
    cudaError_t e = cudaMemcpyAsync(builds, &E.d.box->out_builds, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return moldy::cuda_fail(e, "get_outer_builds");
    return MOLDY_OK;
}

int moldy_gpu_set_thermostat(moldy_gpu *h, double nose, double rqke) {
    GUARD(h);
    TRY(h->e->set_thermostat(nose, rqke));
}

int moldy_gpu_get_thermostat(moldy_gpu *h, double *out4) {
    GUARD(h);
    if (!out4) return fail(MOLDY_ERR_INVALID, "null argument");
    TRY(h->e->get_thermostat(out4));
}

int moldy_gpu_scalev(moldy_gpu *h) {
    GUARD(h);
    TRY(h->e->scalev());
}

int moldy_fetm_build_tables(int32_t nv, const double *av, const double *rv, int32_t np, const double *ap,
                            const double *rp, int32_t nlookup, double *vee, double *dvee, double *phi,
                            double *dphi, double *emb, double *demb) {
    try {
        if (!av || !rv || !ap || !rp || nlookup < 2) return fail(MOLDY_ERR_INVALID, "null knots or nlookup < 2");
        moldy::HostTables ht;
        int rc = moldy::build_fetm_tables(ht, nv, av, rv, np, ap, rp, 1, nlookup);
        if (rc != MOLDY_OK) return fail(rc, "FETRANSMETAL set-up failed");
        double *out[6] = {vee, dvee, phi, dphi, emb, demb};
        const std::vector<double> *src[6] = {&ht.vee, &ht.dvee, &ht.phi, &ht.dphi, &ht.emb, &ht.demb};
        for (int k = 0; k < 6; ++k)
            if (out[k]) std::memcpy(out[k], src[k]->data(), src[k]->size() * sizeof(double));
        return MOLDY_OK;
    } catch (...) {
        return fail(MOLDY_ERR_CAPACITY, "host allocation failed");
    }
}

int moldy_fetm_knot_vjp(int32_t nv, const double *av, const double *rv, int32_t np, const double *ap,
                        const double *rp, int32_t nlookup, const double *g_vee, const double *g_dvee,
                        const double *g_phi, const double *g_dphi, const double *g_emb, const double *g_demb,
                        double *g_av, double *g_rv, double *g_ap, double *g_rp) {
    try {
        if (!av || !rv || !ap || !rp || nlookup < 2) return fail(MOLDY_ERR_INVALID, "null knots or nlookup < 2");
        moldy::HostTables ht;
        int rc = moldy::build_fetm_tables(ht, nv, av, rv, np, ap, rp, 1, nlookup);
        if (rc != MOLDY_OK) return fail(rc, "FETRANSMETAL set-up failed");
        const double *g[6] = {g_vee, g_dvee, g_phi, g_dphi, g_emb, g_demb};
        rc = moldy::fetm_knot_vjp(ht, g, g_av, g_rv, g_ap, g_rp);
        if (rc != MOLDY_OK) return fail(rc, "knot gradient contraction failed");
        return MOLDY_OK;
    } catch (...) {
        return fail(MOLDY_ERR_CAPACITY, "host allocation failed");
    }
}

const char *moldy_gpu_kernel_name(int32_t kernel) {
    if (kernel < 0 || kernel >= moldy::K_COUNT) return "";
    return moldy::kKernelNames[kernel];
}

}  // extern "C"

namespace moldy {
int engine_create(const moldy_params *p, Engine **out) {
    Engine *e = new Engine(*p);
    int rc = init_engine(*e, p->device);
    if (rc == MOLDY_OK) {
        cudaError_t ce = cudaStreamCreateWithFlags(&e->stream_ref(), cudaStreamNonBlocking);
        if (ce != cudaSuccess) rc = cuda_fail(ce, "cudaStreamCreate");
    }
    if (rc != MOLDY_OK) {
        delete e;
        return rc;
    }
    *out = e;
    return MOLDY_OK;
}
}  // namespace moldy
