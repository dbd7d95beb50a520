// noalloc.cu -- an EAM force evaluation that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a Fortran or C++ code whose device
// memory is owned by another allocator (an OpenACC/OpenMP-offload data region,
// a framework's caching allocator, a pool sized once at start-up), or a code
// path that must not allocate while it runs.  moldy_gpu_force_noalloc takes
// every input and output as a device pointer the caller already owns.  The
// intermediates it needs -- the density of every atom, F'(rho) and the
// per-block partial sums of the energy and virial -- live in one file-scope
// __device__ array of fixed size, so the call itself allocates nothing.
//
// The array is part of the library image: every GPU that loads the library
// holds it (4.3 MiB: 2 x 262,144 doubles plus 296 KiB of partial sums)
// until the process exits.  All calls on a device share it and it keeps the last call's contents; each call clears what must start
// at zero.  Two calls whose work overlaps on the GPU (different streams, or
// different host threads) race on the array and give wrong results.
//
// The host cannot use the array's name as a device address (on the host it
// names a stand-in object), so the first call on each device looks the
// address up with cudaGetSymbolAddress, with that device current, and caches
// it.  That first call should come before any stream capture.  The cached
// address belongs to the device's primary context: a caller that resets the
// device (cudaDeviceReset) or runs in a context of its own between calls
// would get a stale address, and is not supported.
//
// One deliberate difference from embed (src/potential_m.F90:148-169): an
// atom with rho <= 1e-40 gets F = 0 and F'(rho) = 0 here, where the reference
// skips it and keeps its F' from an earlier call.  The array's previous
// contents may belong to another system, so they are not used.
#include <mutex>

#include "engine.h"

namespace moldy {
namespace {

constexpr int kNaMaxAtoms = MOLDY_NOALLOC_MAX_ATOMS;
constexpr int kNaBlocks = 148 * 4;                 // grid of the grid-stride kernels
constexpr int kNaPartials = kPartials;             // doubles per block (block_partials stride)
constexpr int kNaTPA = 8;                          // lanes per atom in the pair passes
// layout of the scratch array (doubles): rho | dafrho | partials | status
constexpr size_t kOffRho = 0;
constexpr size_t kOffDaf = kOffRho + kNaMaxAtoms;
constexpr size_t kOffPart = kOffDaf + kNaMaxAtoms;
constexpr size_t kOffStatus = kOffPart + 2 * (size_t)kNaBlocks * kNaPartials;
constexpr size_t kScratchDoubles = kOffStatus + 8;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];
static_assert(kScratchDoubles * sizeof(double) < (5u << 20), "no-alloc scratch stays under 5 MiB");

// separate-table variants of the lookup_m interpolation (src/lookup_m.F90:307-394)
struct NaTables {
    const double *vee, *dvee, *phi, *dphi, *emb, *demb;
    int nlookup;
    double rmin, rmax, range, reciprange, recipnlkp, recipstep;
    double emin, emax, erange, ereciprange, erecipnlkp, erecipstep;
};

__device__ __forceinline__ double na_interp(const double *t, int n, double x, double xmin,
                                            double xmax, double range, double recipr,
                                            double recipn, double recips) {
    if (x >= xmax) return __ldg(&t[n]);
    int idx = (int)(((double)n * (x - xmin)) * recipr);
    idx = idx < 0 ? 0 : (idx > n - 1 ? n - 1 : idx);
    double xlow = xmin + (range * (double)idx) * recipn;
    double d = (x - xlow) * recips;
    return __ldg(&t[idx]) * (1.0 - d) + __ldg(&t[idx + 1]) * d;
}

__device__ __forceinline__ double na_r(const NaTables &t, const double *tab, double r) {
    return na_interp(tab, t.nlookup, r, t.rmin, t.rmax, t.range, t.reciprange, t.recipnlkp, t.recipstep);
}

__device__ __forceinline__ double na_rho(const NaTables &t, const double *tab, double rho) {
    return na_interp(tab, t.nlookup, rho, t.emin, t.emax, t.erange, t.ereciprange, t.erecipnlkp,
                     t.erecipstep);
}

struct NaArgs {
    int nm, nnbrs, ivol;
    const double *x0, *y0, *z0, *mass;
    const int32_t *nlist, *numn;      // NLIST(nnbrs, nm), 1-based entries
    double b0[9];
    double rcull2;
};

__device__ __forceinline__ bool na_pair(const NaArgs &a, int i, int j, double &dx, double &dy,
                                        double &dz, double &rx, double &ry, double &rz, double &r2) {
    dx = a.x0[i] - a.x0[j];
    dy = a.y0[i] - a.y0[j];
    dz = a.z0[i] - a.z0[j];
    min_image(a.ivol, dx, dy, dz);
    const double *b = a.b0;
    rx = b[0] * dx + b[3] * dy + b[6] * dz;
    ry = b[1] * dx + b[4] * dy + b[7] * dz;
    rz = b[2] * dx + b[5] * dy + b[8] * dz;
    r2 = rx * rx + ry * ry + rz * rz;
    return r2 <= a.rcull2;
}

// pass 1: rho_i and rho_j over the half list (rhoset, src/dynamics_m.F90:497-579)
__global__ void __launch_bounds__(256) k_na_density(NaArgs a, NaTables t, double *__restrict__ scratch) {
    double *rho = scratch + kOffRho;
    double *status = scratch + kOffStatus;
    constexpr int GPW = 32 / kNaTPA;
    const int l = threadIdx.x % kNaTPA, lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int base = warp * GPW; base < a.nm; base += nwarps * GPW) {
        const int g = base + lane / kNaTPA;
        const bool active = g < a.nm;
        double rho_i = 0.0;
        if (active) {
            int n = a.numn[g];
            if (n < 0 || n > a.nnbrs) {   // malformed NUMN: record it, use the clamped count
                if (l == 0) status[1] = 1.0;
                n = n < 0 ? 0 : a.nnbrs;
            }
            const int32_t *row = a.nlist + (size_t)g * a.nnbrs;
            for (int k = l; k < n; k += kNaTPA) {
                int j = row[k] - 1;
                if (j < 0 || j >= a.nm) { status[0] = 1.0; continue; }
                double dx, dy, dz, rx, ry, rz, r2;
                if (!na_pair(a, g, j, dx, dy, dz, rx, ry, rz, r2)) continue;
                double phi = na_r(t, t.phi, sqrt(r2));
                atomicAdd(&rho[j], phi);
                rho_i += phi;
            }
        }
#pragma unroll
        for (int o = kNaTPA / 2; o > 0; o >>= 1) rho_i += __shfl_xor_sync(0xffffffffu, rho_i, o);
        if (active && l == 0) atomicAdd(&rho[g], rho_i);
    }
}

// embedding (src/potential_m.F90:148-169): F'(rho) per atom, sum of F(rho)
__global__ void __launch_bounds__(256) k_na_embed(NaArgs a, NaTables t, double *__restrict__ scratch) {
    const double *rho = scratch + kOffRho;
    double *daf = scratch + kOffDaf;
    double *part = scratch + kOffPart;
    double v[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nm; i += gridDim.x * blockDim.x) {
        double r = rho[i];
        double d = 0.0;
        if (r > 1e-40) {
            v[0] += na_rho(t, t.emb, r);
            d = na_rho(t, t.demb, r);
        }
        daf[i] = d;
    }
    block_partials<1>(v, part, 0);
}

// pass 2: pair + embedding forces and the virial (src/dynamics_m.F90:235-346)
__global__ void __launch_bounds__(256)
k_na_pairs(NaArgs a, NaTables t, double *__restrict__ scratch, double *__restrict__ fx,
           double *__restrict__ fy, double *__restrict__ fz) {
    const double *daf = scratch + kOffDaf;
    double *part = scratch + kOffPart + (size_t)kNaBlocks * kNaPartials;
    double v[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) v[k] = 0.0;
    constexpr int GPW = 32 / kNaTPA;
    const int l = threadIdx.x % kNaTPA, lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int base = warp * GPW; base < a.nm; base += nwarps * GPW) {
        const int g = base + lane / kNaTPA;
        const bool active = g < a.nm;
        double fxi = 0.0, fyi = 0.0, fzi = 0.0;
        if (active) {
            int n = a.numn[g];
            n = n < 0 ? 0 : (n > a.nnbrs ? a.nnbrs : n);
            const int32_t *row = a.nlist + (size_t)g * a.nnbrs;
            const double fa = daf[g];
            const double ma = a.mass ? a.mass[g] : 1.0;
            for (int k = l; k < n; k += kNaTPA) {
                int j = row[k] - 1;
                if (j < 0 || j >= a.nm) continue;
                double dx, dy, dz, rx, ry, rz, r2;
                if (!na_pair(a, g, j, dx, dy, dz, rx, ry, rz, r2)) continue;
                double r = sqrt(r2), rr = 1.0 / r;
                double vee = na_r(t, t.vee, r), dvee = na_r(t, t.dvee, r), dphi = na_r(t, t.dphi, r);
                double fp = -dvee * rr - (dphi * fa + dphi * daf[j]) * rr;
                v[0] += vee;
                if (ma > 0.1 || (a.mass && ma + a.mass[j] > 0.1)) {
                    v[1] += dx * rx * fp; v[2] += dx * ry * fp; v[3] += dx * rz * fp;
                    v[4] += dy * rx * fp; v[5] += dy * ry * fp; v[6] += dy * rz * fp;
                    v[7] += dz * rx * fp; v[8] += dz * ry * fp; v[9] += dz * rz * fp;
                }
                double ddx = -(dx * fp), ddy = -(dy * fp), ddz = -(dz * fp);
                atomicAdd(&fx[j], ddx);
                atomicAdd(&fy[j], ddy);
                atomicAdd(&fz[j], ddz);
                fxi += ddx; fyi += ddy; fzi += ddz;
            }
        }
#pragma unroll
        for (int o = kNaTPA / 2; o > 0; o >>= 1) {
            fxi += __shfl_xor_sync(0xffffffffu, fxi, o);
            fyi += __shfl_xor_sync(0xffffffffu, fyi, o);
            fzi += __shfl_xor_sync(0xffffffffu, fzi, o);
        }
        if (active && l == 0) {
            atomicAdd(&fx[g], -fxi);
            atomicAdd(&fy[g], -fyi);
            atomicAdd(&fz[g], -fzi);
        }
    }
    block_partials<10>(v, part, 0);
}

// energy and virial into the caller's 10 doubles: pe, tp (column-major)
__global__ void __launch_bounds__(256) k_na_finalize(const double *__restrict__ scratch, int nblk,
                                                     double *__restrict__ out10) {
    __shared__ double sm[256][11];
    const double *pe = scratch + kOffPart, *pf = scratch + kOffPart + (size_t)kNaBlocks * kNaPartials;
    double acc[11];
    for (int k = 0; k < 11; ++k) acc[k] = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
        acc[0] += pe[(size_t)b * kNaPartials];
        for (int k = 0; k < 10; ++k) acc[1 + k] += pf[(size_t)b * kNaPartials + k];
    }
    for (int k = 0; k < 11; ++k) sm[threadIdx.x][k] = acc[k];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int k = 0; k < 11; ++k) sm[threadIdx.x][k] += sm[threadIdx.x + w][k];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out10[0] = sm[0][0] + sm[0][1];
        for (int k = 0; k < 9; ++k) out10[1 + k] = sm[0][2 + k];
    }
}

std::mutex g_na_mutex;
double *g_na_ptr[64] = {nullptr};

}  // namespace

int noalloc_scratch_ptr(double **out, std::string &err) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { err = std::string("cudaGetDevice: ") + cudaGetErrorString(e); return MOLDY_ERR_CUDA; }
    if (dev < 0 || dev >= 64) { err = "device ordinal above 63"; return MOLDY_ERR_INVALID; }
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return MOLDY_ERR_CUDA;
        }
        g_na_ptr[dev] = (double *)p;
    }
    *out = g_na_ptr[dev];
    return MOLDY_OK;
}

int force_noalloc(int nm, int nnbrs, int ivol, const double *x0, const double *y0, const double *z0,
                  const double *mass, const double *b0, const int32_t *nlist, const int32_t *numn,
                  int nlookup, double rmin, double rmax, double rhomin, double rhomax,
                  const double *vee, const double *dvee, const double *phi, const double *dphi,
                  const double *emb, const double *demb, double *fx, double *fy, double *fz,
                  double *energy_virial, cudaStream_t s, std::string &err) {
    if (nm < 1 || nm > kNaMaxAtoms) {
        err = "nm must be in 1.." + std::to_string(kNaMaxAtoms) + " (MOLDY_NOALLOC_MAX_ATOMS)";
        return MOLDY_ERR_CAPACITY;
    }
    if (nnbrs < 1 || nlookup < 2 || ivol < 0 || ivol > 5) { err = "bad nnbrs, nlookup or ivol"; return MOLDY_ERR_INVALID; }
    if (!x0 || !y0 || !z0 || !b0 || !nlist || !numn || !vee || !dvee || !phi || !dphi || !emb ||
        !demb || !fx || !fy || !fz || !energy_virial) {
        err = "null pointer argument";
        return MOLDY_ERR_INVALID;
    }
    if (!(rmax > rmin) || !(rhomax > rhomin)) { err = "empty table range"; return MOLDY_ERR_INVALID; }
    double *scratch = nullptr;
    int rc = noalloc_scratch_ptr(&scratch, err);
    if (rc != MOLDY_OK) return rc;

    NaArgs a;
    a.nm = nm; a.nnbrs = nnbrs; a.ivol = ivol;
    a.x0 = x0; a.y0 = y0; a.z0 = z0; a.mass = mass; a.nlist = nlist; a.numn = numn;
    for (int k = 0; k < 9; ++k) a.b0[k] = b0[k];
    a.rcull2 = 1.0e300;   // every listed pair is evaluated
    NaTables t;
    t.vee = vee; t.dvee = dvee; t.phi = phi; t.dphi = dphi; t.emb = emb; t.demb = demb;
    t.nlookup = nlookup;
    t.rmin = rmin; t.rmax = rmax; t.range = rmax - rmin;
    t.reciprange = 1.0 / t.range; t.recipnlkp = 1.0 / (double)nlookup;
    t.recipstep = (double)nlookup / t.range;
    t.emin = rhomin; t.emax = rhomax; t.erange = rhomax - rhomin;
    t.ereciprange = 1.0 / t.erange; t.erecipnlkp = 1.0 / (double)nlookup;
    t.erecipstep = (double)nlookup / t.erange;

    cudaError_t e;
    // the density and the status word start at zero; forces are accumulated
    if ((e = cudaMemsetAsync(scratch + kOffRho, 0, sizeof(double) * nm, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(scratch + kOffStatus, 0, sizeof(double) * 8, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(fx, 0, sizeof(double) * nm, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(fy, 0, sizeof(double) * nm, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(fz, 0, sizeof(double) * nm, s)) != cudaSuccess) {
        err = std::string("cudaMemsetAsync: ") + cudaGetErrorString(e);
        return MOLDY_ERR_CUDA;
    }
    k_na_density<<<kNaBlocks, 256, 0, s>>>(a, t, scratch);
    k_na_embed<<<kNaBlocks, 256, 0, s>>>(a, t, scratch);
    k_na_pairs<<<kNaBlocks, 256, 0, s>>>(a, t, scratch, fx, fy, fz);
    k_na_finalize<<<1, 256, 0, s>>>(scratch, kNaBlocks, energy_virial);
    if ((e = cudaGetLastError()) != cudaSuccess) {
        err = std::string("launch: ") + cudaGetErrorString(e);
        return MOLDY_ERR_CUDA;
    }
    double status[2] = {0.0, 0.0};
    if ((e = cudaMemcpyAsync(status, scratch + kOffStatus, 2 * sizeof(double), cudaMemcpyDeviceToHost, s)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        err = std::string("synchronize: ") + cudaGetErrorString(e);
        return MOLDY_ERR_CUDA;
    }
    if (status[1] != 0.0) {
        err = "NUMN holds a count outside 0..nnbrs (those rows were clamped)";
        return MOLDY_ERR_INVALID;
    }
    if (status[0] != 0.0) {
        err = "neighbour list holds an atom index outside 1..nm (those pairs were skipped)";
        return MOLDY_ERR_INVALID;
    }
    return MOLDY_OK;
}

}  // namespace moldy
