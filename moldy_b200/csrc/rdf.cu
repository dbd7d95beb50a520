// rdf.cu -- radial distribution function and Ackland-Jones local structure
// (analysis_m::rdf, src/analysis_m.F90:497-760) from the device state.
//
// Histogram (analysis_m.F90:580-608).  mode 0 bins the pairs of the half
// neighbour list as it stands with rsq <= (maxbin/binsperangstrom)**2
// (integer division, as the reference writes it); mode 1 bins every pair of
// atoms, the older form of the routine that wrote the reference's shipped
// bcc-iron rdf.dat.  ibin = int(r * binsperangstrom); pairs with
// ibin > maxbin are dropped, vacancies (atomic number 0) skipped.  Every
// block keeps its histogram in shared memory (global atomics when it does not
// fit) and adds it to the global one with integer atomics, so the counts do
// not depend on scheduling.  Mode 1 bins the atoms into cells at least half
// the largest binned radius wide and walks 5 cells per direction (all cells
// of a direction with fewer than 5).
//
// Ackland-Jones (analysis_m.F90:644-757).  Each atom first collects its
// neighbours inside 1.45 rn(si,sj)^2 (the full list: its half-list row plus
// the rows that hold it, or in mode 1 every atom from a cell grid), then one
// thread per atom bins the bond angles of every neighbour pair into chi and
// assigns the class with the reference's single-precision scores.  The
// counts do not depend on the order of a neighbour list, so the lists are
// filled with atomics.  Every distance is computed with separately rounded
// products and sums, as the reference's build evaluates it.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "engine.h"

namespace moldy {
namespace {

constexpr int kRdfThreads = 256;
constexpr int kNearCap = 32;          // neighbours inside the Ackland-Jones cutoff per atom
constexpr int kMaxSpecies = 8;
constexpr int kSmemHistBytes = 48 * 1024;

// pr_get_realsep2_from_dx (src/parrinellorahman_m.F90:184-212)
__device__ __forceinline__ double sep2(const double *b, int ivol, double dx, double dy, double dz) {
    min_image(ivol, dx, dy, dz);
    double rx = __dadd_rn(__dadd_rn(__dmul_rn(b[0], dx), __dmul_rn(b[3], dy)), __dmul_rn(b[6], dz));
    double ry = __dadd_rn(__dadd_rn(__dmul_rn(b[1], dx), __dmul_rn(b[4], dy)), __dmul_rn(b[7], dz));
    double rz = __dadd_rn(__dadd_rn(__dmul_rn(b[2], dx), __dmul_rn(b[5], dy)), __dmul_rn(b[8], dz));
    return __dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz));
}

__device__ __forceinline__ double pair_sep2(const double *b, int ivol, const double4 &p, const double4 &q) {
    return sep2(b, ivol, __dsub_rn(p.x, q.x), __dsub_rn(p.y, q.y), __dsub_rn(p.z, q.z));
}

__device__ __forceinline__ int species_of(const int32_t *spec, int i) { return spec ? spec[i] : 0; }

struct HistArgs {
    const double4 *pos;
    const BoxState *box;
    const int32_t *znum, *spec;
    int nm, ivol, nspec, maxbin, bpa;
    int nnbrs;                         // mode 0: the half list's row stride
    double rsqmax;                     // mode 0 bound on rsq
    unsigned long long *hist, *natoms, *nclose;
};

template <bool SMEM>
__device__ __forceinline__ void hist_add(const HistArgs &a, unsigned int *sh, int ibin, int si, int sj) {
    const int k = (ibin * a.nspec + si) * a.nspec + sj;
    if (SMEM) atomicAdd(&sh[k], 1u);
    else atomicAdd(&a.hist[k], 1ULL);
}

// one pair (i, j) of the histogram: skip vacancies, bin r
template <bool SMEM>
__device__ __forceinline__ void bin_pair(const HistArgs &a, const double *b, unsigned int *sh, const double4 &pi,
                                         int si, int j, bool bounded, unsigned int &close) {
    if (a.znum[j] == 0) return;
    const double rsq = pair_sep2(b, a.ivol, pi, a.pos[j]);
    if (bounded && rsq > a.rsqmax) return;
    const double r = __dsqrt_rn(rsq);
    const int ibin = (int)__dmul_rn(r, (double)a.bpa);
    if (r <= 2.0) close += 1;                      // the routine's "too close" warning
    if (ibin > a.maxbin) return;
    hist_add<SMEM>(a, sh, ibin, si, species_of(a.spec, j));
}

template <bool SMEM>
__device__ void flush_hist(const HistArgs &a, unsigned int *sh, unsigned int close, unsigned int *sclose,
                           unsigned int *snat) {
    atomicAdd(sclose, close);
    __syncthreads();
    if (threadIdx.x < a.nspec && snat[threadIdx.x]) atomicAdd(&a.natoms[threadIdx.x], (unsigned long long)snat[threadIdx.x]);
    if (SMEM) {
        const int nh = (a.maxbin + 1) * a.nspec * a.nspec;
        for (int k = threadIdx.x; k < nh; k += blockDim.x)
            if (sh[k]) atomicAdd(&a.hist[k], (unsigned long long)sh[k]);
    }
    if (threadIdx.x == 0 && *sclose) atomicAdd(a.nclose, (unsigned long long)*sclose);
}

template <bool SMEM>
__device__ void init_block(const HistArgs &a, unsigned int *sh, unsigned int *sclose, double *b, unsigned int *snat) {
    if (threadIdx.x < kMaxSpecies) snat[threadIdx.x] = 0u;
    if (SMEM) {
        const int nh = (a.maxbin + 1) * a.nspec * a.nspec;
        for (int k = threadIdx.x; k < nh; k += blockDim.x) sh[k] = 0u;
    }
    if (threadIdx.x < 9) b[threadIdx.x] = a.box->b0[threadIdx.x];
    if (threadIdx.x == 0) *sclose = 0u;
    __syncthreads();
}

// mode 0: the half-list rows (src/analysis_m.F90:580-608).  The lanes of a
// warp walk their rows in step; lanes whose pairs fall in the same bin are
// grouped with __match_any_sync and one of them adds the group's count, since
// the pairs of neighbouring atoms crowd into the same few shell bins.
template <bool SMEM>
__global__ void __launch_bounds__(kRdfThreads)
k_rdf_list(HistArgs a, const int32_t *__restrict__ nlist, const int32_t *__restrict__ numn) {
    extern __shared__ unsigned int sh[];
    __shared__ double b[9];
    __shared__ unsigned int sclose, snat[kMaxSpecies];
    init_block<SMEM>(a, sh, &sclose, b, snat);
    const int lane = threadIdx.x & 31;
    unsigned int close = 0;
    // block-uniform loop: every lane takes part in every __match_any_sync
    for (int base = blockIdx.x * blockDim.x; base < a.nm; base += gridDim.x * blockDim.x) {
        const int i = base + threadIdx.x;
        const bool live = i < a.nm && a.znum[i] != 0;
        const int si = live ? species_of(a.spec, i) : 0;
        if (live) atomicAdd(&snat[si], 1u);
        const double4 pi = live ? a.pos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
        const int n = live ? numn[i] : 0;
        const int nmax = __reduce_max_sync(0xffffffffu, n);
        // four row entries gathered before they are evaluated
        for (int k0 = 0; k0 < nmax; k0 += 4) {
            int jj[4];
            double4 pp[4];
            int zz[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) jj[u] = k0 + u < n ? nlist[(size_t)i * a.nnbrs + k0 + u] : -1;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int j = jj[u] >= 0 ? jj[u] : 0;
                pp[u] = a.pos[j];
                zz[u] = a.znum[j];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (k0 + u >= nmax) break;                 // warp-uniform
                int key = -1;
                if (jj[u] >= 0 && zz[u] != 0) {
                    const double rsq = pair_sep2(b, a.ivol, pi, pp[u]);
                    if (!(rsq > a.rsqmax)) {
                        const double r = __dsqrt_rn(rsq);
                        const int ibin = (int)__dmul_rn(r, (double)a.bpa);
                        if (r <= 2.0) close += 1;
                        if (ibin <= a.maxbin) key = (ibin * a.nspec + si) * a.nspec + species_of(a.spec, jj[u]);
                    }
                }
                const unsigned int m = __match_any_sync(0xffffffffu, key);
                if (key >= 0 && lane == __ffs(m) - 1) {
                    if (SMEM) atomicAdd(&sh[key], (unsigned int)__popc(m));
                    else atomicAdd(&a.hist[key], (unsigned long long)__popc(m));
                }
            }
        }
    }
    flush_hist<SMEM>(a, sh, close, &sclose, snat);
}

// ------------------------------------------------------------ cell grid --
struct Grid {
    int nc[3], off0[3], noff[3];       // cells per direction; first stencil offset and offsets per direction
    int ncell;
    const int32_t *start, *atoms;      // cell_start[ncell + 1], atoms in cell order
};

__device__ __forceinline__ int grid_coord(double x, int n) {
    const double u = x - floor(x);
    int c = (int)(u * (double)n);
    return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

__device__ __forceinline__ int grid_cell(const Grid &g, const double4 &p) {
    return grid_coord(p.x, g.nc[0]) + g.nc[0] * (grid_coord(p.y, g.nc[1]) + g.nc[1] * grid_coord(p.z, g.nc[2]));
}

__global__ void k_grid_count(int nm, const double4 *__restrict__ pos, Grid g, int32_t *__restrict__ cell_of,
                             int32_t *__restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nm) return;
    const int c = grid_cell(g, pos[i]);
    cell_of[i] = c;
    atomicAdd(&count[c], 1);
}

__global__ void k_grid_fill(int nm, const int32_t *__restrict__ cell_of, const int32_t *__restrict__ start,
                            int32_t *__restrict__ cursor, int32_t *__restrict__ atoms) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nm) return;
    const int c = cell_of[i];
    atoms[start[c] + atomicAdd(&cursor[c], 1)] = i;
}

// visits every atom of the stencil cells around position p
template <typename F>
__device__ __forceinline__ void for_stencil(const Grid &g, const double4 &p, F &&visit) {
    const int cx = grid_coord(p.x, g.nc[0]), cy = grid_coord(p.y, g.nc[1]), cz = grid_coord(p.z, g.nc[2]);
    for (int kz = 0; kz < g.noff[2]; ++kz) {
        int iz = g.noff[2] == g.nc[2] ? kz : cz + g.off0[2] + kz;
        iz = iz < 0 ? iz + g.nc[2] : (iz >= g.nc[2] ? iz - g.nc[2] : iz);
        for (int ky = 0; ky < g.noff[1]; ++ky) {
            int iy = g.noff[1] == g.nc[1] ? ky : cy + g.off0[1] + ky;
            iy = iy < 0 ? iy + g.nc[1] : (iy >= g.nc[1] ? iy - g.nc[1] : iy);
            for (int kx = 0; kx < g.noff[0]; ++kx) {
                int ix = g.noff[0] == g.nc[0] ? kx : cx + g.off0[0] + kx;
                ix = ix < 0 ? ix + g.nc[0] : (ix >= g.nc[0] ? ix - g.nc[0] : ix);
                const int c = ix + g.nc[0] * (iy + g.nc[1] * iz);
                for (int s = g.start[c]; s < g.start[c + 1]; ++s) visit(g.atoms[s]);
            }
        }
    }
}

// mode 1: every pair j < i
template <bool SMEM>
__global__ void __launch_bounds__(kRdfThreads)
k_rdf_all(HistArgs a, Grid g) {
    extern __shared__ unsigned int sh[];
    __shared__ double b[9];
    __shared__ unsigned int sclose, snat[kMaxSpecies];
    init_block<SMEM>(a, sh, &sclose, b, snat);
    unsigned int close = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nm; i += gridDim.x * blockDim.x) {
        if (a.znum[i] == 0) continue;
        atomicAdd(&snat[species_of(a.spec, i)], 1u);
        const double4 pi = a.pos[i];
        const int si = species_of(a.spec, i);
        for_stencil(g, pi, [&](int j) {
            if (j < i) bin_pair<SMEM>(a, b, sh, pi, si, j, false, close);
        });
    }
    flush_hist<SMEM>(a, sh, close, &sclose, snat);
}

// ------------------------------------------------------- Ackland-Jones --
struct AjArgs {
    const double4 *pos;
    const BoxState *box;
    const int32_t *spec;
    int nm, ivol, nspec;
    int nnbrs;                               // mode 0: the half list's row stride
    double thr[kMaxSpecies * kMaxSpecies];   // 1.45 rn(si,sj)^2 with the single-precision 1.45
    int32_t *ncount, *near;                  // near[i * kNearCap + k]
    int32_t *flags;                          // [0]: an atom had more than kNearCap neighbours
};

__device__ __forceinline__ void near_add(const AjArgs &a, int i, int j) {
    const int k = atomicAdd(&a.ncount[i], 1);
    if (k < kNearCap) a.near[(size_t)i * kNearCap + k] = j;
    else atomicExch(&a.flags[0], 1);
}

// mode 0: the full list of analysis_m.F90:562-578 from the half-list rows
__global__ void __launch_bounds__(kRdfThreads)
k_aj_near_list(AjArgs a, const int32_t *__restrict__ nlist, const int32_t *__restrict__ numn) {
    __shared__ double b[9];
    if (threadIdx.x < 9) b[threadIdx.x] = a.box->b0[threadIdx.x];
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nm; i += gridDim.x * blockDim.x) {
        const double4 pi = a.pos[i];
        const int si = species_of(a.spec, i);
        const int n = numn[i];
        for (int k = 0; k < n; ++k) {
            const int j = nlist[(size_t)i * a.nnbrs + k];
            const int sj = species_of(a.spec, j);
            // the same rsq from either end: the image rule and the rounding are symmetric
            const double rsq = pair_sep2(b, a.ivol, pi, a.pos[j]);
            if (!(rsq > a.thr[si * a.nspec + sj])) near_add(a, i, j);
            if (!(rsq > a.thr[sj * a.nspec + si])) near_add(a, j, i);
        }
    }
}

// mode 1: every other atom from the cell grid
__global__ void __launch_bounds__(kRdfThreads)
k_aj_near_all(AjArgs a, Grid g) {
    __shared__ double b[9];
    if (threadIdx.x < 9) b[threadIdx.x] = a.box->b0[threadIdx.x];
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nm; i += gridDim.x * blockDim.x) {
        const double4 pi = a.pos[i];
        const int si = species_of(a.spec, i);
        for_stencil(g, pi, [&](int j) {
            if (j == i) return;
            const double rsq = pair_sep2(b, a.ivol, pi, a.pos[j]);
            if (!(rsq > a.thr[si * a.nspec + species_of(a.spec, j)])) near_add(a, i, j);
        });
    }
}

// the eight ctheta windows of analysis_m.F90:695-714 (-1: the unused band)
__device__ __forceinline__ int chi_bin(double ct) {
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

// analysis_m.F90:716-751 in single precision: 0 unknown, 1 bcc, 2 fcc, 3 hcp, 4 icosahedral
__device__ int aj_assign(const int *chi, int nn) {
    float bccscore = __fmul_rn(0.35f, (float)chi[4]);
    bccscore = __fdiv_rn(bccscore, (float)(chi[5] + chi[6] + chi[7] - chi[4]));
    const float fcchcp = __fdiv_rn(fabsf(__fsub_rn(24.0f, (float)chi[6])), 24.0f);
    const int t = chi[0] + chi[1] - 6;
    float fccscore = __fdiv_rn(__fmul_rn(0.61f, (float)((t < 0 ? -t : t) + chi[2])), 6.0f);
    float hcpscore = __fdiv_rn(__fadd_rn(fabsf(__fsub_rn((float)chi[0], 3.0f)),
                                         fabsf(__fsub_rn((float)(chi[0] + chi[1] + chi[2] + chi[3]), 9.0f))),
                               12.0f);
    const double icoscore = (double)chi[4];
    if (nn > 11) {
        if (chi[0] == 7) bccscore = 0.0f;
        if (chi[0] == 6) fccscore = 0.0f;
        if (chi[0] == 3) hcpscore = 0.0f;
    }
    if (chi[7] > 0) return 0;
    if (icoscore < 3.0) return nn != 12 ? 0 : 4;
    if ((double)bccscore <= (double)fcchcp) return nn < 11 ? 0 : 1;
    if (nn != 12) return 0;
    return (double)fccscore < (double)hcpscore ? 2 : 3;
}

__global__ void __launch_bounds__(kRdfThreads)
k_aj_classify(AjArgs a, int32_t *__restrict__ aj, int32_t *__restrict__ nnout, int32_t *__restrict__ chiout) {
    __shared__ double b[9];
    if (threadIdx.x < 9) b[threadIdx.x] = a.box->b0[threadIdx.x];
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nm; i += gridDim.x * blockDim.x) {
        int n = a.ncount[i];
        n = n < kNearCap ? n : kNearCap;
        int chi[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        const int32_t *nb = a.near + (size_t)i * kNearCap;
        const double4 pi = a.pos[i];
        // rsq from the centre, as the routine computes it (x0(i) - x0(j))
        double nr[kNearCap];
        for (int p = 0; p < n; ++p) nr[p] = pair_sep2(b, a.ivol, pi, a.pos[nb[p]]);
        for (int p = 0; p < n; ++p) {
            const int j = nb[p];
            const double rsqj = nr[p];
            const double4 pj = a.pos[j];
            for (int q = p + 1; q < n; ++q) {
                const int k = nb[q];
                const double rsqk = nr[q];
                const double rsq = pair_sep2(b, a.ivol, a.pos[k], pj);
                const double ct = __ddiv_rn(__ddiv_rn(__dsub_rn(__dadd_rn(rsqj, rsqk), rsq), 2.0),
                                            __dsqrt_rn(__dmul_rn(rsqj, rsqk)));
                const int c = chi_bin(ct);
                if (c >= 0) chi[c] += 1;
            }
        }
        aj[i] = aj_assign(chi, n);
        nnout[i] = n;
        if (chiout)
            for (int c = 0; c < 8; ++c) chiout[8 * (size_t)i + c] = chi[c];
    }
}

}  // namespace

// --------------------------------------------------------------- host side
namespace {

#define RCHECK(x)                                                             \
    do {                                                                      \
        int rc_ = (x);                                                        \
        if (rc_ != MOLDY_OK) return rc_;                                      \
    } while (0)
#define RCUDA(x, what)                                                        \
    do {                                                                      \
        cudaError_t e_ = (x);                                                 \
        if (e_ != cudaSuccess) {                                              \
            cudaGetLastError();                                               \
            return set_last_error(MOLDY_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
        }                                                                     \
    } while (0)

// Carves 256-byte aligned pieces out of the engine's analysis scratch.
struct Carve {
    size_t off = 0;
    char *base = nullptr;
    template <typename T>
    T *take(size_t n) {
        off = (off + 255) & ~(size_t)255;
        T *p = base ? (T *)(base + off) : nullptr;
        off += std::max<size_t>(n, 1) * sizeof(T);
        return p;
    }
};

int reserve(DeviceState &d, size_t bytes) {
    if (bytes <= d.rdf_bytes) return MOLDY_OK;
    if (d.rdf) cudaFree(d.rdf);
    d.rdf = nullptr;
    d.rdf_bytes = 0;
    cudaError_t e = cudaMalloc(&d.rdf, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        d.rdf = nullptr;
        return set_last_error(MOLDY_ERR_CUDA, std::string("cudaMalloc analysis scratch: ") + cudaGetErrorString(e));
    }
    d.rdf_bytes = bytes;
    return MOLDY_OK;
}

// Cell grid at least radius/2 wide per direction (5 cells per direction in
// the stencil, all of them where fewer); every pair inside radius must have
// one image only, so each box width must exceed 2 radius.
int grid_shape(const double *b0, double radius, Grid &g) {
    const double vol = b0[0] * (b0[4] * b0[8] - b0[7] * b0[5]) + b0[1] * (b0[5] * b0[6] - b0[3] * b0[8]) +
                       b0[2] * (b0[3] * b0[7] - b0[4] * b0[6]);
    long long ncell = 1;
    for (int d = 0; d < 3; ++d) {
        const double *p = b0 + 3 * ((d + 1) % 3), *q = b0 + 3 * ((d + 2) % 3);
        const double cx = p[1] * q[2] - p[2] * q[1], cy = p[2] * q[0] - p[0] * q[2], cz = p[0] * q[1] - p[1] * q[0];
        const double w = std::fabs(vol) / std::sqrt(cx * cx + cy * cy + cz * cz);
        if (!(w > 2.0 * radius))
            return set_last_error(MOLDY_ERR_INVALID, "box narrower than twice the largest pair distance analysed");
        int n = (int)std::floor(w / (0.5 * radius));
        n = std::max(1, std::min(n, 512));
        g.nc[d] = n;
        if (n >= 5) { g.off0[d] = -2; g.noff[d] = 5; }
        else { g.off0[d] = 0; g.noff[d] = n; }
        ncell *= n;
    }
    g.ncell = (int)ncell;
    return MOLDY_OK;
}

void grid_take(Carve &c, Grid &g, int nm, int32_t **cell_of, int32_t **count, int32_t **cursor) {
    g.start = c.take<int32_t>((size_t)g.ncell + 1);
    g.atoms = c.take<int32_t>(nm);
    *cell_of = c.take<int32_t>(nm);
    *count = c.take<int32_t>(2 * (size_t)g.ncell);
    *cursor = *count + g.ncell;
}

int grid_fill(Grid &g, int nm, const double4 *pos, int32_t *cell_of, int32_t *count, int32_t *cursor,
              cudaStream_t s) {
    RCUDA(cudaMemsetAsync(count, 0, 2 * (size_t)g.ncell * sizeof(int32_t), s), "analysis cells");
    const int nb = (nm + 255) / 256;
    k_grid_count<<<nb, 256, 0, s>>>(nm, pos, g, cell_of, count);
    launch_exclusive_scan(count, (int32_t *)g.start, g.ncell, s);
    k_grid_fill<<<nb, 256, 0, s>>>(nm, cell_of, g.start, cursor, (int32_t *)g.atoms);
    return MOLDY_OK;
}

int check_species(const int32_t *species, int nm, int nspec) {
    if (nspec < 1 || nspec > kMaxSpecies || (!species && nspec != 1))
        return set_last_error(MOLDY_ERR_INVALID, "nspec out of range (1..8; 1 without a species array)");
    if (species)
        for (int i = 0; i < nm; ++i)
            if (species[i] < 0 || species[i] >= nspec)
                return set_last_error(MOLDY_ERR_INVALID, "species index of atom " + std::to_string(i) + " out of range");
    return MOLDY_OK;
}

int host_box(const DeviceState &d, cudaStream_t s, double *b0) {
    BoxState hb;
    RCUDA(cudaMemcpyAsync(&hb, d.box, sizeof(BoxState), cudaMemcpyDeviceToHost, s), "box");
    RCUDA(cudaStreamSynchronize(s), "box");
    for (int k = 0; k < 9; ++k) b0[k] = hb.b0[k];
    return MOLDY_OK;
}

}  // namespace

int Engine::rdf(int mode, int maxbin, int bpa, const int32_t *species, int nspec, uint64_t *hist, int64_t *natoms,
                int64_t *nclose) {
    RCHECK(check_ready());
    if (mode != 0 && mode != 1) return set_last_error(MOLDY_ERR_INVALID, "rdf mode is 0 (neighbour list) or 1 (all pairs)");
    if (maxbin < 1 || maxbin > 1000000 || bpa < 1)
        return set_last_error(MOLDY_ERR_INVALID, "maxbin and binsperangstrom >= 1");
    if (!hist) return set_last_error(MOLDY_ERR_INVALID, "null histogram");
    if (mode == 0 && !list_ready_) return set_last_error(MOLDY_ERR_ORDER, "the neighbour list has not been built");
    const int nm = prm.nm;
    RCHECK(check_species(species, nm, nspec));
    cudaStream_t s = stream_;
    const size_t nh = (size_t)(maxbin + 1) * nspec * nspec;
    Grid g;
    if (mode == 1) {
        double b0[9];
        RCHECK(host_box(d, s, b0));
        RCHECK(grid_shape(b0, (double)(maxbin + 1) / (double)bpa, g));
    }
    // size the scratch, then carve it
    int32_t *cell_of = nullptr, *count = nullptr, *cursor = nullptr;
    Carve c;
    c.take<unsigned long long>(nh + nspec + 1);
    if (species) c.take<int32_t>(nm);
    if (mode == 1) grid_take(c, g, nm, &cell_of, &count, &cursor);
    RCHECK(reserve(d, c.off));
    c = Carve();
    c.base = (char *)d.rdf;
    unsigned long long *dh = c.take<unsigned long long>(nh + nspec + 1);
    int32_t *dsp = species ? c.take<int32_t>(nm) : nullptr;
    if (mode == 1) grid_take(c, g, nm, &cell_of, &count, &cursor);
    RCUDA(cudaMemsetAsync(dh, 0, (nh + nspec + 1) * sizeof(unsigned long long), s), "analysis histogram");
    if (species) RCUDA(cudaMemcpyAsync(dsp, species, nm * sizeof(int32_t), cudaMemcpyHostToDevice, s), "species");
    HistArgs a;
    a.pos = d.pos; a.box = d.box; a.znum = d.znum; a.spec = dsp;
    a.nm = nm; a.ivol = prm.ivol; a.nspec = nspec; a.maxbin = maxbin; a.bpa = bpa; a.nnbrs = prm.nnbrs;
    const int q = maxbin / bpa;
    a.rsqmax = (double)(q * q);
    a.hist = dh; a.natoms = dh + nh; a.nclose = a.natoms + nspec;
    const size_t smem = nh * sizeof(unsigned int);
    const bool use_smem = smem <= (size_t)kSmemHistBytes;
    const int nb = std::max(1, std::min((nm + kRdfThreads - 1) / kRdfThreads, 4 * 148));
    if (mode == 0) {
        if (use_smem) k_rdf_list<true><<<nb, kRdfThreads, smem, s>>>(a, d.nlist, d.numn);
        else k_rdf_list<false><<<nb, kRdfThreads, 0, s>>>(a, d.nlist, d.numn);
        prof.launches[K_RDF] += 1;
    } else {
        RCHECK(grid_fill(g, nm, d.pos, cell_of, count, cursor, s));
        if (use_smem) k_rdf_all<true><<<nb, kRdfThreads, smem, s>>>(a, g);
        else k_rdf_all<false><<<nb, kRdfThreads, 0, s>>>(a, g);
        prof.launches[K_RDF] += 4;
    }
    std::vector<unsigned long long> h(nh + nspec + 1);
    RCUDA(cudaMemcpyAsync(h.data(), dh, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s),
          "analysis histogram");
    RCUDA(cudaStreamSynchronize(s), "rdf");
    RCUDA(cudaGetLastError(), "rdf");
    for (size_t k = 0; k < nh; ++k) hist[k] = h[k];
    if (natoms)
        for (int k = 0; k < nspec; ++k) natoms[k] = (int64_t)h[nh + k];
    if (nclose) *nclose = (int64_t)h[nh + nspec];
    return MOLDY_OK;
}

int Engine::ackland_jones(int mode, const int32_t *species, int nspec, const double *rn, int32_t *aj, int32_t *nn,
                          int32_t *chi) {
    RCHECK(check_ready());
    if (mode != 0 && mode != 1) return set_last_error(MOLDY_ERR_INVALID, "mode is 0 (neighbour list) or 1 (all atoms)");
    if (!rn || !aj || !nn) return set_last_error(MOLDY_ERR_INVALID, "null argument");
    if (mode == 0 && !list_ready_) return set_last_error(MOLDY_ERR_ORDER, "the neighbour list has not been built");
    const int nm = prm.nm;
    RCHECK(check_species(species, nm, nspec));
    cudaStream_t s = stream_;
    AjArgs a;
    double rmax = 0.0;
    for (int k = 0; k < nspec * nspec; ++k) {
        if (!(rn[k] >= 0.0) || !std::isfinite(rn[k]))
            return set_last_error(MOLDY_ERR_INVALID, "rn must be finite and >= 0");
        a.thr[k] = (double)1.45f * (rn[k] * rn[k]);
        rmax = std::max(rmax, std::sqrt(a.thr[k]));
    }
    Grid g;
    if (mode == 1) {
        double b0[9];
        RCHECK(host_box(d, s, b0));
        RCHECK(grid_shape(b0, std::max(rmax, 1e-3), g));
    }
    int32_t *cell_of = nullptr, *count = nullptr, *cursor = nullptr;
    Carve c;
    c.take<int32_t>(nm);                                 // species
    c.take<int32_t>(nm);                                 // neighbour counts
    c.take<int32_t>((size_t)nm * kNearCap);              // neighbours
    c.take<int32_t>(1);                                  // flag
    c.take<int32_t>((size_t)nm * 10);                    // aj, nn, chi
    if (mode == 1) grid_take(c, g, nm, &cell_of, &count, &cursor);
    RCHECK(reserve(d, c.off));
    c = Carve();
    c.base = (char *)d.rdf;
    int32_t *dsp = c.take<int32_t>(nm);
    a.ncount = c.take<int32_t>(nm);
    a.near = c.take<int32_t>((size_t)nm * kNearCap);
    a.flags = c.take<int32_t>(1);
    int32_t *o = c.take<int32_t>((size_t)nm * 10);
    if (mode == 1) grid_take(c, g, nm, &cell_of, &count, &cursor);
    if (species) RCUDA(cudaMemcpyAsync(dsp, species, nm * sizeof(int32_t), cudaMemcpyHostToDevice, s), "species");
    RCUDA(cudaMemsetAsync(a.ncount, 0, nm * sizeof(int32_t), s), "analysis counts");
    RCUDA(cudaMemsetAsync(a.flags, 0, sizeof(int32_t), s), "analysis flag");
    a.pos = d.pos; a.box = d.box; a.spec = species ? dsp : nullptr;
    a.nm = nm; a.ivol = prm.ivol; a.nspec = nspec; a.nnbrs = prm.nnbrs;
    const int blocks = std::max(1, std::min((nm + kRdfThreads - 1) / kRdfThreads, 8 * 148));
    if (mode == 0) {
        k_aj_near_list<<<blocks, kRdfThreads, 0, s>>>(a, d.nlist, d.numn);
        prof.launches[K_RDF] += 1;
    } else {
        RCHECK(grid_fill(g, nm, d.pos, cell_of, count, cursor, s));
        k_aj_near_all<<<blocks, kRdfThreads, 0, s>>>(a, g);
        prof.launches[K_RDF] += 4;
    }
    k_aj_classify<<<blocks, kRdfThreads, 0, s>>>(a, o, o + nm, chi ? o + 2 * (size_t)nm : nullptr);
    prof.launches[K_RDF] += 1;
    int32_t flag = 0;
    RCUDA(cudaMemcpyAsync(&flag, a.flags, sizeof(int32_t), cudaMemcpyDeviceToHost, s), "analysis flag");
    RCUDA(cudaMemcpyAsync(aj, o, nm * sizeof(int32_t), cudaMemcpyDeviceToHost, s), "classes");
    RCUDA(cudaMemcpyAsync(nn, o + nm, nm * sizeof(int32_t), cudaMemcpyDeviceToHost, s), "coordination");
    if (chi)
        RCUDA(cudaMemcpyAsync(chi, o + 2 * (size_t)nm, 8 * (size_t)nm * sizeof(int32_t), cudaMemcpyDeviceToHost, s),
              "angle counts");
    RCUDA(cudaStreamSynchronize(s), "ackland_jones");
    RCUDA(cudaGetLastError(), "ackland_jones");
    if (flag)
        return set_last_error(MOLDY_ERR_CAPACITY, "an atom has more than " + std::to_string(kNearCap) +
                                                      " neighbours inside the Ackland-Jones cutoff");
    return MOLDY_OK;
}

}  // namespace moldy
