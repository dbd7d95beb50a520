// batch.cu -- many independent supercells of uneven size in one set of
// launches: energy, forces and virial by neighbour-cell tiles, and the device
// conjugate-gradient quench.  No counterpart in the reference's API; each
// system's results are those of force() + energy_calc()
// (src/dynamics_m.F90:135-483) and its quench is quench()/VA14CD/derivs
// (src/quench_m.F90:100-551) at a fixed box.
//
// Layout.  Atoms of all systems are concatenated, each system's in the
// reference's order, and system s owns the slots [atom0, atom0 + nm) of the
// cell order too, so one system's list can be rebuilt without moving another
// system's.  A system's cells are at least its list radius rv = rc + skin wide
// (perpendicular to the cell faces).
//
// Lists.  One block per system checks the largest displacement since the
// system's last build; past half the skin (or after a box change) the same
// block bins, scans, fills and sorts the system's cells, and every evaluated
// system copies its positions into cell order.  For a rebuilt system one warp
// per cell stages the 27 (fewer for grids under 3 cells) surrounding cells in
// shared memory and writes each home atom's compact row of the candidates
// inside rv.  The density and force passes run one thread per atom over its
// row and keep the pairs inside rc.  Each pair is evaluated from both ends, so
// there are no atomics and every sum has a fixed order.
//
// Tables.  The batch always runs in lookup mode (uselookup = .true.): the
// passes interpolate the tables directly; energy_calc's exact pair function
// is the one analytic evaluation.
//
// Pairs.  The reference sums over its Verlet list (pairs within rnear at the
// last rebuild); every pair beyond the table cut contributes exactly zero, so
// a complete set of the pairs inside the cut gives the same sums.  A pair
// inside rc now was inside rv at the last build while no atom has moved more
// than half the skin since.
//
// The quench keeps VA14CD's state per system in device memory.  One block per
// system runs the state machine between function evaluations; a round is the
// list check, the tile passes and one control launch, captured once in a
// CUDA graph and replayed until every system has finished.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"

namespace moldy {
namespace {

constexpr int kTileWarps = 4;     // cells (warps) per block
constexpr int kTileCap = 256;     // staged candidates per warp
constexpr int kCgThreads = 512;   // control block
constexpr int kPrepThreads = 256; // list check and binning block

struct BSys {
    int atom0, nm, cell0, ncell;
    int nc[3], nst[3];            // cells per dimension; stencil offsets per dimension (1, 2 or 3)
    int active;                   // evaluated in the next round
    int rebuild;                  // list rebuilt in this evaluation (set by k_prepare)
    int stale;                    // list invalid: rebuild at the next evaluation
    int pad;
    double b0[9], tg[9], vol;
    double rv2;                   // squared list radius
    double hs2;                   // squared half skin: rebuild once an atom moved farther
};

// VA14CD state of one system (src/quench_m.F90:323-551)
struct CgState {
    double f, xnew, dgstep, fmin, dginit, xmin, finit, gsinit, gmin, gm, xbound, clt, gnew;
    double ggstar, beta, gamden, gsumsq, pe, last_fmax;
    int itcrs, maxfnk, noerr, iflag, iretry, iterc, maxfnc, label, done, pad;
};

struct TileArgs {
    const BSys *sys;
    const int32_t *cell_sys, *cell_start, *sorted;
    const double4 *spos;          // cell order: x, y, z, mass
    const double *sfp;            // cell order: F'(rho)
    int ncell;
    int cap;                      // staged candidates per warp (<= kTileCap)
    double rc2;                   // pairs at or beyond sqrt(rc2) contribute zero
};

__device__ __forceinline__ int stencil_off(int k, int nst) { return nst == 3 ? k - 1 : k; }

__device__ __forceinline__ int wrapc(int c, int n) { return c < 0 ? c + n : (c >= n ? c - n : c); }

// Stages the candidates of cell c (the union of its stencil cells, in stencil
// order) into the warp's tile; returns the count.  pre[0..ns] holds the prefix
// of the stencil-cell sizes, cs[0..ns) their first sorted slot.
template <bool FP>
__device__ int stage_tile(const TileArgs &a, const BSys &S, int c, double4 *tp, double *tf, int *ti, int *pre,
                          int *cs) {
    const int lane = threadIdx.x & 31;
    const int local = c - S.cell0;
    const int cx = local % S.nc[0], cy = (local / S.nc[0]) % S.nc[1], cz = local / (S.nc[0] * S.nc[1]);
    const int ns = S.nst[0] * S.nst[1] * S.nst[2];
    int cnt = 0, start = 0;
    if (lane < ns) {
        int kx = lane % S.nst[0], ky = (lane / S.nst[0]) % S.nst[1], kz = lane / (S.nst[0] * S.nst[1]);
        int ix = wrapc(cx + stencil_off(kx, S.nst[0]), S.nc[0]);
        int iy = wrapc(cy + stencil_off(ky, S.nst[1]), S.nc[1]);
        int iz = wrapc(cz + stencil_off(kz, S.nst[2]), S.nc[2]);
        int cc = S.cell0 + ix + S.nc[0] * (iy + S.nc[1] * iz);
        start = a.cell_start[cc];
        cnt = a.cell_start[cc + 1] - start;
    }
    // inclusive scan of the counts over the lanes
    int inc = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane < ns) { pre[lane + 1] = inc; cs[lane] = start; }
    if (lane == 0) pre[0] = 0;
    const int total = __shfl_sync(0xffffffffu, inc, 31);
    __syncwarp();
    const int nstage = total < a.cap ? total : a.cap;
    for (int k = lane; k < nstage; k += 32) {
        int q = 0;
        while (pre[q + 1] <= k) ++q;
        int slot = cs[q] + (k - pre[q]);
        tp[k] = a.spos[slot];
        if (FP) tf[k] = a.sfp[slot];
        ti[k] = slot;
    }
    __syncwarp();
    return total;
}

// candidate k of the staged tile, or from global memory past the tile's capacity
template <bool FP>
__device__ __forceinline__ void candidate(const TileArgs &a, int k, const double4 *tp, const double *tf,
                                          const int *ti, const int *pre, const int *cs, double4 &p, double &fp,
                                          int &slot) {
    if (k < a.cap) {
        p = tp[k];
        fp = FP ? tf[k] : 0.0;
        slot = ti[k];
    } else {
        int q = 0;
        while (pre[q + 1] <= k) ++q;
        slot = cs[q] + (k - pre[q]);
        p = a.spos[slot];
        fp = FP ? a.sfp[slot] : 0.0;
    }
}

__device__ __forceinline__ void pair_u(const double *b, double dx, double dy, double dz, double &ux, double &uy,
                                       double &uz) {
    ux = b[0] * dx + b[3] * dy + b[6] * dz;
    uy = b[1] * dx + b[4] * dy + b[7] * dz;
    uz = b[2] * dx + b[5] * dy + b[8] * dz;
}

template <int LPH>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
    for (int o = LPH / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------ block reductions --
// fixed-order sum over the block, returned to every thread
__device__ double block_sum(double v, double *sh) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        double x = lane < nw ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[32] = x;
    }
    __syncthreads();
    return sh[32];
}

__device__ double block_max(double v, double *sh) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        double x = lane < nw ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_down_sync(0xffffffffu, x, o));
        if (lane == 0) sh[32] = x;
    }
    __syncthreads();
    return sh[32];
}

// ------------------------------------------------------ lists and binning --
// One block per system.  An evaluated system whose list is stale, or one of
// whose atoms moved more than half the skin since the last build (a pair can
// only come inside rc after that), rebuilds: its atoms are binned into its
// cells, the cell sizes scanned into slot ranges starting at atom0, every
// cell filled and sorted by atom index.  Every evaluated system then copies
// its positions and masses into cell order.
// The list check and rebuild of one active system by the whole block (any
// block size up to 1024); todo, when given, receives the rebuilt cells for
// the tile screen.  Every atom's cell-order copy goes to spos when all_spos,
// else only a rebuilt system's (the tile screen reads it).  Returns whether
// the system was rebuilt (the same in every thread).
__device__ int prepare_system(BSys &S, const double *__restrict__ X, const double *__restrict__ mass,
                              double *__restrict__ Xb, int32_t *__restrict__ cell_of,
                              int32_t *__restrict__ cell_count, int32_t *__restrict__ cell_start,
                              int32_t *__restrict__ cursor, int32_t *__restrict__ sorted,
                              double4 *__restrict__ spos, unsigned long long *__restrict__ stats,
                              int32_t *__restrict__ todo, int32_t *__restrict__ ntodo, bool all_spos) {
    __shared__ double sh[33];
    __shared__ int wsum[32];
    __shared__ int todo0;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
    const int a0 = S.atom0, nm = S.nm;
    int rebuild = S.stale;
    if (!rebuild) {
        double m = 0.0;
#pragma unroll 4
        for (int i = tid; i < nm; i += nt) {
            const size_t a = 3 * (size_t)(a0 + i);
            double rx, ry, rz;
            pair_u(S.b0, X[a] - Xb[a], X[a + 1] - Xb[a + 1], X[a + 2] - Xb[a + 2], rx, ry, rz);
            m = fmax(m, rx * rx + ry * ry + rz * rz);
        }
        rebuild = block_max(m, sh) > S.hs2;
    }
    __syncthreads();   // every thread has read S.stale
    if (tid == 0) {
        S.rebuild = rebuild;
        S.stale = 0;
        atomicAdd(&stats[1], 1ULL);
        if (rebuild) {
            atomicAdd(&stats[0], 1ULL);
            if (todo) todo0 = atomicAdd(ntodo, S.ncell);
        }
    }
    if (rebuild) {
        for (int i = tid; i < nm; i += nt) {
            const int a = a0 + i;
            int ic[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double x = X[3 * (size_t)a + d];
                Xb[3 * (size_t)a + d] = x;
                const double u = x - floor(x);
                const int c = (int)(u * (double)S.nc[d]);
                ic[d] = c < 0 ? 0 : (c >= S.nc[d] ? S.nc[d] - 1 : c);
            }
            const int c = S.cell0 + ic[0] + S.nc[0] * (ic[1] + S.nc[1] * ic[2]);
            cell_of[a] = c;
            atomicAdd(&cell_count[c], 1);
        }
        __syncthreads();
        // exclusive scan of the cell sizes; the counts are taken (and zeroed
        // for the next build) with atomics, which read them where they were added
        int carry = a0;
        for (int c0 = 0; c0 < S.ncell; c0 += nt) {
            const int cl = c0 + tid;
            const int v = cl < S.ncell ? atomicExch(&cell_count[S.cell0 + cl], 0) : 0;
            int inc = v;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            if (lane == 31) wsum[w] = inc;
            __syncthreads();
            if (w == 0) {
                int x = lane < nw ? wsum[lane] : 0;
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= o) x += y;
                }
                if (lane < nw) wsum[lane] = x;
            }
            __syncthreads();
            if (cl < S.ncell) {
                cell_start[S.cell0 + cl] = carry + (w > 0 ? wsum[w - 1] : 0) + inc - v;
                cursor[S.cell0 + cl] = 0;
            }
            carry += wsum[nw - 1];
            __syncthreads();
        }
        for (int i = tid; i < nm; i += nt) {
            const int a = a0 + i, c = cell_of[a];
            sorted[cell_start[c] + atomicAdd(&cursor[c], 1)] = a;
        }
        __syncthreads();
        // ascending atom order inside each cell; the cells join the tile screen's work
        for (int cl = tid; cl < S.ncell; cl += nt) {
            const int c = S.cell0 + cl;
            if (todo) todo[todo0 + cl] = c;
            const int s0 = cell_start[c], s1 = cl + 1 < S.ncell ? cell_start[c + 1] : a0 + nm;
            for (int i = s0 + 1; i < s1; ++i) {
                const int v = sorted[i];
                int j = i - 1;
                while (j >= s0 && sorted[j] > v) { sorted[j + 1] = sorted[j]; --j; }
                sorted[j + 1] = v;
            }
        }
        __syncthreads();
    }
    if (rebuild || all_spos) {
        for (int hs = a0 + tid; hs < a0 + nm; hs += nt) {
            const int a = sorted[hs];
            spos[hs] = make_double4(X[3 * (size_t)a], X[3 * (size_t)a + 1], X[3 * (size_t)a + 2], mass[a]);
        }
    }
    __syncthreads();
    return rebuild;
}

__global__ void __launch_bounds__(kPrepThreads)
k_prepare(BSys *__restrict__ sys, const double *__restrict__ X, const double *__restrict__ mass,
          double *__restrict__ Xb, int32_t *__restrict__ cell_of, int32_t *__restrict__ cell_count,
          int32_t *__restrict__ cell_start, int32_t *__restrict__ cursor, int32_t *__restrict__ sorted,
          double4 *__restrict__ spos, unsigned long long *__restrict__ stats, int32_t *__restrict__ todo,
          int32_t *__restrict__ ntodo) {
    BSys &S = sys[blockIdx.x];
    if (!S.active) {
        if (threadIdx.x == 0) S.rebuild = 0;
        return;
    }
    prepare_system(S, X, mass, Xb, cell_of, cell_count, cell_start, cursor, sorted, spos, stats, todo, ntodo,
                   true);
}

// ------------------------------------------------------------ tile passes --
// The tile screen finds, for every home atom of a cell of a rebuilt system,
// the candidates inside the list radius and writes their cell-order slots
// into the atom's compact row (entry-major, alist[e * ntot + slot]) in
// candidate order.  LPH lanes
// serve one home atom: they test LPH candidates at a time and place the hits
// with one warp ballot, so no lane waits on another's pair arithmetic.
// The compact rows of the home atoms of cell c by one warp, with the warp's
// tile (tp, ti: cap entries; pre, cs: 28); returns the longest row seen when
// it exceeds pair_cap, else 0.
template <int LPH>
__device__ int screen_cell(const TileArgs &a, int c, int ntot, int pair_cap, int32_t *__restrict__ alist,
                           int32_t *__restrict__ cnt_out, double4 *tp, int *ti, int *pre, int *cs) {
    const int lane = threadIdx.x & 31;
    const int g = lane / LPH, gl = lane % LPH;
    const unsigned gmask = (LPH == 32 ? 0xffffffffu : ((1u << LPH) - 1u)) << (g * LPH);
    const unsigned below = (1u << lane) - 1u;
    int overflow = 0;
    const BSys &S = a.sys[a.cell_sys[c]];
    const int h0 = a.cell_start[c], h1 = a.cell_start[c + 1];
    if (h1 == h0) return 0;
    double b[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) b[k] = S.b0[k];
    const double rv2 = S.rv2;
    const int total = stage_tile<false>(a, S, c, tp, nullptr, ti, pre, cs);
    for (int hb = h0; hb < h1; hb += 32 / LPH) {
        const int hs = hb + g;
        const bool live = hs < h1;
        const double4 ph = live ? a.spos[hs] : make_double4(0.0, 0.0, 0.0, 0.0);
        int cnt = 0;
        // every lane of the warp runs the same number of rounds (ballots are warp-wide)
        for (int k0 = 0; k0 < total; k0 += LPH) {
            const int k = k0 + gl;
            bool hit = false;
            int slot = -1;
            if (live && k < total) {
                double4 p; double fpk;
                candidate<false>(a, k, tp, nullptr, ti, pre, cs, p, fpk, slot);
                if (slot != hs) {
                    double dx = ph.x - p.x, dy = ph.y - p.y, dz = ph.z - p.z;
                    dx = dx - round(dx); dy = dy - round(dy); dz = dz - round(dz);
                    double ux, uy, uz;
                    pair_u(b, dx, dy, dz, ux, uy, uz);
                    hit = (ux * ux + uy * uy + uz * uz) < rv2;
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit) & gmask;
            if (hit) {
                const int e = cnt + __popc(m & below);
                if (e < pair_cap) alist[(size_t)e * ntot + hs] = slot;
            }
            cnt += __popc(m);
        }
        if (live && gl == 0) {
            cnt_out[hs] = cnt;
            if (cnt > pair_cap) overflow = max(overflow, cnt);
        }
    }
    __syncwarp();   // the next cell restages the warp's tile
    return overflow;
}

template <int LPH>
__global__ void __launch_bounds__(32 * kTileWarps)
k_tile_screen(TileArgs a, int ntot, int pair_cap, int32_t *__restrict__ alist, int32_t *__restrict__ cnt_out,
              int32_t *__restrict__ flags, const int32_t *__restrict__ todo, const int32_t *__restrict__ ntodo) {
    __shared__ double4 tpos[kTileWarps][kTileCap];
    __shared__ int tidx[kTileWarps][kTileCap];
    __shared__ int tpre[kTileWarps][28], tcs[kTileWarps][28];
    const int w = threadIdx.x >> 5;
    const int nwork = *ntodo;
    int overflow = 0;
    // one warp per cell of the rebuilt systems (warp-uniform loop)
    for (int t = blockIdx.x * kTileWarps + w; t < nwork; t += gridDim.x * kTileWarps)
        overflow = max(overflow, screen_cell<LPH>(a, todo[t], ntot, pair_cap, alist, cnt_out, tpos[w], tidx[w],
                                                  tpre[w], tcs[w]));
    if (overflow) { atomicExch(&flags[0], 1); atomicMax(&flags[1], overflow); }
}

__device__ __forceinline__ void pair_uf(const float *b, float dx, float dy, float dz, float &ux, float &uy,
                                        float &uz) {
    ux = b[0] * dx + b[3] * dy + b[6] * dz;
    uy = b[1] * dx + b[4] * dy + b[7] * dz;
    uz = b[2] * dx + b[5] * dy + b[8] * dz;
}

// fractional difference to the nearest image (round is Fortran NINT)
__device__ __forceinline__ void frac_diff(const double4 &p, const double4 &q, double &dx, double &dy, double &dz) {
    dx = p.x - q.x; dy = p.y - q.y; dz = p.z - q.z;
    dx = dx - round(dx); dy = dy - round(dy); dz = dz - round(dz);
}

// rho_i over the pairs of the compact row inside rc (rhoset), then F and F'
// (embed, src/potential_m.F90:148-169), and the atom's energy_calc energy
// F + sum V_src/2 with the exact pair function at the FP64 distance
// (src/dynamics_m.F90:412-483); one thread per atom in cell order, which
// gathers B row entries before it evaluates them.  MIXED takes rho's
// separation B0 d, distance and table interpolation in FP32 from the FP64
// difference and sums rho_i in FP64.  Entries are summed in row order at
// every B.
template <bool MIXED, int B, bool ECALC>
__global__ void __launch_bounds__(256)
k_cl_density(TileArgs a, Tables t, int ntot, int pair_cap, const int32_t *__restrict__ alist,
             const int32_t *__restrict__ cnt, double *__restrict__ sfp, double *__restrict__ rho_out,
             double *__restrict__ afrho_out, double *__restrict__ fp_out, double *__restrict__ en_calc,
             const int32_t *__restrict__ slot_sys, int32_t *__restrict__ ntodo) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *ntodo = 0;   // the tile screen before this pass has read it
    const float rc2f = (float)a.rc2;
    for (int hs = blockIdx.x * blockDim.x + threadIdx.x; hs < ntot; hs += gridDim.x * blockDim.x) {
        const BSys &S = a.sys[slot_sys[hs]];
        if (!S.active) continue;
        double b[9];
        float bf[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) { b[k] = S.b0[k]; bf[k] = (float)b[k]; }
        const double4 ph = a.spos[hs];
        int n = cnt[hs];
        n = n < pair_cap ? n : pair_cap;
        double rho = 0.0, ec = 0.0;
        for (int e0 = 0; e0 < n; e0 += B) {
            int jj[B];
#pragma unroll
            for (int u = 0; u < B; ++u) jj[u] = e0 + u < n ? alist[(size_t)(e0 + u) * ntot + hs] : hs;
            double4 pp[B];
#pragma unroll
            for (int u = 0; u < B; ++u) pp[u] = ldg4(&a.spos[jj[u]]);
#pragma unroll
            for (int u = 0; u < B; ++u) {
                if (e0 + u >= n) continue;
                double dx, dy, dz;
                frac_diff(ph, pp[u], dx, dy, dz);
                if (MIXED) {
                    float ux, uy, uz;
                    pair_uf(bf, (float)dx, (float)dy, (float)dz, ux, uy, uz);
                    const float r2 = ux * ux + uy * uy + uz * uz;
                    if (!(r2 < rc2f)) continue;
                    rho += (double)lookup_phif(t, r2 * rsqrt_ftz(r2));
                    if (ECALC) {
                        double vx, vy, vz;
                        pair_u(b, dx, dy, dz, vx, vy, vz);
                        ec += 0.5 * fetm_vee(t, sqrt(vx * vx + vy * vy + vz * vz));
                    }
                } else {
                    double ux, uy, uz;
                    pair_u(b, dx, dy, dz, ux, uy, uz);
                    const double r2 = ux * ux + uy * uy + uz * uz;
                    if (!(r2 < a.rc2)) continue;
                    const double r = sqrt(r2);
                    rho += lookup_phi(t, r);
                    if (ECALC) ec += 0.5 * fetm_vee(t, r);
                }
            }
        }
        double f = 0.0, fd = 0.0;
        if (rho > 1e-40) {
            double2 e2 = lookup_e2(t, rho);
            f = e2.x; fd = e2.y;
        }
        sfp[hs] = fd;
        const int at = a.sorted[hs];
        rho_out[at] = rho;
        afrho_out[at] = f;
        fp_out[at] = fd;
        if (ECALC) en_calc[at] = f + ec;
    }
}

// Forces on each atom (the pair loop of force(), src/dynamics_m.F90:232-318),
// its force-routine energy F + sum V/2, and with VIR the symmetric per-atom
// moment S = sum d d^T fp / 2 over pairs with m_i + m_j > 0.1 (stored xx, yy,
// zz, xy, xz, yz), from which the virial sum (B0 d) d^T fp / 2 is B0 S; one
// thread per atom, B row entries gathered at a time.  MIXED takes the
// separation, the table interpolation and the pair force in FP32 and sums in
// FP64.
template <bool MIXED, int B, bool VIR>
__global__ void __launch_bounds__(256)
k_cl_forces(TileArgs a, Tables t, int ntot, int pair_cap, const int32_t *__restrict__ alist,
            const int32_t *__restrict__ cnt, const int32_t *__restrict__ slot_sys, const double *__restrict__ afrho,
            double *__restrict__ fout, double *__restrict__ en_force, double *__restrict__ vir) {
    const float rc2f = (float)a.rc2;
    for (int hs = blockIdx.x * blockDim.x + threadIdx.x; hs < ntot; hs += gridDim.x * blockDim.x) {
        const BSys &S = a.sys[slot_sys[hs]];
        if (!S.active) continue;
        double b[9];
        float bf[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) { b[k] = S.b0[k]; bf[k] = (float)b[k]; }
        const double4 ph = a.spos[hs];
        const double fph = a.sfp[hs];
        int n = cnt[hs];
        n = n < pair_cap ? n : pair_cap;
        double fx = 0.0, fy = 0.0, fz = 0.0, ef = 0.0;
        double v[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = 0.0;
        for (int e0 = 0; e0 < n; e0 += B) {
            int jj[B];
#pragma unroll
            for (int u = 0; u < B; ++u) jj[u] = e0 + u < n ? alist[(size_t)(e0 + u) * ntot + hs] : hs;
            double4 pp[B];
            double fq[B];
#pragma unroll
            for (int u = 0; u < B; ++u) { pp[u] = ldg4(&a.spos[jj[u]]); fq[u] = a.sfp[jj[u]]; }
#pragma unroll
            for (int u = 0; u < B; ++u) {
                if (e0 + u >= n) continue;
                double dx, dy, dz;
                frac_diff(ph, pp[u], dx, dy, dz);
                double fpair, vee;
                if (MIXED) {
                    float uxf, uyf, uzf;
                    pair_uf(bf, (float)dx, (float)dy, (float)dz, uxf, uyf, uzf);
                    const float r2 = uxf * uxf + uyf * uyf + uzf * uzf;
                    if (!(r2 < rc2f)) continue;
                    const float rr = rsqrt_ftz(r2), r = r2 * rr;
                    const float4 q = lookup_r4f(t, r);
                    fpair = (double)(-(q.y + q.w * ((float)fph + (float)fq[u])) * rr);
                    vee = (double)q.x;
                } else {
                    double ux, uy, uz;
                    pair_u(b, dx, dy, dz, ux, uy, uz);
                    const double r2 = ux * ux + uy * uy + uz * uz;
                    if (!(r2 < a.rc2)) continue;
                    const double r = sqrt(r2);
                    const double4 q = lookup_r4(t, r);     // V, V', phi, phi'
                    const double rr = 1.0 / r;
                    fpair = -q.y * rr - (q.w * fph + q.w * fq[u]) * rr;
                    vee = q.x;
                }
                fx += dx * fpair; fy += dy * fpair; fz += dz * fpair;
                ef += 0.5 * vee;
                if (VIR && (ph.w + pp[u].w) > 0.1) {
                    const double hf = 0.5 * fpair;
                    v[0] += dx * dx * hf; v[1] += dy * dy * hf; v[2] += dz * dz * hf;
                    v[3] += dx * dy * hf; v[4] += dx * dz * hf; v[5] += dy * dz * hf;
                }
            }
        }
        const int at = a.sorted[hs];
        fout[3 * (size_t)at] = fx;
        fout[3 * (size_t)at + 1] = fy;
        fout[3 * (size_t)at + 2] = fz;
        en_force[at] = afrho[at] + ef;
        if (VIR) {
#pragma unroll
            for (int k = 0; k < 6; ++k) vir[6 * (size_t)at + k] = v[k];
        }
    }
}

// ------------------------------------------------ persistent evaluation --
// One launch evaluates every active system in mixed precision: the force
// routine's energy, the forces and the virial (energy_calc's exact energies
// are left to the per-pass kernels).  A resident grid of blocks takes systems
// from a queue in descending size.  For each system the block
//   1. checks the list and, past half the skin, rebuilds it: binning as
//      k_prepare, then the compact rows with the block's warps over the
//      system's cells as k_tile_screen (the warps' tiles in the shared memory
//      that the records use afterwards);
//   2. stages the system's atoms in cell order as fixed-point records (x, y,
//      z, F'(rho) as float) in shared memory, so every neighbour read of the
//      two passes is a shared-memory load;
//   3. runs the density pass (rho, F, F') and the force pass with LPA lanes
//      per atom: lane g takes the row entries g, g + LPA, ...; the lanes'
//      FP64 sums are combined by shuffles in a fixed order;
//   4. reduces the system's energy, largest force and virial in a fixed
//      order (the results of k_sys_reduce).
// Separations come from the 32-bit fixed-point difference (the integer
// difference is the minimum image); distances, table interpolation and pair
// terms run in FP32, and every sum accumulates in FP64.  Pairs enter the
// virial without the mass filter: the path runs only when every atom is
// heavier than 0.05, so every pair passes m_i + m_j > 0.1.
constexpr int kEvalThreads = 512;
constexpr int kEvalWarps = kEvalThreads / 32;
constexpr int kEvalGather = 4;       // row entries a lane loads before it uses any

struct EvalArgs {
    BSys *sys;
    const int32_t *order;            // systems by descending size
    int nsys, ntot, pair_cap;
    int32_t *queue;                  // [0] next system, [1] blocks done (both zero between launches)
    const double *X, *mass;
    double *Xb;
    int32_t *cell_of, *cell_count, *cell_start, *cursor, *sorted;
    double4 *spos;
    unsigned long long *stats;
    const int32_t *cell_sys;
    int32_t *alist, *pcnt, *flags;
    int ncell, cap;
    double rc2;
    double *f, *rho, *afrho, *fp, *en_force, *sysout;
};

// sum over the LPA lanes of an atom's group, the same in every lane
template <int LPA>
__device__ __forceinline__ double lanes_sum(double v) {
#pragma unroll
    for (int o = LPA / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// fractional difference of two records in fixed-point units (FP32) and r^2
__device__ __forceinline__ float rec_sep(const float *bq, const int4 &qi, const int4 &qj, float &dx, float &dy,
                                         float &dz) {
    dx = fix_to_float((int32_t)((uint32_t)qi.x - (uint32_t)qj.x));
    dy = fix_to_float((int32_t)((uint32_t)qi.y - (uint32_t)qj.y));
    dz = fix_to_float((int32_t)((uint32_t)qi.z - (uint32_t)qj.z));
    const float ux = fmaf(bq[6], dz, fmaf(bq[3], dy, bq[0] * dx));
    const float uy = fmaf(bq[7], dz, fmaf(bq[4], dy, bq[1] * dx));
    const float uz = fmaf(bq[8], dz, fmaf(bq[5], dy, bq[2] * dx));
    return fmaf(uz, uz, fmaf(uy, uy, ux * ux));
}

template <int LPH, int LPA>
__global__ void __launch_bounds__(kEvalThreads, 1)
k_batch_eval(EvalArgs a, Tables t) {
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ int tpre[kEvalWarps][28], tcs[kEvalWarps][28];
    __shared__ double shr[33];
    __shared__ int s_next;
    int4 *rec = reinterpret_cast<int4 *>(dsm);
    const int tid = threadIdx.x, w = tid >> 5;
    const float rc2f = (float)a.rc2;
    constexpr int kAtomsPerRound = kEvalThreads / LPA;
    const int g = tid % LPA;
    int overflow = 0;
    for (;;) {
        if (tid == 0) s_next = atomicAdd(&a.queue[0], 1);
        __syncthreads();
        const int k = s_next;
        __syncthreads();                       // s_next is rewritten only after every thread read it
        if (k >= a.nsys) break;
        const int sid = a.order[k];
        BSys &S = a.sys[sid];
        if (!S.active) continue;
        // 1. list check, rebuild when due
        const int rebuilt = prepare_system(S, a.X, a.mass, a.Xb, a.cell_of, a.cell_count, a.cell_start, a.cursor,
                                           a.sorted, a.spos, a.stats, nullptr, nullptr, false);
        if (rebuilt) {
            TileArgs ta;
            ta.sys = a.sys; ta.cell_sys = a.cell_sys; ta.cell_start = a.cell_start; ta.sorted = a.sorted;
            ta.spos = a.spos; ta.sfp = nullptr; ta.ncell = a.ncell; ta.cap = a.cap; ta.rc2 = a.rc2;
            double4 *tp = reinterpret_cast<double4 *>(dsm) + (size_t)w * a.cap;
            int *ti = reinterpret_cast<int *>(reinterpret_cast<double4 *>(dsm) + (size_t)kEvalWarps * a.cap) +
                      (size_t)w * a.cap;
            for (int c = S.cell0 + w; c < S.cell0 + S.ncell; c += kEvalWarps)
                overflow = max(overflow, screen_cell<LPH>(ta, c, a.ntot, a.pair_cap, a.alist, a.pcnt, tp, ti,
                                                          tpre[w], tcs[w]));
            __syncthreads();                   // rows written; the tiles' memory is reused below
        }
        const int a0 = S.atom0, nm = S.nm;
        double b[9];
        float bq[9];                           // B0 per fixed-point unit
#pragma unroll
        for (int q = 0; q < 9; ++q) { b[q] = S.b0[q]; bq[q] = (float)(b[q] * kFixUnit); }
        // 2. the system's records in cell order
#pragma unroll 4
        for (int i = tid; i < nm; i += kEvalThreads) {
            const size_t at = 3 * (size_t)a.sorted[a0 + i];
            rec[i] = make_int4(fix32(a.X[at]), fix32(a.X[at + 1]), fix32(a.X[at + 2]), 0);
        }
        __syncthreads();
        // 3a. density, F and F'
        for (int i0 = 0; i0 < nm; i0 += kAtomsPerRound) {
            const int i = i0 + tid / LPA;
            const bool live = i < nm;
            const int hs = a0 + (live ? i : 0);
            const int4 qi = rec[live ? i : 0];
            int n = live ? a.pcnt[hs] : 0;
            n = n < a.pair_cap ? n : a.pair_cap;
            double rho = 0.0;
            for (int e0 = g; e0 < n; e0 += kEvalGather * LPA) {
                int jj[kEvalGather];
#pragma unroll
                for (int u = 0; u < kEvalGather; ++u) {
                    const int e = e0 + u * LPA;
                    jj[u] = e < n ? a.alist[(size_t)e * a.ntot + hs] - a0 : -1;
                }
#pragma unroll
                for (int u = 0; u < kEvalGather; ++u) {
                    if (jj[u] < 0) continue;
                    const int4 qj = rec[jj[u]];
                    float dx, dy, dz;
                    const float r2 = rec_sep(bq, qi, qj, dx, dy, dz);
                    if (r2 < rc2f) rho += (double)lookup_phif(t, r2 * rsqrt_ftz(r2));
                }
            }
            rho = lanes_sum<LPA>(rho);
            if (live && g == 0) {
                double fe = 0.0, fd = 0.0;
                if (rho > 1e-40) {
                    const double2 e2 = lookup_e2(t, rho);
                    fe = e2.x; fd = e2.y;
                }
                rec[i].w = __float_as_int((float)fd);
                const int at = a.sorted[hs];
                a.rho[at] = rho;
                a.afrho[at] = fe;
                a.fp[at] = fd;
            }
        }
        __syncthreads();
        // 3b. forces, force-routine energy, virial moments
        double sef = 0.0, sfm = 0.0, sv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int i0 = 0; i0 < nm; i0 += kAtomsPerRound) {
            const int i = i0 + tid / LPA;
            const bool live = i < nm;
            const int hs = a0 + (live ? i : 0);
            const int4 qi = rec[live ? i : 0];
            const float fpi = __int_as_float(qi.w);
            int n = live ? a.pcnt[hs] : 0;
            n = n < a.pair_cap ? n : a.pair_cap;
            double fx = 0.0, fy = 0.0, fz = 0.0, ef = 0.0, v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            for (int e0 = g; e0 < n; e0 += kEvalGather * LPA) {
                int jj[kEvalGather];
#pragma unroll
                for (int u = 0; u < kEvalGather; ++u) {
                    const int e = e0 + u * LPA;
                    jj[u] = e < n ? a.alist[(size_t)e * a.ntot + hs] - a0 : -1;
                }
#pragma unroll
                for (int u = 0; u < kEvalGather; ++u) {
                    if (jj[u] < 0) continue;
                    const int4 qj = rec[jj[u]];
                    float dx, dy, dz;
                    const float r2 = rec_sep(bq, qi, qj, dx, dy, dz);
                    if (!(r2 < rc2f)) continue;
                    const float rr = rsqrt_ftz(r2), r = r2 * rr;
                    const float4 q = lookup_r4f(t, r);
                    const float fpair = -(q.y + q.w * (fpi + __int_as_float(qj.w))) * rr;
                    fx += (double)(dx * fpair);
                    fy += (double)(dy * fpair);
                    fz += (double)(dz * fpair);
                    ef += (double)q.x;
                    const float hf = 0.5f * fpair;
                    const float hx = dx * hf, hy = dy * hf;
                    v[0] += (double)(dx * hx); v[1] += (double)(dy * hy); v[2] += (double)(dz * (dz * hf));
                    v[3] += (double)(dy * hx); v[4] += (double)(dz * hx); v[5] += (double)(dz * hy);
                }
            }
            fx = lanes_sum<LPA>(fx); fy = lanes_sum<LPA>(fy); fz = lanes_sum<LPA>(fz);
            ef = lanes_sum<LPA>(ef);
#pragma unroll
            for (int q = 0; q < 6; ++q) v[q] = lanes_sum<LPA>(v[q]);
            if (live && g == 0) {
                // fixed-point units to box lengths (exact scalings)
                fx *= kFixUnit; fy *= kFixUnit; fz *= kFixUnit;
                const int at = a.sorted[hs];
                a.f[3 * (size_t)at] = fx;
                a.f[3 * (size_t)at + 1] = fy;
                a.f[3 * (size_t)at + 2] = fz;
                const double eat = a.afrho[at] + 0.5 * ef;
                a.en_force[at] = eat;
                sef += eat;
#pragma unroll
                for (int q = 0; q < 6; ++q) sv[q] += v[q] * (kFixUnit * kFixUnit);
                double rx, ry, rz;
                pair_u(b, fx, fy, fz, rx, ry, rz);
                sfm = fmax(sfm, sqrt(rx * rx + ry * ry + rz * rz));
            }
        }
        // 4. the system's sums (block reductions in a fixed order)
        double o[13];
        o[0] = 0.0;
        o[1] = block_sum(sef, shr);
        o[2] = block_max(sfm, shr);
        o[3] = S.vol;
        double sm[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) sm[q] = block_sum(sv[q], shr);
        const double S9[9] = {sm[0], sm[3], sm[4], sm[3], sm[1], sm[5], sm[4], sm[5], sm[2]};   // S(c, b) at c + 3b
        for (int p = 0; p < 3; ++p)
            for (int bb = 0; bb < 3; ++bb)
                o[4 + p + 3 * bb] = b[p] * S9[3 * bb] + b[p + 3] * S9[1 + 3 * bb] + b[p + 6] * S9[2 + 3 * bb];
        if (tid == 0)
            for (int q = 0; q < 13; ++q) a.sysout[13 * (size_t)sid + q] = o[q];
        __syncthreads();                       // the records are restaged for the next system
    }
    if (overflow) { atomicExch(&a.flags[0], 1); atomicMax(&a.flags[1], overflow); }
    // the last block to finish resets the queue for the next launch
    if (tid == 0) {
        __threadfence();
        if (atomicAdd(&a.queue[1], 1) == (int)gridDim.x - 1) {
            a.queue[0] = 0;
            a.queue[1] = 0;
            __threadfence();
        }
    }
}

// per-system sums of one evaluation: pe (energy_calc), pe (force), virial,
// largest real force
__global__ void __launch_bounds__(kCgThreads)
k_sys_reduce(const BSys *__restrict__ sys, const double *__restrict__ en_calc, const double *__restrict__ en_force,
             const double *__restrict__ vir, const double *__restrict__ f, int with_vir, double *__restrict__ out) {
    __shared__ double sh[33];
    const BSys &S = sys[blockIdx.x];
    double ec = 0.0, ef = 0.0, fm = 0.0, v[6] = {0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < S.nm; i += blockDim.x) {
        const int at = S.atom0 + i;
        ec += en_calc[at];
        ef += en_force[at];
        if (with_vir)
            for (int k = 0; k < 6; ++k) v[k] += vir[6 * (size_t)at + k];
        double gx = f[3 * (size_t)at], gy = f[3 * (size_t)at + 1], gz = f[3 * (size_t)at + 2];
        double rx, ry, rz;
        pair_u(S.b0, gx, gy, gz, rx, ry, rz);
        fm = fmax(fm, sqrt(rx * rx + ry * ry + rz * rz));
    }
    double o[13];
    o[0] = block_sum(ec, sh);
    o[1] = block_sum(ef, sh);
    o[2] = block_max(fm, sh);
    o[3] = S.vol;
    // virial B0 S from the summed symmetric moment S
    double sm[6];
    for (int k = 0; k < 6; ++k) sm[k] = with_vir ? block_sum(v[k], sh) : 0.0;
    const double S9[9] = {sm[0], sm[3], sm[4], sm[3], sm[1], sm[5], sm[4], sm[5], sm[2]};   // S(c, b) at c + 3b
    for (int a = 0; a < 3; ++a)
        for (int bb = 0; bb < 3; ++bb)
            o[4 + a + 3 * bb] = S.b0[a] * S9[3 * bb] + S.b0[a + 3] * S9[1 + 3 * bb] + S.b0[a + 6] * S9[2 + 3 * bb];
    if (threadIdx.x == 0)
        for (int k = 0; k < 13; ++k) out[13 * (size_t)blockIdx.x + k] = o[k];
}

// --------------------------------------------------------- CG control --
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }

// --------------------------------------------------------- force matching --
// The force-matching loss of one evaluation of every system against
// reference real forces and stresses, and its adjoint with respect to the six
// lookup tables (no counterpart in the reference).  The differentiated
// quantities are those write_energy_forces_stress prints
// (src/dynamics_m.F90:588-619): F = B0 f and sigma(i,j) = -sum_k b0(j,k)
// tp(i,k) / vol.  With dL/dF_i = gF_i and dL/dsigma_s = G_s, per pair (i,j)
// inside the table cut, u = B0 d, r = |u|:
//   lam_ij = (gF_i - gF_j) . u - u^T G_s u / vol_s  [m_i + m_j > 0.1]   (= dL/dfp_ij)
//   mu_i = dL/dF'_i = sum_j -lam_ij DP(r_ij) / r_ij
//   nu_i = dL/drho_i = mu_i De'(rho_i)          (slope of the interpolant)
//   dL/dDV(r) = -lam / r,  dL/dDP(r) = -lam (F'_i + F'_j) / r,  dL/dP(r) = nu_i + nu_j,
//   dL/dDe(rho_i) = mu_i,  dL/dV = dL/dEm = 0 (the loss holds no energy),
// each table node receiving its interpolation weight times these.  Every row
// holds both directions, so each atom forms its own mu and nu from its row,
// with no atomics; a table histogram takes each pair once (from the lower
// slot).  Only pairs inside the table cut enter: they carry every table
// node below the cut, and with it every knot derivative (the Fe-Fe forms and
// their knot derivatives vanish at and beyond the largest knot).  rho comes
// from the forward pass (per atom), F' from its cell-order copy.

// Loss and dL/dF, dL/dsigma of one evaluation; one block per system.  gF
// goes to cell order (slot hs) for the pair passes.
__global__ void __launch_bounds__(kCgThreads)
k_fm_loss(const BSys *__restrict__ sys, const double *__restrict__ f, const double *__restrict__ fref,
          const double *__restrict__ sref, const double *__restrict__ sysout, const int32_t *__restrict__ sorted,
          double wf, double ws, double *__restrict__ gF, double *__restrict__ gS, double *__restrict__ loss) {
    __shared__ double sh[33];
    const BSys &S = sys[blockIdx.x];
    double lf = 0.0;
    for (int hs = S.atom0 + threadIdx.x; hs < S.atom0 + S.nm; hs += blockDim.x) {
        const size_t at = 3 * (size_t)sorted[hs];
        double fx, fy, fz;
        pair_u(S.b0, f[at], f[at + 1], f[at + 2], fx, fy, fz);
        const double dx = fx - fref[at], dy = fy - fref[at + 1], dz = fz - fref[at + 2];
        lf += dx * dx + dy * dy + dz * dz;
        gF[3 * (size_t)hs] = 2.0 * wf * dx;
        gF[3 * (size_t)hs + 1] = 2.0 * wf * dy;
        gF[3 * (size_t)hs + 2] = 2.0 * wf * dz;
    }
    lf = block_sum(lf, sh);
    if (threadIdx.x == 0) {
        const double *o = sysout + 13 * (size_t)blockIdx.x;
        const double *tp = o + 4;
        double ls = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double sg = 0.0;
                for (int k = 0; k < 3; ++k) sg -= S.b0[j + 3 * k] * tp[i + 3 * k];
                sg /= o[3];
                const double d = sg - sref[9 * (size_t)blockIdx.x + i + 3 * j];
                ls += d * d;
                gS[9 * (size_t)blockIdx.x + i + 3 * j] = 2.0 * ws * d;
            }
        loss[blockIdx.x] = wf * lf + ws * ls;
    }
}

// index and weights of the lookup_m interpolation (src/lookup_m.F90:322-341)
// below the table end
__device__ __forceinline__ int fm_weights(double x, double xmin, double range, double recipr, double recipn,
                                          double recips, int n, double &w1) {
    int idx = (int)(((double)n * (x - xmin)) * recipr);
    idx = idx < 0 ? 0 : (idx > n - 1 ? n - 1 : idx);
    const double xlow = xmin + (range * (double)idx) * recipn;
    w1 = (x - xlow) * recips;
    return idx;
}

__device__ __forceinline__ void fm_hist(double *h, int k, double c, double w1) {
    atomicAdd(&h[k], c * (1.0 - w1));
    atomicAdd(&h[k + 1], c * w1);
}

__device__ __forceinline__ void fm_flush(const double *h, double *g, int nb) {
    __syncthreads();
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        const double v = h[k];
        if (v != 0.0) atomicAdd(&g[k], v);
    }
}

// the pair geometry of slot hs and row entry j: u = B0 d, r; false beyond the cut
__device__ __forceinline__ bool fm_pair(const BSys &S, const double4 &ph, const double4 &pj, double rc2,
                                        double &ux, double &uy, double &uz, double &r) {
    double dx, dy, dz;
    frac_diff(ph, pj, dx, dy, dz);
    pair_u(S.b0, dx, dy, dz, ux, uy, uz);
    const double r2 = ux * ux + uy * uy + uz * uz;
    if (!(r2 < rc2)) return false;
    r = sqrt(r2);
    return true;
}

// lam per pair; mu_i; dL/d dvee and dL/d dphi
__global__ void __launch_bounds__(256)
k_fm_pairs_a(TileArgs a, Tables t, int ntot, int pair_cap, const int32_t *__restrict__ alist,
             const int32_t *__restrict__ cnt, const int32_t *__restrict__ slot_sys, const double *__restrict__ gF,
             const double *__restrict__ gS, double *__restrict__ mu, double *__restrict__ g_dvee,
             double *__restrict__ g_dphi, int nbr) {
    extern __shared__ double sh[];
    double *hdv = sh, *hdp = sh + nbr;
    for (int k = threadIdx.x; k < 2 * nbr; k += blockDim.x) sh[k] = 0.0;
    __syncthreads();
    const double rmin = t.vp_rmin, range = t.vp_range, recipr = t.vp_reciprange, recipn = t.vp_recipnlkp,
                 recips = t.vp_recipstep;
    for (int hs = blockIdx.x * blockDim.x + threadIdx.x; hs < ntot; hs += gridDim.x * blockDim.x) {
        const int s = slot_sys[hs];
        const BSys &S = a.sys[s];
        const double4 ph = a.spos[hs];
        const double fph = a.sfp[hs];
        const double gx = gF[3 * (size_t)hs], gy = gF[3 * (size_t)hs + 1], gz = gF[3 * (size_t)hs + 2];
        const double *G = gS + 9 * (size_t)s;
        const double ivol = 1.0 / S.vol;
        int n = cnt[hs];
        n = n < pair_cap ? n : pair_cap;
        double m = 0.0;
        for (int e = 0; e < n; ++e) {
            const int j = alist[(size_t)e * ntot + hs];
            const double4 pj = a.spos[j];
            double ux, uy, uz, r;
            if (!fm_pair(S, ph, pj, a.rc2, ux, uy, uz, r)) continue;
            double w1;
            const int q = fm_weights(r, rmin, range, recipr, recipn, recips, t.nlookup, w1);
            const double dp = t.r4[q].w * (1.0 - w1) + t.r4[q + 1].w * w1;
            double lam = (gx - gF[3 * (size_t)j]) * ux + (gy - gF[3 * (size_t)j + 1]) * uy +
                         (gz - gF[3 * (size_t)j + 2]) * uz;
            if (ph.w + pj.w > 0.1)
                lam -= ivol * (ux * (G[0] * ux + G[3] * uy + G[6] * uz) + uy * (G[1] * ux + G[4] * uy + G[7] * uz) +
                               uz * (G[2] * ux + G[5] * uy + G[8] * uz));
            const double rr = 1.0 / r;
            m -= lam * dp * rr;
            if (hs < j) {
                fm_hist(hdv, q, -lam * rr, w1);
                fm_hist(hdp, q, -lam * (fph + a.sfp[j]) * rr, w1);
            }
        }
        mu[hs] = m;
    }
    fm_flush(hdv, g_dvee, nbr);
    fm_flush(hdp, g_dphi, nbr);
}

// nu_i = mu_i De'(rho_i) and dL/d demb per atom
__global__ void __launch_bounds__(256)
k_fm_atoms(Tables t, int ntot, const int32_t *__restrict__ sorted, const double *__restrict__ rho,
           const double *__restrict__ mu, double *__restrict__ nu, double *__restrict__ g_demb) {
    extern __shared__ double sh[];
    const int nb = t.nlookup + 1;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) sh[k] = 0.0;
    __syncthreads();
    for (int hs = blockIdx.x * blockDim.x + threadIdx.x; hs < ntot; hs += gridDim.x * blockDim.x) {
        const double r = rho[sorted[hs]];
        double v = 0.0;
        if (r > 1e-40) {
            if (r >= t.e_rmax) {
                atomicAdd(&sh[t.nlookup], mu[hs]);   // the last node alone, zero slope
            } else {
                double w1;
                const int q = fm_weights(r, t.e_rmin, t.e_range, t.e_reciprange, t.e_recipnlkp, t.e_recipstep,
                                         t.nlookup, w1);
                v = mu[hs] * (t.e2[q + 1].y - t.e2[q].y) * t.e_recipstep;
                fm_hist(sh, q, mu[hs], w1);
            }
        }
        nu[hs] = v;
    }
    fm_flush(sh, g_demb, nb);
}

// dL/d phi = nu_i + nu_j per pair
__global__ void __launch_bounds__(256)
k_fm_pairs_c(TileArgs a, Tables t, int ntot, int pair_cap, const int32_t *__restrict__ alist,
             const int32_t *__restrict__ cnt, const int32_t *__restrict__ slot_sys, const double *__restrict__ nu,
             double *__restrict__ g_phi, int nbr) {
    extern __shared__ double sh[];
    for (int k = threadIdx.x; k < nbr; k += blockDim.x) sh[k] = 0.0;
    __syncthreads();
    for (int hs = blockIdx.x * blockDim.x + threadIdx.x; hs < ntot; hs += gridDim.x * blockDim.x) {
        const BSys &S = a.sys[slot_sys[hs]];
        const double4 ph = a.spos[hs];
        const double nui = nu[hs];
        int n = cnt[hs];
        n = n < pair_cap ? n : pair_cap;
        for (int e = 0; e < n; ++e) {
            const int j = alist[(size_t)e * ntot + hs];
            if (!(hs < j)) continue;
            double ux, uy, uz, r;
            if (!fm_pair(S, ph, a.spos[j], a.rc2, ux, uy, uz, r)) continue;
            double w1;
            const int q = fm_weights(r, t.vp_rmin, t.vp_range, t.vp_reciprange, t.vp_recipnlkp, t.vp_recipstep,
                                     t.nlookup, w1);
            fm_hist(sh, q, nui + nu[j], w1);
        }
    }
    fm_flush(sh, g_phi, nbr);
}


struct CgVecs {
    double *X, *G, *D, *GS, *XX, *GG, *DR, *DGR;
};

// One block per system, the largest systems first (order).  On entry after
// an evaluation it finishes derivs
// (pe = sum of energy_calc energies, g = -tg f, f = pe + press vol) and runs
// VA14CD until it needs the next function value (it then leaves x set and
// marks the system active) or returns (the system is done).  Scalars are
// computed identically by every thread; vector sums use fixed-order block
// reductions.  The statement labels follow src/quench_m.F90:323-551.
__global__ void __launch_bounds__(kCgThreads)
k_cg(BSys *__restrict__ sys, CgState *__restrict__ cg, CgVecs v, const double *__restrict__ fvec,
     const double *__restrict__ en_calc, double press, int maxfn, int criterion, double fmax_tol,
     int *__restrict__ n_active, const int32_t *__restrict__ order) {
    __shared__ double sh[33];
    const int sid = order[blockIdx.x];
    BSys &S = sys[sid];
    CgState st = cg[sid];
    if (st.done) return;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int n = 3 * S.nm;            // atom variables; the nine box variables stay 0 in g and d
    const int nref = n + 9;            // N of VA14CD
    const size_t base = 3 * (size_t)S.atom0;
    double *X = v.X + base, *G = v.G + base, *D = v.D + base, *GS = v.GS + base;
    double *XX = v.XX + base, *GG = v.GG + base, *DR = v.DR + base, *DGR = v.DGR + base;
    const double dfn = 0.1, acc = 5.0e-7 * (double)S.nm;
    double c = 0.0, dtest, gamma, toplin, xold;
    int guard = 0;

    if (st.label == 0) {
        st.xnew = 0.0; st.dgstep = 0.0; st.itcrs = 0; st.maxfnk = 0; st.fmin = 0.0; st.dginit = 0.0;
        st.xmin = 0.0; st.finit = 0.0; st.gsinit = 0.0; st.gmin = 0.0; st.gm = 0.0; st.xbound = 0.0;
        st.clt = 0.0; st.gnew = 0.0; st.ggstar = 0.0; st.beta = 0.0; st.noerr = 0; st.gamden = 0.0;
        st.iflag = 0; st.iretry = -2; st.iterc = 0; st.maxfnc = 1; st.gsumsq = 0.0;
        goto CALLF;
    }
    {
        // derivs (src/quench_m.F90:215-313) for the evaluation just made
        double pe = 0.0, fm = 0.0;
        const double *tg = S.tg;
        #pragma unroll 4
        for (int i = tid; i < S.nm; i += nt) {
            const size_t at = (size_t)S.atom0 + i;
            pe += en_calc[at];
            double fx = fvec[3 * at], fy = fvec[3 * at + 1], fz = fvec[3 * at + 2];
            G[3 * i] = (-tg[0] * fx - tg[3] * fy - tg[6] * fz);
            G[3 * i + 1] = (-tg[1] * fx - tg[4] * fy - tg[7] * fz);
            G[3 * i + 2] = (-tg[2] * fx - tg[5] * fy - tg[8] * fz);
            double rx, ry, rz;
            pair_u(S.b0, fx, fy, fz, rx, ry, rz);
            fm = fmax(fm, sqrt(rx * rx + ry * ry + rz * rz));
        }
        st.pe = block_sum(pe, sh);
        st.last_fmax = block_max(fm, sh);
        st.f = st.pe + press * S.vol;
    }
    goto L190_AFTER;

L10:
    st.xnew = fabs(dfn + dfn) / st.gsumsq;
    st.dgstep = -st.gsumsq;
L20:
    st.itcrs = nref + 1;
L30:
    if (++guard > 100000) { st.iflag = 4; goto DONE; }
    if (st.maxfnk >= st.maxfnc) goto L50;
    st.f = st.fmin;
    #pragma unroll 4
    for (int i = tid; i < n; i += nt) { X[i] = XX[i]; G[i] = GG[i]; }
    __syncthreads();
L50:
    if (st.iflag > 0) goto DONE;
    if (st.itcrs <= nref) goto L70;
    #pragma unroll 4
    for (int i = tid; i < n; i += nt) D[i] = -G[i];
    __syncthreads();
L70:
    st.iterc = st.iterc + 1;
    {
        double s = 0.0;
        #pragma unroll 4
        for (int i = tid; i < n; i += nt) { GS[i] = G[i]; s += D[i] * G[i]; }
        st.dginit = block_sum(s, sh);
    }
    if (st.dginit >= 0.0) goto L320;
    st.xmin = 0.0;
    st.fmin = st.f;
    st.finit = st.f;
    st.gsinit = st.gsumsq;
    st.gmin = st.dginit;
    st.gm = st.dginit;
    st.xbound = -1.0;
    st.xnew = st.xnew * dmin(1.0, st.dgstep / st.dginit);
    st.dgstep = st.dginit;
L170:
    if (++guard > 100000) { st.iflag = 4; goto DONE; }
    c = st.xnew - st.xmin;
    {
        double s = 0.0;
        #pragma unroll 4
        for (int i = tid; i < n; i += nt) {
            X[i] = XX[i] + c * D[i];
            s += fabs(X[i] - XX[i]);
        }
        dtest = block_sum(s, sh);
    }
    if (dtest <= 0.0) st.clt = 0.7;
    if (dtest <= 0.0) goto L300;
    if (dmax(st.xbound, st.xmin - c) < 0.0) st.clt = 0.1;
    st.maxfnc = st.maxfnc + 1;
    goto CALLF;

L190_AFTER:
    if (st.maxfnc <= 1) goto L210;
    {
        double s = 0.0;
        #pragma unroll 4
        for (int i = tid; i < n; i += nt) s += D[i] * G[i];
        st.gnew = block_sum(s, sh);
    }
    if (st.f < st.fmin) goto L210;
    if (st.f > st.fmin) goto L250;
    if (fabs(st.gnew) > fabs(st.gmin)) goto L250;
L210:
    st.maxfnk = st.maxfnc;
    {
        double s = 0.0;
        #pragma unroll 4
        for (int i = tid; i < n; i += nt) s += G[i] * G[i];
        st.gsumsq = block_sum(s, sh);
    }
    if (criterion == 1 ? !(st.last_fmax <= fmax_tol) : (st.gsumsq > acc)) goto L250;
    goto DONE;
L250:
    if (st.maxfnc != maxfn) goto L270;
    st.iflag = 1;
    goto L30;
L270:
    if (st.maxfnk < st.maxfnc) goto L300;
    #pragma unroll 4
    for (int i = tid; i < n; i += nt) { XX[i] = X[i]; GG[i] = G[i]; }
    __syncthreads();
    if (st.maxfnc <= 1) goto L10;
    st.gm = st.gnew;
    if (st.gm <= st.dginit) goto L310;
    {
        double s = 0.0;
        #pragma unroll 4
        for (int i = tid; i < n; i += nt) s += GS[i] * G[i];
        st.ggstar = block_sum(s, sh);
    }
    st.beta = (st.gsumsq - st.ggstar) / (st.gm - st.dginit);
L300:
    if (fabs(st.gm) > st.clt * fabs(st.dginit)) goto L310;
    if (fabs(st.gm * st.beta) <= st.clt * st.gsumsq) goto L380;
L310:
    st.clt = st.clt + 0.3;
    if (st.clt <= 0.8) goto L340;
L320:
    st.iretry = -st.iretry;
    if (min(st.iretry, st.maxfnk) >= 2) goto L20;
    st.noerr = st.noerr + 1;
    if (st.noerr < 5) goto L20;
    st.iflag = 2;
    goto L30;
L340:
    xold = st.xnew;
    st.xnew = 0.5 * (st.xmin + xold);
    if (st.maxfnk < st.maxfnc) goto L350;
    if (st.gmin * st.gnew <= 0.0) goto L350;
    st.xnew = 10.0 * xold;
    if (st.xbound >= 0.0) st.xnew = 0.5 * (xold + st.xbound);
L350:
    toplin = (3.0 * st.gnew + st.gmin - 4.0 * (st.f - st.fmin) / (xold - st.xmin));
    c = st.gnew - toplin * (xold - st.xnew) / (xold - st.xmin);
    if (st.maxfnk < st.maxfnc) goto L360;
    if (st.gmin * st.gnew <= 0.0) st.xbound = st.xmin;
    st.xmin = xold;
    st.fmin = st.f;
    st.gmin = st.gnew;
    goto L370;
L360:
    st.xbound = xold;
L370:
    if (c * st.gmin >= 0.0) goto L170;
    st.xnew = (st.xmin * c - st.xnew * st.gmin) / (c - st.gmin);
    goto L170;
L380:
    if (dmin(st.f, st.fmin) < st.finit) goto L390;
    if (st.gsumsq >= st.gsinit) goto L320;
L390:
    if (st.itcrs >= nref) goto L420;
    if (fabs(st.ggstar) >= 0.2 * st.gsumsq) goto L420;
    {
        double s1 = 0.0, s2 = 0.0;
        #pragma unroll 4
        for (int i = tid; i < n; i += nt) { s1 += GG[i] * DGR[i]; s2 += GG[i] * DR[i]; }
        gamma = block_sum(s1, sh);
        c = block_sum(s2, sh);
    }
    gamma = gamma / st.gamden;
    if (fabs(st.beta * st.gm + gamma * c) >= 0.2 * st.gsumsq) goto L420;
    #pragma unroll 4
    for (int i = tid; i < n; i += nt) D[i] = -GG[i] + st.beta * D[i] + gamma * DR[i];
    __syncthreads();
    st.itcrs = st.itcrs + 1;
    goto L30;
L420:
    st.itcrs = 2;
    st.gamden = st.gm - st.dginit;
    #pragma unroll 4
    for (int i = tid; i < n; i += nt) {
        DR[i] = D[i];
        DGR[i] = GG[i] - GS[i];
        D[i] = -GG[i] + st.beta * D[i];
    }
    __syncthreads();
    goto L30;

CALLF:
    __syncthreads();
    if (tid == 0) {
        st.label = 1;
        cg[sid] = st;
        S.active = 1;
        atomicAdd(n_active, 1);
    }
    return;
DONE:
    __syncthreads();
    if (tid == 0) {
        st.done = 1;
        cg[sid] = st;
        S.active = 0;
    }
}

// deinterleaved copy of the variables x(3i-2..3i) <-> x0, y0, z0
__global__ void k_pack(int ntot, const double *__restrict__ x, const double *__restrict__ y,
                       const double *__restrict__ z, double *__restrict__ X) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= ntot) return;
    X[3 * (size_t)a] = x[a]; X[3 * (size_t)a + 1] = y[a]; X[3 * (size_t)a + 2] = z[a];
}

__global__ void k_unpack(int ntot, const double *__restrict__ X, double *__restrict__ x, double *__restrict__ y,
                         double *__restrict__ z) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= ntot) return;
    x[a] = X[3 * (size_t)a]; y[a] = X[3 * (size_t)a + 1]; z[a] = X[3 * (size_t)a + 2];
}

// marks every system active (v) and, with stale, its list invalid
__global__ void k_set_active(int nsys, BSys *sys, int v, int stale) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    sys[s].active = v;
    if (stale) sys[s].stale = 1;
}

}  // namespace

constexpr int kTileCapMax = kTileCap;

// =============================================================== engine ====
class BatchEngine {
  public:
    int nsys = 0, ntot = 0, ncell = 0, device = 0;
    double press = 0.0;
    int lph = 8;                        // lanes per home atom in the tile screen
    int gather = 4;                     // row entries a thread gathers at a time in the per-atom passes
    bool mixed = false;                 // FP32 separations, tables and pair forces in the per-atom passes
    int nsm = 148;
    int cap = kTileCap;                 // staged candidates per warp
    std::vector<int> natoms, atom0;
    std::vector<BSys> hsys;
    HostTables ht;
    Tables tab;
    double rcut = 0.0;
    double skin = 0.3;                  // list radius rcut + skin (less where a box is too narrow)
    bool potential_set = false, state_set = false, boxes_set = false, pos_set = false;
    cudaStream_t stream = nullptr;
    // device buffers
    BSys *sys = nullptr;
    int32_t *atom_sys = nullptr, *cell_sys = nullptr, *cell_of = nullptr, *cell_count = nullptr;
    int32_t *cell_start = nullptr, *cursor = nullptr, *sorted = nullptr, *n_active = nullptr;
    double *X = nullptr, *Xb = nullptr, *mass = nullptr, *f = nullptr, *rho = nullptr, *afrho = nullptr, *fp = nullptr;
    double *en_calc = nullptr, *en_force = nullptr, *vir = nullptr, *sfp = nullptr, *sysout = nullptr;
    double *cgv = nullptr;              // G, D, GS, XX, GG, DR, DGR (3*ntot each)
    int32_t *alist = nullptr, *pcnt = nullptr, *flags = nullptr;
    unsigned long long *stats = nullptr;   // system list builds, system evaluations
    int32_t *todo = nullptr, *ntodo = nullptr;   // cells of the systems rebuilt in this evaluation
    int32_t *cg_order = nullptr;                 // systems by descending size
    int pair_cap = 48;                  // compact-row entries per atom
    double4 *spos = nullptr;
    CgState *cg = nullptr;
    double4 *tab_r4 = nullptr;
    double2 *tab_e2 = nullptr;
    float4 *tab_r4f = nullptr;
    float2 *tab_e2f = nullptr;
    void *tab_aux = nullptr;
    double *stage = nullptr;            // host-to-device staging (3*ntot)
    int *host_active = nullptr;         // pinned
    cudaGraphExec_t graph = nullptr;
    int graph_lph = -1, graph_cap = -1, graph_maxfn = -1, graph_criterion = -1, graph_gather = -1;
    double graph_fmax = -1.0;
    long long launches = 0;

    ~BatchEngine();
    int init(int n, const int32_t *na, double p, int dev);
    int set_fetm(int nv, const double *av, const double *rv, int np, const double *ap, const double *rp,
                 int nlookup);
    int set_state(const double *x0, const double *y0, const double *z0, const double *b0, const double *m);
    int layout();
    int set_skin(double sk);
    int get_state(double *x0, double *y0, double *z0);
    int force(double *out13);
    int quench(int maxfn, int criterion, double fmax, double *out8);
    int autotune(int nreps, double *times_ms, int32_t *chosen);
    // force matching: references (device), dL/dF in cell order, dL/dsigma,
    // per-system loss, mu, nu and the six table gradients; allocated on first use
    double *fm_fref = nullptr, *fm_sref = nullptr, *fm_gF = nullptr, *fm_gS = nullptr, *fm_loss = nullptr;
    double *fm_mu = nullptr, *fm_nu = nullptr, *fm_grads = nullptr;
    int fm_nb = 0;
    bool fm_refs = false;
    int set_references(const double *fref_xyz, const double *sref);
    int force_matching(double wf, double ws, double *loss, double *grads);
    int get_array(const double *dev, int stride, double *a, double *b, double *c);
    int copy_xyz(double *dev, const double *src, double *dst);
    // ecalc: also energy_calc's per-atom energies (exact pair function), which
    // the quench needs and a plain force evaluation only when asked
    // ev (5 events, may be null): recorded before k_prepare, the tile screen,
    // the density pass and the force pass, and after the force pass
    void queue_evaluation(bool with_vir, bool use_mixed, bool ecalc, cudaEvent_t *ev = nullptr);
    int kernel_times(int rebuild, double *ms4);
    bool ecalc = true;                  // moldy_gpu_batch_force computes energy_calc's energies
    int ready();
    int take_overflow();
    // persistent evaluation (k_batch_eval): one launch per force call in
    // mixed precision without energy_calc, when every atom is heavier than
    // 0.05 and the largest system's records fit in shared memory
    bool persistent = true;             // use it where it applies
    int lpa = 2;                        // lanes per atom in its passes (1, 2, 4)
    bool all_heavy = true;
    int max_atoms = 0;
    size_t smem_optin = 0;
    int32_t *queue = nullptr;           // [0] next system, [1] blocks done
    bool en_calc_zero = false;          // en_calc holds zeros (no energy_calc since the last clear)
    int eval_grid = 0;                  // resident blocks of the persistent launch
    // the force evaluation's launches (activity flags, persistent evaluation)
    // captured once and replayed; recaptured when a choice or a buffer changes
    cudaGraphExec_t fgraph = nullptr;
    int fg_lph = -1, fg_lpa = -1, fg_cap = -1;
    void drop_force_graph() {
        if (fgraph) { cudaGraphExecDestroy(fgraph); fgraph = nullptr; }
    }
    int eval_prepare();
    size_t eval_smem() const {
        return std::max((size_t)max_atoms * sizeof(int4), (size_t)kEvalWarps * (size_t)cap * (sizeof(double4) + sizeof(int)));
    }
    bool persistent_applies() const {
        return persistent && mixed && !ecalc && all_heavy && eval_smem() + 8192 <= smem_optin;
    }
    int queue_persistent(bool prepare = true);
    int eval_times(double *ms2);
    int evaluate_once(bool with_reduce);
};

#define BCHECK(call)                                                      \
    do {                                                                  \
        int rc_ = (call);                                                 \
        if (rc_ != MOLDY_OK) return rc_;                                  \
    } while (0)
#define BCUDA(call, what)                                                 \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) {                                          \
            cudaGetLastError();                                           \
            return set_last_error(MOLDY_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
        }                                                                 \
    } while (0)

template <typename T>
static int balloc(T **p, size_t n, const char *what) {
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return set_last_error(MOLDY_ERR_CUDA, std::string("cudaMalloc ") + what + ": " + cudaGetErrorString(e));
    }
    return MOLDY_OK;
}

BatchEngine::~BatchEngine() {
    cudaSetDevice(device);
    if (graph) cudaGraphExecDestroy(graph);
    drop_force_graph();
    void *bufs[] = {sys, atom_sys, cell_sys, cell_of, cell_count, cell_start, cursor, sorted, n_active, X, Xb,
                    mass, f, rho, afrho, fp, en_calc, en_force, vir, sfp, sysout, cgv, spos, cg, tab_r4, tab_e2,
                    tab_r4f, tab_e2f, tab_aux, stage, alist, pcnt, flags, stats, todo, ntodo, cg_order,
                    fm_fref, fm_sref, fm_gF, fm_gS, fm_loss, fm_mu, fm_nu, fm_grads, queue};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (host_active) cudaFreeHost(host_active);
    if (stream) cudaStreamDestroy(stream);
}

int BatchEngine::init(int n, const int32_t *na, double p, int dev) {
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_last_error(MOLDY_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    if (dev < 0 || dev >= ndev) return set_last_error(MOLDY_ERR_INVALID, "device ordinal out of range");
    BCUDA(cudaSetDevice(dev), "cudaSetDevice");
    cudaDeviceProp prop;
    BCUDA(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
    if (prop.major != 10) return set_last_error(MOLDY_ERR_NO_DEVICE, "kernels are built for sm_100a only");
    device = dev;
    nsm = prop.multiProcessorCount;
    smem_optin = prop.sharedMemPerBlockOptin;
    nsys = n;
    press = p;
    natoms.assign(na, na + n);
    atom0.resize(n);
    long long tot = 0;
    for (int s = 0; s < n; ++s) {
        if (na[s] < 2) return set_last_error(MOLDY_ERR_INVALID, "every system needs at least 2 atoms");
        atom0[s] = (int)tot;
        tot += na[s];
    }
    if (tot > (1LL << 28)) return set_last_error(MOLDY_ERR_CAPACITY, "more than 2^28 atoms in one batch");
    ntot = (int)tot;
    max_atoms = *std::max_element(na, na + n);
    BCUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
    size_t nt = (size_t)ntot;
    BCHECK(balloc(&sys, n, "systems"));
    BCHECK(balloc(&atom_sys, nt, "atom_sys"));
    BCHECK(balloc(&cell_of, nt, "cell_of"));
    BCHECK(balloc(&sorted, nt, "sorted"));
    BCHECK(balloc(&n_active, 1, "n_active"));
    BCHECK(balloc(&X, 3 * nt, "X"));
    BCHECK(balloc(&Xb, 3 * nt, "build positions"));
    BCHECK(balloc(&mass, nt, "mass"));
    BCHECK(balloc(&f, 3 * nt, "f"));
    BCHECK(balloc(&rho, nt, "rho"));
    BCHECK(balloc(&afrho, nt, "afrho"));
    BCHECK(balloc(&fp, nt, "fp"));
    BCHECK(balloc(&en_calc, nt, "en_calc"));
    BCHECK(balloc(&en_force, nt, "en_force"));
    BCHECK(balloc(&vir, 6 * nt, "virial moments"));
    BCHECK(balloc(&sfp, nt, "sfp"));
    BCHECK(balloc(&spos, nt, "spos"));
    BCHECK(balloc(&sysout, 13 * (size_t)n, "system results"));
    BCHECK(balloc(&cgv, 7 * 3 * nt, "CG vectors"));
    BCHECK(balloc(&cg, n, "CG state"));
    BCHECK(balloc(&stage, 3 * nt, "staging"));
    BCHECK(balloc(&alist, nt * (size_t)pair_cap, "compact list"));
    BCHECK(balloc(&pcnt, nt, "compact counts"));
    BCHECK(balloc(&flags, 2, "flags"));
    BCUDA(cudaMemset(flags, 0, 2 * sizeof(int32_t)), "flags");
    BCHECK(balloc(&stats, 2, "list statistics"));
    BCHECK(balloc(&ntodo, 1, "screen work count"));
    BCHECK(balloc(&queue, 2, "system queue"));
    BCUDA(cudaMemset(queue, 0, 2 * sizeof(int32_t)), "system queue");
    BCUDA(cudaMemset(ntodo, 0, sizeof(int32_t)), "screen work count");
    BCUDA(cudaMemset(stats, 0, 2 * sizeof(unsigned long long)), "list statistics");
    BCUDA(cudaMallocHost((void **)&host_active, sizeof(int)), "pinned");
    std::vector<int32_t> as(nt);
    for (int s = 0; s < n; ++s)
        for (int i = 0; i < na[s]; ++i) as[atom0[s] + i] = s;
    BCUDA(cudaMemcpy(atom_sys, as.data(), nt * sizeof(int32_t), cudaMemcpyHostToDevice), "atom_sys");
    std::vector<int32_t> ord(n);
    for (int k = 0; k < n; ++k) ord[k] = k;
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return na[x] > na[y]; });
    BCHECK(balloc(&cg_order, n, "system order"));
    BCUDA(cudaMemcpy(cg_order, ord.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice), "system order");
    std::vector<double> m(nt, 55.845);
    BCUDA(cudaMemcpy(mass, m.data(), nt * sizeof(double), cudaMemcpyHostToDevice), "mass");
    hsys.assign(n, BSys());
    return MOLDY_OK;
}

int BatchEngine::set_fetm(int nv, const double *av, const double *rv, int np, const double *ap, const double *rp,
                          int nlookup) {
    if (!av || !rv || !ap || !rp) return set_last_error(MOLDY_ERR_INVALID, "null coefficient pointer");
    int rc = build_fetm_tables(ht, nv, av, rv, np, ap, rp, 1, nlookup);
    if (rc != MOLDY_OK) return set_last_error(rc, "FETRANSMETAL set-up failed");
    double rcull = 0.0;
    BCHECK(upload_device_tables(ht, &tab_r4, &tab_r4f, &tab_e2, &tab_e2f, &tab_aux, tab, &rcull));
    drop_force_graph();   // the graph holds the table descriptor and the cut
    // every pair beyond the table cut and the pair function's knots contributes zero
    double r = rcull < 1e150 ? rcull : 0.0;
    for (int i = 0; i < nv; ++i) r = std::max(r, rv[i] * (1.0 + 1e-12));
    if (!(r > 0.0) || r > 1e100) return set_last_error(MOLDY_ERR_UNSUPPORTED, "tables without a finite cut");
    rcut = r;
    potential_set = true;
    if (boxes_set) return layout();
    return MOLDY_OK;
}

int BatchEngine::set_state(const double *x0, const double *y0, const double *z0, const double *b0,
                           const double *m) {
    if (!potential_set) return set_last_error(MOLDY_ERR_ORDER, "set the potential before the state");
    size_t nt = (size_t)ntot;
    if (x0 && y0 && z0) {
        BCUDA(cudaMemcpyAsync(stage, x0, nt * sizeof(double), cudaMemcpyHostToDevice, stream), "x0");
        BCUDA(cudaMemcpyAsync(stage + nt, y0, nt * sizeof(double), cudaMemcpyHostToDevice, stream), "y0");
        BCUDA(cudaMemcpyAsync(stage + 2 * nt, z0, nt * sizeof(double), cudaMemcpyHostToDevice, stream), "z0");
        k_pack<<<(ntot + 255) / 256, 256, 0, stream>>>(ntot, stage, stage + nt, stage + 2 * nt, X);
    }
    if (m) {
        BCUDA(cudaMemcpyAsync(mass, m, nt * sizeof(double), cudaMemcpyHostToDevice, stream), "mass");
        all_heavy = *std::min_element(m, m + nt) > 0.05;
    }
    if (b0) {
        for (int s = 0; s < nsys; ++s) {
            BSys &S = hsys[s];
            const double *b = b0 + 9 * (size_t)s;
            for (int k = 0; k < 9; ++k) S.b0[k] = b[k];
            double vol = b[0] * (b[4] * b[8] - b[7] * b[5]) + b[1] * (b[5] * b[6] - b[3] * b[8]) +
                         b[2] * (b[3] * b[7] - b[4] * b[6]);
            if (!(std::fabs(vol) > 0.0)) return set_last_error(MOLDY_ERR_SINGULAR_BOX, "singular box");
            S.vol = vol;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double t = 0.0;
                    for (int k = 0; k < 3; ++k) t += b[k + 3 * i] * b[k + 3 * j];
                    S.tg[i + 3 * j] = t;
                }
        }
        boxes_set = true;
        BCHECK(layout());
    }
    if (x0 && y0 && z0) pos_set = true;
    state_set = pos_set && boxes_set;
    BCUDA(cudaStreamSynchronize(stream), "set_state");
    BCUDA(cudaGetLastError(), "set_state");
    return MOLDY_OK;
}

// Per-system list radius and cell grid from the boxes: rv = rcut + skin,
// less where a box is narrower than 2 rv (every pair inside rv must have a
// unique minimum image), and cells at least rv wide perpendicular to each
// face.  Every list is marked stale.
int BatchEngine::layout() {
    int cell = 0;
    std::vector<int32_t> csys;
    for (int s = 0; s < nsys; ++s) {
        BSys &S = hsys[s];
        const double *b = S.b0;
        double w[3];
        for (int d = 0; d < 3; ++d) {
            const double *p = b + 3 * ((d + 1) % 3), *q = b + 3 * ((d + 2) % 3);
            double cx = p[1] * q[2] - p[2] * q[1], cy = p[2] * q[0] - p[0] * q[2], cz = p[0] * q[1] - p[1] * q[0];
            w[d] = std::fabs(S.vol) / std::sqrt(cx * cx + cy * cy + cz * cz);
            if (!(w[d] > 2.0 * rcut))
                return set_last_error(MOLDY_ERR_INVALID, "system " + std::to_string(s) +
                                                             ": box narrower than twice the interaction range");
        }
        const double wmin = std::min(w[0], std::min(w[1], w[2]));
        const double rv = std::max(rcut, std::min(rcut + skin, 0.5 * wmin * (1.0 - 1e-9)));
        const double half = 0.5 * (rv - rcut);
        S.rv2 = rv * rv;
        // a small margin keeps rounding in the displacement from hiding a crossing
        S.hs2 = half * half * (1.0 - 1e-6);
        for (int d = 0; d < 3; ++d) {
            int nc = (int)std::floor(w[d] / rv);
            nc = std::max(1, std::min(nc, 1024));
            S.nc[d] = nc;
            S.nst[d] = nc >= 3 ? 3 : nc;
        }
        S.atom0 = atom0[s];
        S.nm = natoms[s];
        S.cell0 = cell;
        S.ncell = S.nc[0] * S.nc[1] * S.nc[2];
        S.active = 1;
        S.rebuild = 0;
        S.stale = 1;
        cell += S.ncell;
        csys.insert(csys.end(), S.ncell, s);
    }
    if (cell != ncell) {
        void *bufs[] = {cell_sys, cell_count, cell_start, cursor, todo};
        for (void *bp : bufs)
            if (bp) cudaFree(bp);
        cell_sys = cell_count = cell_start = cursor = todo = nullptr;
        ncell = cell;
        BCHECK(balloc(&todo, ncell, "screen work"));
        BCHECK(balloc(&cell_sys, ncell, "cell_sys"));
        BCHECK(balloc(&cell_count, ncell, "cell_count"));
        BCHECK(balloc(&cell_start, ncell + 1, "cell_start"));
        BCHECK(balloc(&cursor, ncell, "cursor"));
        if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
        drop_force_graph();
    }
    BCUDA(cudaMemsetAsync(cell_count, 0, ncell * sizeof(int32_t), stream), "cell_count");
    // every build writes atom0 as the first slot of a system's first cell, and
    // the end of a system's last cell is the next system's first slot
    std::vector<int32_t> cs(ncell + 1, 0);
    for (int s = 0; s < nsys; ++s) cs[hsys[s].cell0] = atom0[s];
    cs[ncell] = ntot;
    BCUDA(cudaMemcpyAsync(cell_start, cs.data(), cs.size() * sizeof(int32_t), cudaMemcpyHostToDevice, stream),
          "cell_start");
    BCUDA(cudaMemcpyAsync(cell_sys, csys.data(), csys.size() * sizeof(int32_t), cudaMemcpyHostToDevice, stream),
          "cell_sys");
    BCUDA(cudaMemcpyAsync(sys, hsys.data(), nsys * sizeof(BSys), cudaMemcpyHostToDevice, stream), "systems");
    BCUDA(cudaStreamSynchronize(stream), "layout");
    return MOLDY_OK;
}

int BatchEngine::set_skin(double sk) {
    if (!(sk >= 0.0) || sk > 10.0) return set_last_error(MOLDY_ERR_INVALID, "skin must be in [0, 10]");
    skin = sk;
    if (boxes_set) return layout();
    return MOLDY_OK;
}

int BatchEngine::ready() {
    if (!potential_set) return set_last_error(MOLDY_ERR_ORDER, "the potential is not set");
    if (!state_set) return set_last_error(MOLDY_ERR_ORDER, "positions and boxes are not set");
    return MOLDY_OK;
}

template <int LPH>
static void launch_screen(const BatchEngine &E, const TileArgs &a, cudaStream_t s) {
    // a persistent grid over the cells of the rebuilt systems (6 blocks of
    // 37 KB shared memory fit one SM)
    const int nb = std::max(1, std::min((E.ncell + kTileWarps - 1) / kTileWarps, 6 * E.nsm));
    k_tile_screen<LPH><<<nb, 32 * kTileWarps, 0, s>>>(a, E.ntot, E.pair_cap, E.alist, E.pcnt, E.flags, E.todo,
                                                     E.ntodo);
}

template <bool MIXED, int B>
static void launch_passes(const BatchEngine &E, const TileArgs &a, bool with_vir, bool ecalc, cudaStream_t s,
                          cudaEvent_t *ev) {
    const int nbs = grid_blocks(E.ntot, 256);
    // a system's slots are its atoms' index range, so atom_sys is the slot's system
    if (ecalc)
        k_cl_density<MIXED, B, true><<<nbs, 256, 0, s>>>(a, E.tab, E.ntot, E.pair_cap, E.alist, E.pcnt, E.sfp,
                                                         E.rho, E.afrho, E.fp, E.en_calc, E.atom_sys, E.ntodo);
    else
        k_cl_density<MIXED, B, false><<<nbs, 256, 0, s>>>(a, E.tab, E.ntot, E.pair_cap, E.alist, E.pcnt, E.sfp,
                                                          E.rho, E.afrho, E.fp, E.en_calc, E.atom_sys, E.ntodo);
    if (ev) cudaEventRecord(ev[3], s);
    if (with_vir)
        k_cl_forces<MIXED, B, true><<<nbs, 256, 0, s>>>(a, E.tab, E.ntot, E.pair_cap, E.alist, E.pcnt, E.atom_sys,
                                                        E.afrho, E.f, E.en_force, E.vir);
    else
        k_cl_forces<MIXED, B, false><<<nbs, 256, 0, s>>>(a, E.tab, E.ntot, E.pair_cap, E.alist, E.pcnt, E.atom_sys,
                                                         E.afrho, E.f, E.en_force, E.vir);
}

template <bool MIXED>
static void launch_passes_b(const BatchEngine &E, const TileArgs &a, bool with_vir, bool ecalc, cudaStream_t s,
                            cudaEvent_t *ev) {
    switch (E.gather) {
        case 1: launch_passes<MIXED, 1>(E, a, with_vir, ecalc, s, ev); break;
        case 2: launch_passes<MIXED, 2>(E, a, with_vir, ecalc, s, ev); break;
        default: launch_passes<MIXED, 4>(E, a, with_vir, ecalc, s, ev); break;
    }
}

// list check (and rebuild) and the tile passes for the systems marked active
void BatchEngine::queue_evaluation(bool with_vir, bool use_mixed, bool ecalc, cudaEvent_t *ev) {
    cudaStream_t s = stream;
    if (ecalc) en_calc_zero = false;
    if (ev) cudaEventRecord(ev[0], s);
    k_prepare<<<nsys, kPrepThreads, 0, s>>>(sys, X, mass, Xb, cell_of, cell_count, cell_start, cursor, sorted, spos,
                                           stats, todo, ntodo);
    if (ev) cudaEventRecord(ev[1], s);
    TileArgs a;
    a.sys = sys; a.cell_sys = cell_sys; a.cell_start = cell_start; a.sorted = sorted;
    a.spos = spos; a.sfp = sfp; a.ncell = ncell; a.cap = cap; a.rc2 = rcut * rcut;
    switch (lph) {
        case 4: launch_screen<4>(*this, a, s); break;
        case 16: launch_screen<16>(*this, a, s); break;
        case 32: launch_screen<32>(*this, a, s); break;
        default: launch_screen<8>(*this, a, s); break;
    }
    if (ev) cudaEventRecord(ev[2], s);
    if (use_mixed)
        launch_passes_b<true>(*this, a, with_vir, ecalc, s, ev);
    else
        launch_passes_b<false>(*this, a, with_vir, ecalc, s, ev);
    if (ev) cudaEventRecord(ev[4], s);
    launches += 4;
}

// compact-row overflow of the last evaluations: grows the rows, marks every
// list stale (the caller evaluates again) and returns the largest row seen,
// or 0
int BatchEngine::take_overflow() {
    int32_t h[2] = {0, 0};
    if (cudaMemcpy(h, flags, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    if (!h[0]) return 0;
    cudaMemset(flags, 0, sizeof(h));
    int need = h[1] + 8;
    if (alist) cudaFree(alist);
    alist = nullptr;
    if (balloc(&alist, (size_t)ntot * (size_t)need, "compact list") != MOLDY_OK) return -1;
    pair_cap = need;
    if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
    drop_force_graph();
    k_set_active<<<(nsys + 255) / 256, 256, 0, stream>>>(nsys, sys, 1, 1);
    if (cudaStreamSynchronize(stream) != cudaSuccess) return -1;
    return h[1];
}

// The launches of one force evaluation of every system: the persistent
// launch where it applies (captured with the activity flags in a graph and
// replayed), else the list check, tile screen, per-atom passes and
// (with_reduce) the per-system sums
int BatchEngine::evaluate_once(bool with_reduce) {
    if (!ecalc && !en_calc_zero) {
        BCUDA(cudaMemsetAsync(en_calc, 0, (size_t)ntot * sizeof(double), stream), "en_calc");
        en_calc_zero = true;
    }
    if (ecalc) en_calc_zero = false;
    if (persistent_applies()) {
        if (!fgraph || fg_lph != lph || fg_lpa != lpa || fg_cap != cap) {
            drop_force_graph();
            BCHECK(eval_prepare());
            cudaGraph_t g = nullptr;
            BCUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "capture");
            k_set_active<<<(nsys + 255) / 256, 256, 0, stream>>>(nsys, sys, 1, 0);
            const int rc = queue_persistent(false);
            cudaError_t e = cudaStreamEndCapture(stream, &g);
            if (rc != MOLDY_OK || e != cudaSuccess) {
                cudaGetLastError();
                if (g) cudaGraphDestroy(g);
                return rc != MOLDY_OK ? rc
                                      : set_last_error(MOLDY_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
            }
            e = cudaGraphInstantiate(&fgraph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                cudaGetLastError();
                fgraph = nullptr;
                return set_last_error(MOLDY_ERR_CUDA, std::string("graph: ") + cudaGetErrorString(e));
            }
            fg_lph = lph; fg_lpa = lpa; fg_cap = cap;
            launches -= 1;   // captured, not run; counted per replay below
        }
        BCUDA(cudaGraphLaunch(fgraph, stream), "graph launch");
        launches += 2;
        return MOLDY_OK;
    }
    k_set_active<<<(nsys + 255) / 256, 256, 0, stream>>>(nsys, sys, 1, 0);
    ++launches;
    queue_evaluation(true, mixed, ecalc);
    if (with_reduce) {
        k_sys_reduce<<<nsys, kCgThreads, 0, stream>>>(sys, en_calc, en_force, vir, f, 1, sysout);
        ++launches;
    }
    return MOLDY_OK;
}

using EvalKernel = void (*)(EvalArgs, Tables);

template <int LPH>
static EvalKernel eval_kernel_l(int lpa) {
    return lpa == 1 ? k_batch_eval<LPH, 1> : (lpa == 4 ? k_batch_eval<LPH, 4> : k_batch_eval<LPH, 2>);
}

// the instantiation for the tile screen's lanes per home atom (4 runs as 8)
// and the lanes per atom
static EvalKernel eval_kernel(int lph, int lpa) {
    switch (lph) {
        case 16: return eval_kernel_l<16>(lpa);
        case 32: return eval_kernel_l<32>(lpa);
        default: return eval_kernel_l<8>(lpa);
    }
}

// shared memory opt-in and resident grid of the current instantiation
int BatchEngine::eval_prepare() {
    EvalKernel kern = eval_kernel(lph, lpa);
    const size_t smem = eval_smem();
    BCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "eval smem");
    int per_sm = 0;
    BCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kEvalThreads, smem), "eval occupancy");
    eval_grid = std::max(1, std::min(nsys, std::max(1, per_sm) * nsm));
    return MOLDY_OK;
}

int BatchEngine::queue_persistent(bool prepare) {
    if (prepare) BCHECK(eval_prepare());
    EvalArgs a;
    a.sys = sys; a.order = cg_order; a.nsys = nsys; a.ntot = ntot; a.pair_cap = pair_cap; a.queue = queue;
    a.X = X; a.mass = mass; a.Xb = Xb; a.cell_of = cell_of; a.cell_count = cell_count; a.cell_start = cell_start;
    a.cursor = cursor; a.sorted = sorted; a.spos = spos; a.stats = stats; a.cell_sys = cell_sys;
    a.alist = alist; a.pcnt = pcnt; a.flags = flags; a.ncell = ncell; a.cap = cap; a.rc2 = rcut * rcut;
    a.f = f; a.rho = rho; a.afrho = afrho; a.fp = fp; a.en_force = en_force; a.sysout = sysout;
    eval_kernel(lph, lpa)<<<eval_grid, kEvalThreads, eval_smem(), stream>>>(a, tab);
    ++launches;
    return MOLDY_OK;
}

// Device times of the persistent evaluation: ms2[0] with every list current,
// ms2[1] with every list rebuilt (binning and compact rows in the same launch)
int BatchEngine::eval_times(double *ms2) {
    BCHECK(ready());
    if (!persistent_applies())
        return set_last_error(MOLDY_ERR_UNSUPPORTED, "the persistent evaluation does not apply (FP64, energy_calc, "
                                                     "an atom of mass <= 0.05, or a system too large)");
    cudaEvent_t e0, e1;
    BCUDA(cudaEventCreate(&e0), "event");
    BCUDA(cudaEventCreate(&e1), "event");
    for (int r = 0; r < 2; ++r) {
        k_set_active<<<(nsys + 255) / 256, 256, 0, stream>>>(nsys, sys, 1, r);
        ++launches;
        cudaEventRecord(e0, stream);
        BCHECK(queue_persistent());
        cudaEventRecord(e1, stream);
        BCUDA(cudaEventSynchronize(e1), "eval times");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms2) ms2[r] = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    BCUDA(cudaGetLastError(), "eval times");
    if (take_overflow() != 0) return set_last_error(MOLDY_ERR_CAPACITY, "compact rows grew; time again");
    return MOLDY_OK;
}

int BatchEngine::force(double *out13) {
    BCHECK(ready());
    for (int attempt = 0;; ++attempt) {
        BCHECK(evaluate_once(true));
        BCUDA(cudaStreamSynchronize(stream), "batch force");
        BCUDA(cudaGetLastError(), "batch force");
        int ov = take_overflow();
        if (ov < 0) return set_last_error(MOLDY_ERR_CUDA, "compact list re-allocation failed");
        if (ov == 0) break;
        if (attempt >= 2) return set_last_error(MOLDY_ERR_CAPACITY, "compact list keeps overflowing");
    }
    if (out13)
        BCUDA(cudaMemcpy(out13, sysout, 13 * (size_t)nsys * sizeof(double), cudaMemcpyDeviceToHost), "results");
    return MOLDY_OK;
}

// Chooses the tile shape and the gather width on the live configuration:
// the lanes per home atom of the tile screen (4, 8, 16, 32) by evaluations
// that rebuild every list, then the row entries gathered at a time by the
// per-atom passes (1, 2, 4) by evaluations with current lists, then, where
// the persistent evaluation applies, its lanes per atom (1, 2, 4), each the
// mean of nreps evaluations in the current precision.  times_ms (10 values)
// gets those means in that order, chosen (3 values) the choice (lanes per
// atom 0 when not tuned).  Positions and boxes are left as they were; the
// lists are current afterwards.
int BatchEngine::autotune(int nreps, double *times_ms, int32_t *chosen) {
    BCHECK(ready());
    if (nreps < 1) nreps = 1;
    cudaEvent_t e0, e1;
    BCUDA(cudaEventCreate(&e0), "event");
    BCUDA(cudaEventCreate(&e1), "event");
    auto evaluate = [&](bool rebuild) {
        k_set_active<<<(nsys + 255) / 256, 256, 0, stream>>>(nsys, sys, 1, rebuild ? 1 : 0);
        queue_evaluation(true, mixed, ecalc);
        k_sys_reduce<<<nsys, kCgThreads, 0, stream>>>(sys, en_calc, en_force, vir, f, 1, sysout);
        launches += 3;
    };
    auto timed = [&](bool rebuild) -> double {
        double total = 0.0;
        for (int r = 0; r < nreps; ++r) {
            if (rebuild) k_set_active<<<(nsys + 255) / 256, 256, 0, stream>>>(nsys, sys, 1, 1);
            cudaEventRecord(e0, stream);
            evaluate(false);
            cudaEventRecord(e1, stream);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            total += ms;
        }
        return total / nreps;
    };
    const int lanes[4] = {4, 8, 16, 32}, gathers[3] = {1, 2, 4};
    double t[7];
    evaluate(true);   // rows sized before timing
    BCUDA(cudaStreamSynchronize(stream), "autotune");
    if (take_overflow() < 0) return set_last_error(MOLDY_ERR_CUDA, "compact list re-allocation failed");
    int bl = 0;
    for (int k = 0; k < 4; ++k) {
        lph = lanes[k];
        t[k] = timed(true);
        if (t[k] < t[bl]) bl = k;
    }
    lph = lanes[bl];
    evaluate(true);
    int bg = 0;
    for (int k = 0; k < 3; ++k) {
        gather = gathers[k];
        t[4 + k] = timed(false);
        if (t[4 + k] < t[4 + bg]) bg = k;
    }
    gather = gathers[bg];
    // lanes per atom of the persistent evaluation (lists current)
    double tp[3] = {0.0, 0.0, 0.0};
    const bool pers = persistent_applies();
    if (pers) {
        const int lanes_a[3] = {1, 2, 4};
        int bp = 0;
        for (int k = 0; k < 3; ++k) {
            lpa = lanes_a[k];
            // one untimed launch first: the variant's first launch also loads it
            k_set_active<<<(nsys + 255) / 256, 256, 0, stream>>>(nsys, sys, 1, 0);
            ++launches;
            BCHECK(queue_persistent());
            double total = 0.0;
            for (int r = 0; r < nreps; ++r) {
                k_set_active<<<(nsys + 255) / 256, 256, 0, stream>>>(nsys, sys, 1, 0);
                ++launches;
                cudaEventRecord(e0, stream);
                BCHECK(queue_persistent());
                cudaEventRecord(e1, stream);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                total += ms;
            }
            tp[k] = total / nreps;
            if (tp[k] < tp[bp]) bp = k;
        }
        lpa = lanes_a[bp];
    }
    if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    BCUDA(cudaStreamSynchronize(stream), "autotune");
    BCUDA(cudaGetLastError(), "autotune");
    if (take_overflow() != 0) return set_last_error(MOLDY_ERR_CAPACITY, "compact rows grew during tuning; run again");
    if (times_ms) {
        for (int k = 0; k < 7; ++k) times_ms[k] = t[k];
        for (int k = 0; k < 3; ++k) times_ms[7 + k] = tp[k];
    }
    if (chosen) { chosen[0] = lph; chosen[1] = gather; chosen[2] = pers ? lpa : 0; }
    return MOLDY_OK;
}

// Reference real forces (interleaved x, y, z per atom, atom order) and
// stresses (9 per system, sigma(i,j) at i + 3 j) for force_matching.
int BatchEngine::set_references(const double *fref_xyz, const double *sref) {
    if (!fref_xyz || !sref) return set_last_error(MOLDY_ERR_INVALID, "null reference array");
    const size_t nt = (size_t)ntot;
    if (!fm_fref) {
        BCHECK(balloc(&fm_fref, 3 * nt, "reference forces"));
        BCHECK(balloc(&fm_sref, 9 * (size_t)nsys, "reference stresses"));
        BCHECK(balloc(&fm_gF, 3 * nt, "dL/dF"));
        BCHECK(balloc(&fm_gS, 9 * (size_t)nsys, "dL/dsigma"));
        BCHECK(balloc(&fm_loss, nsys, "loss"));
        BCHECK(balloc(&fm_mu, nt, "mu"));
        BCHECK(balloc(&fm_nu, nt, "nu"));
    }
    BCUDA(cudaMemcpyAsync(fm_fref, fref_xyz, 3 * nt * sizeof(double), cudaMemcpyHostToDevice, stream), "references");
    BCUDA(cudaMemcpyAsync(fm_sref, sref, 9 * (size_t)nsys * sizeof(double), cudaMemcpyHostToDevice, stream),
          "references");
    BCUDA(cudaStreamSynchronize(stream), "references");
    fm_refs = true;
    return MOLDY_OK;
}

// One FP64 evaluation of every system, the loss
//   L_s = w_f sum_i |F_i - F_i^ref|^2 + w_s |sigma_s - sigma_s^ref|^2
// per system into loss[nsys], and dL/d(table) of L = sum_s L_s into
// grads[6 (nlookup + 1)] (vee, dvee, phi, dphi, emb, demb).
int BatchEngine::force_matching(double wf, double ws, double *loss, double *grads) {
    BCHECK(ready());
    if (!fm_refs) return set_last_error(MOLDY_ERR_ORDER, "set the references first (moldy_gpu_batch_set_references)");
    const int n = tab.nlookup, nb = n + 1, nbr = tab.nr;
    if (fm_nb != nb) {
        if (fm_grads) cudaFree(fm_grads);
        fm_grads = nullptr;
        BCHECK(balloc(&fm_grads, 6 * (size_t)nb, "table gradients"));
        fm_nb = nb;
    }
    // the forward in FP64, energy_calc not needed
    for (int attempt = 0;; ++attempt) {
        k_set_active<<<(nsys + 255) / 256, 256, 0, stream>>>(nsys, sys, 1, 0);
        queue_evaluation(true, false, false);
        k_sys_reduce<<<nsys, kCgThreads, 0, stream>>>(sys, en_calc, en_force, vir, f, 1, sysout);
        launches += 2;
        BCUDA(cudaStreamSynchronize(stream), "force matching");
        int ov = take_overflow();
        if (ov < 0) return set_last_error(MOLDY_ERR_CUDA, "compact list re-allocation failed");
        if (ov == 0) break;
        if (attempt >= 2) return set_last_error(MOLDY_ERR_CAPACITY, "compact list keeps overflowing");
    }
    cudaStream_t s = stream;
    k_fm_loss<<<nsys, kCgThreads, 0, s>>>(sys, f, fm_fref, fm_sref, sysout, sorted, wf, ws, fm_gF, fm_gS, fm_loss);
    BCUDA(cudaMemsetAsync(fm_grads, 0, 6 * (size_t)nb * sizeof(double), s), "table gradients");
    TileArgs a;
    a.sys = sys; a.cell_sys = cell_sys; a.cell_start = cell_start; a.sorted = sorted;
    a.spos = spos; a.sfp = sfp; a.ncell = ncell; a.cap = cap; a.rc2 = rcut * rcut;
    const size_t smem_r = 2 * (size_t)nbr * sizeof(double), smem_e = (size_t)nb * sizeof(double);
    BCUDA(cudaFuncSetAttribute(k_fm_pairs_a, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_r), "smem");
    BCUDA(cudaFuncSetAttribute(k_fm_atoms, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_e), "smem");
    BCUDA(cudaFuncSetAttribute(k_fm_pairs_c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(smem_r / 2)),
          "smem");
    // histogram kernels: two blocks per SM, so each flush serves many atoms
    const int g = std::min(grid_blocks(ntot, 256), 2 * nsm);
    // vee and emb get no gradient: the loss holds no energy
    double *gdv = fm_grads + nb, *gp = fm_grads + 2 * nb, *gdp = fm_grads + 3 * nb, *gde = fm_grads + 5 * nb;
    k_fm_pairs_a<<<g, 256, smem_r, s>>>(a, tab, ntot, pair_cap, alist, pcnt, atom_sys, fm_gF, fm_gS, fm_mu, gdv, gdp,
                                       nbr);
    k_fm_atoms<<<g, 256, smem_e, s>>>(tab, ntot, sorted, rho, fm_mu, fm_nu, gde);
    k_fm_pairs_c<<<g, 256, smem_r / 2, s>>>(a, tab, ntot, pair_cap, alist, pcnt, atom_sys, fm_nu, gp, nbr);
    launches += 4;
    BCUDA(cudaGetLastError(), "force matching launch");
    if (loss) BCUDA(cudaMemcpyAsync(loss, fm_loss, (size_t)nsys * sizeof(double), cudaMemcpyDeviceToHost, s), "loss");
    if (grads)
        BCUDA(cudaMemcpyAsync(grads, fm_grads, 6 * (size_t)nb * sizeof(double), cudaMemcpyDeviceToHost, s), "grads");
    BCUDA(cudaStreamSynchronize(s), "force matching");
    return MOLDY_OK;
}

// The four launches of one evaluation of every system, timed with CUDA
// events on the batch's stream: the list check (k_prepare), the tile screen,
// the density pass and the force pass, in ms; rebuild = 1 rebuilds every
// list first.  The per-system reduction is not included.
int BatchEngine::kernel_times(int rebuild, double *ms4) {
    BCHECK(ready());
    cudaEvent_t ev[5];
    for (auto &e : ev) BCUDA(cudaEventCreate(&e), "event");
    k_set_active<<<(nsys + 255) / 256, 256, 0, stream>>>(nsys, sys, 1, rebuild ? 1 : 0);
    queue_evaluation(true, mixed, ecalc, ev);
    k_sys_reduce<<<nsys, kCgThreads, 0, stream>>>(sys, en_calc, en_force, vir, f, 1, sysout);
    launches += 2;
    BCUDA(cudaStreamSynchronize(stream), "kernel times");
    for (int k = 0; k < 4; ++k) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
        if (ms4) ms4[k] = ms;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (take_overflow() != 0) return set_last_error(MOLDY_ERR_CAPACITY, "compact rows grew; time again");
    return MOLDY_OK;
}

int BatchEngine::get_array(const double *dev, int stride, double *a, double *b, double *c) {
    size_t nt = (size_t)ntot;
    if (stride == 3) {
        k_unpack<<<(ntot + 255) / 256, 256, 0, stream>>>(ntot, dev, stage, stage + nt, stage + 2 * nt);
        double *outs[3] = {a, b, c};
        for (int k = 0; k < 3; ++k)
            if (outs[k])
                BCUDA(cudaMemcpyAsync(outs[k], stage + k * nt, nt * sizeof(double), cudaMemcpyDeviceToHost, stream),
                      "copy back");
    } else if (a) {
        BCUDA(cudaMemcpyAsync(a, dev, nt * sizeof(double), cudaMemcpyDeviceToHost, stream), "copy back");
    }
    BCUDA(cudaStreamSynchronize(stream), "copy back");
    return MOLDY_OK;
}

int BatchEngine::get_state(double *x0, double *y0, double *z0) { return get_array(X, 3, x0, y0, z0); }

// interleaved x(3i-2..3i) straight to or from the device arrays
int BatchEngine::copy_xyz(double *dev, const double *src, double *dst) {
    const size_t bytes = 3 * (size_t)ntot * sizeof(double);
    if (src) {
        BCUDA(cudaMemcpyAsync(dev, src, bytes, cudaMemcpyHostToDevice, stream), "positions");
        pos_set = true;
        state_set = pos_set && boxes_set;
    }
    if (dst) BCUDA(cudaMemcpyAsync(dst, dev, bytes, cudaMemcpyDeviceToHost, stream), "copy back");
    BCUDA(cudaStreamSynchronize(stream), "interleaved copy");
    return MOLDY_OK;
}

int BatchEngine::quench(int maxfn, int criterion, double fmax, double *out8) {
    BCHECK(ready());
    if (maxfn < 1) return set_last_error(MOLDY_ERR_INVALID, "maxfn < 1");
    cudaStream_t s = stream;
    size_t nt3 = 3 * (size_t)ntot;
    CgVecs v;
    v.X = X; v.G = cgv; v.D = cgv + nt3; v.GS = cgv + 2 * nt3; v.XX = cgv + 3 * nt3; v.GG = cgv + 4 * nt3;
    v.DR = cgv + 5 * nt3; v.DGR = cgv + 6 * nt3;
    BCUDA(cudaMemsetAsync(cgv, 0, 7 * nt3 * sizeof(double), s), "CG vectors");
    BCUDA(cudaMemsetAsync(cg, 0, nsys * sizeof(CgState), s), "CG state");
    BCUDA(cudaMemsetAsync(n_active, 0, sizeof(int), s), "counter");
    // first pass: every system asks for its first function value
    k_cg<<<nsys, kCgThreads, 0, s>>>(sys, cg, v, f, en_calc, press, maxfn, criterion, fmax, n_active,
                                         cg_order);
    launches += 1;
    BCUDA(cudaGetLastError(), "quench start");
    // one round: evaluate the active systems, then advance every state machine
    if (!graph || graph_lph != lph || graph_cap != cap || graph_maxfn != maxfn || graph_criterion != criterion ||
        graph_fmax != fmax || graph_gather != gather) {
        if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
        cudaGraph_t g = nullptr;
        BCUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "capture");
        // FP64 passes: the line search compares energies that differ in the
        // seventh digit, below the rounding of FP32 distances
        queue_evaluation(false, false, true);
        cudaMemsetAsync(n_active, 0, sizeof(int), s);
        k_cg<<<nsys, kCgThreads, 0, s>>>(sys, cg, v, f, en_calc, press, maxfn, criterion, fmax, n_active,
                                         cg_order);
        cudaError_t e = cudaStreamEndCapture(s, &g);
        if (e != cudaSuccess) {
            cudaGetLastError();
            if (g) cudaGraphDestroy(g);
            return set_last_error(MOLDY_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
        }
        e = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            cudaGetLastError();
            graph = nullptr;
            return set_last_error(MOLDY_ERR_CUDA, std::string("graph: ") + cudaGetErrorString(e));
        }
        graph_lph = lph; graph_cap = cap; graph_maxfn = maxfn; graph_criterion = criterion; graph_fmax = fmax;
        graph_gather = gather;
        launches -= 4;   // captured, not run; counted per replay below
    }
    // VA14CD evaluates at most maxfn times; a few rounds more let every
    // system reach its return
    const int rounds = maxfn + 8;
    for (int r = 0; r < rounds; ++r) {
        BCUDA(cudaGraphLaunch(graph, s), "graph launch");
        launches += 5;
        if ((r & 7) == 7 || r == rounds - 1) {
            BCUDA(cudaMemcpyAsync(host_active, n_active, sizeof(int), cudaMemcpyDeviceToHost, s), "counter");
            BCUDA(cudaStreamSynchronize(s), "quench");
            if (*host_active == 0) break;
        }
    }
    BCUDA(cudaStreamSynchronize(s), "quench");
    BCUDA(cudaGetLastError(), "quench");
    std::vector<CgState> hs(nsys);
    BCUDA(cudaMemcpy(hs.data(), cg, nsys * sizeof(CgState), cudaMemcpyDeviceToHost), "CG state");
    int unfinished = 0;
    for (int k = 0; k < nsys; ++k) {
        const CgState &c = hs[k];
        if (!c.done) ++unfinished;
        if (out8) {
            double *o = out8 + 8 * (size_t)k;
            o[0] = c.f; o[1] = c.pe; o[2] = c.gsumsq; o[3] = c.last_fmax;
            o[4] = c.maxfnc; o[5] = c.iterc; o[6] = c.done ? c.iflag : 5; o[7] = 0.0;
        }
    }
    // leave every system active for later force calls
    k_set_active<<<(nsys + 255) / 256, 256, 0, s>>>(nsys, sys, 1, 0);
    BCUDA(cudaStreamSynchronize(s), "quench");
    int ov = take_overflow();
    if (ov != 0)
        return set_last_error(MOLDY_ERR_CAPACITY, "an atom had " + std::to_string(ov) +
                                                      " neighbours inside the cut, more than a compact row held; "
                                                      "the rows have been grown, quench again");
    if (unfinished) return set_last_error(MOLDY_ERR_CAPACITY, std::to_string(unfinished) + " systems did not finish");
    return MOLDY_OK;
}

}  // namespace moldy

// ================================================================ C ABI ====
struct moldy_batch {
    moldy::BatchEngine *e;
};

#define BGUARD(h)                                                                      \
    do {                                                                               \
        if (!(h) || !(h)->e) return moldy::set_last_error(MOLDY_ERR_INVALID, "null handle"); \
        cudaSetDevice((h)->e->device);                                                \
    } while (0)
#define BTRY(expr)                                                                     \
    try {                                                                              \
        return (expr);                                                                 \
    } catch (...) {                                                                    \
        return moldy::set_last_error(MOLDY_ERR_CAPACITY, "host allocation failed");    \
    }

extern "C" {

int moldy_gpu_batch_create(int32_t nsys, const int32_t *natoms, double press, int32_t device, moldy_batch **out) {
    if (!out || !natoms || nsys < 1) return moldy::set_last_error(MOLDY_ERR_INVALID, "invalid arguments");
    *out = nullptr;
    try {
        moldy::BatchEngine *e = new moldy::BatchEngine();
        int rc = e->init(nsys, natoms, press, device);
        if (rc != MOLDY_OK) { delete e; return rc; }
        *out = new moldy_batch{e};
        return MOLDY_OK;
    } catch (...) {
        return moldy::set_last_error(MOLDY_ERR_CAPACITY, "host allocation failed");
    }
}

int moldy_gpu_batch_destroy(moldy_batch *h) {
    if (!h) return MOLDY_OK;
    delete h->e;
    delete h;
    return MOLDY_OK;
}

int moldy_gpu_batch_set_fetm_fe(moldy_batch *h, int32_t nv, const double *av, const double *rv, int32_t np,
                                const double *ap, const double *rp, int32_t nlookup) {
    BGUARD(h);
    BTRY(h->e->set_fetm(nv, av, rv, np, ap, rp, nlookup));
}

int moldy_gpu_batch_set_state(moldy_batch *h, const double *x0, const double *y0, const double *z0,
                              const double *b0, const double *mass) {
    BGUARD(h);
    BTRY(h->e->set_state(x0, y0, z0, b0, mass));
}

int moldy_gpu_batch_get_state(moldy_batch *h, double *x0, double *y0, double *z0) {
    BGUARD(h);
    BTRY(h->e->get_state(x0, y0, z0));
}

int moldy_gpu_batch_force(moldy_batch *h, double *out13) {
    BGUARD(h);
    BTRY(h->e->force(out13));
}

int moldy_gpu_batch_get_forces(moldy_batch *h, double *fx, double *fy, double *fz) {
    BGUARD(h);
    BTRY(h->e->get_array(h->e->f, 3, fx, fy, fz));
}

int moldy_gpu_batch_set_positions(moldy_batch *h, const double *xyz) {
    BGUARD(h);
    if (!h->e->potential_set) return moldy::set_last_error(MOLDY_ERR_ORDER, "set the potential before the state");
    if (!xyz) return moldy::set_last_error(MOLDY_ERR_INVALID, "null positions");
    BTRY(h->e->copy_xyz(h->e->X, xyz, nullptr));
}

int moldy_gpu_batch_get_forces_xyz(moldy_batch *h, double *fxyz) {
    BGUARD(h);
    if (!fxyz) return moldy::set_last_error(MOLDY_ERR_INVALID, "null output");
    BTRY(h->e->copy_xyz(h->e->f, nullptr, fxyz));
}

int moldy_gpu_batch_get_energies(moldy_batch *h, double *en_calc, double *en_force) {
    BGUARD(h);
    int rc = h->e->get_array(h->e->en_calc, 1, en_calc, nullptr, nullptr);
    if (rc != MOLDY_OK) return rc;
    return h->e->get_array(h->e->en_force, 1, en_force, nullptr, nullptr);
}

int moldy_gpu_batch_get_density(moldy_batch *h, double *rho, double *afrho, double *dafrho) {
    BGUARD(h);
    int rc = h->e->get_array(h->e->rho, 1, rho, nullptr, nullptr);
    if (rc == MOLDY_OK) rc = h->e->get_array(h->e->afrho, 1, afrho, nullptr, nullptr);
    if (rc == MOLDY_OK) rc = h->e->get_array(h->e->fp, 1, dafrho, nullptr, nullptr);
    return rc;
}

int moldy_gpu_batch_quench(moldy_batch *h, int32_t maxfn, int32_t criterion, double fmax, double *out8) {
    BGUARD(h);
    BTRY(h->e->quench(maxfn, criterion, fmax, out8));
}

int moldy_gpu_batch_set_tiles(moldy_batch *h, int32_t lanes, int32_t staged) {
    BGUARD(h);
    if (lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32)
        return moldy::set_last_error(MOLDY_ERR_INVALID, "lanes per atom must be 4, 8, 16 or 32");
    if (staged < 0 || staged > moldy::kTileCapMax)
        return moldy::set_last_error(MOLDY_ERR_INVALID, "staged candidates out of range");
    h->e->lph = lanes;
    h->e->cap = staged;
    return MOLDY_OK;
}

int moldy_gpu_batch_autotune(moldy_batch *h, int32_t nreps, double *times_ms, int32_t *chosen) {
    BGUARD(h);
    BTRY(h->e->autotune(nreps, times_ms, chosen));
}

int moldy_gpu_batch_set_references(moldy_batch *h, const double *fref_xyz, const double *sref) {
    BGUARD(h);
    BTRY(h->e->set_references(fref_xyz, sref));
}

int moldy_gpu_batch_force_matching(moldy_batch *h, double w_force, double w_stress, double *loss,
                                   double *table_grads) {
    BGUARD(h);
    BTRY(h->e->force_matching(w_force, w_stress, loss, table_grads));
}

int moldy_gpu_batch_kernel_times(moldy_batch *h, int32_t rebuild, double *ms4) {
    BGUARD(h);
    BTRY(h->e->kernel_times(rebuild, ms4));
}

int moldy_gpu_batch_set_energy_calc(moldy_batch *h, int32_t enable) {
    BGUARD(h);
    h->e->ecalc = enable != 0;
    return MOLDY_OK;
}

int moldy_gpu_batch_set_precision(moldy_batch *h, int32_t mixed) {
    BGUARD(h);
    if (mixed != 0 && mixed != 1) return moldy::set_last_error(MOLDY_ERR_INVALID, "mixed must be 0 or 1");
    h->e->mixed = mixed == 1;
    return MOLDY_OK;
}

int moldy_gpu_batch_set_persistent(moldy_batch *h, int32_t enable) {
    BGUARD(h);
    h->e->persistent = enable != 0;
    return MOLDY_OK;
}

int moldy_gpu_batch_set_atom_lanes(moldy_batch *h, int32_t lanes) {
    BGUARD(h);
    if (lanes != 1 && lanes != 2 && lanes != 4)
        return moldy::set_last_error(MOLDY_ERR_INVALID, "lanes per atom must be 1, 2 or 4");
    h->e->lpa = lanes;
    return MOLDY_OK;
}

int moldy_gpu_batch_persistent_applies(moldy_batch *h, int32_t *applies) {
    BGUARD(h);
    if (!applies) return moldy::set_last_error(MOLDY_ERR_INVALID, "null pointer");
    *applies = h->e->persistent_applies() ? 1 : 0;
    return MOLDY_OK;
}

int moldy_gpu_batch_eval_times(moldy_batch *h, double *ms2) {
    BGUARD(h);
    BTRY(h->e->eval_times(ms2));
}

int moldy_gpu_batch_set_gather(moldy_batch *h, int32_t entries) {
    BGUARD(h);
    if (entries != 1 && entries != 2 && entries != 4)
        return moldy::set_last_error(MOLDY_ERR_INVALID, "row entries gathered at a time must be 1, 2 or 4");
    h->e->gather = entries;
    return MOLDY_OK;
}

int moldy_gpu_batch_set_skin(moldy_batch *h, double skin) {
    BGUARD(h);
    BTRY(h->e->set_skin(skin));
}

int moldy_gpu_batch_row_entries(moldy_batch *h, int64_t *total) {
    BGUARD(h);
    if (!total) return moldy::set_last_error(MOLDY_ERR_INVALID, "null output");
    const int nt = h->e->ntot;
    std::vector<int32_t> c(nt);
    cudaError_t e = cudaMemcpy(c.data(), h->e->pcnt, nt * sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return moldy::set_last_error(MOLDY_ERR_CUDA, std::string("row entries: ") + cudaGetErrorString(e));
    }
    long long t = 0;
    for (int k = 0; k < nt; ++k) t += std::min(c[k], h->e->pair_cap);
    *total = (int64_t)t;
    return MOLDY_OK;
}

int moldy_gpu_batch_list_stats(moldy_batch *h, int64_t *out2) {
    BGUARD(h);
    if (!out2) return moldy::set_last_error(MOLDY_ERR_INVALID, "null output");
    unsigned long long v[2] = {0, 0};
    cudaError_t e = cudaMemcpy(v, h->e->stats, sizeof(v), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return moldy::set_last_error(MOLDY_ERR_CUDA, std::string("list statistics: ") + cudaGetErrorString(e));
    }
    out2[0] = (int64_t)v[0];
    out2[1] = (int64_t)v[1];
    return MOLDY_OK;
}

int moldy_gpu_batch_launches(moldy_batch *h, int64_t *launches) {
    BGUARD(h);
    if (launches) *launches = h->e->launches;
    return MOLDY_OK;
}

int moldy_gpu_batch_get_stream(moldy_batch *h, void **stream) {
    BGUARD(h);
    if (stream) *stream = (void *)h->e->stream;
    return MOLDY_OK;
}

}  // extern "C"
