// nlist.cu -- the hybrid Verlet half list (update_neighbourlist,
// src/neighbourlist_m.F90:103-276) built on the GPU.
//
// One block (two warps) owns one link cell.  It stages the atoms of the
// reference's half stencil in shared memory: the home cell, then the 13
// further cells in the reference's order (dz in {0,+1}; at dz=0 dy in {0,+1};
// at dz=0,dy=0 dx in {0,+1}; otherwise dx,dy in {-1,0,+1}), each cell's
// atoms in chain order.  Each lane takes one home atom i; the candidates
// after i form NLIST(:, i), entry for entry as the reference's walk appends
// them.  Candidates past the staging capacity are read from global memory.
// Each atom's reverse row (the atoms j with i in NLIST(:, j), i's own cell
// before i, then the 13 mirror cells, each in chain order) is gathered
// afterwards from keep bits the build leaves per staged candidate.  NLIST is
// stored as the reference holds NLIST(nnbrs, nm): atom i's row at i*nnbrs,
// its entries contiguous, so that a lane appending to its own row fills
// whole 32-byte sectors (a cell's atoms have scattered ids, so rows stored
// entry-major took partial-sector writes, 3x the row bytes in DRAM traffic).
// The reverse rows, written one thread per atom in atom order, are stored
// entry-major (entry k of atom j at k*nm + j): a warp's stores of one entry
// index are then contiguous.  The exact distance test
// uses separately rounded products and sums (no FMA), as the Fortran
// evaluates pr_get_realsep_from_dx, so r < rnear gives the same pair set.
// In a fully periodic box an FP32 distance decides first (from positions
// relative to the home cell's centre, or from the fixed-point difference; see
// k_build_nlist): its error is bounded far inside kNlBand, so a candidate more
// than kNlBand from rnear is taken or left by it alone, and only the others
// take the exact FP64 test.
#include "engine.h"

namespace moldy {

// (dx, dy, dz) offsets of the half stencil in the reference's loop order;
// rows 14..26 are the mirror (backward) half, in the negated order
__constant__ int8_t c_stencil[27][3] = {
    {0, 0, 0}, {1, 0, 0},
    {-1, 1, 0}, {0, 1, 0}, {1, 1, 0},
    {-1, -1, 1}, {0, -1, 1}, {1, -1, 1},
    {-1, 0, 1}, {0, 0, 1}, {1, 0, 1},
    {-1, 1, 1}, {0, 1, 1}, {1, 1, 1},
    {-1, 0, 0},
    {1, -1, 0}, {0, -1, 0}, {-1, -1, 0},
    {1, 1, -1}, {0, 1, -1}, {-1, 1, -1},
    {1, 0, -1}, {0, 0, -1}, {-1, 0, -1},
    {1, -1, -1}, {0, -1, -1}, {-1, -1, -1}};

__device__ __forceinline__ int wrap(int j, int n) { return j < 0 ? j + n : (j >= n ? j - n : j); }

constexpr int kNlStage = 384;   // staged candidates per home cell (its 14 half-stencil cells hold ~310
                                // on average); the rest are read from global memory
constexpr int kNlChunks = kNlStage / 32;
constexpr double kNlBand = 1.0e-3;   // A; the FP32 test decides outside rnear -+ this

// Pre-test of a candidate.  PERIODIC = false (boxes not periodic in all three
// directions): the exact FP64 test for every candidate.  PERIODIC = true: an
// FP32 distance decides outside the band rnear -+ kNlBand, in one of two
// forms chosen per launch on the device:
//  fixed point   the FP32 distance from the 32-bit fixed-point difference
//                (the integer difference is the minimum image);
//  cell relative the FP32 distance between Cartesian positions c relative to
//                the home cell's centre, computed once per staged candidate
//                instead of once per (home atom, candidate).  A staged
//                candidate is kept as (-2c, |c|^2), so that r^2 - t =
//                (|c|^2 - (t - |a|^2)) - 2 a.c costs three fused multiply-adds
//                per pair.  It needs at least 4 cells per direction, so that
//                every staged candidate lies within 1.5 cells, less than half
//                a box, of the centre and its fixed-point offset from it is
//                its own minimum image (the pair's difference is then the
//                minimum image too), and a stencil reach R (centre to the far
//                corner of a stencil cell) for which the FP32 error stays far
//                inside the band: the positions carry under 8 ulp of R per
//                component (under 1.7e-6 R in a distance) and the expansion
//                under 27 ulp of R^2 (under 0.8e-6 R^2 / rnear in a distance
//                near rnear); their sum must stay under kNlBand / 8.
__device__ __forceinline__ bool cell_relative_ok(double reach, double rnear) {
    return 1.7e-6 * reach + 0.8e-6 * reach * reach / rnear < 0.125 * kNlBand;
}

// Shared state of one block's candidate tests
struct NlStage {
    const int4 *srec;       // staged records (fixed point, or (-2c, |c|^2) as float bits)
    const int *sid;         // staged atom ids
    const int *sbase, *sstart;
    const int32_t *cell_atoms;
    const int4 *posq;
    const double4 *pos;
    const float *bs;        // B0 per fixed-point unit
    const double *b;        // B0
    int staged, ivol;
    double rnear;
    float rlo2, rhi2;
};

// The exact test r(a, j) < rnear with separately rounded products and sums,
// as pr_get_realsep_from_dx evaluates it (out of line: rare)
__device__ __noinline__ bool nl_exact(const double4 *__restrict__ pos, const double *b, int ivol, double rnear,
                                      double4 pa, int j) {
    const double4 pj = pos[j];
    double dx = __dsub_rn(pa.x, pj.x), dy = __dsub_rn(pa.y, pj.y), dz = __dsub_rn(pa.z, pj.z);
    min_image(ivol, dx, dy, dz);
    return realsep_exact(b, dx, dy, dz) < rnear;
}

// Cartesian position of a fixed-point point relative to the fixed-point
// origin o, in FP32 (the integer difference is the minimum image)
__device__ __forceinline__ float3 fix_rel(const float *bs, int4 q, int4 o) {
    const float dx = __int2float_rn((int32_t)((uint32_t)q.x - (uint32_t)o.x));
    const float dy = __int2float_rn((int32_t)((uint32_t)q.y - (uint32_t)o.y));
    const float dz = __int2float_rn((int32_t)((uint32_t)q.z - (uint32_t)o.z));
    return make_float3(fmaf(bs[6], dz, fmaf(bs[3], dy, bs[0] * dx)),
                       fmaf(bs[7], dz, fmaf(bs[4], dy, bs[1] * dx)),
                       fmaf(bs[8], dz, fmaf(bs[5], dy, bs[2] * dx)));
}

// r(a, candidate kk) < rnear, decided as the reference evaluates it: the FP32
// pre-test outside the band, the exact FP64 separation (separately rounded
// products and sums) inside it; j receives the candidate's atom id.  The
// exact test is symmetric bit for bit (negating a difference is exact), so
// the forward and backward rows describe the same pair set.  ar is the home
// atom's cell-relative position (cell-relative form), qa its fixed-point one.
template <bool PERIODIC>
__device__ __forceinline__ bool nl_take(const NlStage &S, int kk, const double4 &pa, const int4 &qa,
                                        const float3 &ar, bool rel, const int4 &cen, int &j) {
    const bool staged = kk < S.staged;
    if (staged) {
        j = S.sid[kk];
    } else {
        int s = 0;
        while (S.sbase[s + 1] <= kk) ++s;
        j = S.cell_atoms[S.sstart[s] + (kk - S.sbase[s])];
    }
    if (PERIODIC) {
        float3 r;
        if (rel) {
            float3 cr;
            if (staged) {
                const int4 rec = S.srec[kk];
                cr = make_float3(-0.5f * __int_as_float(rec.x), -0.5f * __int_as_float(rec.y),
                                 -0.5f * __int_as_float(rec.z));
            } else {
                cr = fix_rel(S.bs, S.posq[j], cen);
            }
            r = make_float3(ar.x - cr.x, ar.y - cr.y, ar.z - cr.z);
        } else {
            r = fix_rel(S.bs, qa, staged ? S.srec[kk] : S.posq[j]);
        }
        const float r2 = fmaf(r.z, r.z, fmaf(r.y, r.y, r.x * r.x));
        if (r2 < S.rlo2) return true;
        if (r2 > S.rhi2) return false;
    }
    return nl_exact(S.pos, S.b, S.ivol, S.rnear, pa, j);
}

// a / b for a >= 0, b > 0: below 2^24 an FP32 quotient corrected by one in
// either direction (the FP32 estimate is then within one of the true quotient)
__device__ __forceinline__ int div_small(int a, int b) {
    if (a >= (1 << 24)) return a / b;
    int q = __float2int_rz(__fdividef((float)a, (float)b));
    q -= (q * b > a) ? 1 : 0;
    q += ((q + 1) * b <= a) ? 1 : 0;
    return q;
}

// bits [0, x) of a word, x in [0, 32]
__device__ __forceinline__ unsigned low_bits(int x) { return x >= 32 ? ~0u : (1u << x) - 1u; }

// The transpose of a 32x32 bit matrix held one row per lane (bit c of lane
// l's word is element (l, c)): lane l receives column l.  Five butterfly
// stages swap blocks of 16, 8, 4, 2 and 1 bits between lanes l and l ^ j.
__device__ __forceinline__ unsigned transpose_lanes(unsigned x, int lane) {
    unsigned m = 0x0000ffffu;
#pragma unroll
    for (int j = 16; j > 0; j >>= 1, m ^= m << j) {
        const unsigned y = __shfl_xor_sync(0xffffffffu, x, j);
        x = (lane & j) ? (((y >> j) & m) | (x & ~m)) : ((x & m) | ((y & m) << j));
    }
    return x;
}

// Two warps per link cell stage the atoms of the reference's half stencil:
// the home cell, then the 13 further cells, each cell's atoms in chain order.
// Each lane then takes one home atom a (the cell's atoms 32 at a time) and,
// over the staged candidates in order, every lane reading the same candidate
// (a shared-memory broadcast), builds NLIST(:, a): the candidates after a,
// in the reference's order (entry for entry).  In the cell-relative form the
// two warps first test alternate chunks of 32 candidates into keep masks (one
// word per home atom and chunk, in shared memory); then warp 0 appends the
// kept candidates of the first half of the chunks and warp 1 those of the
// second half, from the count of the first half on.  The reverse rows come
// afterwards from the finished rows (k_rev_scatter, k_rev_sort).
template <bool PERIODIC>
__global__ void __launch_bounds__(64, 20)
k_build_nlist(Params p, const double4 *__restrict__ pos, const int4 *__restrict__ posq,
              const BoxState *__restrict__ box,
              const int32_t *__restrict__ cell_start, const int32_t *__restrict__ cell_count,
              const int32_t *__restrict__ cell_atoms, int32_t *__restrict__ nlist,
              int32_t *__restrict__ numn, uint32_t *__restrict__ revmask, int32_t *__restrict__ flags) {
    // per staged candidate: its fixed-point position (fixed-point form) or
    // (-2c, |c|^2) of its cell-relative Cartesian position c as float bits
    // (cell-relative form), and its atom id
    __shared__ int4 srec[kNlStage];
    __shared__ int sid[kNlStage];
    // keep masks of each chunk of 32 candidates (forward candidates only),
    // per home atom (lane); per warp the chunks with some; warp 1's counts
    __shared__ unsigned smask[kNlChunks][32];
    __shared__ unsigned snz[2][32];
    __shared__ int scount[32];
    __shared__ uint8_t scell[kNlStage];   // half-stencil cell (0..13) of each staged candidate
    __shared__ int sbase[28], sstart[27];
    __shared__ double sb[9];
    __shared__ int4 scen;     // the home cell's centre in fixed point; w: cell-relative form
    const int c = blockIdx.x;
    const int L0 = cell_count[c];
    if (L0 == 0) return;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int cx = c % p.nlcx, cy = (c / p.nlcx) % p.nlcy, cz = c / (p.nlcx * p.nlcy);
    if (warp == 0) {
        if (lane < 9) sb[lane] = box->b0[lane];
        int cnt = 0, st = 0;
        if (lane < 14) {   // the home cell and the 13 further cells of the half stencil
            const int jx = wrap(cx + c_stencil[lane][0], p.nlcx);
            const int jy = wrap(cy + c_stencil[lane][1], p.nlcy);
            const int jz = wrap(cz + c_stencil[lane][2], p.nlcz);
            const int jp = jx + p.nlcx * (jy + p.nlcy * jz);
            st = cell_start[jp];
            cnt = cell_count[jp];
        }
        // inclusive scan of the cell sizes over the lanes
        int inc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        if (lane < 14) { sbase[lane + 1] = inc; sstart[lane] = st; }
        if (lane == 0) sbase[0] = 0;
        __syncwarp();
        if (PERIODIC) {
            // lanes 0-7: distance from the centre to corner `lane` of the 27
            // cells; lanes 0-2: the centre's fixed-point coordinate `lane`
            // (fractional (i + 1/2) / nlc - 1/2: a cell holds x - nint(x) in
            // [i/nlc - 1/2, (i+1)/nlc - 1/2))
            double r = 0.0;
            if (lane < 8) {
                const double f0 = (lane & 1 ? 1.5 : -1.5) / p.nlcx, f1 = (lane & 2 ? 1.5 : -1.5) / p.nlcy,
                             f2 = (lane & 4 ? 1.5 : -1.5) / p.nlcz;
                double r2 = 0.0;
                for (int i = 0; i < 3; ++i) {
                    const double v = sb[i] * f0 + sb[3 + i] * f1 + sb[6 + i] * f2;
                    r2 += v * v;
                }
                r = sqrt(r2);
            }
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
            const int ci = lane == 0 ? cx : (lane == 1 ? cy : cz);
            const int nl = lane == 0 ? p.nlcx : (lane == 1 ? p.nlcy : p.nlcz);
            const int cc = fix32((ci + 0.5) / nl - 0.5);
            const int c0 = __shfl_sync(0xffffffffu, cc, 0), c1 = __shfl_sync(0xffffffffu, cc, 1),
                      c2 = __shfl_sync(0xffffffffu, cc, 2);
            if (lane == 0) {
                const bool rel = p.nlcx >= 4 && p.nlcy >= 4 && p.nlcz >= 4 && cell_relative_ok(r, p.rnear);
                scen = make_int4(c0, c1, c2, rel ? 1 : 0);
            }
        }
    }
    __syncthreads();
    const int4 cen = PERIODIC ? scen : make_int4(0, 0, 0, 0);
    const bool rel = PERIODIC && cen.w != 0;
    float bs[9];   // B0 per fixed-point unit
#pragma unroll
    for (int k = 0; k < 9; ++k) bs[k] = (float)(sb[k] * kFixUnit);
    const int fwd_end = sbase[14], total = fwd_end;
    const int staged = total < kNlStage ? total : kNlStage;
    // staging: the ids (each cell's atoms are contiguous in cell_atoms):
    // thread t copies atom t of every cell, 27 independent predicated loads
    // in flight at once, then the atoms past 64 of crowded cells; then the
    // records slot by slot, again several independent loads per thread
#pragma unroll
    for (int sc = 0; sc < 14; ++sc) {
        const int kb = sbase[sc], n = min(sbase[sc + 1], staged) - kb;
        if (t < n) { sid[kb + t] = cell_atoms[sstart[sc] + t]; scell[kb + t] = (uint8_t)sc; }
    }
    for (int sc = 0; sc < 14; ++sc) {
        const int kb = sbase[sc], n = min(sbase[sc + 1], staged) - kb;
        for (int i = t + 64; i < n; i += 64) { sid[kb + i] = cell_atoms[sstart[sc] + i]; scell[kb + i] = (uint8_t)sc; }
    }
    // more home atoms than the reverse-row masks hold: the reverse rows are
    // formed by the scatter-and-sort path instead
    if (t == 0 && L0 > 32 * kRevRounds) atomicExch(&flags[12], 1);
    __syncthreads();
    if (PERIODIC) {
#pragma unroll 5
        for (int k = t; k < staged; k += 64) {
            const int4 qj = posq[sid[k]];
            if (rel) {
                const float3 v = fix_rel(bs, qj, cen);
                srec[k] = make_int4(__float_as_int(-2.0f * v.x), __float_as_int(-2.0f * v.y),
                                    __float_as_int(-2.0f * v.z),
                                    __float_as_int(fmaf(v.z, v.z, fmaf(v.y, v.y, v.x * v.x))));
            } else {
                srec[k] = qj;
            }
        }
    }
    // records past the staged candidates, up to the next multiple of 32: far
    // away, so the chunked tests below need no bound check
    if (rel) {
        const int pad_end = min((staged + 31) & ~31, kNlStage);
        for (int k = staged + t; k < pad_end; k += 64) {
            srec[k] = make_int4(0, 0, 0, __float_as_int(1.0e30f));
            sid[k] = -1;
        }
    }
    __syncthreads();
    NlStage S;
    S.srec = srec; S.sid = sid; S.sbase = sbase; S.sstart = sstart; S.cell_atoms = cell_atoms;
    S.posq = posq; S.pos = pos; S.bs = bs; S.b = sb; S.staged = staged; S.ivol = p.ivol; S.rnear = p.rnear;
    S.rlo2 = (float)((p.rnear - kNlBand) * (p.rnear - kNlBand));
    S.rhi2 = (float)((p.rnear + kNlBand) * (p.rnear + kNlBand));
    const size_t nm = (size_t)p.nm;
    const int cap = p.nnbrs;
    const bool fwd_warp = warp == 0;
    for (int q0 = 0; q0 < L0; q0 += 32) {
        if (q0 > 0) __syncthreads();             // the previous round's masks are read
        const int q = q0 + lane;                 // this lane's home atom: staged slot q
        const bool live = q < L0;
        const bool home_staged = q < staged;
        const int a = live ? (home_staged ? sid[q] : cell_atoms[sstart[0] + q]) : 0;
        const double4 pa = live ? pos[a] : make_double4(0.0, 0.0, 0.0, 0.0);
        int4 qa = make_int4(0, 0, 0, 0);         // fixed point (fixed-point form)
        float3 ar = make_float3(0.f, 0.f, 0.f);  // cell relative (cell-relative form)
        float a2 = 0.f;
        if (PERIODIC && live) {
            if (rel) {
                if (home_staged) {
                    const int4 rec = srec[q];
                    ar = make_float3(-0.5f * __int_as_float(rec.x), -0.5f * __int_as_float(rec.y),
                                     -0.5f * __int_as_float(rec.z));
                    a2 = __int_as_float(rec.w);
                } else {
                    ar = fix_rel(bs, posq[a], cen);
                }
            } else {
                qa = home_staged ? srec[q] : posq[a];
            }
        }
        // the row of a: entry n at base[n] (atom-major)
        int32_t *const base = nlist + (size_t)a * cap;
        int n = 0;
        int kk = 0;
        if (rel && min(L0, q0 + 32) <= staged) {   // every live lane's home atom staged
            const int nch = (staged + 31) >> 5;
            // keep masks of the candidates after q: warp w tests chunks w,
            // w + 2, ... into those below rnear + band (m) and below rnear -
            // band (mlo); the exact test settles those in between here, so the
            // masks hold the final pairs
            const float thi = S.rhi2 - a2, dlt = S.rhi2 - S.rlo2;
            unsigned nzf = 0u;
            for (int ch = warp; ch < nch; ch += 2) {
                const int k0 = ch << 5;
                unsigned m = 0u, mlo = 0u;
#pragma unroll
                for (int b = 0; b < 32; ++b) {
                    const int4 rec = srec[k0 + b];
                    // s = r^2 - (rnear + band)^2
                    const float s = fmaf(ar.z, __int_as_float(rec.z),
                                         fmaf(ar.y, __int_as_float(rec.y),
                                              fmaf(ar.x, __int_as_float(rec.x), __int_as_float(rec.w) - thi)));
                    m = __funnelshift_l(__float_as_uint(s), m, 1);            // (m << 1) | sign(s)
                    mlo = __funnelshift_l(__float_as_uint(s + dlt), mlo, 1);
                }
                const unsigned after = ~low_bits(min(max(q + 1 - k0, 0), 32));
                m = live ? __brev(m) & after : 0u;                           // bit b: candidate k0 + b
                unsigned band = m & ~__brev(mlo);
                while (band) {                                               // rare
                    const int b = __ffs(band) - 1;
                    band &= band - 1u;
                    if (!nl_exact(pos, sb, p.ivol, p.rnear, pa, sid[k0 + b])) m &= ~(1u << b);
                }
                smask[ch][lane] = m;
                nzf |= m ? 1u << ch : 0u;
            }
            snz[warp][lane] = nzf;
            __syncthreads();
            // for each staged candidate j, the home atoms of this round whose
            // rows hold it: the chunk's keep bits transposed across the lanes
            const int round = q0 >> 5;
            if (round < kRevRounds) {
                for (int ch = warp; ch < nch; ch += 2) {
                    const int k = (ch << 5) + lane;
                    const unsigned colm = transpose_lanes(smask[ch][lane], lane);
                    if (k < staged)
                        revmask[(size_t)(scell[k] * kRevRounds + round) * nm + sid[k]] = colm;
                }
            }
            // appends: warp 0 the chunks [0, mid), warp 1 the chunks [mid,
            // nch) from the count of warp 0's entries on.  Each lane walks its
            // kept candidates over its chunks in one loop, so the warp runs
            // as many iterations as its longest share of a row takes
            const int mid = (nch + 1) >> 1;
            unsigned chunks = (snz[0][lane] | snz[1][lane]) & (fwd_warp ? low_bits(mid) : ~low_bits(mid));
            if (!fwd_warp)
                for (int ch = 0; ch < mid; ++ch) n += __popc(smask[ch][lane]);
            unsigned m = 0u;
            int k0 = 0;
            while (m | chunks) {
                if (m == 0u) {
                    const int ch = __ffs(chunks) - 1;
                    chunks &= chunks - 1u;
                    k0 = ch << 5;
                    m = smask[ch][lane];
                }
                const int k = k0 + __ffs(m) - 1;
                m &= m - 1u;
                if (n < cap) base[n] = sid[k];
                ++n;
            }
            // warp 1's count is the row's
            if (!fwd_warp) scount[lane] = n;
            __syncthreads();
            n = scount[lane];
            kk = staged;
        }
        // the rest: candidates beyond the staging, every candidate of the
        // fixed-point form and of boxes not periodic in all three directions
        if (fwd_warp) {
            const int round = q0 >> 5;
            for (int k = kk; k < fwd_end; ++k) {
                int j = 0;
                const bool take = live && k > q && nl_take<PERIODIC>(S, k, pa, qa, ar, rel, cen, j);
                if (take && n < cap) base[n] = j;
                n += take ? 1 : 0;
                // this candidate's column of the reverse-row masks
                const unsigned colm = __ballot_sync(0xffffffffu, take);
                if (lane == 0 && round < kRevRounds) {
                    int sc = 0;
                    while (sbase[sc + 1] <= k) ++sc;
                    const int jk = k < staged ? sid[k] : cell_atoms[sstart[sc] + (k - sbase[sc])];
                    revmask[(size_t)(sc * kRevRounds + round) * nm + jk] = colm;
                }
            }
            if (live) {
                numn[a] = n < cap ? n : cap;
                if (n > cap) {
                    atomicExch(&flags[0], 1);
                    atomicMax(&flags[2], a + 1);
                }
            }
        }
    }
}

// Reverse rows: row j holds the atoms i with j in NLIST(:, i) -- j's own cell
// first, then the 13 mirror cells of the half stencil in order, each cell in
// chain order, the order in which a full-stencil walk from j's cell meets them.
// The half-list build leaves, per atom j and half-stencil rank r, the home
// atoms of the source cell (j's cell minus forward offset r) whose rows hold
// j, as bits over the source cell's chain positions (32 per round); one thread
// per atom expands them in rank, round and bit order.  A link cell fuller
// than the masks hold (flag 12) leaves the rows to the scatter-and-sort path.
__global__ void __launch_bounds__(256)
k_rev_gather(Params p, const int32_t *__restrict__ ic, const int32_t *__restrict__ cell_start,
             const int32_t *__restrict__ cell_count, const int32_t *__restrict__ cell_atoms,
             const uint32_t *__restrict__ revmask, int32_t *__restrict__ rlist, int32_t *__restrict__ numr,
             int32_t *__restrict__ flags) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.nm) return;
    if (flags[12]) {   // the fallback counts from zero
        numr[j] = 0;
        return;
    }
    const size_t nm = (size_t)p.nm;
    const int cap = p.nnbrs;
    const int cj = ic[j];
    const int nxy = p.nlcx * p.nlcy;
    const int jz = div_small(cj, nxy), rxy = cj - jz * nxy;
    const int jy = div_small(rxy, p.nlcx), jx = rxy - jy * p.nlcx;
    // the 14 source cells' sizes and starts, then their first-round words, all
    // loads issued before any is used
    int cnt[14], st[14];
#pragma unroll
    for (int r = 0; r < 14; ++r) {
        const int sx = wrap(jx - c_stencil[r][0], p.nlcx), sy = wrap(jy - c_stencil[r][1], p.nlcy),
                  sz = wrap(jz - c_stencil[r][2], p.nlcz);
        const int cs = sx + p.nlcx * (sy + p.nlcy * sz);
        cnt[r] = cell_count[cs];
        st[r] = cell_start[cs];
    }
    unsigned w0[14];
#pragma unroll
    for (int r = 0; r < 14; ++r) w0[r] = cnt[r] > 0 ? revmask[(size_t)(r * kRevRounds) * nm + j] : 0u;
    int n = 0;
#pragma unroll
    for (int r = 0; r < 14; ++r) {
        for (int round = 0; round < kRevRounds && 32 * round < cnt[r]; ++round) {
            unsigned m = round == 0 ? w0[r] : revmask[(size_t)(r * kRevRounds + round) * nm + j];
            while (m) {
                const int L = __ffs(m) - 1;
                m &= m - 1u;
                if (n < cap) rlist[(size_t)n * nm + j] = cell_atoms[st[r] + 32 * round + L];
                ++n;
            }
        }
    }
    numr[j] = n < cap ? n : cap;
    if (n > cap) { atomicExch(&flags[10], 1); atomicMax(&flags[11], n); }
}

// The fallback for link cells fuller than the masks hold: each forward entry
// (i -> j) enters i into j's reverse row at a position taken from a counter;
// then each row is sorted by cell (as seen from j) and chain position.
__global__ void __launch_bounds__(256)
k_rev_scatter(int nm, int cap, const int32_t *__restrict__ nlist, const int32_t *__restrict__ numn,
              int32_t *__restrict__ rlist, int32_t *__restrict__ numr, const int32_t *__restrict__ flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nm || !flags[12]) return;
    int n = numn[i];
    n = n < cap ? n : cap;
    for (int e = 0; e < n; ++e) {
        const int j = nlist[(size_t)i * cap + e];
        const int r = atomicAdd(&numr[j], 1);
        if (r < cap) rlist[(size_t)r * nm + j] = i;
    }
}

constexpr int kRevLocal = 96;   // reverse-row entries sorted in registers / local memory

__global__ void __launch_bounds__(256)
k_rev_sort(Params p, const int32_t *__restrict__ ic, const int32_t *__restrict__ cell_pos,
           int32_t *__restrict__ rlist, int32_t *__restrict__ numr, int32_t *__restrict__ flags) {
    // rank of each cell offset (dx, dy, dz), at (dx+1) + 3 (dy+1) + 9 (dz+1),
    // in a reverse row: 0 for the own cell, 1 + r for mirror offset r of the
    // half stencil (rows 14..26 of the stencil table)
    __shared__ int8_t srank[27];
    if (threadIdx.x < 27) srank[threadIdx.x] = -1;
    __syncthreads();
    if (threadIdx.x < 14) {
        const int r = threadIdx.x == 0 ? 0 : 13 + threadIdx.x;   // own cell, then rows 14..26
        const int idx = (c_stencil[r][0] + 1) + 3 * (c_stencil[r][1] + 1) + 9 * (c_stencil[r][2] + 1);
        srank[idx] = (int8_t)threadIdx.x;
    }
    __syncthreads();
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.nm || !flags[12]) return;
    const size_t nm = (size_t)p.nm;
    const int cap = p.nnbrs;
    int n = numr[j];
    if (n > cap) {
        atomicExch(&flags[10], 1);
        atomicMax(&flags[11], n);
        n = cap;
        numr[j] = cap;
    }
    const int cj = ic[j];
    const int jx = cj % p.nlcx, jy = (cj / p.nlcx) % p.nlcy, jz = cj / (p.nlcx * p.nlcy);
    auto key = [&](int i) {
        const int ci = ic[i];
        int dx = ci % p.nlcx - jx, dy = (ci / p.nlcx) % p.nlcy - jy, dz = ci / (p.nlcx * p.nlcy) - jz;
        dx = dx > 1 ? dx - p.nlcx : (dx < -1 ? dx + p.nlcx : dx);
        dy = dy > 1 ? dy - p.nlcy : (dy < -1 ? dy + p.nlcy : dy);
        dz = dz > 1 ? dz - p.nlcz : (dz < -1 ? dz + p.nlcz : dz);
        return ((int)srank[(dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)] << 20) | cell_pos[i];
    };
    int32_t *row = rlist + j;
    if (n <= kRevLocal) {
        int kv[kRevLocal], iv[kRevLocal];
        for (int e = 0; e < n; ++e) {
            const int i = row[(size_t)e * nm];
            const int kk = key(i);
            int m = e - 1;
            while (m >= 0 && kv[m] > kk) { kv[m + 1] = kv[m]; iv[m + 1] = iv[m]; --m; }
            kv[m + 1] = kk;
            iv[m + 1] = i;
        }
        for (int e = 0; e < n; ++e) row[(size_t)e * nm] = iv[e];
    } else {
        // long rows (crowded cells): insertion sort in place
        for (int e = 1; e < n; ++e) {
            const int i = row[(size_t)e * nm];
            const int kk = key(i);
            int m = e - 1;
            while (m >= 0 && key(row[(size_t)m * nm]) > kk) { row[(size_t)(m + 1) * nm] = row[(size_t)m * nm]; --m; }
            row[(size_t)(m + 1) * nm] = i;
        }
    }
}

// The box of a half-list build (B0 and rnear |B0^-1|_F) beside the
// positions' snapshot, for the rule that keeps the outer list across the
// next half-list rebuild
__global__ void k_half_box(Params p, BoxState *__restrict__ box) {
    if (threadIdx.x != 0) return;
    double b0[9], inv[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) b0[k] = box->b0[k];
    const double dh = mat_invert(b0, inv) ? p.rnear * frob(inv) : 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) box->bhalf[k] = b0[k];
    box->dmax_half = dh;
}

void launch_build_nlist(DeviceState &d, const Params &p, cudaStream_t s) {
    cudaMemcpyAsync(d.xhalf, d.posq, (size_t)p.nm * sizeof(int4), cudaMemcpyDeviceToDevice, s);
    k_half_box<<<1, 32, 0, s>>>(p, d.box);
    cudaMemsetAsync(d.flags + 12, 0, sizeof(int32_t), s);
    if (p.ivol == 0 || p.ivol == 1 || p.ivol == 4)
        k_build_nlist<true><<<p.ncell, 64, 0, s>>>(p, d.pos, d.posq, d.box, d.cell_start, d.cell_count,
                                                   d.cell_atoms, d.nlist, d.numn, d.revmask, d.flags);
    else
        k_build_nlist<false><<<p.ncell, 64, 0, s>>>(p, d.pos, d.posq, d.box, d.cell_start, d.cell_count,
                                                    d.cell_atoms, d.nlist, d.numn, d.revmask, d.flags);
    const int nb = (p.nm + 255) / 256;
    k_rev_gather<<<nb, 256, 0, s>>>(p, d.ic, d.cell_start, d.cell_count, d.cell_atoms, d.revmask, d.rlist,
                                    d.numr, d.flags);
    // the fallback (a link cell fuller than the masks hold): both return at once otherwise
    k_rev_scatter<<<nb, 256, 0, s>>>(p.nm, p.nnbrs, d.nlist, d.numn, d.rlist, d.numr, d.flags);
    k_rev_sort<<<nb, 256, 0, s>>>(p, d.ic, d.cell_pos, d.rlist, d.numr, d.flags);
}

// NLIST(nnbrs, nm) with 1-based entries; unused slots are zero.  ATOM_MAJOR:
// rows stored as NLIST itself (the half list), else entry-major (the reverse
// rows).
template <bool ATOM_MAJOR>
__global__ void k_export_nlist(int nm, int nnbrs, const int32_t *__restrict__ rows,
                               const int32_t *__restrict__ cnt, int32_t *__restrict__ out) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)nm * nnbrs) return;
    int a = (int)(e / nnbrs), k = (int)(e % nnbrs);
    out[e] = k < cnt[a] ? (ATOM_MAJOR ? rows[e] : rows[(size_t)k * nm + a]) + 1 : 0;
}

void launch_export_nlist(const int32_t *rows, const int32_t *cnt, bool atom_major, const Params &p, int32_t *out,
                         cudaStream_t s) {
    long long n = (long long)p.nm * p.nnbrs;
    int nb = (int)((n + 255) / 256);
    if (atom_major) k_export_nlist<true><<<nb, 256, 0, s>>>(p.nm, p.nnbrs, rows, cnt, out);
    else k_export_nlist<false><<<nb, 256, 0, s>>>(p.nm, p.nnbrs, rows, cnt, out);
}

}  // namespace moldy
