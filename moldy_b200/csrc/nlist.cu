// nlist.cu -- the hybrid Verlet half list (update_neighbourlist,
// src/neighbourlist_m.F90:103-276) built on the GPU.
//
// One block owns one link cell.  It stages the atoms of the 14 cells of the
// reference's half stencil in shared memory, in the reference's order (dz in
// {0,+1}; at dz=0 dy in {0,+1}; at dz=0,dy=0 dx in {0,+1}; otherwise dx,dy in
// {-1,0,+1}), each cell's atoms in chain order, the home cell first.  Each
// warp then takes home atoms i in turn and walks the staged candidates from
// the one after i: the rest of i's own cell, then the other 13 cells.  Lanes
// test 32 candidates at a time and a ballot appends the accepted ones in
// order, so NLIST(:, i) matches the reference entry for entry.  Candidates
// past the staging capacity are read from global memory.  The list is
// stored entry-major (entry k of atom i at k*nm + i) so that the per-step
// passes, one thread per atom, read it in contiguous 128-byte rows; the export
// transposes it to the reference's NLIST(nnbrs, nm).  The distance
// test uses separately rounded products and sums (no FMA), as the Fortran
// evaluates pr_get_realsep_from_dx, so r < rnear gives the same pair set.
// In a fully periodic box an FP32 distance decides first (from positions
// relative to the home cell's centre, or from the fixed-point difference; see
// k_build_nlist): it is within 1e-4 A of the exact one, so a candidate more
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

constexpr int kNlStage = 640;   // staged candidates per home cell (27 cells)
constexpr double kNlBand = 1.0e-3;   // A; the FP32 test decides outside rnear -+ this

// Pre-test of a candidate.  PERIODIC = false (boxes not periodic in all three
// directions): the exact FP64 test for every candidate.  PERIODIC = true: an
// FP32 distance decides outside the band rnear -+ kNlBand, in one of two
// forms chosen per launch on the device:
//  fixed point   the FP32 distance from the 32-bit fixed-point difference
//                (the integer difference is the minimum image);
//  cell relative the FP32 distance between Cartesian positions relative to
//                the home cell's centre, computed once per staged candidate
//                instead of once per (home atom, candidate).  It needs at least
//                4 cells per direction, so that every staged candidate lies
//                within 1.5 cells, less than half a box, of the centre and its
//                fixed-point offset from it is its own minimum image (the
//                pair's difference is then the minimum image too), and a
//                stencil reach (centre to the far corner of a stencil cell)
//                under 150 A: the FP32 error is then a few units in the last
//                place of 150 A, under 1e-4 A, far inside the band.
__device__ double stencil_reach(const double *b, int nlcx, int nlcy, int nlcz) {
    double m = 0.0;
    for (int k = 0; k < 8; ++k) {
        const double f0 = (k & 1 ? 1.5 : -1.5) / nlcx, f1 = (k & 2 ? 1.5 : -1.5) / nlcy,
                     f2 = (k & 4 ? 1.5 : -1.5) / nlcz;
        double r2 = 0.0;
        for (int i = 0; i < 3; ++i) {
            const double c = b[i] * f0 + b[3 + i] * f1 + b[6 + i] * f2;
            r2 += c * c;
        }
        m = fmax(m, sqrt(r2));
    }
    return m;
}

// Shared state of one block's candidate tests
struct NlStage {
    const int4 *sqc;        // staged fixed-point or cell-relative positions, atom id in w
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

// r(a, candidate kk) < rnear, decided as the reference evaluates it: the FP32
// pre-test outside the band, the exact FP64 separation (separately rounded
// products and sums) inside it; j receives the candidate's atom id.  The
// exact test is symmetric bit for bit (negating a difference is exact), so
// the forward and backward rows describe the same pair set.
template <bool PERIODIC>
__device__ __forceinline__ bool nl_take(const NlStage &S, int kk, const double4 &pa, const int4 &qa, bool rel_a,
                                        bool rel, const int4 &cen, int &j) {
    int4 qj = make_int4(0, 0, 0, 0);
    const bool staged = kk < S.staged;
    if (staged) {
        j = S.sqc[kk].w;
    } else {
        int s = 0;
        while (S.sbase[s + 1] <= kk) ++s;
        j = S.cell_atoms[S.sstart[s] + (kk - S.sbase[s])];
    }
    if (PERIODIC) {
        // the staged copy is in the home atom's form (cell relative when rel),
        // else the fixed-point position from global memory
        qj = staged && (rel_a || !rel) ? S.sqc[kk] : S.posq[j];
        float rx, ry, rz;
        if (rel_a && staged) {   // both cell relative
            rx = __int_as_float(qa.x) - __int_as_float(qj.x);
            ry = __int_as_float(qa.y) - __int_as_float(qj.y);
            rz = __int_as_float(qa.z) - __int_as_float(qj.z);
        } else {
            // fixed-point difference (taken from the cell centre when the home
            // atom is cell relative and the candidate lies beyond the staging)
            const int4 qi = rel_a ? cen : qa;
            const float dx = __int2float_rn((int32_t)((uint32_t)qi.x - (uint32_t)qj.x));
            const float dy = __int2float_rn((int32_t)((uint32_t)qi.y - (uint32_t)qj.y));
            const float dz = __int2float_rn((int32_t)((uint32_t)qi.z - (uint32_t)qj.z));
            const float *bs = S.bs;
            rx = fmaf(bs[6], dz, fmaf(bs[3], dy, bs[0] * dx));
            ry = fmaf(bs[7], dz, fmaf(bs[4], dy, bs[1] * dx));
            rz = fmaf(bs[8], dz, fmaf(bs[5], dy, bs[2] * dx));
            if (rel_a) { rx += __int_as_float(qa.x); ry += __int_as_float(qa.y); rz += __int_as_float(qa.z); }
        }
        const float r2 = fmaf(rz, rz, fmaf(ry, ry, rx * rx));
        if (r2 < S.rlo2) return true;
        if (r2 > S.rhi2) return false;
    }
    return nl_exact(S.pos, S.b, S.ivol, S.rnear, pa, j);
}

// One warp per link cell stages the atoms of the 27 surrounding cells: the
// home cell, the 13 cells of the reference's half stencil, then the 13 mirror
// cells, each cell's atoms in chain order.  Each lane then takes one home atom
// a (the cell's atoms 32 at a time) and walks the staged candidates in order,
// every lane reading the same candidate (a shared-memory broadcast), and
// appends to
//   row(a)      NLIST(:, a): the half-stencil candidates after a in staging
//               order, in the reference's order (entry for entry);
//   reverse(a)  the atoms j with a in row(j): a's own cell before a, then the
//               mirror cells, in staging order.
template <bool PERIODIC>
__global__ void __launch_bounds__(32)
k_build_nlist(Params p, const double4 *__restrict__ pos, const int4 *__restrict__ posq,
              const BoxState *__restrict__ box,
              const int32_t *__restrict__ cell_start, const int32_t *__restrict__ cell_count,
              const int32_t *__restrict__ cell_atoms, int32_t *__restrict__ nlist,
              int32_t *__restrict__ numn, int32_t *__restrict__ rlist, int32_t *__restrict__ numr,
              int32_t *__restrict__ flags) {
    // per staged candidate: its fixed-point position (fixed-point form) or its
    // cell-relative Cartesian position as float bits (cell-relative form) in
    // x, y, z, and its atom id in w
    __shared__ int4 sqc[kNlStage];
    __shared__ int sbase[28], sstart[27];
    __shared__ double sb[9];
    const int c = blockIdx.x;
    const int L0 = cell_count[c];
    if (L0 == 0) return;
    const int lane = threadIdx.x;
    const int cx = c % p.nlcx, cy = (c / p.nlcx) % p.nlcy, cz = c / (p.nlcx * p.nlcy);
    if (lane < 9) sb[lane] = box->b0[lane];
    int cnt = 0, st = 0;
    if (lane < 27) {
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
    if (lane < 27) { sbase[lane + 1] = inc; sstart[lane] = st; }
    if (lane == 0) sbase[0] = 0;
    __syncwarp();
    const bool rel = PERIODIC && p.nlcx >= 4 && p.nlcy >= 4 && p.nlcz >= 4 &&
                     stencil_reach(sb, p.nlcx, p.nlcy, p.nlcz) < 150.0;
    float bs[9];   // B0 per fixed-point unit
#pragma unroll
    for (int k = 0; k < 9; ++k) bs[k] = (float)(sb[k] * kFixUnit);
    // the home cell's centre in fixed point: fractional (ix + 1/2) / nlc - 1/2
    // per direction (a cell holds x - nint(x) in [ix/nlc - 1/2, (ix+1)/nlc - 1/2))
    int4 cen = make_int4(0, 0, 0, 0);
    if (rel) {
        cen.x = fix32((cx + 0.5) / p.nlcx - 0.5);
        cen.y = fix32((cy + 0.5) / p.nlcy - 0.5);
        cen.z = fix32((cz + 0.5) / p.nlcz - 0.5);
    }
    const int fwd_end = sbase[14], total = sbase[27];
    const int staged = total < kNlStage ? total : kNlStage;
    // two phases of independent loads: the atom ids, then their positions
#pragma unroll 4
    for (int k = lane; k < staged; k += 32) {
        int sc = 0;
        while (sbase[sc + 1] <= k) ++sc;
        sqc[k].w = cell_atoms[sstart[sc] + (k - sbase[sc])];
    }
    __syncwarp();
    if (PERIODIC) {
#pragma unroll 4
        for (int k = lane; k < staged; k += 32) {
            const int j = sqc[k].w;
            const int4 qj = posq[j];
            if (rel) {
                const float dx = __int2float_rn((int32_t)((uint32_t)qj.x - (uint32_t)cen.x));
                const float dy = __int2float_rn((int32_t)((uint32_t)qj.y - (uint32_t)cen.y));
                const float dz = __int2float_rn((int32_t)((uint32_t)qj.z - (uint32_t)cen.z));
                sqc[k] = make_int4(__float_as_int(fmaf(bs[6], dz, fmaf(bs[3], dy, bs[0] * dx))),
                                   __float_as_int(fmaf(bs[7], dz, fmaf(bs[4], dy, bs[1] * dx))),
                                   __float_as_int(fmaf(bs[8], dz, fmaf(bs[5], dy, bs[2] * dx))), j);
            } else {
                sqc[k] = make_int4(qj.x, qj.y, qj.z, j);
            }
        }
    }
    // records past the staged candidates, up to the next multiple of 32: far
    // away, so the chunked walk below needs no bound check
    if (PERIODIC && rel) {
        const int pad_end = (staged + 31) & ~31;
        for (int k = staged + lane; k < pad_end && k < kNlStage; k += 32)
            sqc[k] = make_int4(__float_as_int(1.0e30f), __float_as_int(1.0e30f), __float_as_int(1.0e30f), -1);
    }
    __syncwarp();
    NlStage S;
    S.sqc = sqc; S.sbase = sbase; S.sstart = sstart; S.cell_atoms = cell_atoms;
    S.posq = posq; S.pos = pos; S.bs = bs; S.b = sb; S.staged = staged; S.ivol = p.ivol; S.rnear = p.rnear;
    S.rlo2 = (float)((p.rnear - kNlBand) * (p.rnear - kNlBand));
    S.rhi2 = (float)((p.rnear + kNlBand) * (p.rnear + kNlBand));
    const size_t nm = (size_t)p.nm;
    int over = 0;
    for (int q0 = 0; q0 < L0; q0 += 32) {
        const int q = q0 + lane;                 // this lane's home atom: staged slot q
        const bool live = q < L0;
        const int a = live ? cell_atoms[sstart[0] + q] : 0;
        const double4 pa = live ? pos[a] : make_double4(0.0, 0.0, 0.0, 0.0);
        int4 qa = make_int4(0, 0, 0, 0);   // fixed point, or the cell-relative position's bits
        if (PERIODIC && live) qa = q < staged ? sqc[q] : posq[a];
        const bool rel_a = rel && q < staged;
        const float ax = __int_as_float(qa.x), ay = __int_as_float(qa.y), az = __int_as_float(qa.z);
        // every append below is predicated, with no branch: entry n of a row
        // sits at n * nm + a (entry-major)
        int nf = 0, nr = 0;
        const int cap = p.nnbrs;
        auto append = [&](bool take, bool fwd, int j) {
            const int n = fwd ? nf : nr;
            int32_t *base = fwd ? nlist : rlist;
            if (take && n < cap) base[(size_t)n * nm + a] = j;
            nf += (take && fwd) ? 1 : 0;
            nr += (take && !fwd) ? 1 : 0;
        };
        int kk = 0;
        if (rel && min(L0, q0 + 32) <= staged) {   // cell relative, every live lane's atom staged
            // 32 candidates at a time: every lane tests its home atom against
            // each (a shared-memory broadcast) into a keep mask and a mask of
            // those in the band around rnear, then appends its kept ones in
            // order, so the append work is paid per kept pair only
            for (int k0 = 0; k0 < staged; k0 += 32) {
                unsigned tm = 0u, um = 0u;
#pragma unroll
                for (int b = 0; b < 32; ++b) {
                    const int4 cq = sqc[k0 + b];
                    const float rx = ax - __int_as_float(cq.x), ry = ay - __int_as_float(cq.y),
                                rz = az - __int_as_float(cq.z);
                    const float r2 = fmaf(rz, rz, fmaf(ry, ry, rx * rx));
                    tm |= (r2 < S.rlo2 ? 1u : 0u) << b;
                    um |= (r2 <= S.rhi2 ? 1u : 0u) << b;
                }
                um &= ~tm;                                   // in the band: the exact test decides
                const unsigned self = (q >= k0 && q < k0 + 32) ? (1u << (q - k0)) : 0u;
                tm = live ? tm & ~self : 0u;
                um = live ? um & ~self : 0u;
                while (um) {
                    const int b = __ffs(um) - 1;
                    um &= um - 1;
                    if (nl_exact(pos, sb, p.ivol, p.rnear, pa, sqc[k0 + b].w)) tm |= 1u << b;
                }
                while (tm) {
                    const int b = __ffs(tm) - 1;
                    tm &= tm - 1;
                    const int c = k0 + b;
                    append(true, c > q && c < fwd_end, sqc[c].w);
                }
            }
            kk = staged;
        }
        // the rest: candidates beyond the staging, every candidate of the
        // fixed-point form and of boxes not periodic in all three directions
        for (; kk < total; ++kk) {
            int j = 0;
            const bool take = live && kk != q && nl_take<PERIODIC>(S, kk, pa, qa, rel_a, rel, cen, j);
            append(take, kk > q && kk < fwd_end, j);
        }
        if (live) {
            numn[a] = nf < p.nnbrs ? nf : p.nnbrs;
            numr[a] = nr < p.nnbrs ? nr : p.nnbrs;
            if (nf > p.nnbrs) {
                atomicExch(&flags[0], 1);
                atomicMax(&flags[2], a + 1);
            }
            if (nr > p.nnbrs) over = max(over, nr);
        }
    }
    if (over) { atomicExch(&flags[10], 1); atomicMax(&flags[11], over); }
}

void launch_build_nlist(DeviceState &d, const Params &p, cudaStream_t s) {
    if (p.ivol == 0 || p.ivol == 1 || p.ivol == 4)
        k_build_nlist<true><<<p.ncell, 32, 0, s>>>(p, d.pos, d.posq, d.box, d.cell_start, d.cell_count,
                                                   d.cell_atoms, d.nlist, d.numn, d.rlist, d.numr, d.flags);
    else
        k_build_nlist<false><<<p.ncell, 32, 0, s>>>(p, d.pos, d.posq, d.box, d.cell_start, d.cell_count,
                                                    d.cell_atoms, d.nlist, d.numn, d.rlist, d.numr, d.flags);
}

// NLIST(nnbrs, nm) with 1-based entries; unused slots are zero
__global__ void k_export_nlist(int nm, int nnbrs, const int32_t *__restrict__ nlist,
                               const int32_t *__restrict__ numn, int32_t *__restrict__ out) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)nm * nnbrs) return;
    int a = (int)(e / nnbrs), k = (int)(e % nnbrs);
    out[e] = k < numn[a] ? nlist[(size_t)k * nm + a] + 1 : 0;
}

void launch_export_nlist(const DeviceState &d, const Params &p, int32_t *out, cudaStream_t s) {
    long long n = (long long)p.nm * p.nnbrs;
    int nb = (int)((n + 255) / 256);
    k_export_nlist<<<nb, 256, 0, s>>>(p.nm, p.nnbrs, d.nlist, d.numn, out);
}

}  // namespace moldy
