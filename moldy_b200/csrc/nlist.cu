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
// In a fully periodic box an FP32 distance from the fixed-point positions
// decides first: it is within 1e-5 A of the exact one, so a candidate more
// than kNlBand from rnear is taken or left by it alone, and only the others
// take the exact FP64 test.
#include "engine.h"

namespace moldy {

// (dx, dy, dz) offsets of the half stencil in the reference's loop order
__constant__ int8_t c_stencil[14][3] = {
    {0, 0, 0}, {1, 0, 0},
    {-1, 1, 0}, {0, 1, 0}, {1, 1, 0},
    {-1, -1, 1}, {0, -1, 1}, {1, -1, 1},
    {-1, 0, 1}, {0, 0, 1}, {1, 0, 1},
    {-1, 1, 1}, {0, 1, 1}, {1, 1, 1}};

__device__ __forceinline__ int wrap(int j, int n) { return j < 0 ? j + n : (j >= n ? j - n : j); }

constexpr int kNlStage = 640;   // staged candidates per home cell
constexpr int kNlWarps = 4;
constexpr double kNlBand = 1.0e-3;   // A; the FP32 test decides outside rnear -+ this

template <bool FIX>
__global__ void __launch_bounds__(32 * kNlWarps)
k_build_nlist(Params p, const double4 *__restrict__ pos, const int4 *__restrict__ posq,
              const BoxState *__restrict__ box,
              const int32_t *__restrict__ cell_start, const int32_t *__restrict__ cell_count,
              const int32_t *__restrict__ cell_atoms, int32_t *__restrict__ nlist,
              int32_t *__restrict__ numn, int32_t *__restrict__ flags) {
    __shared__ double sx[kNlStage], sy[kNlStage], sz[kNlStage];
    __shared__ int sj[kNlStage];
    __shared__ int4 sq[FIX ? kNlStage : 1];
    __shared__ int sbase[15], sstart[14];
    __shared__ double sb[9];
    const int c = blockIdx.x;
    const int L0 = cell_count[c];
    if (L0 == 0) return;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid < 9) sb[tid] = box->b0[tid];
    if (tid < 14) {
        const int cx = c % p.nlcx, cy = (c / p.nlcx) % p.nlcy, cz = c / (p.nlcx * p.nlcy);
        const int jx = wrap(cx + c_stencil[tid][0], p.nlcx);
        const int jy = wrap(cy + c_stencil[tid][1], p.nlcy);
        const int jz = wrap(cz + c_stencil[tid][2], p.nlcz);
        const int jp = jx + p.nlcx * (jy + p.nlcy * jz);
        sstart[tid] = cell_start[jp];
        sbase[tid + 1] = cell_count[jp];
    }
    __syncthreads();
    if (tid == 0) {
        sbase[0] = 0;
        for (int k = 1; k <= 14; ++k) sbase[k] += sbase[k - 1];
    }
    __syncthreads();
    const int total = sbase[14];
    const int staged = total < kNlStage ? total : kNlStage;
    for (int k = tid; k < staged; k += blockDim.x) {
        int s = 0;
        while (sbase[s + 1] <= k) ++s;
        const int j = cell_atoms[sstart[s] + (k - sbase[s])];
        const double4 pj = pos[j];
        sx[k] = pj.x; sy[k] = pj.y; sz[k] = pj.z; sj[k] = j;
        if (FIX) sq[k] = posq[j];
    }
    __syncthreads();
    double b[9];
    float bs[9];   // B0 per fixed-point unit
#pragma unroll
    for (int k = 0; k < 9; ++k) { b[k] = sb[k]; bs[k] = (float)(sb[k] * kFixUnit); }
    const float rlo2 = (float)((p.rnear - kNlBand) * (p.rnear - kNlBand));
    const float rhi2 = (float)((p.rnear + kNlBand) * (p.rnear + kNlBand));
    const unsigned lt = (1u << lane) - 1u;
    // home atom q sits at staged slot q (the home cell is staged first)
    for (int q = w; q < L0; q += kNlWarps) {
        const int a = cell_atoms[sstart[0] + q];
        const double4 pa = pos[a];
        const int4 qa = FIX ? posq[a] : make_int4(0, 0, 0, 0);
        int count = 0;
        for (int k0 = q + 1; k0 < total; k0 += 32) {
            const int kk = k0 + lane;
            bool take = false;
            int j = 0;
            if (kk < total) {
                double qx, qy, qz;
                int4 qj;
                if (kk < staged) {
                    qx = sx[kk]; qy = sy[kk]; qz = sz[kk]; j = sj[kk];
                    if (FIX) qj = sq[kk];
                } else {
                    int s = 0;
                    while (sbase[s + 1] <= kk) ++s;
                    j = cell_atoms[sstart[s] + (kk - sbase[s])];
                    const double4 pj = pos[j];
                    qx = pj.x; qy = pj.y; qz = pj.z;
                    if (FIX) qj = posq[j];
                }
                bool exact = true;
                if (FIX) {
                    const float dx = fix_to_float((int32_t)((uint32_t)qa.x - (uint32_t)qj.x));
                    const float dy = fix_to_float((int32_t)((uint32_t)qa.y - (uint32_t)qj.y));
                    const float dz = fix_to_float((int32_t)((uint32_t)qa.z - (uint32_t)qj.z));
                    const float rx = fmaf(bs[6], dz, fmaf(bs[3], dy, bs[0] * dx));
                    const float ry = fmaf(bs[7], dz, fmaf(bs[4], dy, bs[1] * dx));
                    const float rz = fmaf(bs[8], dz, fmaf(bs[5], dy, bs[2] * dx));
                    const float r2 = fmaf(rz, rz, fmaf(ry, ry, rx * rx));
                    if (r2 < rlo2) { take = true; exact = false; }
                    else if (r2 > rhi2) exact = false;
                }
                if (exact) {
                    double dx = __dsub_rn(pa.x, qx), dy = __dsub_rn(pa.y, qy), dz = __dsub_rn(pa.z, qz);
                    min_image(p.ivol, dx, dy, dz);
                    const double r = realsep_exact(b, dx, dy, dz);
                    take = r < p.rnear;
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, take);
            if (take) {
                const int slot = count + __popc(bal & lt);
                if (slot < p.nnbrs) nlist[(size_t)slot * p.nm + a] = j;
            }
            count += __popc(bal);
        }
        if (lane == 0) {
            numn[a] = count < p.nnbrs ? count : p.nnbrs;
            if (count > p.nnbrs) {
                atomicExch(&flags[0], 1);
                atomicMax(&flags[2], a + 1);
            }
        }
    }
}

void launch_build_nlist(DeviceState &d, const Params &p, cudaStream_t s) {
    if (p.ivol == 0 || p.ivol == 1 || p.ivol == 4)
        k_build_nlist<true><<<p.ncell, 32 * kNlWarps, 0, s>>>(p, d.pos, d.posq, d.box, d.cell_start, d.cell_count,
                                                              d.cell_atoms, d.nlist, d.numn, d.flags);
    else
        k_build_nlist<false><<<p.ncell, 32 * kNlWarps, 0, s>>>(p, d.pos, d.posq, d.box, d.cell_start, d.cell_count,
                                                               d.cell_atoms, d.nlist, d.numn, d.flags);
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
