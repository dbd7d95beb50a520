// nlist.cu -- the hybrid Verlet half list (update_neighbourlist,
// src/neighbourlist_m.F90:103-276) built on the GPU.
//
// One warp owns one atom i.  It walks the 14 cells of the reference's half
// stencil in the reference's order (dz in {0,+1}; at dz=0 dy in {0,+1}; at
// dz=0,dy=0 dx in {0,+1}; otherwise dx,dy in {-1,0,+1}), and inside each cell
// the atoms in chain order; in i's own cell only the atoms after i.  Lanes
// test 32 candidates at a time and a ballot appends the accepted ones in
// order, so NLIST(:, i) matches the reference entry for entry.  The list is
// stored entry-major (entry k of atom i at k*nm + i) so that the per-step
// passes, one thread per atom, read it in contiguous 128-byte rows; the export
// transposes it to the reference's NLIST(nnbrs, nm).  The distance
// test uses separately rounded products and sums (no FMA), as the Fortran
// evaluates pr_get_realsep_from_dx, so r < rnear gives the same pair set.
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

__global__ void __launch_bounds__(256)
k_build_nlist(Params p, const double4 *__restrict__ pos, const BoxState *__restrict__ box,
              const int32_t *__restrict__ ic, const int32_t *__restrict__ cell_pos,
              const int32_t *__restrict__ cell_start, const int32_t *__restrict__ cell_count,
              const int32_t *__restrict__ cell_atoms, int32_t *__restrict__ nlist,
              int32_t *__restrict__ numn, int32_t *__restrict__ flags) {
    __shared__ double sb[9];
    if (threadIdx.x < 9) sb[threadIdx.x] = box->b0[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (a >= p.nm) return;
    double b[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) b[k] = sb[k];
    const int c = ic[a];
    const int q = cell_pos[a];
    const int cx = c % p.nlcx, cy = (c / p.nlcx) % p.nlcy, cz = c / (p.nlcx * p.nlcy);
    const double4 pa = pos[a];
    int count = 0;
    const unsigned lt = (1u << lane) - 1u;
    for (int s = 0; s < 14; ++s) {
        int jx = wrap(cx + c_stencil[s][0], p.nlcx);
        int jy = wrap(cy + c_stencil[s][1], p.nlcy);
        int jz = wrap(cz + c_stencil[s][2], p.nlcz);
        int jp = jx + p.nlcx * (jy + p.nlcy * jz);
        int L = cell_count[jp];
        const int32_t *seg = cell_atoms + cell_start[jp];
        int k0 = (jp == c) ? q + 1 : 0;
        for (int k = k0; k < L; k += 32) {
            int kk = k + lane;
            bool take = false;
            int j = 0;
            if (kk < L) {
                j = seg[kk];
                double4 pj = pos[j];
                double dx = __dsub_rn(pa.x, pj.x), dy = __dsub_rn(pa.y, pj.y), dz = __dsub_rn(pa.z, pj.z);
                min_image(p.ivol, dx, dy, dz);
                double r = realsep_exact(b, dx, dy, dz);
                take = r < p.rnear;
            }
            unsigned bal = __ballot_sync(0xffffffffu, take);
            if (take) {
                int slot = count + __popc(bal & lt);
                if (slot < p.nnbrs) nlist[(size_t)slot * p.nm + a] = j;
            }
            count += __popc(bal);
        }
    }
    if (lane == 0) {
        numn[a] = count < p.nnbrs ? count : p.nnbrs;
        if (count > p.nnbrs) {
            atomicExch(&flags[0], 1);
            atomicMax(&flags[2], a + 1);
        }
    }
}

void launch_build_nlist(DeviceState &d, const Params &p, cudaStream_t s) {
    long long threads = (long long)p.nm * 32;
    int nb = (int)((threads + 255) / 256);
    k_build_nlist<<<nb, 256, 0, s>>>(p, d.pos, d.box, d.ic, d.cell_pos, d.cell_start, d.cell_count,
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
