// cells.cu -- link cells (linkcell_m) on the GPU.
//
// The reference keeps each link cell as a circular singly-linked chain
// (l0 = chain start, link = successor, src/linkcell_m.F90:61-64).  Here a cell
// is a CSR segment listing its atoms in chain traversal order starting at l0.
// linkup (src/linkcell_m.F90:122-198) inserts atoms in index order, so every
// segment is ascending.  relink (src/linkcell_m.F90:215-274) is a sequential
// loop over atoms; its effect on one cell depends only on the removals from
// and insertions into that cell, taken in atom-index order, so each cell is
// replayed independently (one warp per cell, k_relink_cells):
//   remove x: the chain start moves to x's successor;
//   insert i: i goes right after the current start and becomes the start.
// The cells' segments are placed by an exclusive scan of their sizes.
#include "engine.h"

namespace moldy {

__global__ void k_assign_cells(const double4 *__restrict__ pos, int nm, int nlcx, int nlcy,
                               int nlcz, int32_t *__restrict__ ic_out,
                               int32_t *__restrict__ count) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nm) return;
    double4 p = pos[a];
    int ix = cell_coord(p.x, nlcx), iy = cell_coord(p.y, nlcy), iz = cell_coord(p.z, nlcz);
    int c = ix + nlcx * iy + nlcx * nlcy * iz;
    ic_out[a] = c;
    if (count) atomicAdd(&count[c], 1);
}

__global__ void k_fill_cells(const int32_t *__restrict__ ic, int nm,
                             const int32_t *__restrict__ start, int32_t *__restrict__ cursor,
                             int32_t *__restrict__ atoms) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nm) return;
    int c = ic[a];
    int k = atomicAdd(&cursor[c], 1);
    atoms[start[c] + k] = a;
}

// ascending order inside each cell = linkup's chain order
__global__ void k_sort_cells(int ncell, const int32_t *__restrict__ start,
                             const int32_t *__restrict__ count, int32_t *__restrict__ atoms,
                             int32_t *__restrict__ cell_pos) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    int32_t *seg = atoms + start[c];
    int n = count[c];
    for (int i = 1; i < n; ++i) {
        int v = seg[i], k = i - 1;
        while (k >= 0 && seg[k] > v) { seg[k + 1] = seg[k]; --k; }
        seg[k + 1] = v;
    }
    for (int i = 0; i < n; ++i) cell_pos[seg[i]] = i;
}

// single-block exclusive scan: out[0..n-1] exclusive sums, out[n] total.
// Thread t sums the contiguous segment [t per, (t + 1) per) with its loads
// independent of one another, the block scans the segment sums, then each
// thread writes its segment's prefixes (the second read hits the cache).
__global__ void __launch_bounds__(1024)
k_exclusive_scan(const int32_t *__restrict__ in, int32_t *__restrict__ out, int n) {
    __shared__ int32_t wsum[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int b0 = min(n, (int)threadIdx.x * per), b1 = min(n, b0 + per);
    int v = 0;
#pragma unroll 8
    for (int i = b0; i < b1; ++i) v += in[i];
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < nw ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) wsum[lane] = w;
    }
    __syncthreads();
    int run = (warp > 0 ? wsum[warp - 1] : 0) + x - v;   // exclusive prefix of this segment
    for (int i = b0; i < b1; ++i) {
        out[i] = run;
        run += in[i];
    }
    if (threadIdx.x == blockDim.x - 1) out[n] = run;
}

// Multi-block exclusive scan for n up to 2^31: block sums of tiles of
// kScanTile elements, a scan of the block sums, then each block's tile scanned
// from its offset; every load and store is coalesced.  scratch holds
// ceil(n / kScanTile) ints.
constexpr int kScanTile = 2048;   // 256 threads x 8 contiguous elements

__device__ __forceinline__ int block_excl_scan256(int v, int *wsum, int &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < 8 ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < 8) wsum[lane] = w;
    }
    __syncthreads();
    total = wsum[7];
    const int r = (warp > 0 ? wsum[warp - 1] : 0) + x - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(256) k_scan_reduce(const int32_t *__restrict__ in, int n, int32_t *__restrict__ bsum) {
    __shared__ int wsum[8];
    const int base = blockIdx.x * kScanTile;
    int v = 0;
#pragma unroll
    for (int k = 0; k < kScanTile / 256; ++k) {
        const int i = base + k * 256 + threadIdx.x;
        if (i < n) v += in[i];
    }
    int total = 0;
    block_excl_scan256(v, wsum, total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(256) k_scan_blocks(int32_t *__restrict__ bsum, int nb, int32_t *__restrict__ out,
                                                      int n) {
    __shared__ int wsum[8];
    int carry = 0;
    for (int b0 = 0; b0 < nb; b0 += 256) {
        const int i = b0 + threadIdx.x;
        const int v = i < nb ? bsum[i] : 0;
        int total = 0;
        const int e = block_excl_scan256(v, wsum, total);
        if (i < nb) bsum[i] = carry + e;
        carry += total;
    }
    if (threadIdx.x == 0) out[n] = carry;
}

__global__ void __launch_bounds__(256) k_scan_apply(const int32_t *__restrict__ in, int32_t *__restrict__ out, int n,
                                                     const int32_t *__restrict__ bsum) {
    __shared__ int wsum[8];
    const int base = blockIdx.x * kScanTile + threadIdx.x * 8;
    int v[8];
    int sum = 0;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        v[u] = base + u < n ? in[base + u] : 0;
        sum += v[u];
    }
    int total = 0;
    int run = bsum[blockIdx.x] + block_excl_scan256(sum, wsum, total);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        if (base + u < n) out[base + u] = run;
        run += v[u];
    }
}

void launch_exclusive_scan(const int32_t *in, int32_t *out, int n, cudaStream_t s, int32_t *scratch) {
    if (!scratch) {
        k_exclusive_scan<<<1, 1024, 0, s>>>(in, out, n);
        return;
    }
    const int nb = (n + kScanTile - 1) / kScanTile;
    k_scan_reduce<<<nb, 256, 0, s>>>(in, n, scratch);
    k_scan_blocks<<<1, 256, 0, s>>>(scratch, nb, out, n);
    k_scan_apply<<<nb, 256, 0, s>>>(in, out, n, scratch);
}

void launch_linkup(DeviceState &d, const Params &p, cudaStream_t s) {
    int nb = (p.nm + kAtomThreads - 1) / kAtomThreads;
    int nbc = (p.ncell + kAtomThreads - 1) / kAtomThreads;
    cudaMemsetAsync(d.cell_count, 0, sizeof(int32_t) * p.ncell, s);
    k_assign_cells<<<nb, kAtomThreads, 0, s>>>(d.pos, p.nm, p.nlcx, p.nlcy, p.nlcz, d.ic, d.cell_count);
    launch_exclusive_scan(d.cell_count, d.cell_start, p.ncell, s, d.scan_tmp);
    cudaMemsetAsync(d.new_count, 0, sizeof(int32_t) * p.ncell, s);
    k_fill_cells<<<nb, kAtomThreads, 0, s>>>(d.ic, p.nm, d.cell_start, d.new_count, d.cell_atoms);
    k_sort_cells<<<nbc, kAtomThreads, 0, s>>>(p.ncell, d.cell_start, d.cell_count, d.cell_atoms,
                                              d.cell_pos);
}

// ------------------------------------------------------------------ relink --
__global__ void k_relink_assign(const double4 *__restrict__ pos, int nm, int nlcx, int nlcy,
                                int nlcz, const int32_t *__restrict__ ic,
                                int32_t *__restrict__ ic_new, int32_t *__restrict__ arr_count) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nm) return;
    double4 p = pos[a];
    int ix = cell_coord(p.x, nlcx), iy = cell_coord(p.y, nlcy), iz = cell_coord(p.z, nlcz);
    int c = ix + nlcx * iy + nlcx * nlcy * iz;
    ic_new[a] = c;
    if (c != ic[a]) atomicAdd(&arr_count[c], 1);
}

__global__ void k_relink_arrivals(int nm, const int32_t *__restrict__ ic,
                                  const int32_t *__restrict__ ic_new,
                                  const int32_t *__restrict__ arr_start,
                                  int32_t *__restrict__ cursor, int32_t *__restrict__ arr_list) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nm) return;
    int c = ic_new[a];
    if (c == ic[a]) return;
    int k = atomicAdd(&cursor[c], 1);
    arr_list[arr_start[c] + k] = a;
}

// Replays relink's chain surgery for one cell (src/linkcell_m.F90:215-274).
// The reference visits the atoms in index order; an atom that changed cell
// is unlinked from its old chain (the chain start moves to its successor)
// and linked into its new cell's chain after the start, becoming the start.
// Per cell that is a merge, in atom-index order, of its departures and its
// arrivals.  The working sequence W holds the circular chain order; st is the
// position of the chain start.  On return W holds the new chain from its
// start (st = 0).  Serial form, one thread: W has room for the old atoms plus
// all arrivals.
__device__ void relink_cell_serial(int c, int L, int32_t *W, const int32_t *__restrict__ ic,
                                   const int32_t *__restrict__ ic_new, int32_t *A, int na, int &Lout) {
    for (int i = 1; i < na; ++i) {   // arrivals in atom-index order
        int v = A[i], k = i - 1;
        while (k >= 0 && A[k] > v) { A[k + 1] = A[k]; --k; }
        A[k + 1] = v;
    }
    int st = 0, ia = 0, last = -1;
    const int kInf = 0x7fffffff;
    for (;;) {
        int lmin = kInf, lpos = -1;
        for (int k = 0; k < L; ++k) {
            int x = W[k];
            if (x > last && x < lmin && ic[x] == c && ic_new[x] != c) { lmin = x; lpos = k; }
        }
        int nxt = ia < na ? A[ia] : kInf;
        if (lmin == kInf && nxt == kInf) break;
        if (lmin < nxt) {            // remove lmin; start moves to its successor
            for (int k = lpos; k < L - 1; ++k) W[k] = W[k + 1];
            --L;
            st = (L == 0) ? 0 : (lpos < L ? lpos : 0);
            last = lmin;
        } else {                     // insert after the start; it becomes the start
            if (L == 0) {
                W[0] = nxt; L = 1; st = 0;
            } else {
                for (int k = L; k > st + 1; --k) W[k] = W[k - 1];
                W[st + 1] = nxt;
                ++L;
                st = st + 1;
            }
            ++ia;
        }
    }
    // rotate so that the chain starts at W[0] (through the free tail of W)
    for (int r = 0; r < st; ++r) {
        const int x = W[0];
        for (int k = 0; k < L - 1; ++k) W[k] = W[k + 1];
        W[L - 1] = x;
    }
    Lout = L;
}

// One warp per cell.  When the old atoms and the arrivals fit in 64 slots,
// lane k holds slots k and 32 + k of W, and each event is a warp minimum and
// one shuffle shift of both halves; otherwise lane 0 runs the serial form.
// (Link cells span two or three lattice planes per direction, so in bcc
// crystals they hold 16 to 54 atoms.)  Writes the new chain (from its start)
// to the cell's work segment and its length to new_count.
__global__ void __launch_bounds__(256)
k_relink_cells(int ncell, const int32_t *__restrict__ cell_start, const int32_t *__restrict__ cell_count,
               const int32_t *__restrict__ cell_atoms, const int32_t *__restrict__ ic,
               const int32_t *__restrict__ ic_new, const int32_t *__restrict__ arr_start,
               int32_t *__restrict__ arr_count_rot, int32_t *__restrict__ arr_list, int32_t *__restrict__ work,
               int32_t *__restrict__ new_count) {
    const int lane = threadIdx.x & 31;
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= ncell) return;   // warp-uniform
    int L = cell_count[c];
    const int32_t *old = cell_atoms + cell_start[c];
    int32_t *W = work + cell_start[c] + arr_start[c];
    const int na = arr_count_rot[c];
    int32_t *A = arr_list + arr_start[c];
    const unsigned full = 0xffffffffu;
    if (L + na > 64) {
        if (lane == 0) {
            for (int k = 0; k < L; ++k) W[k] = old[k];
            int Ln = 0;
            relink_cell_serial(c, L, W, ic, ic_new, A, na, Ln);
            new_count[c] = Ln;
            arr_count_rot[c] = 0;
        }
        return;
    }
    const int kInf = 0x7fffffff;
    const int hi = 32 + lane;   // this lane's second slot
    // slot k: W[k] and whether it departs
    int w0 = lane < L ? old[lane] : kInf, w1 = hi < L ? old[hi] : kInf;
    bool d0 = lane < L && ic_new[w0] != c, d1 = hi < L && ic_new[w1] != c;
    // this lane's arrivals (at most two), taken in atom-index order
    int a0 = lane < na ? A[lane] : kInf, a1 = hi < na ? A[hi] : kInf;
    int st = 0;
    for (;;) {
        const int lmin = __reduce_min_sync(full, min(d0 ? w0 : kInf, d1 ? w1 : kInf));
        const int nxt = __reduce_min_sync(full, min(a0, a1));
        if (lmin == kInf && nxt == kInf) break;
        if (lmin < nxt) {            // remove lmin; start moves to its successor
            const unsigned b0 = __ballot_sync(full, d0 && w0 == lmin);
            const unsigned b1 = __ballot_sync(full, d1 && w1 == lmin);
            const int lpos = b0 ? __ffs(b0) - 1 : 32 + __ffs(b1) - 1;
            // every slot from lpos on takes the next slot's content
            const int w0n = __shfl_down_sync(full, w0, 1), w1n = __shfl_down_sync(full, w1, 1);
            const bool d0n = __shfl_down_sync(full, d0, 1), d1n = __shfl_down_sync(full, d1, 1);
            const int w32 = __shfl_sync(full, w1, 0);
            const bool d32 = __shfl_sync(full, d1, 0);
            if (lane >= lpos) { w0 = lane < 31 ? w0n : w32; d0 = lane < 31 ? d0n : d32; }
            if (hi >= lpos) { w1 = lane < 31 ? w1n : kInf; d1 = lane < 31 ? d1n : false; }
            --L;
            st = (L == 0) ? 0 : (lpos < L ? lpos : 0);
        } else {                     // insert after the start; it becomes the start
            if (a0 == nxt) a0 = kInf;   // taken
            else if (a1 == nxt) a1 = kInf;
            if (L == 0) {
                if (lane == 0) { w0 = nxt; d0 = false; }
                L = 1;
                st = 0;
            } else {
                const int pos = st + 1;
                // every slot after pos, up to L, takes the previous slot's content
                const int w0p = __shfl_up_sync(full, w0, 1), w1p = __shfl_up_sync(full, w1, 1);
                const bool d0p = __shfl_up_sync(full, d0, 1), d1p = __shfl_up_sync(full, d1, 1);
                const int w31 = __shfl_sync(full, w0, 31);
                const bool d31 = __shfl_sync(full, d0, 31);
                if (lane > pos && lane <= L) { w0 = w0p; d0 = d0p; }
                if (lane == pos) { w0 = nxt; d0 = false; }
                if (hi > pos && hi <= L) { w1 = lane == 0 ? w31 : w1p; d1 = lane == 0 ? d31 : d1p; }
                if (hi == pos) { w1 = nxt; d1 = false; }
                ++L;
                st = pos;
            }
        }
    }
    // the new chain from its start
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int i = lane + 32 * h;
        const int src = L > 0 ? (st + i) % L : 0;
        const int x0 = __shfl_sync(full, w0, src & 31), x1 = __shfl_sync(full, w1, src & 31);
        if (i < L) W[i] = src < 32 ? x0 : x1;
    }
    if (lane == 0) { new_count[c] = L; arr_count_rot[c] = 0; }
}

// One warp per cell: the new chain (rotated by rot[c] < L) into the cell's
// segment of the new cell lists, and each atom's chain position.
__global__ void __launch_bounds__(256)
k_relink_write(int ncell, int nm, const int32_t *__restrict__ cell_start,
               const int32_t *__restrict__ arr_start,
               const int32_t *__restrict__ rot, const int32_t *__restrict__ work,
               const int32_t *__restrict__ new_count,
               const int32_t *__restrict__ new_start, int32_t *__restrict__ atoms2,
               int32_t *__restrict__ cell_pos, int32_t *__restrict__ flags) {
    const int lane = threadIdx.x & 31;
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= ncell) return;   // warp-uniform
    const int L = new_count[c], st = rot[c];
    const int base = new_start[c];
    if (L < 0 || base < 0 || base + L > nm || st < 0 || (L > 0 && st >= L)) {   // inconsistent: record, skip
        if (lane == 0) atomicExch(&flags[1], 1);
        return;
    }
    const int32_t *W = work + cell_start[c] + arr_start[c];
    int32_t *out = atoms2 + base;
    for (int k = lane; k < L; k += 32) {
        const int j = st + k < L ? st + k : st + k - L;
        const int x = W[j];
        if (x < 0 || x >= nm) { atomicExch(&flags[1], 1); continue; }
        out[k] = x;
        cell_pos[x] = k;
    }
}

void launch_relink(DeviceState &d, const Params &p, cudaStream_t s) {
    int nb = (p.nm + kAtomThreads - 1) / kAtomThreads;
    cudaMemsetAsync(d.arr_count, 0, sizeof(int32_t) * p.ncell, s);
    k_relink_assign<<<nb, kAtomThreads, 0, s>>>(d.pos, p.nm, p.nlcx, p.nlcy, p.nlcz, d.ic, d.ic_new,
                                                d.arr_count);
    launch_exclusive_scan(d.arr_count, d.arr_start, p.ncell, s, d.scan_tmp);
    cudaMemsetAsync(d.new_count, 0, sizeof(int32_t) * p.ncell, s);
    k_relink_arrivals<<<nb, kAtomThreads, 0, s>>>(p.nm, d.ic, d.ic_new, d.arr_start, d.new_count,
                                                  d.arr_list);
    const int nbw = (p.ncell + 7) / 8;   // one warp per cell, 8 per block
    k_relink_cells<<<nbw, 256, 0, s>>>(p.ncell, d.cell_start, d.cell_count, d.cell_atoms, d.ic,
                                       d.ic_new, d.arr_start, d.arr_count, d.arr_list, d.work,
                                       d.new_count);
    launch_exclusive_scan(d.new_count, d.new_start, p.ncell, s, d.scan_tmp);
    k_relink_write<<<(p.ncell + 7) / 8, 256, 0, s>>>(p.ncell, p.nm, d.cell_start, d.arr_start,
                                                d.arr_count, d.work, d.new_count, d.new_start,
                                                d.cell_atoms2, d.cell_pos, d.flags);
    // commit (copies keep buffer addresses fixed for graph capture)
    cudaMemcpyAsync(d.cell_atoms, d.cell_atoms2, sizeof(int32_t) * p.nm, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(d.cell_start, d.new_start, sizeof(int32_t) * (p.ncell + 1),
                    cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(d.cell_count, d.new_count, sizeof(int32_t) * p.ncell, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(d.ic, d.ic_new, sizeof(int32_t) * p.nm, cudaMemcpyDeviceToDevice, s);
}

// -------------------------------------------------------------- export -----
__global__ void k_export_cells(int ncell, const int32_t *__restrict__ start,
                               const int32_t *__restrict__ count,
                               const int32_t *__restrict__ atoms, int32_t *__restrict__ l0,
                               int32_t *__restrict__ link) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    int n = count[c];
    const int32_t *seg = atoms + start[c];
    l0[c] = n > 0 ? seg[0] + 1 : 0;
    for (int k = 0; k < n; ++k) link[seg[k]] = seg[(k + 1) % n] + 1;
}

void launch_export_linkcells(const DeviceState &d, const Params &p, int32_t *l0, int32_t *link,
                             cudaStream_t s) {
    int nbc = (p.ncell + kAtomThreads - 1) / kAtomThreads;
    k_export_cells<<<nbc, kAtomThreads, 0, s>>>(p.ncell, d.cell_start, d.cell_count, d.cell_atoms,
                                                l0, link);
}

}  // namespace moldy
