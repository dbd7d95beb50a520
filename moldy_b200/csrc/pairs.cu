// pairs.cu -- the per-step pair passes over a compact list of interacting pairs.
//
// The reference evaluates every pair of its half list twice per step (rhoset
// and force, src/dynamics_m.F90:235-346, 524-569).  Only the pairs closer than
// the last nonzero table node contribute (about 7 of the ~44 listed per atom
// in bcc Fe at rnear = 6.3 A); the others add exact zeros.  So each step:
//
//  k_screen   walks each atom's half-list row, keeps the pairs inside the
//             table range and writes them into a compact FULL list: j into
//             i's own list (in row order) and i into j's reverse list (one
//             int atomic per pair).  Both lists are entry-major like the half
//             list, so one thread per atom reads contiguous rows.  In FP64 mode an FP32 distance with a
//             margin that bounds its rounding error pre-selects candidates and
//             the exact FP64 distance decides, so the kept set equals the set
//             an all-FP64 test keeps.
//  k_density  rho_i = sum_j phi(r_ij) over the compact full list (no atomics),
//             then F(rho_i), F'(rho_i) (embed) and the kinetic stress tk.
//  k_forces   f_i = sum_j dx_ij fp_ij over the same list (no atomics); energy
//             and virial take half of every directed pair; the velocity-Verlet
//             second half (src/quench_m.F90:606-622) is applied in the epilogue.
//
// Each pair is thus evaluated from both ends (2x the pair arithmetic of a half
// list) but no floating-point atomic is issued, and all sums for one atom are
// taken by one group of lanes.  MIXED = true runs distances, tables and pair
// forces in FP32 (differences of FP64 positions rounded to FP32) and keeps
// every accumulation, rho, F and F' in FP64.
#include "engine.h"

namespace moldy {


// L2 prefetch of one address (no register result; the address is always
// inside an allocated buffer)
__device__ __forceinline__ void prefetch_l2(const void *ptr) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
}

template <bool MIXED>
__device__ __forceinline__ void fsep(const float *bf, int ivol, float dx, float dy, float dz,
                                     float &rx, float &ry, float &rz, float &r2,
                                     float &odx, float &ody, float &odz) {
    if (ivol == 0 || ivol == 1 || ivol == 4) {
        dx -= rintf(dx); dy -= rintf(dy); dz -= rintf(dz);
    } else if (ivol == 2) {
        dx -= rintf(dx); dy -= rintf(dy);
    } else if (ivol == 5) {
        dz -= rintf(dz);
    }
    rx = fmaf(bf[6], dz, fmaf(bf[3], dy, bf[0] * dx));
    ry = fmaf(bf[7], dz, fmaf(bf[4], dy, bf[1] * dx));
    rz = fmaf(bf[8], dz, fmaf(bf[5], dy, bf[2] * dx));
    r2 = fmaf(rz, rz, fmaf(ry, ry, rx * rx));
    odx = dx; ody = dy; odz = dz;
}

// --------------------------------------------------------------- screen --
// Squared screening radius for the FP32 pre-selection.  The FP32 copy of a
// fractional coordinate is off by at most 2^-24 |x|; for |x| < 5 (positions
// are never wrapped) the FP32 distance is then within 2e-6 |B0|_F + 1e-4 A of
// the FP64 one.  rintf and NINT pick different images only at |dx| = 1/2,
// i.e. at half a box width; when half the narrowest width is not beyond the
// screening radius every pair goes to the FP64 test.
__device__ float screen_radius2(const double *b, double rcull2) {
    double nf = 0.0;
    for (int k = 0; k < 9; ++k) nf += b[k] * b[k];
    double rs = sqrt(rcull2) + 2.0e-6 * sqrt(nf) + 1.0e-4;
    double vol = fabs(b[0] * (b[4] * b[8] - b[7] * b[5]) - b[3] * (b[1] * b[8] - b[7] * b[2]) +
                      b[6] * (b[1] * b[5] - b[4] * b[2]));
    double wmin = 1e300;
    for (int k = 0; k < 3; ++k) {   // width across the face spanned by the other two box vectors
        const double *u = b + 3 * ((k + 1) % 3), *w = b + 3 * ((k + 2) % 3);
        double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
        double a = sqrt(cx * cx + cy * cy + cz * cz);
        if (a > 0.0) wmin = fmin(wmin, vol / a);
    }
    if (!(0.5 * wmin > rs * (1.0 + 1e-6))) return 3.0e38f;
    return (float)(rs * rs);
}

// Keeps pair (a, j) iff its distance is inside the table range.  In FP64 mode
// the FP32 distance decides outright when it is farther than the error bound
// from the cut (rin2 .. rscreen2 is the only band that needs the FP64 test).
template <bool MIXED, int B, bool PF>
__global__ void __launch_bounds__(256)
k_screen(Params p, Tables t, const double4 *__restrict__ pos, const float4 *__restrict__ posf,
         const BoxState *__restrict__ box, const int32_t *__restrict__ nlist,
         const int32_t *__restrict__ numn, const int32_t *__restrict__ mlist,
         const int32_t *__restrict__ mid_cnt, int32_t *__restrict__ alist,
         int32_t *__restrict__ own_cnt, int32_t *__restrict__ rev_cnt) {
    __shared__ double sb[9];
    __shared__ float srs2, srin2;
    if (threadIdx.x < 9) sb[threadIdx.x] = box->b0[threadIdx.x];
    __syncthreads();
    if (threadIdx.x == 0) {
        srs2 = screen_radius2(sb, t.rcull2);
        // inner edge of the band: rcull minus the same error bound
        float rs = sqrtf(srs2), rc = (float)sqrt(t.rcull2);
        float rin = rc - (rs - rc);
        srin2 = (srs2 > 1e37f || rin <= 0.f) ? -1.f : rin * rin;
    }
    __syncthreads();
    const float rscreen2 = MIXED ? t.rcull2f : srs2;
    const float rin2 = srin2;
    double b[9];
    float bf[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { b[k] = sb[k]; bf[k] = (float)sb[k]; }
    const int nm = p.nm;
    const size_t stride = (size_t)nm;
    const int astride = gridDim.x * blockDim.x;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += astride) {
        if (PF && a + astride < nm) {   // next atom of this thread: its rows into L2
            const int an = a + astride;
#pragma unroll
            for (int u = 0; u < 16; ++u) prefetch_l2(&mlist[(size_t)u * stride + an]);
            prefetch_l2(&mid_cnt[an]);
            prefetch_l2(&posf[an]);
        }
        // the intermediate row (pairs within r_mid at its build), or the full
        // half-list row when that row overflowed
        const int mc = mid_cnt[a];
        const int n = mc >= 0 ? mc : numn[a];
        const int32_t *col = (mc >= 0 ? mlist : nlist) + a;
        const float4 pf = posf[a];
        int cnt = 0;
        for (int k0 = 0; k0 < n; k0 += B) {
            int jj[B];
#pragma unroll
            for (int u = 0; u < B; ++u) jj[u] = (k0 + u < n) ? __ldg(&col[(size_t)(k0 + u) * stride]) : -1;
            float4 qq[B];
#pragma unroll
            for (int u = 0; u < B; ++u) qq[u] = __ldg(&posf[jj[u] >= 0 ? jj[u] : a]);
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const int j = jj[u];
                if (j < 0) continue;
                float rx, ry, rz, r2, dx, dy, dz;
                fsep<MIXED>(bf, p.ivol, pf.x - qq[u].x, pf.y - qq[u].y, pf.z - qq[u].z, rx, ry, rz,
                            r2, dx, dy, dz);
                if (r2 > rscreen2) continue;
                bool keep = true;
                if (!MIXED && !(r2 < rin2)) {
                    const double4 pa = pos[a];
                    const double4 qd = pos[j];
                    double ex = pa.x - qd.x, ey = pa.y - qd.y, ez = pa.z - qd.z;
                    min_image(p.ivol, ex, ey, ez);
                    double sx = b[0] * ex + b[3] * ey + b[6] * ez;
                    double sy = b[1] * ex + b[4] * ey + b[7] * ez;
                    double sz = b[2] * ex + b[5] * ey + b[8] * ez;
                    keep = (sx * sx + sy * sy + sz * sz) <= t.rcull2;
                }
                if (keep) {
                    if (cnt < p.own_cap) alist[(size_t)cnt * stride + a] = j;
                    ++cnt;
                    int rs = atomicAdd(&rev_cnt[j], 1);
                    if (rs < p.rev_cap) alist[((size_t)p.own_cap + rs) * stride + j] = a;
                }
            }
        }
        own_cnt[a] = cnt;
    }
}

// the compact list of atom a: own entries 0..no-1 then reverse entries
// 0..nr-1, stored entry-major at (e * nm + a) and ((own_cap + e) * nm + a)
__device__ __forceinline__ void alist_counts(const Params &p, const int32_t *own_cnt, const int32_t *rev_cnt,
                                             int a, int &no, int &nr, bool &over) {
    no = own_cnt[a];
    nr = rev_cnt[a];
    over = no > p.own_cap || nr > p.rev_cap;
    no = no < p.own_cap ? no : p.own_cap;
    nr = nr < p.rev_cap ? nr : p.rev_cap;
}

__device__ __forceinline__ size_t alist_index(const Params &p, int e, int no, int a, int nm) {
    return (size_t)(e < no ? e : p.own_cap + (e - no)) * (size_t)nm + a;
}

// -------------------------------------------------------------- density --
// rho_i = sum phi over the compact row; embed; M = sum m x1 x1^T for kinten
template <bool MIXED, bool EXACT, int B, bool PF>
__global__ void __launch_bounds__(256)
k_density_full(Params p, Tables t, const double4 *__restrict__ pos, double4 *__restrict__ pos2,
               const BoxState *__restrict__ box, const int32_t *__restrict__ alist,
               const int32_t *__restrict__ own_cnt, const int32_t *__restrict__ rev_cnt,
               double *__restrict__ rho, double *__restrict__ afrho, double *__restrict__ dafrho,
               const double *__restrict__ x1, const double *__restrict__ mass,
               const int32_t *__restrict__ znum, double *__restrict__ partials,
               int32_t *__restrict__ flags) {
    __shared__ double sb[9];
    if (threadIdx.x < 9) sb[threadIdx.x] = box->b0[threadIdx.x];
    __syncthreads();
    double b[9];
    float bf[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { b[k] = sb[k]; bf[k] = (float)sb[k]; }
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = 0.0;
    const int nm = p.nm;
    const int astride = gridDim.x * blockDim.x;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += astride) {
        if (PF && a + astride < nm) {
            const int an = a + astride;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                prefetch_l2(&alist[(size_t)u * nm + an]);
                prefetch_l2(&alist[(size_t)(p.own_cap + u) * nm + an]);
            }
            prefetch_l2(&own_cnt[an]); prefetch_l2(&rev_cnt[an]); prefetch_l2(&pos[an]);
            prefetch_l2(&dafrho[an]); prefetch_l2(&mass[an]); prefetch_l2(&znum[an]);
            prefetch_l2(&x1[an]); prefetch_l2(&x1[nm + an]); prefetch_l2(&x1[2 * nm + an]);
        }
        int no, nr;
        bool over;
        alist_counts(p, own_cnt, rev_cnt, a, no, nr, over);
        v[7] += (double)(no + nr);
        if (over) {
            atomicExch(&flags[3], 1);
            atomicMax(&flags[4], max(own_cnt[a], rev_cnt[a]));
        }
        const double4 pa = pos[a];
        double rho_a = 0.0;
        const int ne = no + nr;
        for (int e0 = 0; e0 < ne; e0 += B) {
            int jj[B];
#pragma unroll
            for (int u = 0; u < B; ++u) jj[u] = (e0 + u < ne) ? alist[alist_index(p, e0 + u, no, a, nm)] : -1;
            double4 qq[B];
#pragma unroll
            for (int u = 0; u < B; ++u) qq[u] = pos[jj[u] >= 0 ? jj[u] : a];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                if (jj[u] < 0) continue;
                double dx = pa.x - qq[u].x, dy = pa.y - qq[u].y, dz = pa.z - qq[u].z;
                if (MIXED) {
                    float rx, ry, rz, r2, fx, fy, fz;
                    fsep<true>(bf, p.ivol, (float)dx, (float)dy, (float)dz, rx, ry, rz, r2, fx, fy, fz);
                    rho_a += (double)lookup_phif(t, sqrtf(r2));
                } else {
                    min_image(p.ivol, dx, dy, dz);
                    double rx = b[0] * dx + b[3] * dy + b[6] * dz;
                    double ry = b[1] * dx + b[4] * dy + b[7] * dz;
                    double rz = b[2] * dx + b[5] * dy + b[8] * dz;
                    double r = sqrt(rx * rx + ry * ry + rz * rz);
                    rho_a += EXACT ? fetm_phi(t, r) : lookup_phi(t, r);
                }
            }
        }
        // embed (src/potential_m.F90:148-169): rho <= 1e-40 keeps the old values
        double fd = dafrho[a];
        if (rho_a > 1e-40) {
            double2 e = EXACT ? embed_funcs(t, rho_a) : lookup_e2(t, rho_a);
            afrho[a] = e.x;
            dafrho[a] = e.y;
            fd = e.y;
            v[0] += e.x;
        }
        rho[a] = rho_a;
        pos2[a] = make_double4(pa.x, pa.y, pa.z, fd);
        // kinten (src/thermostat_m.F90:138-157) as tk = B0 M / dt^2, M = sum m x1 x1^T
        if (znum[a] != 0) {
            double m = mass[a];
            double ux = x1[a], uy = x1[nm + a], uz = x1[2 * nm + a];
            v[1] += m * ux * ux; v[2] += m * uy * uy; v[3] += m * uz * uz;
            v[4] += m * ux * uy; v[5] += m * ux * uz; v[6] += m * uy * uz;
        }
    }
    block_partials<8>(v, partials, 0);
}

// --------------------------------------------------------------- forces --
// f_i = sum dx fp over the compact row; pe and the virial moment
// D = sum d d^T fp / 2 (tp = B0 D); mode 1 adds the velocity-Verlet second half
template <bool MIXED, bool EXACT, int B, bool PF>
__global__ void __launch_bounds__(256)
k_forces(Params p, Tables t, const double4 *__restrict__ pos2, const BoxState *__restrict__ box,
         const int32_t *__restrict__ alist, const int32_t *__restrict__ own_cnt,
         const int32_t *__restrict__ rev_cnt, const double *__restrict__ mass,
         const int32_t *__restrict__ znum, const double *__restrict__ del2,
         double *__restrict__ f, double *__restrict__ x1, double *__restrict__ x2,
         double *__restrict__ stress, double *__restrict__ partials, int mode) {
    __shared__ double sb[9], stg[9];
    if (threadIdx.x < 9) {
        sb[threadIdx.x] = box->b0[threadIdx.x];
        stg[threadIdx.x] = box->tgid[threadIdx.x];
    }
    __syncthreads();
    double b[9];
    float bf[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { b[k] = sb[k]; bf[k] = (float)sb[k]; }
    double v[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) v[k] = 0.0;
    const int nm = p.nm;
    const int astride = gridDim.x * blockDim.x;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += astride) {
        if (PF && a + astride < nm) {
            const int an = a + astride;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                prefetch_l2(&alist[(size_t)u * nm + an]);
                prefetch_l2(&alist[(size_t)(p.own_cap + u) * nm + an]);
            }
            prefetch_l2(&own_cnt[an]); prefetch_l2(&rev_cnt[an]); prefetch_l2(&pos2[an]);
            prefetch_l2(&mass[an]);
            if (mode == 1) {
                prefetch_l2(&x1[an]); prefetch_l2(&x1[nm + an]); prefetch_l2(&x1[2 * nm + an]);
                prefetch_l2(&x2[an]); prefetch_l2(&x2[nm + an]); prefetch_l2(&x2[2 * nm + an]);
                prefetch_l2(&del2[an]); prefetch_l2(&znum[an]);
            }
        }
        int no, nr;
        bool over;
        alist_counts(p, own_cnt, rev_cnt, a, no, nr, over);
        const double4 pa = pos2[a];
        const double ma = mass[a];
        double fxa = 0.0, fya = 0.0, fza = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
        const int ne = no + nr;
        for (int e0 = 0; e0 < ne; e0 += B) {
            int jj[B];
#pragma unroll
            for (int u = 0; u < B; ++u) jj[u] = (e0 + u < ne) ? alist[alist_index(p, e0 + u, no, a, nm)] : -1;
            double4 qq[B];
#pragma unroll
            for (int u = 0; u < B; ++u) qq[u] = pos2[jj[u] >= 0 ? jj[u] : a];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const int j = jj[u];
                if (j < 0) continue;
                const double4 q = qq[u];
                double dx = pa.x - q.x, dy = pa.y - q.y, dz = pa.z - q.z;
                double fp, vee, rx, ry, rz;
                if (MIXED) {
                    float frx, fry, frz, r2, ex, ey, ez;
                    fsep<true>(bf, p.ivol, (float)dx, (float)dy, (float)dz, frx, fry, frz, r2, ex, ey, ez);
                    float r = sqrtf(r2), rr = 1.0f / r;
                    float4 tv = lookup_r4f(t, r);
                    fp = (double)(-(tv.y + tv.w * ((float)pa.w + (float)q.w)) * rr);
                    vee = (double)tv.x;
                    dx = (double)ex; dy = (double)ey; dz = (double)ez;
                    rx = (double)frx; ry = (double)fry; rz = (double)frz;
                } else {
                    min_image(p.ivol, dx, dy, dz);
                    rx = b[0] * dx + b[3] * dy + b[6] * dz;
                    ry = b[1] * dx + b[4] * dy + b[7] * dz;
                    rz = b[2] * dx + b[5] * dy + b[8] * dz;
                    double r = sqrt(rx * rx + ry * ry + rz * rz);
                    double rr = 1.0 / r;
                    double4 tv = EXACT ? pair_funcs(t, r) : lookup_r4(t, r);    // vee, dvee, phi, dphi
                    fp = -tv.y * rr - (tv.w * pa.w + tv.w * q.w) * rr;
                    vee = tv.x;
                }
                fxa += dx * fp; fya += dy * fp; fza += dz * fp;
                v[0] += vee;
                if (ma > 0.1 || ma + mass[j] > 0.1) {
                    v[1] += dx * dx * fp; v[2] += dy * dy * fp; v[3] += dz * dz * fp;
                    v[4] += dx * dy * fp; v[5] += dx * dz * fp; v[6] += dy * dz * fp;
                }
                if (p.atomstress && e0 + u < no) { sx += rx * fp; sy += ry * fp; sz += rz * fp; }
            }
        }
        f[a] = fxa; f[nm + a] = fya; f[2 * nm + a] = fza;
        if (p.atomstress) { stress[a] = sx; stress[nm + a] = sy; stress[2 * nm + a] = sz; }
        if (mode == 1) {
            // velocity Verlet second half (src/quench_m.F90:606-622), previous tgid
            double ux = x1[a], uy = x1[nm + a], uz = x1[2 * nm + a];
            double wx = x2[a], wy = x2[nm + a], wz = x2[2 * nm + a];
            double hx = ux + wx, hy = uy + wy, hz = uz + wz;
            if (!(znum[a] == 0 || ma < 0.1)) {
                double s0 = 0.0, s1 = 0.0, s2 = 0.0;
                if (p.ivol == 0) {
                    s0 = stg[0] * ux + stg[3] * uy + stg[6] * uz;
                    s1 = stg[1] * ux + stg[4] * uy + stg[7] * uz;
                    s2 = stg[2] * ux + stg[5] * uy + stg[8] * uz;
                }
                if (p.ivol == 4) s2 = stg[8] * uz;
                double d2 = del2[a];
                wx = d2 * fxa - 0.5 * s0;
                wy = d2 * fya - 0.5 * s1;
                wz = d2 * fza - 0.5 * s2;
                x2[a] = wx; x2[nm + a] = wy; x2[2 * nm + a] = wz;
            }
            x1[a] = hx + wx; x1[nm + a] = hy + wy; x1[2 * nm + a] = hz + wz;
        }
    }
    // every directed pair carries half of the pair energy and virial
#pragma unroll
    for (int k = 0; k < 7; ++k) v[k] *= 0.5;
    block_partials<7>(v, partials, 0);
}

// ------------------------------------------------------ intermediate list --
// The screen walks, per atom, the half-list pairs that were within
// r_mid = r_cut + skin when the intermediate list was last built.  A pair
// left out was farther than r_mid - eps then (eps bounds the FP32 distance
// error); since then its distance can have shrunk by at most
// 2 max_i |B0 (x_i - x_i,build)| + |B0 - B0_build|_F dmax, with dmax = rnear
// |B0_build^-1|_F bounding the fractional separation of any listed pair.  The
// list is rebuilt before that bound reaches the screening radius, and after
// every half-list rebuild and every force call outside velocity Verlet, so
// the screen keeps exactly the pairs a walk over the whole half list keeps.
__device__ double frob(const double *m) {
    double s = 0.0;
    for (int k = 0; k < 9; ++k) s += m[k] * m[k];
    return sqrt(s);
}

__global__ void k_mid_decide(Params p, BoxState *__restrict__ box, double rmid, double rcut,
                             int force, int apply_box) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    BoxState &B = *box;
    if (apply_box) {   // velocityverlet box half (src/quench_m.F90:582-589)
        if (p.ivol == 4) {
            MAT(B.b1, 3, 3) = MAT(B.b1, 3, 3) + MAT(B.b2, 3, 3);
            MAT(B.b0, 3, 3) = MAT(B.b0, 3, 3) + MAT(B.b1, 3, 3);
        }
        if (p.ivol < 1) {
            for (int k = 0; k < 9; ++k) B.b1[k] = B.b1[k] + B.b2[k];
            for (int k = 0; k < 9; ++k) B.b0[k] = B.b0[k] + B.b1[k];
        }
    }
    double md = sqrt(__longlong_as_double((long long)B.maxdisp2));
    B.maxdisp2 = 0ull;
    double eps = 2.0e-6 * frob(B.b0) + 1.0e-4;
    double db[9], inv[9];
    for (int k = 0; k < 9; ++k) db[k] = B.b0[k] - B.bbuild[k];
    bool ok = mat_invert(B.bbuild, inv);
    double dmax = ok ? p.rnear * frob(inv) : 1e300;
    double shrink = 2.0 * md + frob(db) * dmax;
    int need = force || !ok || !(shrink < rmid - eps - (rcut + eps));
    B.mid_rebuild = need;
    if (need) {
        for (int k = 0; k < 9; ++k) B.bbuild[k] = B.b0[k];
        B.mid_builds += 1;
    }
}

__global__ void __launch_bounds__(256)
k_mid_build(Params p, double rmid, const double4 *__restrict__ pos, const float4 *__restrict__ posf,
            const BoxState *__restrict__ box, const int32_t *__restrict__ nlist,
            const int32_t *__restrict__ numn, int32_t *__restrict__ mlist,
            int32_t *__restrict__ mid_cnt, double4 *__restrict__ xbuild) {
    __shared__ double sb[9];
    __shared__ float skeep2;
    __shared__ int sneed;
    if (threadIdx.x < 9) sb[threadIdx.x] = box->b0[threadIdx.x];
    if (threadIdx.x == 0) sneed = box->mid_rebuild;
    __syncthreads();
    if (!sneed) return;
    if (threadIdx.x == 0) {
        float keep = (float)(rmid + 2.0 * (2.0e-6 * frob(sb) + 1.0e-4));
        // when a box is too small for the FP32 screen, keep every listed pair
        skeep2 = screen_radius2(sb, rmid * rmid) > 1e37f ? 3.0e38f : keep * keep;
    }
    __syncthreads();
    float bf[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) bf[k] = (float)sb[k];
    const float keep2 = skeep2;
    const int nm = p.nm;
    const size_t stride = (size_t)nm;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += gridDim.x * blockDim.x) {
        const int n = numn[a];
        const int32_t *col = nlist + a;
        const float4 pf = posf[a];
        int cnt = 0;
#pragma unroll 4
        for (int k = 0; k < n; ++k) {
            const int j = __ldg(&col[(size_t)k * stride]);
            const float4 q = __ldg(&posf[j]);
            float rx, ry, rz, r2, dx, dy, dz;
            fsep<true>(bf, p.ivol, pf.x - q.x, pf.y - q.y, pf.z - q.z, rx, ry, rz, r2, dx, dy, dz);
            if (r2 <= keep2) {
                if (cnt < kMidCap) mlist[(size_t)cnt * stride + a] = j;
                ++cnt;
            }
        }
        mid_cnt[a] = cnt <= kMidCap ? cnt : -1;
        xbuild[a] = pos[a];
    }
}

void launch_mid_decide(DeviceState &d, const Params &p, double rmid, double rcut, int force,
                       int apply_box, cudaStream_t s) {
    k_mid_decide<<<1, 32, 0, s>>>(p, d.box, rmid, rcut, force, apply_box);
}

void launch_mid_build(DeviceState &d, const Params &p, double rmid, cudaStream_t s) {
    int nb = grid_blocks(p.nm, 256);
    k_mid_build<<<nb, 256, 0, s>>>(p, rmid, d.pos, d.posf, d.box, d.nlist, d.numn, d.mlist,
                                   d.mid_cnt, d.xbuild);
}

// ------------------------------------------------------------ launchers --
// Variant v: bit 0 selects the batch of list entries whose gathers are issued
// before any is used (screen {4, 8}, density and forces {2, 4}); bit 1 adds
// L2 prefetches of the next atom's rows and per-atom data.
void launch_screen(DeviceState &d, const Params &p, const Tables &t, bool mixed, int variant,
                   cudaStream_t s) {
    int nb = grid_blocks(p.nm, 256);
    cudaMemsetAsync(d.rev_cnt, 0, sizeof(int32_t) * p.nm, s);
#define SCREEN_ARGS p, t, d.pos, d.posf, d.box, d.nlist, d.numn, d.mlist, d.mid_cnt, d.alist, \
                    d.own_cnt, d.rev_cnt
#define SCREEN(B, PF)                                                                  \
    do {                                                                               \
        if (mixed) k_screen<true, B, PF><<<nb, 256, 0, s>>>(SCREEN_ARGS);              \
        else k_screen<false, B, PF><<<nb, 256, 0, s>>>(SCREEN_ARGS);                   \
    } while (0)
    switch (variant) {
    case 0: SCREEN(4, false); break;
    case 1: SCREEN(8, false); break;
    case 2: SCREEN(4, true); break;
    default: SCREEN(8, true); break;
    }
#undef SCREEN
#undef SCREEN_ARGS
}

int launch_density_full(DeviceState &d, const Params &p, const Tables &t, bool mixed, int variant,
                        double *partials, cudaStream_t s) {
    int nb = grid_blocks(p.nm, 256);
#define DENSITY_ARGS p, t, d.pos, d.pos2, d.box, d.alist, d.own_cnt, d.rev_cnt, d.rho, d.afrho, \
                     d.dafrho, d.x1, d.mass, d.znum, partials, d.flags
#define DENSITY(B, PF)                                                                          \
    do {                                                                                        \
        if (t.exact) k_density_full<false, true, B, PF><<<nb, 256, 0, s>>>(DENSITY_ARGS);       \
        else if (mixed) k_density_full<true, false, B, PF><<<nb, 256, 0, s>>>(DENSITY_ARGS);    \
        else k_density_full<false, false, B, PF><<<nb, 256, 0, s>>>(DENSITY_ARGS);              \
    } while (0)
    switch (variant) {
    case 0: DENSITY(2, false); break;
    case 1: DENSITY(4, false); break;
    case 2: DENSITY(2, true); break;
    default: DENSITY(4, true); break;
    }
#undef DENSITY
#undef DENSITY_ARGS
    return nb;
}

int launch_forces(DeviceState &d, const Params &p, const Tables &t, bool mixed, int mode,
                  int variant, double *partials, cudaStream_t s) {
    int nb = grid_blocks(p.nm, 256);
#define FORCE_ARGS p, t, d.pos2, d.box, d.alist, d.own_cnt, d.rev_cnt, d.mass, d.znum, d.del2, d.f, \
                   d.x1, d.x2, d.stress, partials, mode
#define FORCES(B, PF)                                                                        \
    do {                                                                                     \
        if (t.exact) k_forces<false, true, B, PF><<<nb, 256, 0, s>>>(FORCE_ARGS);            \
        else if (mixed) k_forces<true, false, B, PF><<<nb, 256, 0, s>>>(FORCE_ARGS);         \
        else k_forces<false, false, B, PF><<<nb, 256, 0, s>>>(FORCE_ARGS);                   \
    } while (0)
    switch (variant) {
    case 0: FORCES(2, false); break;
    case 1: FORCES(4, false); break;
    case 2: FORCES(2, true); break;
    default: FORCES(4, true); break;
    }
#undef FORCES
#undef FORCE_ARGS
    return nb;
}

// list entries the screening pass reads per step: the intermediate row, or
// the half-list row of an atom whose intermediate row overflowed
__global__ void k_count_screened(int nm, const int32_t *__restrict__ mid_cnt, const int32_t *__restrict__ numn,
                                 unsigned long long *__restrict__ out) {
    unsigned long long s = 0;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += gridDim.x * blockDim.x) {
        int mc = mid_cnt[a];
        s += (unsigned long long)(mc >= 0 ? mc : numn[a]);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

void launch_count_screened(const DeviceState &d, const Params &p, unsigned long long *out, cudaStream_t s) {
    cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
    k_count_screened<<<grid_blocks(p.nm, kAtomThreads), kAtomThreads, 0, s>>>(p.nm, d.mid_cnt, d.numn, out);
}

}  // namespace moldy
