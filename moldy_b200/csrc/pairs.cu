// pairs.cu -- the per-step pair passes over a compact list of interacting pairs.
//
// The reference evaluates every pair of its half list twice per step (rhoset
// and force, src/dynamics_m.F90:235-346, 524-569).  Only the pairs closer than
// the last nonzero table node contribute (about 7 of the ~44 listed per atom
// in bcc Fe at rnear = 6.3 A); the others add exact zeros.  The lists:
//
//  outer         a FULL list (both directions) of the half-list pairs within
//                r_out = rcut + outer skin, rebuilt from the half list only when
//                the displacements since its build could bring an unlisted
//                pair within r_mid;
//  intermediate  the outer-list pairs within r_mid = rcut + skin, rebuilt
//                (filtered from the outer rows) only when the displacements
//                since its build could bring an unlisted pair inside the cut;
//  compact       per step, the FULL list of pairs inside the table cut.
//
// Each step runs two passes, one thread per atom, no floating-point atomics:
//
//  k_screen_density  walks the atom's intermediate row, keeps the pairs inside
//             the cut (exact FP64 distance in FP64 mode; FP32 with an error
//             margin and an FP64 decision inside the margin in mixed mode),
//             writes them to its compact row and sums rho_i = sum_j phi(r_ij);
//             then embed and F'(rho) into pos2.w / posq2.w.  (The kinetic
//             moment of kinten is taken by the drift kernel, or k_kinetic
//             outside MD.)
//  k_forces   f_i = sum_j dx_ij fp_ij over the compact row; the pair energy
//             and the virial take each pair once, from the copy in its
//             owner's row (bit 31); the velocity-Verlet second half
//             (src/quench_m.F90:606-622) is applied in the epilogue.
//
// Entries carry the pair's direction in the reference's half list in bit 31
// (set: j is in i's own row), which the per-atom stress of the reference
// (own rows only) needs.  MIXED = true runs distances, tables and pair forces
// in FP32 from 32-bit fixed-point positions (whose integer differences are
// the minimum image) and keeps rho, F, F', the forces, the energy, the virial
// and every other sum in FP64: each pair's FP32 terms are converted once and
// accumulated in FP64.
#include <type_traits>

#include "engine.h"

namespace moldy {

// One wave of resident blocks for the kernel (at 256 threads): every block
// then runs the same number of grid-stride iterations (to within one), and no
// partly filled last wave idles the SMs.  Computed once per instantiation.
template <typename K>
static int one_wave(K kernel) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0) != cudaSuccess) {
        cudaGetLastError();
        per_sm = 0;
    }
    const long long w = (long long)(sms > 0 ? sms : 148) * (per_sm > 0 ? per_sm : 1);
    return (int)(w < kMaxBlocks ? w : kMaxBlocks);
}

#define LAUNCH_WAVE(KERNEL, NB, S, ...)                      \
    do {                                                     \
        static const int wave_ = one_wave(KERNEL);           \
        NB = NB < wave_ ? NB : wave_;                        \
        launch_pdl(KERNEL, NB, 256, S, __VA_ARGS__);         \
    } while (0)



// L2 prefetch of one address (no register result; the address is always
// inside an allocated buffer)
__device__ __forceinline__ void prefetch_l2(const void *ptr) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
}

// Squared FP32 distance of an FP64 fractional difference (any box): the
// difference rounded to FP32 (off by at most 2^-24 |dx|), the minimum image by
// rintf in the periodic directions.
__device__ __forceinline__ float sep2_f32(const float *bf, int ivol, double dxd, double dyd, double dzd) {
    float dx = (float)dxd, dy = (float)dyd, dz = (float)dzd;
    if (ivol == 0 || ivol == 1 || ivol == 4) {
        dx -= rintf(dx); dy -= rintf(dy); dz -= rintf(dz);
    } else if (ivol == 2) {
        dx -= rintf(dx); dy -= rintf(dy);
    } else if (ivol == 5) {
        dz -= rintf(dz);
    }
    const float rx = fmaf(bf[6], dz, fmaf(bf[3], dy, bf[0] * dx));
    const float ry = fmaf(bf[7], dz, fmaf(bf[4], dy, bf[1] * dx));
    const float rz = fmaf(bf[8], dz, fmaf(bf[5], dy, bf[2] * dx));
    return fmaf(rz, rz, fmaf(ry, ry, rx * rx));
}

// Separation of two atoms from their fixed-point coordinates (fully periodic
// box): the 32-bit differences are the minimum image; bs is B0 per fixed-point
// unit.  Returns r^2 and the Cartesian separation, all FP32.
__device__ __forceinline__ float fix_sep(const float *bs, const int4 &qa, const int4 &qj, float &rx, float &ry,
                                         float &rz, float &dx, float &dy, float &dz) {
    dx = fix_to_float((int32_t)((uint32_t)qa.x - (uint32_t)qj.x));
    dy = fix_to_float((int32_t)((uint32_t)qa.y - (uint32_t)qj.y));
    dz = fix_to_float((int32_t)((uint32_t)qa.z - (uint32_t)qj.z));
    rx = fmaf(bs[6], dz, fmaf(bs[3], dy, bs[0] * dx));
    ry = fmaf(bs[7], dz, fmaf(bs[4], dy, bs[1] * dx));
    rz = fmaf(bs[8], dz, fmaf(bs[5], dy, bs[2] * dx));
    return fmaf(rz, rz, fmaf(ry, ry, rx * rx));
}

__device__ __forceinline__ float fix_sep(const float *bs, const int4 &qa, const int4 &qj, float &rx, float &ry,
                                         float &rz) {
    float dx, dy, dz;
    return fix_sep(bs, qa, qj, rx, ry, rz, dx, dy, dz);
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


constexpr int32_t kOwnBit = (int32_t)0x80000000u;
constexpr int32_t kIdMask = 0x7fffffff;

// The exact FP64 test r^2 <= rcull^2 for a pair whose FP32 distance lies in
// the error band around the cut (rare: kept out of line, so its registers do
// not count against the screening loop)
__device__ __noinline__ bool inside_cut_fp64(const double4 *__restrict__ pos, int a, int j, const double *b,
                                             int ivol, double rcull2) {
    const double4 pa = pos[a], qd = pos[j];
    double ex = pa.x - qd.x, ey = pa.y - qd.y, ez = pa.z - qd.z;
    min_image(ivol, ex, ey, ez);
    double sx = b[0] * ex + b[3] * ey + b[6] * ez;
    double sy = b[1] * ex + b[4] * ey + b[7] * ez;
    double sz = b[2] * ex + b[5] * ey + b[8] * ez;
    return (sx * sx + sy * sy + sz * sz) <= rcull2;
}

// Keeps pair (a, j) iff its distance is inside the table range, sums rho_a,
// embeds.  FP64: the exact distance decides.  Mixed: the FP32 distance decides
// outside the band [rin, rscreen] around the cut, the FP64 one inside it.
template <bool MIXED, bool EXACT, int B, bool PF, int MINB>
__global__ void __launch_bounds__(256, MINB)
k_screen_density(Params p, Tables t, const double4 *__restrict__ pos, const int4 *__restrict__ posq,
                 double4 *__restrict__ pos2, int4 *__restrict__ posq2, const BoxState *__restrict__ box,
                 const int32_t *__restrict__ mlist,
                 const int32_t *__restrict__ mid_cnt,
                 int32_t *__restrict__ alist, int32_t *__restrict__ pair_cnt,
                 double *__restrict__ rho, double *__restrict__ afrho, double *__restrict__ dafrho,
                 double *__restrict__ partials, int32_t *__restrict__ flags, int store_rho) {
    grid_dep_wait();   // launched dependent on the step's previous kernel
    __shared__ double sb[9];
    __shared__ float srs2, srin2;
    if (threadIdx.x < 9) sb[threadIdx.x] = box->b0[threadIdx.x];
    __syncthreads();
    if (MIXED && threadIdx.x == 0) {
        srs2 = screen_radius2(sb, t.rcull2);
        float rs = sqrtf(srs2), rc = (float)sqrt(t.rcull2);
        float rin = rc - (rs - rc);
        srin2 = (srs2 > 1e37f || rin <= 0.f) ? -1.f : rin * rin;
    }
    __syncthreads();
    double b[9];
    float bs[9];   // B0 in A per fixed-point unit (mixed)
#pragma unroll
    for (int k = 0; k < 9; ++k) { b[k] = MIXED ? 0.0 : sb[k]; bs[k] = (float)(sb[k] * kFixUnit); }
    const float rscreen2 = MIXED ? srs2 : 0.f, rin2 = MIXED ? srin2 : 0.f;
    double v[2] = {0.0, 0.0};   // embedding energy, directed pairs
    const int nm = p.nm;
    const size_t stride = (size_t)nm;
    const int astride = gridDim.x * blockDim.x;
    int over = 0, over_max = 0;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += astride) {
        if (PF && a + astride < nm) {   // next atom of this thread: its row and data into L2
            const int an = a + astride;
#pragma unroll
            for (int u = 0; u < 16; ++u) prefetch_l2(&mlist[(size_t)u * stride + an]);
            prefetch_l2(&mid_cnt[an]);
            prefetch_l2(MIXED ? (const void *)&posq[an] : (const void *)&pos[an]);
            prefetch_l2(&dafrho[an]);
        }
        const int mc = mid_cnt[a];
        const int n = mc < p.mid_cap ? mc : p.mid_cap;
        const double4 pa = MIXED ? make_double4(0.0, 0.0, 0.0, 0.0) : pos[a];
        const int4 qa = MIXED ? posq[a] : make_int4(0, 0, 0, 0);
        double rho_a = 0.0;
        int cnt = 0;
        for (int k0 = 0; k0 < n; k0 += B) {
            int ee[B];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const int k = k0 + u;
                ee[u] = (k < n) ? __ldg(&mlist[(size_t)k * stride + a]) : -1;
            }
            if (MIXED) {
                int4 qq[B];
#pragma unroll
                for (int u = 0; u < B; ++u) qq[u] = __ldg(&posq[ee[u] != -1 ? (ee[u] & kIdMask) : a]);
#pragma unroll
                for (int u = 0; u < B; ++u) {
                    if (ee[u] == -1) continue;
                    float rx, ry, rz;
                    const float r2 = fix_sep(bs, qa, qq[u], rx, ry, rz);
                    if (r2 > rscreen2) continue;
                    // inside the error band: the FP64 distance decides
                    if (!(r2 < rin2) && !inside_cut_fp64(pos, a, ee[u] & kIdMask, sb, p.ivol, t.rcull2)) continue;
                    rho_a += (double)lookup_phif(t, r2 * rsqrt_ftz(r2));
                    if (cnt < p.pair_cap) alist[(size_t)cnt * stride + a] = ee[u];
                    ++cnt;
                }
            } else {
                double4 qq[B];
#pragma unroll
                for (int u = 0; u < B; ++u) qq[u] = ldg4(&pos[ee[u] != -1 ? (ee[u] & kIdMask) : a]);
#pragma unroll
                for (int u = 0; u < B; ++u) {
                    if (ee[u] == -1) continue;
                    double dx = pa.x - qq[u].x, dy = pa.y - qq[u].y, dz = pa.z - qq[u].z;
                    min_image(p.ivol, dx, dy, dz);
                    double rx = b[0] * dx + b[3] * dy + b[6] * dz;
                    double ry = b[1] * dx + b[4] * dy + b[7] * dz;
                    double rz = b[2] * dx + b[5] * dy + b[8] * dz;
                    double r2 = rx * rx + ry * ry + rz * rz;
                    if (!(r2 <= t.rcull2)) continue;
                    double r = sqrt(r2);
                    rho_a += EXACT ? fetm_phi(t, r) : lookup_phi(t, r);
                    if (cnt < p.pair_cap) alist[(size_t)cnt * stride + a] = ee[u];
                    ++cnt;
                }
            }
        }
        pair_cnt[a] = cnt;
        v[1] += (double)cnt;
        if (cnt > p.pair_cap) { over = 1; over_max = max(over_max, cnt); }
        if (mc > p.mid_cap) { over |= 2; over_max = max(over_max, mc); }
        // embed (src/potential_m.F90:148-169): rho <= 1e-40 keeps the old values
        double fd;
        if (rho_a > 1e-40) {
            double2 e = EXACT ? embed_funcs(t, rho_a) : lookup_e2(t, rho_a);
            afrho[a] = e.x;
            dafrho[a] = e.y;
            fd = e.y;
            v[0] += e.x;
        } else {
            fd = dafrho[a];
        }
        if (store_rho) rho[a] = rho_a;
        if (MIXED) posq2[a] = make_int4(qa.x, qa.y, qa.z, __float_as_int((float)fd));
        else pos2[a] = make_double4(pa.x, pa.y, pa.z, fd);
    }
    if (over & 1) { atomicExch(&flags[3], 1); atomicMax(&flags[4], over_max); }
    if (over & 2) { atomicExch(&flags[5], 1); atomicMax(&flags[6], over_max); }
    block_partials<2>(v, partials, 0);
}

// --------------------------------------------------------------- forces --
// v[1..6] += s * sym(a (x) b) in the order xx, yy, zz, xy, xz, yz
__device__ __forceinline__ void add_sym(double *v, double ax, double ay, double az, double bx, double by,
                                        double bz, double s) {
    v[1] += s * (ax * bx);
    v[2] += s * (ay * by);
    v[3] += s * (az * bz);
    v[4] += (0.5 * s) * (ax * by + ay * bx);
    v[5] += (0.5 * s) * (ax * bz + az * bx);
    v[6] += (0.5 * s) * (ay * bz + az * by);
}

// f_i = sum_j g_ij over the compact row, g_ij = d_ij fp_ij; pe and the
// virial moment D = sum over pairs d d^T fp (tp = B0 D, pairs with
// m_i + m_j <= 0.1 left out, src/dynamics_m.F90:287); mode 1 adds the
// velocity-Verlet second half.
//
// D is formed from per-atom FP64 quantities instead of a per-pair sum: with
// d_ij = x_i - x_j - m_ij (m_ij the periodic image the minimum-image
// convention picks) and g_ji = -g_ij,
//   sum_pairs d_ij (x) g_ij = sum_i x_i (x) f_i - sum_pairs m_ij (x) g_ij,
// and D is symmetric, so sym(x_i (x) f_i) is accumulated per atom and
// sym(m_ij (x) g_ij) / 2 subtracted on both ends of the pairs that cross a
// periodic boundary (a few percent); a pair the mass filter leaves out has
// its whole sym((x_i - x_j) (x) g_ij) / 2 removed the same way.  The two
// ends compute g_ij bit for bit with opposite signs, so this is the pair sum
// up to FP64 rounding of the per-atom terms, and it needs no per-pair
// conversion to FP64 in the mixed pass.  The pair energy is summed from the
// copy in the owner's row.
template <bool MIXED, bool EXACT, int B, bool PF, bool STRESS, int MINB>
__global__ void __launch_bounds__(256, MINB)
k_forces(Params p, Tables t, const double4 *__restrict__ pos2, const int4 *__restrict__ posq2,
         const BoxState *__restrict__ box,
         const int32_t *__restrict__ alist, const int32_t *__restrict__ pair_cnt, const double *__restrict__ mass,
         const int32_t *__restrict__ znum, const double *__restrict__ del2,
         double *__restrict__ f, double *__restrict__ x1, double *__restrict__ x2,
         double *__restrict__ stress, double *__restrict__ partials, int mode) {
    grid_dep_wait();   // launched dependent on the step's previous kernel
    __shared__ double sb[9], stg[9];
    __shared__ int slim[3];
    if (threadIdx.x < 9) {
        sb[threadIdx.x] = box->b0[threadIdx.x];
        stg[threadIdx.x] = box->tgid[threadIdx.x];
    }
    __syncthreads();
    if (MIXED && threadIdx.x == 0) {
        // a pair inside the cut spans at most M_d = rcull |row d of B0^-1|
        // box lengths in direction d; an atom whose fixed-point coordinates
        // all lie within 2^31 - M_d of zero has no pair whose 32-bit
        // difference wraps (crosses a periodic boundary)
        double bi[9];
        const bool ok = mat_invert(sb, bi);
        for (int d = 0; d < 3; ++d) {
            const double rn = sqrt(MAT(bi, d + 1, 1) * MAT(bi, d + 1, 1) + MAT(bi, d + 1, 2) * MAT(bi, d + 1, 2) +
                                   MAT(bi, d + 1, 3) * MAT(bi, d + 1, 3));
            const double m = sqrt(t.rcull2) * rn * (1.0 + 1e-6) * kFixScale + 4.0;
            slim[d] = (ok && m < 2147483000.0) ? (int)(2147483647.0 - m) : -1;
        }
    }
    __syncthreads();
    const int limx = slim[0], limy = slim[1], limz = slim[2];
    double b[9];
    float bs[9];   // B0 in A per fixed-point unit (mixed)
#pragma unroll
    for (int k = 0; k < 9; ++k) { b[k] = sb[k]; bs[k] = (float)(sb[k] * kFixUnit); }
    double v[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) v[k] = 0.0;
    const int nm = p.nm;
    const int astride = gridDim.x * blockDim.x;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += astride) {
        if (PF && a + astride < nm) {
            const int an = a + astride;
#pragma unroll
            for (int u = 0; u < 8; ++u) prefetch_l2(&alist[(size_t)u * nm + an]);
            prefetch_l2(&pair_cnt[an]); prefetch_l2(MIXED ? (const void *)&posq2[an] : (const void *)&pos2[an]);
            prefetch_l2(&mass[an]);
            if (mode == 1) {
                prefetch_l2(&x1[an]); prefetch_l2(&x1[nm + an]); prefetch_l2(&x1[2 * nm + an]);
                prefetch_l2(&x2[an]); prefetch_l2(&x2[nm + an]); prefetch_l2(&x2[2 * nm + an]);
                prefetch_l2(&del2[an]); prefetch_l2(&znum[an]);
            }
        }
        int ne = pair_cnt[a];
        ne = ne < p.pair_cap ? ne : p.pair_cap;
        const double ma = mass[a];
        double fxa = 0.0, fya = 0.0, fza = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
        if constexpr (MIXED) {
            // fixed-point separations, FP32 geometry, tables and pair forces;
            // forces, pair energy and virial accumulate in FP64
            const int4 qa = posq2[a];
            const float fa = __int_as_float(qa.w);
            double gx = 0.0, gy = 0.0, gz = 0.0;   // sum of g = d fp, fixed-point units
            float tx = 0.f, ty = 0.f, tz = 0.f;
            // CORR: the pairs that wrap or that the mass filter leaves out are
            // corrected; a warp takes that path when one of its atoms lies near
            // a face (limits above) or has m <= 0.1
            const bool slow = !(ma > 0.1) || qa.x > limx || qa.x < -limx || qa.y > limy || qa.y < -limy ||
                              qa.z > limz || qa.z < -limz;
            auto row = [&](auto corr) {
            constexpr bool CORR = decltype(corr)::value;
            for (int e0 = 0; e0 < ne; e0 += B) {
                int ee[B];
#pragma unroll
                for (int u = 0; u < B; ++u) ee[u] = (e0 + u < ne) ? alist[(size_t)(e0 + u) * nm + a] : -1;
                int4 qq[B];
#pragma unroll
                for (int u = 0; u < B; ++u) qq[u] = __ldg(&posq2[ee[u] != -1 ? (ee[u] & kIdMask) : a]);
#pragma unroll
                for (int u = 0; u < B; ++u) {
                    if (ee[u] == -1) continue;
                    const int j = ee[u] & kIdMask;
                    const int4 qj = qq[u];
                    // 32-bit differences: the minimum image (wrapping past half a box)
                    const int32_t ex = (int32_t)((uint32_t)qa.x - (uint32_t)qj.x);
                    const int32_t ey = (int32_t)((uint32_t)qa.y - (uint32_t)qj.y);
                    const int32_t ez = (int32_t)((uint32_t)qa.z - (uint32_t)qj.z);
                    const float dx = fix_to_float(ex), dy = fix_to_float(ey), dz = fix_to_float(ez);
                    const float rx = fmaf(bs[6], dz, fmaf(bs[3], dy, bs[0] * dx));
                    const float ry = fmaf(bs[7], dz, fmaf(bs[4], dy, bs[1] * dx));
                    const float rz = fmaf(bs[8], dz, fmaf(bs[5], dy, bs[2] * dx));
                    const float r2 = fmaf(rz, rz, fmaf(ry, ry, rx * rx));
                    const float rr = rsqrt_ftz(r2);
                    const float4 tv = lookup_r4f(t, r2 * rr);    // vee, dvee, phi, dphi
                    const float fp = -(tv.y + tv.w * (fa + __int_as_float(qj.w))) * rr;
                    const float dfx = dx * fp, dfy = dy * fp, dfz = dz * fp;
                    gx += (double)dfx; gy += (double)dfy; gz += (double)dfz;
                    if (ee[u] & kOwnBit) {   // the owner's copy carries the pair energy
                        v[0] += (double)tv.x;
                        if (STRESS) { tx = fmaf(rx, fp, tx); ty = fmaf(ry, fp, ty); tz = fmaf(rz, fp, tz); }
                    }
                    if constexpr (CORR) {
                        // sign bit set: that difference wrapped (a periodic image, m = +-1)
                        const int32_t wx = (qa.x ^ qj.x) & (qa.x ^ ex), wy = (qa.y ^ qj.y) & (qa.y ^ ey),
                                      wz = (qa.z ^ qj.z) & (qa.z ^ ez);
                        const bool excluded = !(ma > 0.1 || ma + mass[j] > 0.1);
                        if ((wx | wy | wz) < 0 || excluded) {
                            // c = m 2^32 (the image), or q_a - q_j exactly when excluded
                            double cx = wx < 0 ? (qa.x >= 0 ? kFixScale : -kFixScale) : 0.0;
                            double cy = wy < 0 ? (qa.y >= 0 ? kFixScale : -kFixScale) : 0.0;
                            double cz = wz < 0 ? (qa.z >= 0 ? kFixScale : -kFixScale) : 0.0;
                            if (excluded) { cx += (double)ex; cy += (double)ey; cz += (double)ez; }
                            add_sym(v, cx, cy, cz, (double)dfx, (double)dfy, (double)dfz, -0.5);
                        }
                    }
                }
            }
            };
            if (__any_sync(__activemask(), slow)) row(std::true_type{});
            else row(std::false_type{});
            add_sym(v, (double)qa.x, (double)qa.y, (double)qa.z, gx, gy, gz, 1.0);
            fxa = gx * kFixUnit; fya = gy * kFixUnit; fza = gz * kFixUnit;
            sx = (double)tx; sy = (double)ty; sz = (double)tz;
        } else {
            const double4 pa = pos2[a];
            // periodic directions of min_image: all for ivol 0, 1, 4; x and y for 2; z for 5
            const bool pxy = p.ivol == 0 || p.ivol == 1 || p.ivol == 4 || p.ivol == 2;
            const bool pz = p.ivol == 0 || p.ivol == 1 || p.ivol == 4 || p.ivol == 5;
            for (int e0 = 0; e0 < ne; e0 += B) {
                int ee[B];
#pragma unroll
                for (int u = 0; u < B; ++u) ee[u] = (e0 + u < ne) ? alist[(size_t)(e0 + u) * nm + a] : -1;
                double4 qq[B];
#pragma unroll
                for (int u = 0; u < B; ++u) qq[u] = ldg4(&pos2[ee[u] != -1 ? (ee[u] & kIdMask) : a]);
#pragma unroll
                for (int u = 0; u < B; ++u) {
                    if (ee[u] == -1) continue;
                    const int j = ee[u] & kIdMask;
                    const double4 q = qq[u];
                    // the minimum image as min_image takes it, keeping the image m
                    const double ux = pa.x - q.x, uy = pa.y - q.y, uz = pa.z - q.z;
                    const double mx = pxy ? round(ux) : 0.0, my = pxy ? round(uy) : 0.0, mz = pz ? round(uz) : 0.0;
                    const double dx = __dsub_rn(ux, mx), dy = __dsub_rn(uy, my), dz = __dsub_rn(uz, mz);
                    const double rx = b[0] * dx + b[3] * dy + b[6] * dz;
                    const double ry = b[1] * dx + b[4] * dy + b[7] * dz;
                    const double rz = b[2] * dx + b[5] * dy + b[8] * dz;
                    const double r = sqrt(rx * rx + ry * ry + rz * rz);
                    const double rr = 1.0 / r;
                    const double4 tv = EXACT ? pair_funcs(t, r) : lookup_r4(t, r);    // vee, dvee, phi, dphi
                    const double fp = -tv.y * rr - (tv.w * pa.w + tv.w * q.w) * rr;
                    const double gxp = dx * fp, gyp = dy * fp, gzp = dz * fp;
                    fxa += gxp; fya += gyp; fza += gzp;
                    if (ee[u] & kOwnBit) {   // the owner's copy carries the pair energy
                        v[0] += tv.x;
                        if (STRESS) { sx += rx * fp; sy += ry * fp; sz += rz * fp; }
                    }
                    const bool excluded = !(ma > 0.1 || ma + mass[j] > 0.1);
                    if (mx != 0.0 || my != 0.0 || mz != 0.0 || excluded) {
                        // c = m, or x_a - x_j when excluded (ux = dx + mx exactly)
                        add_sym(v, excluded ? ux : mx, excluded ? uy : my, excluded ? uz : mz, gxp, gyp, gzp,
                                -0.5);
                    }
                }
            }
            add_sym(v, pa.x, pa.y, pa.z, fxa, fya, fza, 1.0);
        }
        f[a] = fxa; f[nm + a] = fya; f[2 * nm + a] = fza;
        if (STRESS) { stress[a] = sx; stress[nm + a] = sy; stress[2 * nm + a] = sz; }
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
    if (MIXED) {   // the virial moments were summed in fixed-point units^2
#pragma unroll
        for (int k = 1; k < 7; ++k) v[k] *= kFixUnit * kFixUnit;
    }
    // v[1..6] is D; every directed pair entered half of it
    block_partials<7>(v, partials, 0);
}

// ------------------------------------------------ outer and intermediate --
// The screen walks, per atom, a FULL intermediate row: the pairs within
// r_mid = r_cut + skin when the intermediate list was last built.  A pair
// left out was farther than r_mid - eps then (eps bounds the FP32 distance
// error); since then its distance can have shrunk by at most
// 2 max_i |B0 (x_i - x_i,build)| + |B0 - B0_build|_F dmax, with dmax = rnear
// |B0_build^-1|_F bounding the fractional separation of any listed pair.  The
// list is rebuilt before that bound reaches the screening radius, and after
// every half-list rebuild and every force call outside velocity Verlet, so
// the screen keeps exactly the pairs a walk over the whole half list keeps
// (k_mid_decide applies the rule).
//
// The intermediate list is filtered from the outer list (half-list pairs
// within r_out = r_cut + outer skin, both directions), which k_mid_decide has
// rebuilt from the half list whenever the displacements since its own build
// could bring an unlisted pair within r_mid.  The outer build walks, per atom,
// its own half-list row and its reverse half row (the atoms whose rows hold
// it, written by the half-list build) and keeps the pairs within r_out: own
// entries first (flagged in bit 31, in half-list order), then the reverse
// ones in reverse-row order.  Each atom writes only its own row, so there are
// no atomics and every row is the same from run to run.  The intermediate
// build filters each atom's outer row the same way.  Each kernel returns at
// once when k_mid_decide asked for no build.

// FP32 keep radius^2 of a list of radius r: r plus twice the FP32 distance
// error bound, or every pair when the box is too small for the FP32 screen
__device__ float keep_radius2(const double *sb, double r) {
    const float keep = (float)(r + 2.0 * (2.0e-6 * frob(sb) + 1.0e-4));
    return screen_radius2(sb, r * r) > 1e37f ? 3.0e38f : keep * keep;
}

// Appends to atom a's row (entries kept in [cnt, cap), entry-major with
// stride nm) the entries of one source row (n entries, entry k at
// row[k * step]) whose FP32 distance is within keep2; own = bit 31 to set on
// the kept entries.
template <bool FIX, int B>
__device__ __forceinline__ int filter_row(const Params &p, const int32_t *__restrict__ row, size_t step, int n,
                                          int a, const double4 &pa, const int4 &qa, const double4 *__restrict__ pos,
                                          const int4 *__restrict__ posq, const float *bf, float keep2,
                                          int32_t own, int32_t *__restrict__ dst, int cap, int cnt) {
    const size_t stride = (size_t)p.nm;
    for (int k0 = 0; k0 < n; k0 += B) {
        int ee[B];
#pragma unroll
        for (int u = 0; u < B; ++u) ee[u] = (k0 + u < n) ? __ldg(&row[(size_t)(k0 + u) * step]) : -1;
        double4 qq[FIX ? 1 : B];
        int4 qi[FIX ? B : 1];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const int j = ee[u] != -1 ? (ee[u] & kIdMask) : a;
            if (FIX) qi[u] = __ldg(&posq[j]);
            else qq[u] = ldg4(&pos[j]);
        }
#pragma unroll
        for (int u = 0; u < B; ++u) {
            if (ee[u] == -1) continue;
            float rx, ry, rz;
            const float r2 = FIX ? fix_sep(bf, qa, qi[u], rx, ry, rz)
                                 : sep2_f32(bf, p.ivol, pa.x - qq[u].x, pa.y - qq[u].y, pa.z - qq[u].z);
            if (!(r2 <= keep2)) continue;
            if (cnt < cap) dst[(size_t)cnt * stride + a] = ee[u] | own;
            ++cnt;
        }
    }
    return cnt;
}

// Both builds in one pass, each when k_mid_decide asked for it (the launch
// returns at once when it asked for neither).  Each atom first refilters its
// outer row from its own half-list row and its reverse half row (within
// r_out: own entries, flagged in bit 31, then the reverse ones), then its
// intermediate row from that outer row (within r_mid), and measures its
// displacement since the outer build (outdisp2, for the next decision).
// An atom reads and writes only its own rows, so there are no atomics and
// every row is the same from run to run; a row longer than its capacity
// keeps its true count, which the flags (outer) or the screening pass
// (intermediate) report.
template <bool FIX>
__global__ void __launch_bounds__(256, 4)
k_list_build(Params p, double rout, double rmid, const double4 *__restrict__ pos, const int4 *__restrict__ posq,
             BoxState *__restrict__ box, const int32_t *__restrict__ nlist, const int32_t *__restrict__ numn,
             const int32_t *__restrict__ rlist, const int32_t *__restrict__ numr, int32_t *__restrict__ olist,
             int32_t *__restrict__ out_cnt, int4 *__restrict__ xout, const int4 *__restrict__ xhalf,
             int32_t *__restrict__ mlist, int32_t *__restrict__ mid_cnt, int4 *__restrict__ xbuild,
             int32_t *__restrict__ flags) {
    grid_dep_wait();   // launched dependent on the step's previous kernel
    __shared__ double sb[9];
    __shared__ float skeep[2];
    __shared__ int sneed[2];
    if (threadIdx.x < 9) sb[threadIdx.x] = box->b0[threadIdx.x];
    if (threadIdx.x == 0) { sneed[0] = box->out_rebuild; sneed[1] = box->mid_rebuild; }
    __syncthreads();
    const bool need_out = sneed[0] != 0, need_mid = sneed[1] != 0;
    if (!need_out && !need_mid) return;
    if (threadIdx.x == 0) { skeep[0] = keep_radius2(sb, rout); skeep[1] = keep_radius2(sb, rmid); }
    __syncthreads();
    float bf[9];   // B0, per fixed-point unit when FIX
    float bq[9];   // B0 per fixed-point unit, for the displacement
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        bf[k] = (float)(FIX ? sb[k] * kFixUnit : sb[k]);
        bq[k] = (float)(sb[k] * kFixUnit);
    }
    const float keep_out = skeep[0], keep_mid = skeep[1];
    const int nm = p.nm, ocap = p.out_cap, mcap = p.mid_cap;
    int over = 0;
    float d2 = 0.f, dh2 = 0.f;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += gridDim.x * blockDim.x) {
        const double4 pa = pos[a];
        const int4 qa = posq[a];
        if (need_out) {
            dh2 = fmaxf(dh2, fix_disp2(bq, qa, xhalf[a]));
            // the own row is stored atom-major (NLIST(:, a)), the reverse row entry-major
            int cnt = filter_row<FIX, 4>(p, nlist + (size_t)a * p.nnbrs, 1, numn[a], a, pa, qa, pos, posq, bf,
                                         keep_out, kOwnBit, olist, ocap, 0);
            cnt = filter_row<FIX, 4>(p, rlist + a, (size_t)nm, numr[a], a, pa, qa, pos, posq, bf, keep_out, 0, olist,
                                     ocap, cnt);
            out_cnt[a] = cnt;
            if (cnt > ocap) over = max(over, cnt);
            xout[a] = qa;
        }
        if (need_mid) {
            const int nt = out_cnt[a];
            const int n = nt < ocap ? nt : ocap;
            mid_cnt[a] = filter_row<FIX, 4>(p, olist + a, (size_t)nm, n, a, pa, qa, pos, posq, bf, keep_mid, 0, mlist,
                                            mcap, 0);
            xbuild[a] = qa;
            d2 = fmaxf(d2, fix_disp2(bq, qa, xout[a]));
        }
    }
    if (over) { atomicExch(&flags[8], 1); atomicMax(&flags[9], over); }
    __shared__ float wmax[8], hmax[8];
    if (need_out) {
        // the displacement since the source half list's build, block maximum
        // then one atomic per block
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) dh2 = fmaxf(dh2, __shfl_xor_sync(0xffffffffu, dh2, o));
        if ((threadIdx.x & 31) == 0) hmax[threadIdx.x >> 5] = dh2;
        __syncthreads();
        if (threadIdx.x == 0) {
            float m = 0.f;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, hmax[w]);
            atomicMax(&box->halfdisp2, (unsigned long long)__double_as_longlong((double)m));
        }
    }
    if (need_mid) {
        // block maximum, then one atomic per block (non-negative doubles order as their bits)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d2 = fmaxf(d2, __shfl_xor_sync(0xffffffffu, d2, o));
        if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = d2;
        __syncthreads();
        if (threadIdx.x == 0) {
            float m = 0.f;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, wmax[w]);
            atomicMax(&box->outdisp2, (unsigned long long)__double_as_longlong((double)m));
        }
    }
}

// fixed-point separations in a fully periodic box, FP64 differences otherwise;
// the launches exit at once when no build was decided, so their grids are one
// resident wave
void launch_mid_build(DeviceState &d, const Params &p, double rmid, double rout, cudaStream_t s) {
    const bool fix = p.ivol == 0 || p.ivol == 1 || p.ivol == 4;
    int nb = grid_blocks(p.nm, 256);
    if (fix)
        LAUNCH_WAVE(k_list_build<true>, nb, s, p, rout, rmid, d.pos, d.posq, d.box, d.nlist, d.numn, d.rlist,
                    d.numr, d.olist, d.out_cnt, d.xout, d.xhalf, d.mlist, d.mid_cnt, d.xbuild, d.flags);
    else
        LAUNCH_WAVE(k_list_build<false>, nb, s, p, rout, rmid, d.pos, d.posq, d.box, d.nlist, d.numn, d.rlist,
                    d.numr, d.olist, d.out_cnt, d.xout, d.xhalf, d.mlist, d.mid_cnt, d.xbuild, d.flags);
}

// ------------------------------------------------------------ launchers --
// Variant v (0..7): bit 0 selects the batch of list entries whose gathers are
// issued before any is used (screen-density {4, 8}, forces {2, 4}); bit 1 adds
// L2 prefetches of the next atom's rows and per-atom data; bit 2 asks for 3
// resident blocks per SM instead of 2 (fewer registers per thread, more warps
// to hide the gather latency).
template <int B, bool PF, int MINB>
static int sd_variant(DeviceState &d, const Params &p, const Tables &t, bool mixed, double *partials,
                      int store_rho, cudaStream_t s) {
#define SD_ARGS p, t, d.pos, d.posq, d.pos2, d.posq2, d.box, d.mlist, d.mid_cnt, d.alist, d.pair_cnt, \
                d.rho, d.afrho, d.dafrho, partials, d.flags, store_rho
    int nb = grid_blocks(p.nm, 256);
    if (t.exact) LAUNCH_WAVE((k_screen_density<false, true, B, PF, MINB>), nb, s, SD_ARGS);
    else if (mixed) LAUNCH_WAVE((k_screen_density<true, false, B, PF, MINB>), nb, s, SD_ARGS);
    else LAUNCH_WAVE((k_screen_density<false, false, B, PF, MINB>), nb, s, SD_ARGS);
#undef SD_ARGS
    return nb;
}

// The mixed passes take the minimum image from fixed-point differences, which
// needs a box periodic in all three directions; other boxes run in FP64.
static inline bool mixed_applies(const Params &p) { return p.ivol == 0 || p.ivol == 1 || p.ivol == 4; }

int launch_screen_density(DeviceState &d, const Params &p, const Tables &t, bool mixed, int variant,
                          double *partials, cudaStream_t s, bool store_rho) {
    mixed = mixed && mixed_applies(p);
    switch (variant) {
    case 0: return sd_variant<4, true, 4>(d, p, t, mixed, partials, store_rho ? 1 : 0, s);
    case 1: return sd_variant<8, true, 4>(d, p, t, mixed, partials, store_rho ? 1 : 0, s);
    case 2: return sd_variant<4, true, 2>(d, p, t, mixed, partials, store_rho ? 1 : 0, s);
    case 3: return sd_variant<8, true, 2>(d, p, t, mixed, partials, store_rho ? 1 : 0, s);
    case 4: return sd_variant<4, false, 3>(d, p, t, mixed, partials, store_rho ? 1 : 0, s);
    case 5: return sd_variant<8, false, 3>(d, p, t, mixed, partials, store_rho ? 1 : 0, s);
    case 6: return sd_variant<4, true, 3>(d, p, t, mixed, partials, store_rho ? 1 : 0, s);
    default: return sd_variant<8, true, 3>(d, p, t, mixed, partials, store_rho ? 1 : 0, s);
    }
}

template <int B, bool PF, bool STRESS, int MINB>
static int forces_variant(DeviceState &d, const Params &p, const Tables &t, bool mixed, int mode, double *partials,
                          cudaStream_t s) {
#define FORCE_ARGS p, t, d.pos2, d.posq2, d.box, d.alist, d.pair_cnt, d.mass, d.znum, d.del2, d.f, d.x1, d.x2, \
                   d.stress, partials, mode
    int nb = grid_blocks(p.nm, 256);
    if (t.exact) LAUNCH_WAVE((k_forces<false, true, B, PF, STRESS, MINB>), nb, s, FORCE_ARGS);
    else if (mixed) LAUNCH_WAVE((k_forces<true, false, B, PF, STRESS, MINB>), nb, s, FORCE_ARGS);
    else LAUNCH_WAVE((k_forces<false, false, B, PF, STRESS, MINB>), nb, s, FORCE_ARGS);
#undef FORCE_ARGS
    return nb;
}

int launch_forces(DeviceState &d, const Params &p, const Tables &t, bool mixed, int mode,
                  int variant, double *partials, cudaStream_t s) {
    mixed = mixed && mixed_applies(p);
    if (p.atomstress) return forces_variant<2, false, true, 2>(d, p, t, mixed, mode, partials, s);
    switch (variant) {
    case 0: return forces_variant<2, true, false, 4>(d, p, t, mixed, mode, partials, s);
    case 1: return forces_variant<4, true, false, 4>(d, p, t, mixed, mode, partials, s);
    case 2: return forces_variant<2, true, false, 2>(d, p, t, mixed, mode, partials, s);
    case 3: return forces_variant<4, true, false, 2>(d, p, t, mixed, mode, partials, s);
    case 4: return forces_variant<2, false, false, 3>(d, p, t, mixed, mode, partials, s);
    case 5: return forces_variant<4, false, false, 3>(d, p, t, mixed, mode, partials, s);
    case 6: return forces_variant<2, true, false, 3>(d, p, t, mixed, mode, partials, s);
    default: return forces_variant<4, true, false, 3>(d, p, t, mixed, mode, partials, s);
    }
}

// list entries the screening pass reads per step (the full intermediate rows)
__global__ void k_count_screened(int nm, const int32_t *__restrict__ mid_cnt,
                                 unsigned long long *__restrict__ out) {
    unsigned long long s = 0;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += gridDim.x * blockDim.x) {
        s += (unsigned long long)mid_cnt[a];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

void launch_count_screened(const DeviceState &d, const Params &p, unsigned long long *out, cudaStream_t s) {
    cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
    k_count_screened<<<grid_blocks(p.nm, kAtomThreads), kAtomThreads, 0, s>>>(p.nm, d.mid_cnt, out);
}

}  // namespace moldy
