// eam.cu -- the two-pass Finnis-Sinclair/EAM evaluation, the virial and the
// velocity-Verlet / Parrinello-Rahman update (dynamics_m, potential_m,
// thermostat_m::kinten, quench_m::velocityverlet).
//
// The pair passes walk the reference's half list: TPA lanes share one owner
// atom i, each lane takes every TPA-th neighbour j.  Pairs beyond the last
// nonzero table node are skipped (their table values are exactly zero).  The
// j side is scattered with FP64 atomics (the reference uses per-link-cell
// OpenMP locks), the i side is reduced over the lane group and added once.
#include "engine.h"

namespace moldy {

// --------------------------------------------------------- pass 1: density --
// rhoset (src/dynamics_m.F90:497-579): rho_j += phi(r), rho_i += phi(r)
template <int TPA>
__global__ void __launch_bounds__(256)
k_density(Params p, Tables t, const double4 *__restrict__ pos, const BoxState *__restrict__ box,
          const int32_t *__restrict__ nlist, const int32_t *__restrict__ numn,
          double *__restrict__ rho) {
    __shared__ double sb[9];
    if (threadIdx.x < 9) sb[threadIdx.x] = box->b0[threadIdx.x];
    __syncthreads();
    double b[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) b[k] = sb[k];
    constexpr int GPW = 32 / TPA;                      // groups per warp
    const int l = threadIdx.x % TPA;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int base = warp * GPW; base < p.nm; base += nwarps * GPW) {
        const int g = base + lane / TPA;
        const bool active = g < p.nm;
        double rho_i = 0.0;
        if (active) {
            const double4 pa = pos[g];
            const int n = numn[g];
            const int32_t *row = nlist + (size_t)g * p.nnbrs;
            for (int k = l; k < n; k += TPA) {
                int j = row[k];
                double4 pj = pos[j];
                double dx = pa.x - pj.x, dy = pa.y - pj.y, dz = pa.z - pj.z;
                min_image(p.ivol, dx, dy, dz);
                double rx = b[0] * dx + b[3] * dy + b[6] * dz;
                double ry = b[1] * dx + b[4] * dy + b[7] * dz;
                double rz = b[2] * dx + b[5] * dy + b[8] * dz;
                double r2 = rx * rx + ry * ry + rz * rz;
                if (r2 > t.rcull2) continue;
                double phi = density_func(t, sqrt(r2));
                atomicAdd(&rho[j], phi);
                rho_i += phi;
            }
        }
#pragma unroll
        for (int o = TPA / 2; o > 0; o >>= 1) rho_i += __shfl_xor_sync(0xffffffffu, rho_i, o);
        if (active && l == 0) atomicAdd(&rho[g], rho_i);
    }
}

void launch_density(DeviceState &d, const Params &p, const Tables &t, cudaStream_t s) {
    int nb = grid_blocks((long long)p.nm * kPairTPA, 256);
    k_density<kPairTPA><<<nb, 256, 0, s>>>(p, t, d.pos, d.box, d.nlist, d.numn, d.rho);
}

// --------------------------------------------------- embed + kinetic stress --
// embed (src/potential_m.F90:148-169): rho <= 1e-40 keeps the old F, F'.
// kinten (src/thermostat_m.F90:127-164): tk(a,b) += x1_b * m (B0 x1)_a.
// F' is also stored in pos.w for the force pass.
__global__ void __launch_bounds__(256)
k_embed_kinten(Params p, Tables t, double4 *__restrict__ pos, const BoxState *__restrict__ box,
               const double *__restrict__ rho, double *__restrict__ afrho,
               double *__restrict__ dafrho, const double *__restrict__ x1,
               const double *__restrict__ mass, const int32_t *__restrict__ znum,
               double *__restrict__ partials) {
    __shared__ double sb[9];
    if (threadIdx.x < 9) sb[threadIdx.x] = box->b0[threadIdx.x];
    __syncthreads();
    double v[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) v[k] = 0.0;
    const int nm = p.nm;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += gridDim.x * blockDim.x) {
        double r = rho[a];
        double fd = dafrho[a];
        if (r > 1e-40) {
            double2 e = embed_funcs(t, r);
            afrho[a] = e.x;
            dafrho[a] = e.y;
            fd = e.y;
            v[0] += e.x;
        }
        pos[a].w = fd;
        if (znum[a] != 0) {
            double m = mass[a];
            double ux = x1[a], uy = x1[nm + a], uz = x1[2 * nm + a];
            double mvx = (sb[0] * ux + sb[3] * uy + sb[6] * uz) * m;
            double mvy = (sb[1] * ux + sb[4] * uy + sb[7] * uz) * m;
            double mvz = (sb[2] * ux + sb[5] * uy + sb[8] * uz) * m;
            v[1] += ux * mvx; v[2] += ux * mvy; v[3] += ux * mvz;   // tk(:,1)
            v[4] += uy * mvx; v[5] += uy * mvy; v[6] += uy * mvz;   // tk(:,2)
            v[7] += uz * mvx; v[8] += uz * mvy; v[9] += uz * mvz;   // tk(:,3)
        }
    }
    block_partials<10>(v, partials, 0);
}

void launch_embed_kinten(DeviceState &d, const Params &p, const Tables &t, double *partials,
                         cudaStream_t s) {
    int nblocks = grid_blocks(p.nm, kAtomThreads);
    k_embed_kinten<<<nblocks, kAtomThreads, 0, s>>>(p, t, d.pos, d.box, d.rho, d.afrho, d.dafrho,
                                                    d.x1, d.mass, d.znum, partials);
}

// ------------------------------------------------------ pass 2: pair forces --
// force loop (src/dynamics_m.F90:235-346):
//   fp = -dvee/r - (dphi_ij F'_i + dphi_ji F'_j)/r,  f_j += -dx fp,  f_i -= sum(-dx fp)
//   tp(a,b) += dx_b (B0 dx)_a fp  when m_i + m_j > 0.1,  pe += vee.
template <int TPA>
__global__ void __launch_bounds__(256)
k_pair_forces(Params p, Tables t, const double4 *__restrict__ pos, const BoxState *__restrict__ box,
              const int32_t *__restrict__ nlist, const int32_t *__restrict__ numn,
              const double *__restrict__ mass, double *__restrict__ f,
              double *__restrict__ stress, double *__restrict__ partials) {
    __shared__ double sb[9];
    if (threadIdx.x < 9) sb[threadIdx.x] = box->b0[threadIdx.x];
    __syncthreads();
    double b[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) b[k] = sb[k];
    double v[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) v[k] = 0.0;
    constexpr int GPW = 32 / TPA;
    const int l = threadIdx.x % TPA;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nm = p.nm;
    for (int base = warp * GPW; base < nm; base += nwarps * GPW) {
        const int g = base + lane / TPA;
        const bool active = g < nm;
        double fxi = 0.0, fyi = 0.0, fzi = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
        if (active) {
            const double4 pa = pos[g];
            const double ma = mass[g];
            const int n = numn[g];
            const int32_t *row = nlist + (size_t)g * p.nnbrs;
            for (int k = l; k < n; k += TPA) {
                int j = row[k];
                double4 pj = pos[j];
                double dx = pa.x - pj.x, dy = pa.y - pj.y, dz = pa.z - pj.z;
                min_image(p.ivol, dx, dy, dz);
                double rx = b[0] * dx + b[3] * dy + b[6] * dz;
                double ry = b[1] * dx + b[4] * dy + b[7] * dz;
                double rz = b[2] * dx + b[5] * dy + b[8] * dz;
                double r2 = rx * rx + ry * ry + rz * rz;
                if (r2 > t.rcull2) continue;
                double r = sqrt(r2);
                double rr = 1.0 / r;
                double4 tv = pair_funcs(t, r);            // vee, dvee, phi, dphi
                double fpp = -tv.y * rr;
                double fcp = -(tv.w * pa.w + tv.w * pj.w) * rr;
                double fp = fpp + fcp;
                v[0] += tv.x;
                if (p.atomstress) { sx += rx * fp; sy += ry * fp; sz += rz * fp; }
                if (ma > 0.1 || ma + mass[j] > 0.1) {
                    v[1] += dx * rx * fp; v[2] += dx * ry * fp; v[3] += dx * rz * fp;
                    v[4] += dy * rx * fp; v[5] += dy * ry * fp; v[6] += dy * rz * fp;
                    v[7] += dz * rx * fp; v[8] += dz * ry * fp; v[9] += dz * rz * fp;
                }
                double ddx = -(dx * fp), ddy = -(dy * fp), ddz = -(dz * fp);
                atomicAdd(&f[j], ddx);
                atomicAdd(&f[nm + j], ddy);
                atomicAdd(&f[2 * nm + j], ddz);
                fxi += ddx; fyi += ddy; fzi += ddz;
            }
        }
#pragma unroll
        for (int o = TPA / 2; o > 0; o >>= 1) {
            fxi += __shfl_xor_sync(0xffffffffu, fxi, o);
            fyi += __shfl_xor_sync(0xffffffffu, fyi, o);
            fzi += __shfl_xor_sync(0xffffffffu, fzi, o);
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
            sz += __shfl_xor_sync(0xffffffffu, sz, o);
        }
        if (active && l == 0) {
            atomicAdd(&f[g], -fxi);
            atomicAdd(&f[nm + g], -fyi);
            atomicAdd(&f[2 * nm + g], -fzi);
            if (p.atomstress) { stress[g] = sx; stress[nm + g] = sy; stress[2 * nm + g] = sz; }
        }
    }
    block_partials<10>(v, partials, 0);
}

void launch_pair_forces(DeviceState &d, const Params &p, const Tables &t, double *partials,
                        cudaStream_t s) {
    int nb = grid_blocks((long long)p.nm * kPairTPA, 256);
    k_pair_forces<kPairTPA><<<nb, 256, 0, s>>>(p, t, d.pos, d.box, d.nlist, d.numn, d.mass, d.f,
                                               d.stress, partials);
}

// ----------------------------------------------------------- box algebra --
__device__ void mat_cofactor(const double *b, double *tc) {
    // tc as in src/dynamics_m.F90:365-373
    MAT(tc, 1, 1) = MAT(b, 2, 2) * MAT(b, 3, 3) - MAT(b, 2, 3) * MAT(b, 3, 2);
    MAT(tc, 2, 1) = MAT(b, 3, 2) * MAT(b, 1, 3) - MAT(b, 1, 2) * MAT(b, 3, 3);
    MAT(tc, 3, 1) = MAT(b, 1, 2) * MAT(b, 2, 3) - MAT(b, 2, 2) * MAT(b, 1, 3);
    MAT(tc, 1, 2) = MAT(b, 2, 3) * MAT(b, 3, 1) - MAT(b, 3, 3) * MAT(b, 2, 1);
    MAT(tc, 2, 2) = MAT(b, 3, 3) * MAT(b, 1, 1) - MAT(b, 1, 3) * MAT(b, 3, 1);
    MAT(tc, 3, 2) = MAT(b, 1, 3) * MAT(b, 2, 1) - MAT(b, 1, 1) * MAT(b, 2, 3);
    MAT(tc, 1, 3) = MAT(b, 2, 1) * MAT(b, 3, 2) - MAT(b, 3, 1) * MAT(b, 2, 2);
    MAT(tc, 2, 3) = MAT(b, 3, 1) * MAT(b, 1, 2) - MAT(b, 1, 1) * MAT(b, 3, 2);
    MAT(tc, 3, 3) = MAT(b, 1, 1) * MAT(b, 2, 2) - MAT(b, 2, 1) * MAT(b, 1, 2);
}

__device__ double mat_volume(const double *b) {
    // pr_get_metric_tensor (src/parrinellorahman_m.F90:223-227)
    return MAT(b, 1, 1) * (MAT(b, 2, 2) * MAT(b, 3, 3) - MAT(b, 2, 3) * MAT(b, 3, 2)) +
           MAT(b, 2, 1) * (MAT(b, 3, 2) * MAT(b, 1, 3) - MAT(b, 1, 2) * MAT(b, 3, 3)) +
           MAT(b, 3, 1) * (MAT(b, 1, 2) * MAT(b, 2, 3) - MAT(b, 2, 2) * MAT(b, 1, 3));
}

// matrix_invert (src/matrix_m.F90:89-119); returns false for det == 0
__device__ bool mat_invert(const double *a, double *bo) {
    double deta = MAT(a, 1, 1) * (MAT(a, 2, 2) * MAT(a, 3, 3) - MAT(a, 2, 3) * MAT(a, 3, 2));
    deta = deta + MAT(a, 2, 1) * (MAT(a, 3, 2) * MAT(a, 1, 3) - MAT(a, 1, 2) * MAT(a, 3, 3));
    deta = deta + MAT(a, 3, 1) * (MAT(a, 1, 2) * MAT(a, 2, 3) - MAT(a, 1, 3) * MAT(a, 2, 2));
    MAT(bo, 1, 1) = MAT(a, 2, 2) * MAT(a, 3, 3) - MAT(a, 2, 3) * MAT(a, 3, 2);
    MAT(bo, 1, 2) = MAT(a, 3, 1) * MAT(a, 2, 3) - MAT(a, 2, 1) * MAT(a, 3, 3);
    MAT(bo, 1, 3) = MAT(a, 2, 1) * MAT(a, 3, 2) - MAT(a, 3, 1) * MAT(a, 2, 2);
    MAT(bo, 2, 1) = MAT(a, 3, 2) * MAT(a, 1, 3) - MAT(a, 1, 2) * MAT(a, 3, 3);
    MAT(bo, 2, 2) = MAT(a, 1, 1) * MAT(a, 3, 3) - MAT(a, 1, 3) * MAT(a, 3, 1);
    MAT(bo, 2, 3) = MAT(a, 3, 1) * MAT(a, 1, 2) - MAT(a, 1, 1) * MAT(a, 3, 2);
    MAT(bo, 3, 1) = MAT(a, 1, 2) * MAT(a, 2, 3) - MAT(a, 1, 3) * MAT(a, 2, 2);
    MAT(bo, 3, 2) = MAT(a, 2, 1) * MAT(a, 1, 3) - MAT(a, 2, 3) * MAT(a, 1, 1);
    MAT(bo, 3, 3) = MAT(a, 1, 1) * MAT(a, 2, 2) - MAT(a, 1, 2) * MAT(a, 2, 1);
    if (fabs(deta) == 0.0) return false;
    for (int k = 0; k < 9; ++k) bo[k] = bo[k] / deta;
    return true;
}

// matrix_multiply (src/matrix_m.F90:60-79)
__device__ void mat_mul(const double *a, const double *b, double *c) {
    for (int i = 1; i <= 3; ++i) {
        for (int j = 1; j <= 3; ++j) MAT(c, i, j) = 0.0;
        for (int k = 1; k <= 3; ++k)
            for (int j = 1; j <= 3; ++j) MAT(c, i, j) = MAT(c, i, j) + MAT(a, i, k) * MAT(b, k, j);
    }
}

// Sums NV partial columns over nblk blocks in a fixed order into out[NV].
template <int NV>
__device__ void reduce_partials(const double *__restrict__ part, int nblk, double *out) {
    __shared__ double sm[256][NV];
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (int bidx = threadIdx.x; bidx < nblk; bidx += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] += part[(size_t)bidx * kPartials + k];
#pragma unroll
    for (int k = 0; k < NV; ++k) sm[threadIdx.x][k] = acc[k];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
#pragma unroll
            for (int k = 0; k < NV; ++k) sm[threadIdx.x][k] += sm[threadIdx.x + w][k];
        __syncthreads();
    }
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) out[k] = sm[0][k];
    __syncthreads();
}

// mode 0: force only; 1: velocity Verlet second half (box); 2: md_init
__global__ void __launch_bounds__(256)
k_finalize_force(Params p, BoxState *__restrict__ box, const double *__restrict__ part_embed,
                 int nblk_embed, const double *__restrict__ part_force, int nblk_force, int mode) {
    __shared__ double se[10], sf[10];
    reduce_partials<10>(part_embed, nblk_embed, se);
    reduce_partials<10>(part_force, nblk_force, sf);
    if (threadIdx.x != 0) return;
    BoxState &B = *box;
    B.pe_emb = se[0];
    B.pe_pair = sf[0];
    B.pe = se[0] + sf[0];
    for (int k = 0; k < 9; ++k) B.tp[k] = sf[1 + k];
    double dt2 = p.deltat * p.deltat;
    for (int k = 0; k < 9; ++k) B.tk[k] = se[1 + k] / dt2;
    mat_cofactor(B.b0, B.tc);
    for (int k = 0; k < 9; ++k) { B.tgdot[k] = 0.0; B.tg[k] = 0.0; }
    for (int i = 1; i <= 3; ++i)
        for (int k = 1; k <= 3; ++k)
            for (int j = 1; j <= 3; ++j) {
                MAT(B.tg, i, j) = MAT(B.tg, i, j) + MAT(B.b0, k, i) * MAT(B.b0, k, j);
                MAT(B.tgdot, i, j) = MAT(B.tgdot, i, j) + MAT(B.b0, k, i) * MAT(B.b1, k, j) +
                                     MAT(B.b1, k, i) * MAT(B.b0, k, j);
            }
    B.vol = mat_volume(B.b0);
    for (int k = 0; k < 9; ++k) B.fb[k] = B.tk[k] + B.tp[k] - p.press * B.tc[k];
    if (mode == 1) {
        if (p.ivol < 1) {
            for (int k = 0; k < 9; ++k) B.b2[k] = p.bdel2 * B.fb[k];
            for (int k = 0; k < 9; ++k) B.b1[k] = B.b1[k] + B.b2[k];
        }
        if (p.ivol == 4) {
            MAT(B.b2, 3, 3) = p.bdel2 * MAT(B.fb, 3, 3);
            for (int k = 0; k < 9; ++k) B.b1[k] = B.b1[k] + B.b2[k];
        }
    } else if (mode == 2) {
        if (!mat_invert(B.tg, B.tginv)) { B.status = MOLDY_ERR_SINGULAR_BOX; return; }
        mat_mul(B.tginv, B.tgdot, B.tgid);
        for (int k = 0; k < 9; ++k) B.b2[k] = p.bdel2 * B.fb[k];
    }
}

void launch_finalize_force(DeviceState &d, const Params &p, const double *part_embed, int nblk_embed,
                           const double *part_force, int nblk_force, int mode, cudaStream_t s) {
    k_finalize_force<<<1, 256, 0, s>>>(p, d.box, part_embed, nblk_embed, part_force, nblk_force, mode);
}

// ------------------------------------------------------------- integrator --
// velocityverlet first half (src/quench_m.F90:574-589):
//   x1_dt2 = x1 + x2; x0 += x1_dt2; box b1 += b2; b0 += b1 (ivol < 1) or zz only (ivol 4)
__global__ void __launch_bounds__(256)
k_drift(Params p, double4 *__restrict__ pos, const double *__restrict__ x1,
        const double *__restrict__ x2, BoxState *__restrict__ box) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a == 0) {
        BoxState &B = *box;
        if (p.ivol == 4) {
            MAT(B.b1, 3, 3) = MAT(B.b1, 3, 3) + MAT(B.b2, 3, 3);
            MAT(B.b0, 3, 3) = MAT(B.b0, 3, 3) + MAT(B.b1, 3, 3);
        }
        if (p.ivol < 1) {
            for (int k = 0; k < 9; ++k) B.b1[k] = B.b1[k] + B.b2[k];
            for (int k = 0; k < 9; ++k) B.b0[k] = B.b0[k] + B.b1[k];
        }
    }
    if (a >= p.nm) return;
    const int nm = p.nm;
    double4 q = pos[a];
    q.x = q.x + (x1[a] + x2[a]);
    q.y = q.y + (x1[nm + a] + x2[nm + a]);
    q.z = q.z + (x1[2 * nm + a] + x2[2 * nm + a]);
    pos[a] = q;
}

void launch_drift(DeviceState &d, const Params &p, cudaStream_t s) {
    int nb = (p.nm + kAtomThreads - 1) / kAtomThreads;
    k_drift<<<nb, kAtomThreads, 0, s>>>(p, d.pos, d.x1, d.x2, d.box);
}

// velocityverlet second half (src/quench_m.F90:606-622) with the tgid of the
// previous update_therm_avs:  x2 = del2 f - tgid x1 / 2;  x1 = x1_dt2 + x2.
__global__ void __launch_bounds__(256)
k_vv_second_half(Params p, const BoxState *__restrict__ box, const double *__restrict__ f,
                 double *__restrict__ x1, double *__restrict__ x2, const double *__restrict__ del2,
                 const double *__restrict__ mass, const int32_t *__restrict__ znum) {
    __shared__ double tg[9];
    if (threadIdx.x < 9) tg[threadIdx.x] = box->tgid[threadIdx.x];
    __syncthreads();
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= p.nm) return;
    const int nm = p.nm;
    double ux = x1[a], uy = x1[nm + a], uz = x1[2 * nm + a];
    double wx = x2[a], wy = x2[nm + a], wz = x2[2 * nm + a];
    double hx = ux + wx, hy = uy + wy, hz = uz + wz;       // x1_dt2
    if (!(znum[a] == 0 || mass[a] < 0.1)) {
        double sxi = 0.0, syi = 0.0, szi = 0.0;
        if (p.ivol == 0) {
            sxi = tg[0] * ux + tg[3] * uy + tg[6] * uz;
            syi = tg[1] * ux + tg[4] * uy + tg[7] * uz;
            szi = tg[2] * ux + tg[5] * uy + tg[8] * uz;
        }
        if (p.ivol == 4) szi = tg[8] * uz;
        double d2 = del2[a];
        wx = d2 * f[a] - 0.5 * sxi;
        wy = d2 * f[nm + a] - 0.5 * syi;
        wz = d2 * f[2 * nm + a] - 0.5 * szi;
        x2[a] = wx; x2[nm + a] = wy; x2[2 * nm + a] = wz;
    }
    x1[a] = hx + wx; x1[nm + a] = hy + wy; x1[2 * nm + a] = hz + wz;
}

void launch_vv_second_half(DeviceState &d, const Params &p, cudaStream_t s) {
    int nb = (p.nm + kAtomThreads - 1) / kAtomThreads;
    k_vv_second_half<<<nb, kAtomThreads, 0, s>>>(p, d.box, d.f, d.x1, d.x2, d.del2, d.mass, d.znum);
}

// moldin strain-loop preparation (src/moldin.F90:458-471): every atom with a
// species, x2 = del2 f - tgid x1 / 2
__global__ void k_md_init_x2(Params p, const BoxState *__restrict__ box, const double *__restrict__ f,
                             const double *__restrict__ x1, double *__restrict__ x2,
                             const double *__restrict__ del2) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= p.nm) return;
    const double *t = box->tgid;
    const int nm = p.nm;
    double ux = x1[a], uy = x1[nm + a], uz = x1[2 * nm + a];
    double a1 = t[0] * ux + t[3] * uy + t[6] * uz;
    double a2 = t[1] * ux + t[4] * uy + t[7] * uz;
    double a3 = t[2] * ux + t[5] * uy + t[8] * uz;
    double d2 = del2[a];
    x2[a] = d2 * f[a] - 0.5 * a1;
    x2[nm + a] = d2 * f[nm + a] - 0.5 * a2;
    x2[2 * nm + a] = d2 * f[2 * nm + a] - 0.5 * a3;
}

void launch_md_init_x2(DeviceState &d, const Params &p, cudaStream_t s) {
    int nb = (p.nm + kAtomThreads - 1) / kAtomThreads;
    k_md_init_x2<<<nb, kAtomThreads, 0, s>>>(p, d.box, d.f, d.x1, d.x2, d.del2);
}

// ---------------------------------------------------------- thermo sums ----
// update_therm_avs (src/dynamics_m.F90:649-734): tg, tgdot (ivol != 1),
// tgid = tg^-1 tgdot, vol, and per-atom s1 = sum |F|^2, s2 = sum |F|^4,
// s3 = sum m |B0 x1|^2.
__device__ bool therm_box(const Params &p, const BoxState &B, double *tg, double *tgdot,
                          double *tginv, double *tgid, double &vol) {
    for (int k = 0; k < 9; ++k) { tg[k] = 0.0; tgdot[k] = 0.0; }
    for (int i = 1; i <= 3; ++i)
        for (int k = 1; k <= 3; ++k)
            for (int j = 1; j <= 3; ++j) {
                MAT(tg, i, j) = MAT(tg, i, j) + MAT(B.b0, k, i) * MAT(B.b0, k, j);
                if (p.ivol != 1)
                    MAT(tgdot, i, j) = MAT(tgdot, i, j) + MAT(B.b1, k, i) * MAT(B.b0, k, j) +
                                       MAT(B.b0, k, i) * MAT(B.b1, k, j);
            }
    bool ok = mat_invert(tg, tginv);
    mat_mul(tginv, tgdot, tgid);
    vol = mat_volume(B.b0);
    return ok;
}

__global__ void __launch_bounds__(256)
k_therm(Params p, const BoxState *__restrict__ box, const double *__restrict__ x1,
        const double *__restrict__ x2, const double *__restrict__ mass,
        const int32_t *__restrict__ znum, double *__restrict__ partials) {
    __shared__ double sh[9 + 9 + 9];   // tgid, b0, cof(b0)/vol
    if (threadIdx.x == 0) {
        double tg[9], tgdot[9], tginv[9], tgid[9], vol;
        therm_box(p, *box, tg, tgdot, tginv, tgid, vol);
        const double *b = box->b0;
        for (int k = 0; k < 9; ++k) { sh[k] = tgid[k]; sh[9 + k] = b[k]; }
        double *d = sh + 18;   // b0_xxdet ... stored row-major as in the reference names
        d[0] = (MAT(b, 2, 2) * MAT(b, 3, 3) - MAT(b, 2, 3) * MAT(b, 3, 2)) / vol;
        d[1] = (MAT(b, 2, 3) * MAT(b, 3, 1) - MAT(b, 3, 3) * MAT(b, 2, 1)) / vol;
        d[2] = (MAT(b, 2, 1) * MAT(b, 3, 2) - MAT(b, 3, 1) * MAT(b, 2, 2)) / vol;
        d[3] = (MAT(b, 3, 2) * MAT(b, 1, 3) - MAT(b, 1, 2) * MAT(b, 3, 3)) / vol;
        d[4] = (MAT(b, 1, 1) * MAT(b, 3, 3) - MAT(b, 1, 3) * MAT(b, 3, 1)) / vol;
        d[5] = (MAT(b, 3, 1) * MAT(b, 1, 2) - MAT(b, 1, 1) * MAT(b, 3, 2)) / vol;
        d[6] = (MAT(b, 1, 2) * MAT(b, 2, 3) - MAT(b, 2, 2) * MAT(b, 1, 3)) / vol;
        d[7] = (MAT(b, 1, 3) * MAT(b, 2, 1) - MAT(b, 1, 1) * MAT(b, 2, 3)) / vol;
        d[8] = (MAT(b, 1, 1) * MAT(b, 2, 2) - MAT(b, 1, 2) * MAT(b, 2, 1)) / vol;
    }
    __syncthreads();
    double v[3] = {0.0, 0.0, 0.0};
    const int nm = p.nm;
    const double *t = sh, *b = sh + 9, *d = sh + 18;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += gridDim.x * blockDim.x) {
        if (znum[a] == 0) continue;
        double ux = x1[a], uy = x1[nm + a], uz = x1[2 * nm + a];
        double sxi = t[0] * ux + t[3] * uy + t[6] * uz;
        double syi = t[1] * ux + t[4] * uy + t[7] * uz;
        double szi = t[2] * ux + t[5] * uy + t[8] * uz;
        double fxp = 2.0 * x2[a] + sxi, fyp = 2.0 * x2[nm + a] + syi, fzp = 2.0 * x2[2 * nm + a] + szi;
        double fx = d[0] * fxp + d[1] * fyp + d[2] * fzp;
        double fy = d[3] * fxp + d[4] * fyp + d[5] * fzp;
        double fz = d[6] * fxp + d[7] * fyp + d[8] * fzp;
        double f2 = fx * fx + fy * fy + fz * fz;
        v[0] += f2;
        v[1] += f2 * f2;
        double rx = b[0] * ux + b[3] * uy + b[6] * uz;
        double ry = b[1] * ux + b[4] * uy + b[7] * uz;
        double rz = b[2] * ux + b[5] * uy + b[8] * uz;
        v[2] += mass[a] * (rx * rx + ry * ry + rz * rz);
    }
    block_partials<3>(v, partials, 0);
}

int launch_therm(DeviceState &d, const Params &p, cudaStream_t s) {
    int nblocks = grid_blocks(p.nm, kAtomThreads);
    k_therm<<<nblocks, kAtomThreads, 0, s>>>(p, d.box, d.x1, d.x2, d.mass, d.znum, d.partials);
    return nblocks;
}

// reduces the thermo partials and derives the mdloop quantities
// (src/moldin.F90:760-790)
__global__ void __launch_bounds__(256)
k_finalize_therm(Params p, BoxState *__restrict__ box, const double *__restrict__ partials, int nblk) {
    __shared__ double s[3];
    reduce_partials<3>(partials, nblk, s);
    if (threadIdx.x != 0) return;
    BoxState &B = *box;
    double vol;
    if (!therm_box(p, B, B.tg, B.tgdot, B.tginv, B.tgid, vol)) B.status = MOLDY_ERR_SINGULAR_BOX;
    B.vol = vol;
    B.s1 = s[0]; B.s2 = s[1]; B.s3 = s[2];
    const double bk = 1.3806504e-23 / 1.602176487e-19;
    B.ke = s[2] / (p.deltat * p.deltat) / 2.0;
    B.temp = B.ke / (1.5 * bk * (double)p.nm);
    double boxke = 0.0;
    for (int i = 1; i <= 3; ++i)
        for (int j = 1; j <= 3; ++j) boxke = boxke + (MAT(B.b1, i, j) * MAT(B.b1, i, j)) / p.bdel2;
    B.boxke = boxke;
    B.te = B.ke + B.pe;
    B.h = B.te + p.press * B.vol;
    B.th = B.h + boxke;
}

void launch_finalize_therm(DeviceState &d, const Params &p, int nblocks, cudaStream_t s) {
    k_finalize_therm<<<1, 256, 0, s>>>(p, d.box, d.partials, nblocks);
}

// ------------------------------------------------------------ energy_calc --
// src/dynamics_m.F90:412-483: en_atom = F(rho) + half of each exact pair term
__global__ void __launch_bounds__(256)
k_energy_pairs(Params p, Tables t, const double4 *__restrict__ pos, const BoxState *__restrict__ box,
               const int32_t *__restrict__ nlist, const int32_t *__restrict__ numn,
               double *__restrict__ en) {
    __shared__ double sb[9];
    if (threadIdx.x < 9) sb[threadIdx.x] = box->b0[threadIdx.x];
    __syncthreads();
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= p.nm) return;
    const double4 pa = pos[a];
    const int n = numn[a];
    const int32_t *row = nlist + (size_t)a * p.nnbrs;
    double own = 0.0;
    for (int k = 0; k < n; ++k) {
        int j = row[k];
        double4 pj = pos[j];
        double dx = pa.x - pj.x, dy = pa.y - pj.y, dz = pa.z - pj.z;
        min_image(p.ivol, dx, dy, dz);
        double rx = sb[0] * dx + sb[3] * dy + sb[6] * dz;
        double ry = sb[1] * dx + sb[4] * dy + sb[7] * dz;
        double rz = sb[2] * dx + sb[5] * dy + sb[8] * dz;
        double r = sqrt(rx * rx + ry * ry + rz * rz);
        double pp = fetm_vee(t, r) / 2.0;
        if (pp != 0.0) {
            own += pp;
            atomicAdd(&en[j], pp);
        }
    }
    atomicAdd(&en[a], own);
}

void launch_energy_calc(DeviceState &d, const Params &p, const Tables &t, cudaStream_t s) {
    cudaMemcpyAsync(d.en_atom, d.afrho, sizeof(double) * p.nm, cudaMemcpyDeviceToDevice, s);
    int nb = (p.nm + kAtomThreads - 1) / kAtomThreads;
    k_energy_pairs<<<nb, kAtomThreads, 0, s>>>(p, t, d.pos, d.box, d.nlist, d.numn, d.en_atom);
}

}  // namespace moldy
