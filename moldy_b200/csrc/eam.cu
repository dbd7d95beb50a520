// eam.cu -- box algebra, the velocity-Verlet / Parrinello-Rahman update, the
// thermodynamic sums and energy_calc (dynamics_m, thermostat_m::kinten,
// quench_m::velocityverlet).  The pair passes are in pairs.cu.
#include "engine.h"

namespace moldy {

__device__ void therm_prep(const Params &p, const double *b0, const double *b1, BoxState &B);

int stream_blocks(int nm) {
    static const int sms = [] {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n > 0 ? n : 148;
    }();
    const int nb = grid_blocks(nm, kAtomThreads);
    return nb < 4 * sms ? nb : 4 * sms;
}

__device__ void therm_prep(const Params &p, const double *b, const double *b1, BoxState &B);

// The box algebra of k_finalize_force, by one thread on the block's shared
// copy of the box: sr holds the 15 reduced sums (embedding energy, pair
// count; pair energy, virial moments; kinetic moments).
__device__ void finalize_box(const Params &p, BoxState &B, const double *sr, int mode) {
    const double *se = sr, *sf = sr + 2, *sk = sr + 9;
    // the box algebra runs on register copies and is stored once at the end
    double b0[9], b1[9], b2[9], tp[9], tk[9], tc[9], tg[9], tgdot[9], fb[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { b0[k] = B.b0[k]; b1[k] = B.b1[k]; b2[k] = B.b2[k]; }
    B.pe_emb = se[0];
    B.pe_pair = sf[0];
    B.pe = se[0] + sf[0];
    B.npairs = se[1];
    // symmetric moments (xx, yy, zz, xy, xz, yz) -> full 3x3
    double M[9], D[9];
    M[0] = sk[0]; M[4] = sk[1]; M[8] = sk[2]; M[3] = M[1] = sk[3]; M[6] = M[2] = sk[4]; M[7] = M[5] = sk[5];
    D[0] = sf[1]; D[4] = sf[2]; D[8] = sf[3]; D[3] = D[1] = sf[4]; D[6] = D[2] = sf[5]; D[7] = D[5] = sf[6];
    double dt2 = p.deltat * p.deltat;
    mat_mul(b0, D, tp);                           // tp(a,b) = sum r_a d_b fp, r = B0 d
    mat_mul(b0, M, tk);                           // tk(a,b) = sum m (B0 x1)_a x1_b
#pragma unroll
    for (int k = 0; k < 9; ++k) tk[k] = tk[k] / dt2;
    mat_cofactor(b0, tc);
#pragma unroll
    for (int k = 0; k < 9; ++k) { tgdot[k] = 0.0; tg[k] = 0.0; }
#pragma unroll
    for (int i = 1; i <= 3; ++i)
#pragma unroll
        for (int k = 1; k <= 3; ++k)
#pragma unroll
            for (int j = 1; j <= 3; ++j) {
                MAT(tg, i, j) = MAT(tg, i, j) + MAT(b0, k, i) * MAT(b0, k, j);
                MAT(tgdot, i, j) = MAT(tgdot, i, j) + MAT(b0, k, i) * MAT(b1, k, j) + MAT(b1, k, i) * MAT(b0, k, j);
            }
    const double vol = mat_volume(b0);
#pragma unroll
    for (int k = 0; k < 9; ++k) fb[k] = tk[k] + tp[k] - p.press * tc[k];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        B.tp[k] = tp[k]; B.tk[k] = tk[k]; B.tc[k] = tc[k]; B.tg[k] = tg[k]; B.tgdot[k] = tgdot[k]; B.fb[k] = fb[k];
    }
    B.vol = vol;
    if (mode == 1) {
        if (p.ivol < 1) {
#pragma unroll
            for (int k = 0; k < 9; ++k) b2[k] = p.bdel2 * fb[k];
#pragma unroll
            for (int k = 0; k < 9; ++k) b1[k] = b1[k] + b2[k];
        }
        if (p.ivol == 4) {
            MAT(b2, 3, 3) = p.bdel2 * MAT(fb, 3, 3);
#pragma unroll
            for (int k = 0; k < 9; ++k) b1[k] = b1[k] + b2[k];
        }
    } else if (mode == 2) {
        double tginv[9], tgid[9];
        if (!mat_invert(tg, tginv)) { B.status = MOLDY_ERR_SINGULAR_BOX; return; }
        mat_mul(tginv, tgdot, tgid);
#pragma unroll
        for (int k = 0; k < 9; ++k) { B.tginv[k] = tginv[k]; B.tgid[k] = tgid[k]; b2[k] = p.bdel2 * fb[k]; }
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) { B.b1[k] = b1[k]; B.b2[k] = b2[k]; }
    therm_prep(p, b0, b1, B);       // for the update_therm_avs that follows
}

// mode 0: force only; 1: velocity Verlet second half (box); 2: md_init
__global__ void __launch_bounds__(256)
k_finalize_force(Params p, BoxState *__restrict__ box, const double *__restrict__ part_embed,
                 int nblk_embed, const double *__restrict__ part_force, int nblk_force,
                 const double *__restrict__ part_kin, int nblk_kin, int mode) {
    grid_dep_wait();   // launched dependent on the step's previous kernel
    // the box in shared memory, loaded while the partials are summed
    __shared__ BoxState sbox;
    box_load(sbox, box);
    // the three sets of block partials in one pass: each thread issues the
    // loads of all three before adding (per set, the same order as
    // reduce_partials)
    __shared__ double sm[8][15], sr[15];
    double acc[15];
#pragma unroll
    for (int k = 0; k < 15; ++k) acc[k] = 0.0;
    const int nmax = max(nblk_embed, max(nblk_force, nblk_kin));
    for (int b = threadIdx.x; b < nmax; b += blockDim.x) {
        double e[15];
#pragma unroll
        for (int k = 0; k < 2; ++k) e[k] = b < nblk_embed ? part_embed[(size_t)b * kPartials + k] : 0.0;
#pragma unroll
        for (int k = 0; k < 7; ++k) e[2 + k] = b < nblk_force ? part_force[(size_t)b * kPartials + k] : 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k) e[9 + k] = b < nblk_kin ? part_kin[(size_t)b * kPartials + k] : 0.0;
#pragma unroll
        for (int k = 0; k < 15; ++k) acc[k] += e[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 15; ++k) {
        const double w = warp_sum(acc[k]);
        if (lane == 0) sm[warp][k] = w;
    }
    __syncthreads();
    if (warp == 0 && lane < 15) {
        double w = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) w += sm[q][lane];
        sr[lane] = w;
    }
    __syncthreads();
    __syncthreads();
    if (threadIdx.x == 0) finalize_box(p, sbox, sr, mode);
    __syncthreads();
    box_store(box, sbox);
}

void launch_finalize_force(DeviceState &d, const Params &p, const double *part_embed, int nblk_embed,
                           const double *part_force, int nblk_force, const double *part_kin, int nblk_kin,
                           int mode, cudaStream_t s) {
    launch_pdl(k_finalize_force, 1, 256, s, p, d.box, part_embed, nblk_embed, part_force, nblk_force, part_kin, nblk_kin,
                                        mode);
}

// kinten's moment M = sum m x1 x1^T over atoms with a species
// (src/thermostat_m.F90:138-157); tk = B0 M / dt^2 in k_finalize_force
__device__ __forceinline__ void kin_moment(double (&v)[6], double m, double ux, double uy, double uz) {
    v[0] += m * ux * ux; v[1] += m * uy * uy; v[2] += m * uz * uz;
    v[3] += m * ux * uy; v[4] += m * ux * uz; v[5] += m * uy * uz;
}

__global__ void __launch_bounds__(256)
k_kinetic(Params p, const double *__restrict__ x1, const double *__restrict__ mass,
          const int32_t *__restrict__ znum, double *__restrict__ partials) {
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const int nm = p.nm;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += gridDim.x * blockDim.x)
        if (znum[a] != 0) kin_moment(v, mass[a], x1[a], x1[nm + a], x1[2 * nm + a]);
    block_partials<6>(v, partials, 0);
}

int launch_kinetic(DeviceState &d, const Params &p, double *partials, cudaStream_t s) {
    int nb = stream_blocks(p.nm);
    k_kinetic<<<nb, kAtomThreads, 0, s>>>(p, d.x1, d.mass, d.znum, partials);
    return nb;
}

// ---------------------------------------------------------- thermo sums ----
// update_therm_avs (src/dynamics_m.F90:649-734): tg, tgdot (ivol != 1),
// tgid = tg^-1 tgdot, vol, and per-atom s1 = sum |F|^2, s2 = sum |F|^4,
// s3 = sum m |B0 x1|^2.
__device__ __forceinline__ bool therm_box(const Params &p, const double *b0, const double *b1, double *tg,
                                          double *tgdot, double *tginv, double *tgid, double &vol) {
#pragma unroll
    for (int k = 0; k < 9; ++k) { tg[k] = 0.0; tgdot[k] = 0.0; }
#pragma unroll
    for (int i = 1; i <= 3; ++i)
#pragma unroll
        for (int k = 1; k <= 3; ++k)
#pragma unroll
            for (int j = 1; j <= 3; ++j) {
                MAT(tg, i, j) = MAT(tg, i, j) + MAT(b0, k, i) * MAT(b0, k, j);
                if (p.ivol != 1)
                    MAT(tgdot, i, j) = MAT(tgdot, i, j) + MAT(b1, k, i) * MAT(b0, k, j) +
                                       MAT(b0, k, i) * MAT(b1, k, j);
            }
    bool ok = mat_invert(tg, tginv);
    mat_mul(tginv, tgdot, tgid);
    vol = mat_volume(b0);
    return ok;
}

// The box quantities k_therm needs, from the box after the force call:
// tgid = tg^-1 tgdot of the new B1 and cof(B0)/vol (the b0_xxdet ... of
// update_therm_avs); computed once, by one thread, from register copies of
// B0 and B1.
__device__ void therm_prep(const Params &p, const double *b, const double *b1, BoxState &B) {
    double tg[9], tgdot[9], tginv[9], tgid[9], vol, d[9];   // d row-major as in the reference's names
    therm_box(p, b, b1, tg, tgdot, tginv, tgid, vol);
    d[0] = (MAT(b, 2, 2) * MAT(b, 3, 3) - MAT(b, 2, 3) * MAT(b, 3, 2)) / vol;
    d[1] = (MAT(b, 2, 3) * MAT(b, 3, 1) - MAT(b, 3, 3) * MAT(b, 2, 1)) / vol;
    d[2] = (MAT(b, 2, 1) * MAT(b, 3, 2) - MAT(b, 3, 1) * MAT(b, 2, 2)) / vol;
    d[3] = (MAT(b, 3, 2) * MAT(b, 1, 3) - MAT(b, 1, 2) * MAT(b, 3, 3)) / vol;
    d[4] = (MAT(b, 1, 1) * MAT(b, 3, 3) - MAT(b, 1, 3) * MAT(b, 3, 1)) / vol;
    d[5] = (MAT(b, 3, 1) * MAT(b, 1, 2) - MAT(b, 1, 1) * MAT(b, 3, 2)) / vol;
    d[6] = (MAT(b, 1, 2) * MAT(b, 2, 3) - MAT(b, 2, 2) * MAT(b, 1, 3)) / vol;
    d[7] = (MAT(b, 1, 3) * MAT(b, 2, 1) - MAT(b, 1, 1) * MAT(b, 2, 3)) / vol;
    d[8] = (MAT(b, 1, 1) * MAT(b, 2, 2) - MAT(b, 1, 2) * MAT(b, 2, 1)) / vol;
#pragma unroll
    for (int k = 0; k < 9; ++k) { B.th_tgid[k] = tgid[k]; B.th_cof[k] = d[k]; }
}

__global__ void k_therm_prep(Params p, BoxState *__restrict__ box) {
    double b0[9], b1[9];
    for (int k = 0; k < 9; ++k) { b0[k] = box->b0[k]; b1[k] = box->b1[k]; }
    therm_prep(p, b0, b1, *box);
}

// update_therm_avs (src/dynamics_m.F90:649-734), one atom's terms: s1 += |F|^2,
// s2 += |F|^4, s3 += m |B0 x1|^2, with F = cof(B0)/vol (2 x2 + tgid x1); t, b, d
// are tgid, B0 and cof(B0)/vol in shared memory, read at every use (volatile)
// rather than held in 54 registers across the atom loop, which would halve the
// resident warps of the streaming kernels that call this.  The caller skips
// atoms without a species.
__device__ __forceinline__ void therm_terms(double (&v)[3], const volatile double *t, const volatile double *b,
                                            const volatile double *d,
                                            double ma, double ux, double uy, double uz, double wx, double wy,
                                            double wz) {
    double sxi = t[0] * ux + t[3] * uy + t[6] * uz;
    double syi = t[1] * ux + t[4] * uy + t[7] * uz;
    double szi = t[2] * ux + t[5] * uy + t[8] * uz;
    double fxp = 2.0 * wx + sxi, fyp = 2.0 * wy + syi, fzp = 2.0 * wz + szi;
    double fx = d[0] * fxp + d[1] * fyp + d[2] * fzp;
    double fy = d[3] * fxp + d[4] * fyp + d[5] * fzp;
    double fz = d[6] * fxp + d[7] * fyp + d[8] * fzp;
    double f2 = fx * fx + fy * fy + fz * fz;
    v[0] += f2;
    v[1] += f2 * f2;
    double rx = b[0] * ux + b[3] * uy + b[6] * uz;
    double ry = b[1] * ux + b[4] * uy + b[7] * uz;
    double rz = b[2] * ux + b[5] * uy + b[8] * uz;
    v[2] += ma * (rx * rx + ry * ry + rz * rz);
}

// The mdloop quantities (src/moldin.F90:760-790) from the three sums of
// update_therm_avs (s3 = s1, s2, s3), by one thread.  The box has not moved
// since the force evaluation that ended the step.
// rec (may be null): the step's thermo record, kThermoRec doubles in the order
// of moldy_thermo (ke, pe, te, h, th, vol, s1, s2, s3, temp, boxke)
__device__ void therm_store(const Params &p, BoxState &B, const double *s3, double *rec) {
    double b0[9], b1[9], tg[9], tgdot[9], tginv[9], tgid[9], vol;
#pragma unroll
    for (int k = 0; k < 9; ++k) { b0[k] = B.b0[k]; b1[k] = B.b1[k]; }
    if (!therm_box(p, b0, b1, tg, tgdot, tginv, tgid, vol)) B.status = MOLDY_ERR_SINGULAR_BOX;
#pragma unroll
    for (int k = 0; k < 9; ++k) { B.tg[k] = tg[k]; B.tgdot[k] = tgdot[k]; B.tginv[k] = tginv[k]; B.tgid[k] = tgid[k]; }
    B.vol = vol;
    B.s1 = s3[0]; B.s2 = s3[1]; B.s3 = s3[2];
    const double bk = 1.3806504e-23 / 1.602176487e-19;
    B.ke = s3[2] / (p.deltat * p.deltat) / 2.0;
    B.temp = B.ke / (1.5 * bk * (double)p.nm);
    double boxke = 0.0;
    for (int i = 1; i <= 3; ++i)
        for (int j = 1; j <= 3; ++j) boxke = boxke + (MAT(b1, i, j) * MAT(b1, i, j)) / p.bdel2;
    B.boxke = boxke;
    B.te = B.ke + B.pe;
    B.h = B.te + p.press * B.vol;
    B.th = B.h + boxke;
    if (rec) {
        rec[0] = B.ke; rec[1] = B.pe; rec[2] = B.te; rec[3] = B.h; rec[4] = B.th; rec[5] = B.vol;
        rec[6] = B.s1; rec[7] = B.s2; rec[8] = B.s3; rec[9] = B.temp; rec[10] = B.boxke;
    }
}

// Every block's three partial sums of update_therm_avs, in block order, and
// the quantities derived from them (one block)
__global__ void __launch_bounds__(256)
k_therm_finish(Params p, BoxState *__restrict__ box, const double *__restrict__ partials, int nblk,
               double *__restrict__ rec) {
    __shared__ double s3[3];
    reduce_partials<3>(partials, nblk, s3);
    if (threadIdx.x == 0) therm_store(p, *box, s3, rec);
}

// ------------------------------------------------ intermediate-list check --
// therm_nblk > 0: first finish the update_therm_avs that the drift kernel
// took for the step that has just ended (its block partials), before the box
// moves.
// The list-rebuild decisions and the box advance of k_mid_decide, by one
// thread on the block's shared copy of the box.
__device__ void mid_decide_box(const Params &p, BoxState &B, double rmid, double rcut, double rout, int force,
                               int half_build, int apply_box) {
    // register copies; the box is stored back once
    double b0[9], b1[9], b2[9], bb[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { b0[k] = B.b0[k]; b1[k] = B.b1[k]; b2[k] = B.b2[k]; bb[k] = B.bbuild[k]; }
    if (apply_box) {   // velocityverlet box half (src/quench_m.F90:582-589)
        if (p.ivol == 4) {
            MAT(b1, 3, 3) = MAT(b1, 3, 3) + MAT(b2, 3, 3);
            MAT(b0, 3, 3) = MAT(b0, 3, 3) + MAT(b1, 3, 3);
        }
        if (p.ivol < 1) {
#pragma unroll
            for (int k = 0; k < 9; ++k) b1[k] = b1[k] + b2[k];
#pragma unroll
            for (int k = 0; k < 9; ++k) b0[k] = b0[k] + b1[k];
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) { B.b0[k] = b0[k]; B.b1[k] = b1[k]; }
    }
    // displacements are measured in FP32 from fixed-point positions: the
    // factor and the offset cover their rounding
    double md = sqrt(__longlong_as_double((long long)B.maxdisp2)) * (1.0 + 1.0e-5) + 1.0e-6;
    B.maxdisp2 = 0ull;
    double eps = 2.0e-6 * frob(b0) + 1.0e-4;
    // dmax = rnear |B_build^-1|_F bounds the fractional separation of a listed
    // pair; it is stored with each build (0: none yet, or a singular box)
    double db[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) db[k] = b0[k] - bb[k];
    const double dmax = B.dmax_mid;
    double shrink = 2.0 * md + frob(db) * dmax;
    // A half-list rebuild this step (half_build) keeps the outer and
    // intermediate lists when the outer list needs no pair that its own
    // source half list lacked.  A pair missing from that source was farther
    // than rnear at the source's build; at the outer build it was farther
    // than rnear - eps - shrink_h (shrink_h: twice the largest displacement
    // between the two builds, measured by the outer build, plus the box
    // change times the source's dmax).  When that is beyond r_out + eps the
    // pair was left out of the outer list like any pair beyond r_out, and the
    // outer list's own rule below bounds its approach from then on.
    bool keep_lists = false;
    if (half_build) {
        double dbh[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) dbh[k] = B.bout[k] - B.bhalf_out[k];
        const double dh = sqrt(__longlong_as_double((long long)B.halfdisp2)) * (1.0 + 1.0e-5) + 1.0e-6;
        const double shrink_h = 2.0 * dh + frob(dbh) * B.dmax_half_out;
        keep_lists = B.dmax_half_out > 0.0 && B.dmax_out > 0.0 && B.dmax_mid > 0.0 &&
                     shrink_h < p.rnear - eps - (rout + eps);
        double hinv[9];
        const double dh_new = mat_invert(b0, hinv) ? p.rnear * frob(hinv) : 0.0;
#pragma unroll
        for (int k = 0; k < 9; ++k) B.bhalf[k] = b0[k];
        B.dmax_half = dh_new;
    }
    const int forced = force || (half_build && !keep_lists);
    int need = forced || !(dmax > 0.0) || !(shrink < rmid - eps - (rcut + eps));
    int need_out = 0;
    if (need) {
        // The intermediate list is filtered from the outer list, which must
        // then hold every pair within r_mid: a pair left out of it was farther
        // than r_out - eps at its build, and each atom has moved since then by
        // at most its displacement at the last intermediate build (outdisp2)
        // plus its displacement since (md).
        double dbo[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) dbo[k] = b0[k] - B.bout[k];
        const double dmaxo = B.dmax_out;
        const double dout = sqrt(__longlong_as_double((long long)B.outdisp2)) * (1.0 + 1.0e-5) + 1.0e-6 + md;
        const double shrink_out = 2.0 * dout + frob(dbo) * dmaxo;
        need_out = forced || !(dmaxo > 0.0) || !(shrink_out < rout - eps - (rmid + 2.0 * eps));
        double inv[9];
        const double dnew = mat_invert(b0, inv) ? p.rnear * frob(inv) : 0.0;
#pragma unroll
        for (int k = 0; k < 9; ++k) B.bbuild[k] = b0[k];
        B.dmax_mid = dnew;
        B.mid_builds += 1;
        B.outdisp2 = 0ull;   // measured again by the intermediate build
        if (need_out) {
            // the half list this outer list is filtered from, and the
            // displacement since that half list's build (measured by the build)
#pragma unroll
            for (int k = 0; k < 9; ++k) B.bhalf_out[k] = B.bhalf[k];
            B.dmax_half_out = B.dmax_half;
            B.halfdisp2 = 0ull;
#pragma unroll
            for (int k = 0; k < 9; ++k) B.bout[k] = b0[k];
            B.dmax_out = dnew;
            B.out_builds += 1;
        }
    }
    B.mid_rebuild = need;
    B.out_rebuild = need_out;
}

__global__ void __launch_bounds__(256)
k_mid_decide(Params p, BoxState *__restrict__ box, double rmid, double rcut, double rout, int force,
             int half_build, int apply_box, const double *__restrict__ therm_partials, int therm_nblk,
             double *__restrict__ rec, int rec_indexed) {
    grid_dep_wait();   // launched dependent on the step's previous kernel
    __shared__ BoxState sbox;
    box_load(sbox, box);
    __syncthreads();
    if (therm_nblk > 0) {
        __shared__ double s3[3];
        reduce_partials<3>(therm_partials, therm_nblk, s3);
        if (threadIdx.x == 0) {
            // rec_indexed: rec is the first record, and the box says which one
            // this step writes (a replayed step's launches are all alike)
            double *r = rec;
            if (rec_indexed) {
                if (r) r += (size_t)kThermoRec * (size_t)sbox.rec_step;
                sbox.rec_step += 1;
            }
            therm_store(p, sbox, s3, r);
        }
    }
    if (threadIdx.x == 0) mid_decide_box(p, sbox, rmid, rcut, rout, force, half_build, apply_box);
    __syncthreads();
    box_store(box, sbox);
}

void launch_mid_decide(DeviceState &d, const Params &p, double rmid, double rcut, double rout, int force,
                       int half_build, int apply_box, int therm_nblk, double *rec, cudaStream_t s,
                       int rec_indexed) {
    launch_pdl(k_mid_decide, 1, 256, s, p, d.box, rmid, rcut, rout, force, half_build, apply_box, d.partials,
                                   therm_nblk, rec, rec_indexed);
}

__global__ void k_set_rec_step(BoxState *__restrict__ box, int step) { box->rec_step = step; }

// the record index the next indexed k_mid_decide writes
void launch_set_rec_step(DeviceState &d, int step, cudaStream_t s) { k_set_rec_step<<<1, 1, 0, s>>>(d.box, step); }

// ------------------------------------------------------------- integrator --
// velocityverlet first half (src/quench_m.F90:574-589): x1_dt2 = x1 + x2;
// x0 += x1_dt2.  The box half (b1 += b2; b0 += b1 for ivol < 1, zz only for
// ivol 4) is applied by k_mid_decide, which runs next.
//
// THERM: the update_therm_avs of the previous step is taken here too.  x1 and
// x2 are read unchanged from the force evaluation that ended that step, the
// box has not yet moved, and the grid is k_therm's, so the sums are k_therm's
// to the last bit.  The block partials go to therm_partials; k_mid_decide,
// which runs next, finishes them.
template <bool THERM>
__global__ void __launch_bounds__(256, 4)   // the grid is 4 blocks per SM (stream_blocks): one wave
k_drift(Params p, double4 *__restrict__ pos, int4 *__restrict__ posq,
        const double *__restrict__ x1, const double *__restrict__ x2, BoxState *__restrict__ box,
        const int4 *__restrict__ xbuild, const double *__restrict__ mass, const int32_t *__restrict__ znum,
        double *__restrict__ kin_partials, double *__restrict__ therm_partials) {
    grid_dep_wait();   // launched dependent on the step's previous kernel
    // every thread forms the post-drift box exactly as thread 0 stores it
    __shared__ float nbs[9];   // that box per fixed-point unit
    __shared__ double sh[THERM ? 27 : 1];   // tgid, b0, cof(b0)/vol of the previous step
    if (THERM && threadIdx.x < 9) {
        sh[threadIdx.x] = box->th_tgid[threadIdx.x];
        sh[9 + threadIdx.x] = box->b0[threadIdx.x];
        sh[18 + threadIdx.x] = box->th_cof[threadIdx.x];
    }
    if (threadIdx.x == 0) {
        const BoxState &B = *box;
        double b1[9], b0[9];
        for (int k = 0; k < 9; ++k) { b1[k] = B.b1[k]; b0[k] = B.b0[k]; }
        if (p.ivol == 4) {
            MAT(b1, 3, 3) = MAT(b1, 3, 3) + MAT(B.b2, 3, 3);
            MAT(b0, 3, 3) = MAT(b0, 3, 3) + MAT(b1, 3, 3);
        }
        if (p.ivol < 1) {
            for (int k = 0; k < 9; ++k) b1[k] = b1[k] + B.b2[k];
            for (int k = 0; k < 9; ++k) b0[k] = b0[k] + b1[k];
        }
        for (int k = 0; k < 9; ++k) nbs[k] = (float)(b0[k] * kFixUnit);
    }
    __syncthreads();
    float d2 = 0.f;
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double vt[3] = {0.0, 0.0, 0.0};
    const int nm = p.nm;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += gridDim.x * blockDim.x) {
        const double ex = x1[a], ey = x1[nm + a], ez = x1[2 * nm + a];
        const double wx = x2[a], wy = x2[nm + a], wz = x2[2 * nm + a];
    double4 q = pos[a];
        q.x = q.x + (ex + wx);
        q.y = q.y + (ey + wy);
        q.z = q.z + (ez + wz);
        pos[a] = q;
        const int4 qn = make_int4(fix32(q.x), fix32(q.y), fix32(q.z), 0);
        posq[a] = qn;
        d2 = fmaxf(d2, fix_disp2(nbs, qn, xbuild[a]));
        // x1 is not changed by this half of the step: the kinetic moment of
        // the coming force evaluation can be taken here
        if (znum[a] != 0) {
            const double ma = mass[a];
            kin_moment(v, ma, ex, ey, ez);
            if (THERM) therm_terms(vt, sh, sh + 9, sh + 18, ma, ex, ey, ez, wx, wy, wz);
        }
    }
    block_partials<6>(v, kin_partials, 0);
    // block maximum, then one atomic per block (non-negative doubles order as their bits)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d2 = fmaxf(d2, __shfl_xor_sync(0xffffffffu, d2, o));
    __shared__ float wmax[8];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = d2;
    __syncthreads();
    if (threadIdx.x == 0) {
        float m = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, wmax[w]);
        atomicMax(&box->maxdisp2, (unsigned long long)__double_as_longlong((double)m));
    }
    // the sums are finished by k_mid_decide, which runs next
    if (THERM) block_partials<3>(vt, therm_partials, 0);
    // the box itself is advanced afterwards by k_mid_decide, so that no block
    // here can read a box another block has already moved
}

int launch_drift(DeviceState &d, const Params &p, double *kin_partials, bool therm, cudaStream_t s) {
    int nb = stream_blocks(p.nm);
    if (therm)
        launch_pdl(k_drift<true>, nb, kAtomThreads, s, p, d.pos, d.posq, d.x1, d.x2, d.box, d.xbuild, d.mass, d.znum,
                                                  kin_partials, d.partials);
    else
        launch_pdl(k_drift<false>, nb, kAtomThreads, s, p, d.pos, d.posq, d.x1, d.x2, d.box, d.xbuild, d.mass, d.znum,
                                                   kin_partials, nullptr);
    return nb;
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

// update_therm_avs over the atoms with a species, after a force evaluation
// (therm_prep has left tgid and cof(B0)/vol in the box state); block partials
// only, finished by k_therm_finish
__global__ void __launch_bounds__(256)
k_therm(Params p, BoxState *__restrict__ box, const double *__restrict__ x1,
        const double *__restrict__ x2, const double *__restrict__ mass,
        const int32_t *__restrict__ znum, double *__restrict__ partials) {
    __shared__ double sh[9 + 9 + 9];   // tgid, b0, cof(b0)/vol
    if (threadIdx.x < 9) {
        sh[threadIdx.x] = box->th_tgid[threadIdx.x];
        sh[9 + threadIdx.x] = box->b0[threadIdx.x];
        sh[18 + threadIdx.x] = box->th_cof[threadIdx.x];
    }
    __syncthreads();
    double v[3] = {0.0, 0.0, 0.0};
    const int nm = p.nm;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += gridDim.x * blockDim.x) {
        // every load issued before the species test, so none waits on it
        const int z = znum[a];
        const double ux = x1[a], uy = x1[nm + a], uz = x1[2 * nm + a];
        const double wx = x2[a], wy = x2[nm + a], wz = x2[2 * nm + a];
        const double ma = mass[a];
        if (z == 0) continue;
        therm_terms(v, sh, sh + 9, sh + 18, ma, ux, uy, uz, wx, wy, wz);
    }
    block_partials<3>(v, partials, 0);
}

// prep: compute the box quantities first (the call does not follow a force
// evaluation that left them)
int launch_therm(DeviceState &d, const Params &p, bool prep, double *rec, cudaStream_t s) {
    if (prep) k_therm_prep<<<1, 1, 0, s>>>(p, d.box);
    int nblocks = stream_blocks(p.nm);
    k_therm<<<nblocks, kAtomThreads, 0, s>>>(p, d.box, d.x1, d.x2, d.mass, d.znum, d.partials);
    k_therm_finish<<<1, kAtomThreads, 0, s>>>(p, d.box, d.partials, nblocks, rec);
    return nblocks;
}

// ----------------------------------------------------------------- scalev --
// scalev (src/thermostat_m.F90:317-395), the Nose-Hoover Euler thermostat:
// remove the mean of x1 (over all atoms) from the movable atoms, measure their
// kinetic energy, update snhv -= (ke - rqke) / (nose nm) and scale their x1
// by 1 + snhv.  Atoms with Z = 0 or mass < 0.1 are not movable.
__global__ void __launch_bounds__(256)
k_scalev_mean(int nm, const double *__restrict__ x1, double *__restrict__ partials) {
    double v[3] = {0.0, 0.0, 0.0};
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += gridDim.x * blockDim.x) {
        v[0] += x1[a]; v[1] += x1[nm + a]; v[2] += x1[2 * nm + a];
    }
    block_partials<3>(v, partials, 0);
}

__global__ void __launch_bounds__(256)
k_scalev_ke(Params p, const BoxState *__restrict__ box, const double *__restrict__ mean_part, int nblk,
            double *__restrict__ x1, const double *__restrict__ mass, const int32_t *__restrict__ znum,
            double *__restrict__ partials) {
    __shared__ double s[3];
    reduce_partials<3>(mean_part, nblk, s);
    const int nm = p.nm;
    const double fnm = (double)(float)nm;      // float(nm): default REAL
    const double sx = s[0] / fnm, sy = s[1] / fnm, sz = s[2] / fnm;
    const double *b = box->b0;
    double v[1] = {0.0};
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += gridDim.x * blockDim.x) {
        if (znum[a] == 0 || mass[a] < 0.1) continue;
        double ux = x1[a] - sx, uy = x1[nm + a] - sy, uz = x1[2 * nm + a] - sz;
        x1[a] = ux; x1[nm + a] = uy; x1[2 * nm + a] = uz;
        double rx = b[0] * ux + b[3] * uy + b[6] * uz;
        double ry = b[1] * ux + b[4] * uy + b[7] * uz;
        double rz = b[2] * ux + b[5] * uy + b[8] * uz;
        v[0] += mass[a] * (rx * rx + ry * ry + rz * rz);
    }
    block_partials<1>(v, partials, 0);
}

__global__ void __launch_bounds__(256)
k_scalev_finish(Params p, BoxState *__restrict__ box, const double *__restrict__ partials, int nblk, double nose,
                double rqke) {
    __shared__ double s[1];
    reduce_partials<1>(partials, nblk, s);
    if (threadIdx.x != 0) return;
    BoxState &B = *box;
    double ke = s[0] / (p.deltat * p.deltat) / 2.0;
    // snhf keeps its previous value when ke is not positive
    if (ke > 0.0) B.snhf = (ke - rqke) / (nose * (double)p.nm);
    B.snhv = B.snhv - B.snhf;
    B.scalev_ke = ke;
}

__global__ void __launch_bounds__(256)
k_scalev_scale(int nm, const BoxState *__restrict__ box, double *__restrict__ x1, const double *__restrict__ mass,
               const int32_t *__restrict__ znum) {
    const double f = 1.0 + box->snhv;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nm; a += gridDim.x * blockDim.x) {
        if (znum[a] == 0 || mass[a] < 0.1) continue;
        x1[a] = x1[a] * f; x1[nm + a] = x1[nm + a] * f; x1[2 * nm + a] = x1[2 * nm + a] * f;
    }
}

void launch_scalev(DeviceState &d, const Params &p, double nose, double rqke, cudaStream_t s) {
    const int nb = grid_blocks(p.nm, kAtomThreads);
    double *mean_part = d.partials, *ke_part = d.partials + (size_t)kMaxBlocks * kPartials;
    k_scalev_mean<<<nb, kAtomThreads, 0, s>>>(p.nm, d.x1, mean_part);
    k_scalev_ke<<<nb, kAtomThreads, 0, s>>>(p, d.box, mean_part, nb, d.x1, d.mass, d.znum, ke_part);
    k_scalev_finish<<<1, kAtomThreads, 0, s>>>(p, d.box, ke_part, nb, nose, rqke);
    k_scalev_scale<<<nb, kAtomThreads, 0, s>>>(p.nm, d.box, d.x1, d.mass, d.znum);
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
    double own = 0.0;
    for (int k = 0; k < n; ++k) {
        int j = nlist[(size_t)a * p.nnbrs + k];
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
