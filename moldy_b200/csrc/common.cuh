// common.cuh -- device-side types and helpers shared by the MOLDY kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace moldy {

// column-major 3x3 access with Fortran (1-based) indices, as B0(i,j)
#define MAT(a, i, j) ((a)[((i) - 1) + 3 * ((j) - 1)])

constexpr int kPartials = 32;   // doubles of per-block partial sums

// Box tensors and scalar results held on the device so that a step needs no
// host round trip (parrinellorahman_m module data, src/parrinellorahman_m.F90:102-115).
struct BoxState {
    double b0[9], b1[9], b2[9];
    double tgid[9];                // tg^-1 tgdot from the last update_therm_avs
    double tg[9], tgdot[9], tginv[9];
    double tk[9], tp[9], tc[9], fb[9];
    double vol, pe, pe_emb, pe_pair;
    double s1, s2, s3, ke, te, h, th, boxke, temp;
    double maxdisp;
    double npairs;                 // directed interacting pairs in the last density pass
    double bbuild[9];              // B0 when the intermediate list was built
    double snhv, snhf, scalev_ke;  // Nose-Hoover scaling state of scalev and its last KE
    double th_tgid[9], th_cof[9];  // tg^-1 tgdot and cof(B0)/vol of the box k_therm sees
    double bout[9];                // B0 when the outer list was built
    double dmax_mid, dmax_out;     // rnear |B_build^-1|_F of those builds (0: none)
    double bhalf[9], dmax_half;    // B0 and rnear |B0^-1|_F at the last half-list build
    double bhalf_out[9], dmax_half_out;   // the same of the half list the outer list was filtered from
    unsigned long long halfdisp2;  // max |B0 (x - x_half)|^2 at the last outer build (double bits)
    unsigned long long maxdisp2;   // max |B0 (x - x_build)|^2 of the last drift (double bits)
    unsigned long long outdisp2;   // max |B0 (x - x_out)|^2 at the last intermediate build (double bits)
    int32_t mid_rebuild;           // 1: the intermediate list is rebuilt this step
    int32_t mid_builds;            // number of intermediate-list builds so far
    int32_t status;                // nonzero: singular box in a device-side inversion
    int32_t out_rebuild;           // 1: the outer list is rebuilt this step
    int32_t out_builds;            // number of outer-list builds so far
    int32_t rec_step;              // thermo record the next indexed k_mid_decide writes
};

// Per-launch constant parameters.
struct Params {
    double rnear;
    double deltat, press, bdel2;
    int nm, nnbrs, ivol, atomstress;
    int nlcx, nlcy, nlcz, ncell;
    int pair_cap, mid_cap;   // entries per atom of the compact and the intermediate (full) rows
    int out_cap;             // entries per atom of the outer (full) rows
};

// Lookup-table description (lookup_m module data, src/lookup_m.F90:64-78).
struct Tables {
    const double4 *r4;      // per node (vee, dvee, phi, dphi), nodes 0..nr-1
    const double2 *e2;      // per node (emb, demb), nodes 0..nlookup
    const float4 *r4f;      // FP32 copy of r4 for the mixed path, node pairs: [2k] = node k, [2k+1] = node k+1
    const float2 *e2f;
    const double2 *phi2;    // per node k (phi_k, phi_k+1): one load per density lookup
    const float2 *phi2f;
    int nlookup;            // intervals
    int nr;                 // stored r nodes (culled tail removed)
    int idx_cut;            // first node from which all r tables are zero
    int exact;              // 1: evaluate *_src analytically, not from tables
    double vp_rmin, vp_rmax, vp_range, vp_reciprange, vp_recipnlkp, vp_recipstep;
    double e_rmin, e_rmax, e_range, e_reciprange, e_recipnlkp, e_recipstep;
    double rcull2;          // pairs with r^2 above this contribute exactly zero
    float rcull2f;
    float recipstep_f;      // (float) vp_recipstep: node coordinate of r in the FP32 lookups
    float xoff_f;           // (float) (-vp_rmin * vp_recipstep): node coordinate = r * recipstep_f + xoff_f
    float4 tail_f;          // FP32 (vee, dvee, phi, dphi) of the last stored node nr - 1: the
                            // value for r >= rmax (node nlookup) or beyond the culled tail (zero)
    // FETRANSMETAL Fe-Fe analytic data for exact mode / energy_calc
    int nv, np;
    double av[8], rv[8], ap[8], rp[8];
    double bier_cut1, bier_cut2, sc[4], phi_cut1, phi_cut2, bier_a, bier_zed;
};

#ifdef __CUDACC__
// ------------------------------------------------------------- geometry --
// Minimum image exactly as pr_get_realsep_from_dx (src/parrinellorahman_m.F90:149-173):
// NINT rounds half away from zero, which is CUDA's round().
__device__ __forceinline__ void min_image(int ivol, double &dx, double &dy, double &dz) {
    if (ivol == 0 || ivol == 1 || ivol == 4) {
        dx = __dsub_rn(dx, round(dx));
        dy = __dsub_rn(dy, round(dy));
        dz = __dsub_rn(dz, round(dz));
    } else if (ivol == 2) {
        dx = __dsub_rn(dx, round(dx));
        dy = __dsub_rn(dy, round(dy));
    } else if (ivol == 5) {
        dz = __dsub_rn(dz, round(dz));
    }
}

// Real separation with every product and sum rounded separately (no fused
// multiply-add), so that the comparison r < rnear is bit-identical to the
// reference's evaluation order.
__device__ __forceinline__ double realsep_exact(const double *b, double dx, double dy, double dz) {
    double rx = __dadd_rn(__dadd_rn(__dmul_rn(b[0], dx), __dmul_rn(b[3], dy)), __dmul_rn(b[6], dz));
    double ry = __dadd_rn(__dadd_rn(__dmul_rn(b[1], dx), __dmul_rn(b[4], dy)), __dmul_rn(b[7], dz));
    double rz = __dadd_rn(__dadd_rn(__dmul_rn(b[2], dx), __dmul_rn(b[5], dy)), __dmul_rn(b[8], dz));
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz)));
}

// link-cell coordinate of a fractional position (src/linkcell_m.F90:150-152)
__device__ __forceinline__ int cell_coord(double x, int nlc) {
    const double hmeps = 0.4999999999;
    return (int)__dmul_rn(__dadd_rn(__dsub_rn(x, round(x)), hmeps), (double)nlc);
}

// Read-only (non-coherent) 32-byte loads as one 256-bit request (sm_100).
// The address must be 32-byte aligned: every double4 array and the paired
// float4 table are cudaMalloc'd arrays of 32-byte elements.  The data must
// not be written while the kernel runs.
__device__ __forceinline__ double4 ldg4(const double4 *p) {
    double4 v;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w) : "l"(p));
    return v;
}

__device__ __forceinline__ void ldg8f(const float4 *p, float4 &a, float4 &b) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(p));
}

// ------------------------------------------------------- fixed point --
// Fractional coordinates in 32-bit fixed point: one box length is 2^32 units,
// so the difference of two coordinates taken in 32-bit integer arithmetic
// wraps to the minimum image of a periodic direction by itself (within half a
// box; the quantisation is 2^-33 box lengths).  Used by the mixed-precision
// pair passes of fully periodic boxes.
constexpr double kFixScale = 4294967296.0;               // 2^32
constexpr double kFixUnit = 1.0 / 4294967296.0;          // 2^-32

// round(x 2^32) mod 2^32 (ties to even) for |x| < 2^19: one fused multiply-add
// against the bias 1.5 * 2^52 leaves the integer in the low mantissa bits
__device__ __forceinline__ int32_t fix32(double x) {
    return __double2loint(fma(x, kFixScale, 6755399441055744.0));
}

// 1/sqrt(x) of a positive normal x (pair distances: never denormal), with
// no denormal handling
__device__ __forceinline__ float rsqrt_ftz(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// A 32-bit integer as a float, rounded once to nearest (ties to even): the
// conversion instruction, whose throughput the pair passes measured to be
// no limit (about 7 % faster than forming it on the FMA pipe)
__device__ __forceinline__ float fix_to_float(int32_t d) { return __int2float_rn(d); }

// |B0 (x - x_ref)|^2 from fixed-point coordinates (any box: displacements
// since a list build are far below half a box, so the 32-bit difference is
// the displacement itself); bs is B0 per fixed-point unit.  Off from the FP64
// value by less than 1e-6 A^2 for any displacement a list build allows.
__device__ __forceinline__ float fix_disp2(const float *bs, const int4 &q, const int4 &ref) {
    const float dx = fix_to_float((int32_t)((uint32_t)q.x - (uint32_t)ref.x));
    const float dy = fix_to_float((int32_t)((uint32_t)q.y - (uint32_t)ref.y));
    const float dz = fix_to_float((int32_t)((uint32_t)q.z - (uint32_t)ref.z));
    const float rx = fmaf(bs[6], dz, fmaf(bs[3], dy, bs[0] * dx));
    const float ry = fmaf(bs[7], dz, fmaf(bs[4], dy, bs[1] * dx));
    const float rz = fmaf(bs[8], dz, fmaf(bs[5], dy, bs[2] * dx));
    return fmaf(rz, rz, fmaf(ry, ry, rx * rx));
}

// floor(x) of 0 <= x < 2^23 as an integer and as a float, from one round-down
// addition (no conversion unit)
__device__ __forceinline__ int floor_small(float x, float &fl) {
    const float b = __fadd_rd(fminf(x, 8388607.0f), 8388608.0f);
    fl = b - 8388608.0f;
    return __float_as_int(b) - 0x4b000000;
}

// ---------------------------------------------------------- table lookup --
// get_value_from_lookup_veephi (src/lookup_m.F90:307-346) for the four r tables
// at once; returns (vee, dvee, phi, dphi).
__device__ __forceinline__ double4 lookup_r4(const Tables &t, double r) {
    if (r >= t.vp_rmax) {
        int n = t.nlookup < t.nr ? t.nlookup : t.nr - 1;
        return ldg4(&t.r4[n]);
    }
    int idx = (int)(((double)t.nlookup * (r - t.vp_rmin)) * t.vp_reciprange);
    if (idx >= t.nr - 1) return make_double4(0.0, 0.0, 0.0, 0.0);
    idx = idx < 0 ? 0 : idx;   // r below rmin (the reference reads out of bounds)
    double rlow = t.vp_rmin + (t.vp_range * (double)idx) * t.vp_recipnlkp;
    double dr = (r - rlow) * t.vp_recipstep;
    double4 a = ldg4(&t.r4[idx]);
    double4 b = ldg4(&t.r4[idx + 1]);
    double w = 1.0 - dr;
    return make_double4(a.x * w + b.x * dr, a.y * w + b.y * dr, a.z * w + b.z * dr, a.w * w + b.w * dr);
}

__device__ __forceinline__ double lookup_phi(const Tables &t, double r) {
    if (r >= t.vp_rmax) {
        int n = t.nlookup < t.nr ? t.nlookup : t.nr - 1;
        return __ldg(&t.r4[n].z);
    }
    int idx = (int)(((double)t.nlookup * (r - t.vp_rmin)) * t.vp_reciprange);
    if (idx >= t.nr - 1) return 0.0;
    idx = idx < 0 ? 0 : idx;
    double rlow = t.vp_rmin + (t.vp_range * (double)idx) * t.vp_recipnlkp;
    double dr = (r - rlow) * t.vp_recipstep;
    const double2 v = __ldg(&t.phi2[idx]);
    return v.x * (1.0 - dr) + v.y * dr;
}

// get_value_from_lookup_emb (src/lookup_m.F90:356-394) for (emb, demb)
__device__ __forceinline__ double2 lookup_e2(const Tables &t, double rho) {
    if (rho >= t.e_rmax) return __ldg(&t.e2[t.nlookup]);
    int idx = (int)(((double)t.nlookup * (rho - t.e_rmin)) * t.e_reciprange);
    idx = idx < 0 ? 0 : (idx > t.nlookup - 1 ? t.nlookup - 1 : idx);
    double rlow = t.e_rmin + (t.e_range * (double)idx) * t.e_recipnlkp;
    double dr = (rho - rlow) * t.e_recipstep;
    double2 a = __ldg(&t.e2[idx]);
    double2 b = __ldg(&t.e2[idx + 1]);
    double w = 1.0 - dr;
    return make_double2(a.x * w + b.x * dr, a.y * w + b.y * dr);
}

// FP32 lookups for the mixed path, in FP32 index arithmetic.  As
// get_value_from_lookup_veephi (src/lookup_m.F90:322-340): the node
// coordinate x = (r - rmin) n / range comes from one fused multiply-add and
// its interval from a floor on the FMA pipe; at and beyond the last stored
// node (r >= rmax: node nlookup; a culled table: its first all-zero node) the
// value is that node's.  Below rmin the first interval is extrapolated, as
// the FP64 lookups do (the reference reads out of bounds there).  A stored
// interval is its lower node and the FP32 difference to the upper one.
__device__ __forceinline__ float4 lookup_r4f(const Tables &t, float r) {
    const float x = fmaf(r, t.recipstep_f, t.xoff_f);
    float fl;
    const int idx = floor_small(fmaxf(x, 0.f), fl);
    if (idx >= t.nr - 1) return t.tail_f;
    const float dr = x - fl;
    float4 a, b;
    ldg8f(&t.r4f[2 * idx], a, b);
    return make_float4(fmaf(b.x, dr, a.x), fmaf(b.y, dr, a.y), fmaf(b.z, dr, a.z), fmaf(b.w, dr, a.w));
}

__device__ __forceinline__ float lookup_phif(const Tables &t, float r) {
    const float x = fmaf(r, t.recipstep_f, t.xoff_f);
    float fl;
    const int idx = floor_small(fmaxf(x, 0.f), fl);
    if (idx >= t.nr - 1) return t.tail_f.z;
    const float dr = x - fl;
    const float2 v = __ldg(&t.phi2f[idx]);
    return fmaf(v.y, dr, v.x);
}

// ------------------------------------------------ exact FETRANSMETAL Fe-Fe --
// src/fetransmetal.F90:100-159 (vee_src) and 167-219 (dvee_src), Fe-Fe branch;
// the Biersack screening length and prefactor come precomputed from the host.
__device__ __forceinline__ double fetm_biersack(const Tables &t, double r) {
    double x = r / t.bier_a;
    double p = (double)0.1818f * exp(-((double)3.2f * x));
    p = p + (double)0.5099f * exp(-((double)0.9423f * x));
    p = p + (double)0.2802f * exp(-((double)0.4029f * x));
    p = p + (double)0.02817f * exp(-((double)0.2016f * x));
    return t.bier_zed * p / r;
}

__device__ __forceinline__ double fetm_dbiersack(const Tables &t, double r) {
    double a = t.bier_a, x = r / a;
    double s = (1.0 / r + 3.2 / a) * 0.1818 * exp(-(3.2 * x));
    s = s + (1.0 / r + 0.9423 / a) * 0.5099 * exp(-(0.9423 * x));
    s = s + (1.0 / r + 0.4029 / a) * 0.2802 * exp(-(0.4029 * x));
    s = s + (1.0 / r + 0.2016 / a) * 0.02817 * exp(-(0.2016 * x));
    return -((t.bier_zed / r) * s);
}

__device__ __forceinline__ void hermite_log_join(const Tables &t, double r, double &sp, double &ds) {
    double a1 = t.bier_cut1, a2 = t.bier_cut2;
    double vv1 = t.sc[1] / t.sc[0], xx1 = log(t.sc[0]);
    double vv2 = t.sc[3] / t.sc[2], xx2 = log(t.sc[2]);
    double h = a2 - a1;
    double u = (r - a1) / h;
    double h00 = ((2.0 * u) * u) * u - (3.0 * u) * u + 1.0;
    double h10 = (u * u) * u - (2.0 * u) * u + u;
    double h01 = -(((2.0 * u) * u) * u) + (3.0 * u) * u;
    double h11 = (u * u) * u - u * u;
    sp = h00 * xx1 + h10 * vv1 * h + h01 * xx2 + h11 * vv2 * h;
    double d00 = (6.0 * u) * u - 6.0 * u;
    double d10 = (3.0 * u) * u - 4.0 * u + 1.0;
    double d01 = -((6.0 * u) * u) + 6.0 * u;
    double d11 = (3.0 * u) * u - 2.0 * u;
    ds = (d00 * xx1 + d10 * vv1 * h + d01 * xx2 + d11 * vv2 * h) / h;
}

__device__ __forceinline__ double fetm_vee(const Tables &t, double r) {
    if (r > t.bier_cut2) {
        double s = 0.0;
        for (int i = 0; i < t.nv; ++i) {
            double d = t.rv[i] - r;
            if (d >= 0.0) s += t.av[i] * ((d * d) * d);
        }
        return s;
    } else if (r > t.bier_cut1) {
        double sp, ds;
        hermite_log_join(t, r, sp, ds);
        return exp(sp);
    } else if (r < t.bier_cut1) {
        return fetm_biersack(t, r);
    }
    return 0.0;
}

__device__ __forceinline__ double fetm_dvee(const Tables &t, double r) {
    if (r > t.bier_cut2) {
        double s = 0.0;
        for (int i = 0; i < t.nv; ++i) {
            double d = t.rv[i] - r;
            if (d >= 0.0) s -= 3.0 * t.av[i] * (d * d);
        }
        return s;
    } else if (r > t.bier_cut1) {
        double sp, ds;
        hermite_log_join(t, r, sp, ds);
        return ds * exp(sp);
    } else if (r < t.bier_cut1) {
        return fetm_dbiersack(t, r);
    }
    return 0.0;
}

// src/fetransmetal.F90:227-366: phi flat below its maximum
__device__ __forceinline__ double fetm_phi(const Tables &t, double r) {
    if (r < t.phi_cut1) return t.phi_cut2;
    double s = 0.0;
    for (int i = 0; i < t.np; ++i) {
        double d = t.rp[i] - r;
        if (d >= 0.0) s += t.ap[i] * ((d * d) * d);
    }
    return s;
}

__device__ __forceinline__ double fetm_dphi(const Tables &t, double r) {
    if (r < t.phi_cut1) return 0.0;
    double s = 0.0;
    for (int i = 0; i < t.np; ++i) {
        double d = t.rp[i] - r;
        if (d >= 0.0) s -= 3.0 * t.ap[i] * (d * d);
    }
    return s;
}

// (vee, dvee, phi, dphi) at r through the table or the exact functions
__device__ __forceinline__ double4 pair_funcs(const Tables &t, double r) {
    if (t.exact) return make_double4(fetm_vee(t, r), fetm_dvee(t, r), fetm_phi(t, r), fetm_dphi(t, r));
    return lookup_r4(t, r);
}

__device__ __forceinline__ double density_func(const Tables &t, double r) {
    if (t.exact) return fetm_phi(t, r);
    return lookup_phi(t, r);
}

// (F(rho), F'(rho)): src/fetransmetal.F90:375-404 or the emb tables
__device__ __forceinline__ double2 embed_funcs(const Tables &t, double rho) {
    if (t.exact) {
        double f = -(1.0 * sqrt(rho > 0.0 ? rho : 0.0));
        double d = rho > 0.0 ? -(0.5 / sqrt(rho)) : 0.0;
        return make_double2(f, d);
    }
    return lookup_e2(t, rho);
}

// ----------------------------------------------------------- box algebra --
__device__ __forceinline__ void mat_cofactor(const double *b, double *tc) {
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

__device__ __forceinline__ double mat_volume(const double *b) {
    // pr_get_metric_tensor (src/parrinellorahman_m.F90:223-227)
    return MAT(b, 1, 1) * (MAT(b, 2, 2) * MAT(b, 3, 3) - MAT(b, 2, 3) * MAT(b, 3, 2)) +
           MAT(b, 2, 1) * (MAT(b, 3, 2) * MAT(b, 1, 3) - MAT(b, 1, 2) * MAT(b, 3, 3)) +
           MAT(b, 3, 1) * (MAT(b, 1, 2) * MAT(b, 2, 3) - MAT(b, 2, 2) * MAT(b, 1, 3));
}

// matrix_invert (src/matrix_m.F90:89-119); returns false for det == 0
__device__ __forceinline__ bool mat_invert(const double *a, double *bo) {
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
__device__ __forceinline__ void mat_mul(const double *a, const double *b, double *c) {
    for (int i = 1; i <= 3; ++i) {
        for (int j = 1; j <= 3; ++j) MAT(c, i, j) = 0.0;
        for (int k = 1; k <= 3; ++k)
            for (int j = 1; j <= 3; ++j) MAT(c, i, j) = MAT(c, i, j) + MAT(a, i, k) * MAT(b, k, j);
    }
}

// Frobenius norm of a 3x3 matrix
__device__ __forceinline__ double frob(const double *m) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) s += m[k] * m[k];
    return sqrt(s);
}

// ------------------------------------------------------------ reductions --
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of NV values per thread into partials[blockIdx.x*kPartials + off + k].
// Deterministic: fixed shuffle tree, then warps in order.
// Programmatic dependent launch: a step kernel launched with programmatic
// stream serialization (launch_pdl) may be scheduled while the kernel before
// it drains; it waits here, before it reads or writes anything, until that
// kernel has completed and its memory is visible.  A no-op for a kernel
// launched without the attribute.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// The box state of a one-block kernel in shared memory: every thread loads
// a share of it at once (one round of global loads instead of thread 0's
// chain of dependent ones), thread 0 works on the copy, every thread stores
// a share back.  Only one-block kernels that own the box for their whole
// run use these.
__device__ __forceinline__ void box_load(BoxState &s, const BoxState *__restrict__ g) {
    static_assert(sizeof(BoxState) % 8 == 0, "BoxState is copied in 8-byte words");
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(g);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(&s);
    for (int i = threadIdx.x; i < (int)(sizeof(BoxState) / 8); i += blockDim.x) dst[i] = src[i];
}

__device__ __forceinline__ void box_store(BoxState *__restrict__ g, const BoxState &s) {
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(&s);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(g);
    for (int i = threadIdx.x; i < (int)(sizeof(BoxState) / 8); i += blockDim.x) dst[i] = src[i];
}

template <int NV>
__device__ __forceinline__ void block_partials(double (&v)[NV], double *partials, int off) {
    __shared__ double sm[32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double s = warp_sum(v[k]);
        if (lane == 0) sm[warp][k] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = lane < nw ? sm[lane][k] : 0.0;
            s = warp_sum(s);
            if (lane == 0) partials[(size_t)blockIdx.x * kPartials + off + k] = s;
        }
    }
    __syncthreads();
}

// Sums NV partial columns over nblk blocks in a fixed order into out[NV];
// CG reads them through L2 (partials other blocks of the same launch wrote).
template <int NV, bool CG = false>
__device__ __forceinline__ void reduce_partials(const double *__restrict__ part, int nblk, double *out) {
    __shared__ double sm[32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (int bidx = threadIdx.x; bidx < nblk; bidx += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] += CG ? __ldcg(&part[(size_t)bidx * kPartials + k]) : part[(size_t)bidx * kPartials + k];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const double w = warp_sum(acc[k]);
        if (lane == 0) sm[warp][k] = w;
    }
    __syncthreads();
    if (warp == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const double w = warp_sum(lane < nw ? sm[lane][k] : 0.0);
            if (lane == 0) out[k] = w;
        }
    __syncthreads();
}

#endif  // __CUDACC__

}  // namespace moldy
