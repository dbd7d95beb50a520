// adjoint.cu -- gradients of the energy, the real forces and the stress with
// respect to the six lookup tables (vee, dvee, phi, dphi, emb, demb).  There
// is no counterpart in the reference.  The quantities differentiated are the
// ones write_energy_forces_stress prints (src/dynamics_m.F90:588-619): pe, the
// real forces B0 f and sigma(i,j) = -sum_k b0(j,k) tp(i,k) / vol, as force()
// (src/dynamics_m.F90:135-401) computes them with the lookup_m interpolation
// (src/lookup_m.F90:307-394).
//
// Forward, per unordered pair (i,j) of the half list, u = B0 d, r = |u|:
//   rho_i = sum_j P(r_ij),  Fp_i = De(rho_i),  E = sum_i Em(rho_i) + sum_ij V(r_ij)
//   fp_ij = -(DV(r) + DP(r) (Fp_i + Fp_j)) / r
//   F_i = sum_j u_ij fp_ij,  F_j -= u_ij fp_ij,  sigma = -(1/vol) sum_ij u u^T fp_ij [m_i+m_j > 0.1]
// with V, DV, P, DP, Em, De linear interpolations in the tables.  Given
// gE = dL/dE, gF_i = dL/dF_i and gS = dL/dsigma:
//   lam_ij = (gF_i - gF_j) . u_ij - (1/vol) u^T gS u [mass filter]   (= dL/dfp_ij)
//   dL/dDV(r_ij) = -lam/r,  dL/dDP(r_ij) = -lam (Fp_i + Fp_j)/r
//   mu_i  = dL/dFp_i = sum_j -lam_ij DP(r_ij)/r_ij
//   nu_i  = dL/drho_i = mu_i De'(rho_i) + gE Em'(rho_i)     (slopes of the interpolants)
//   dL/dP(r_ij) = nu_i + nu_j,  dL/dV(r_ij) = gE,  dL/dEm(rho_i) = gE,  dL/dDe(rho_i) = mu_i
// and each table node receives its interpolation weight times these.  Every
// listed pair is used, not only those inside the current table cut, so a node
// beyond the cut gets the gradient that a perturbation of it would see.  rho
// is recomputed from the positions in FP64; no per-pair state is stored.
// The three table scatters go through per-block shared-memory histograms.
#include "engine.h"

namespace moldy {
namespace {

// index and weights of the lookup_m interpolation (src/lookup_m.F90:322-341);
// x >= xmax takes node n alone
__device__ __forceinline__ void interp_w(double x, double xmin, double xmax, double range,
                                         double recipr, double recipn, double recips, int n,
                                         int &k, double &w0, double &w1) {
    if (x >= xmax) { k = n; w0 = 1.0; w1 = 0.0; return; }
    int idx = (int)(((double)n * (x - xmin)) * recipr);
    idx = idx < 0 ? 0 : (idx > n - 1 ? n - 1 : idx);
    double xlow = xmin + (range * (double)idx) * recipn;
    double d = (x - xlow) * recips;
    k = idx; w0 = 1.0 - d; w1 = d;
}

__device__ __forceinline__ void r_weights(const AdjointArgs &a, double r, int &k, double &w0, double &w1) {
    interp_w(r, a.rmin, a.rmax, a.rmax - a.rmin, a.r_reciprange, a.recipn, a.r_recipstep, a.n, k, w0, w1);
}
__device__ __forceinline__ void e_weights(const AdjointArgs &a, double rho, int &k, double &w0, double &w1) {
    interp_w(rho, a.emin, a.emax, a.emax - a.emin, a.e_reciprange, a.recipn, a.e_recipstep, a.n, k, w0, w1);
}

__device__ __forceinline__ double tval(const double *t, int k, double w0, double w1, int n) {
    return k >= n ? t[n] : t[k] * w0 + t[k + 1] * w1;
}

struct Box {
    double b[9], inv_vol;
};

__device__ __forceinline__ Box load_box(const BoxState *bs) {
    Box x;
    for (int k = 0; k < 9; ++k) x.b[k] = bs->b0[k];
    x.inv_vol = 1.0 / mat_volume(x.b);
    return x;
}

__device__ __forceinline__ void pair_geom(int ivol, const Box &bx, const double4 &pi, const double4 &pj,
                                          double &ux, double &uy, double &uz, double &r) {
    double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    min_image(ivol, dx, dy, dz);
    const double *b = bx.b;
    ux = b[0] * dx + b[3] * dy + b[6] * dz;
    uy = b[1] * dx + b[4] * dy + b[7] * dz;
    uz = b[2] * dx + b[5] * dy + b[8] * dz;
    r = sqrt(ux * ux + uy * uy + uz * uz);
}

// shared-memory histogram add over bins [0, n]
__device__ __forceinline__ void hist_add(double *h, int k, int n, double c, double w0, double w1) {
    if (k >= n) { atomicAdd(&h[n], c); return; }
    atomicAdd(&h[k], c * w0);
    atomicAdd(&h[k + 1], c * w1);
}

__device__ __forceinline__ void hist_clear(double *h, int nbins) {
    for (int k = threadIdx.x; k < nbins; k += blockDim.x) h[k] = 0.0;
    __syncthreads();
}

__device__ __forceinline__ void hist_flush(const double *h, double *g, int nbins) {
    __syncthreads();
    for (int k = threadIdx.x; k < nbins; k += blockDim.x) {
        double v = h[k];
        if (v != 0.0) atomicAdd(&g[k], v);
    }
}

// rho_i over the half list, both ends, as rhoset accumulates it
// (src/dynamics_m.F90:497-586), from the full phi table
__global__ void __launch_bounds__(256)
k_adj_density(AdjointArgs a, const double4 *__restrict__ pos, const int32_t *__restrict__ nlist,
              const int32_t *__restrict__ numn, const BoxState *__restrict__ bs,
              double *__restrict__ rho) {
    const Box bx = load_box(bs);
    const int nm = a.nm;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += gridDim.x * blockDim.x) {
        const double4 pi = pos[i];
        const int n = numn[i];
        double s = 0.0;
        for (int k = 0; k < n; ++k) {
            const int j = nlist[(size_t)i * a.nnbrs + k];
            double ux, uy, uz, r;
            pair_geom(a.ivol, bx, pi, pos[j], ux, uy, uz, r);
            int q; double w0, w1;
            r_weights(a, r, q, w0, w1);
            double ph = tval(a.phi, q, w0, w1, a.n);
            s += ph;
            atomicAdd(&rho[j], ph);
        }
        atomicAdd(&rho[i], s);
    }
}

// F'(rho_i); an atom with rho <= 1e-40 keeps the value the forward used
// (embed leaves such atoms untouched, src/potential_m.F90:148-169)
__global__ void k_adj_embed(AdjointArgs a, const double *__restrict__ rho,
                            const double *__restrict__ dafrho, double *__restrict__ fpr) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nm) return;
    double r = rho[i];
    double v = dafrho[i];
    if (r > 1e-40) {
        int q; double w0, w1;
        e_weights(a, r, q, w0, w1);
        v = tval(a.demb, q, w0, w1, a.n);
    }
    fpr[i] = v;
}

// lam_ij per pair; mu_i at both ends; dL/d dvee and dL/d dphi
__global__ void __launch_bounds__(256)
k_adj_pairs_a(AdjointArgs a, const double4 *__restrict__ pos, const int32_t *__restrict__ nlist,
              const int32_t *__restrict__ numn, const double *__restrict__ mass,
              const BoxState *__restrict__ bs, const double *__restrict__ fpr,
              const double *__restrict__ gF, double *__restrict__ mu, double *__restrict__ g_dvee,
              double *__restrict__ g_dphi) {
    extern __shared__ double sh[];
    const int nb = a.n + 1;
    double *hdv = sh, *hdp = sh + nb;
    hist_clear(sh, 2 * nb);
    const Box bx = load_box(bs);
    const double *g = a.gs;
    const int nm = a.nm;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += gridDim.x * blockDim.x) {
        const double4 pi = pos[i];
        const double gxi = gF[i], gyi = gF[nm + i], gzi = gF[2 * nm + i];
        const double fi = fpr[i], mi = mass[i];
        const int n = numn[i];
        double mui = 0.0;
        for (int k = 0; k < n; ++k) {
            const int j = nlist[(size_t)i * a.nnbrs + k];
            double ux, uy, uz, r;
            pair_geom(a.ivol, bx, pi, pos[j], ux, uy, uz, r);
            int q; double w0, w1;
            r_weights(a, r, q, w0, w1);
            double dp = tval(a.dphi, q, w0, w1, a.n);
            double lam = (gxi - gF[j]) * ux + (gyi - gF[nm + j]) * uy + (gzi - gF[2 * nm + j]) * uz;
            if (mi + mass[j] > 0.1) {
                double sgu = ux * (g[0] * ux + g[3] * uy + g[6] * uz) +
                             uy * (g[1] * ux + g[4] * uy + g[7] * uz) +
                             uz * (g[2] * ux + g[5] * uy + g[8] * uz);
                lam -= bx.inv_vol * sgu;
            }
            double rr = 1.0 / r;
            double m = -lam * dp * rr;
            mui += m;
            atomicAdd(&mu[j], m);
            hist_add(hdv, q, a.n, -lam * rr, w0, w1);
            hist_add(hdp, q, a.n, -lam * (fi + fpr[j]) * rr, w0, w1);
        }
        atomicAdd(&mu[i], mui);
    }
    hist_flush(hdv, g_dvee, nb);
    hist_flush(hdp, g_dphi, nb);
}

// nu_i, dL/d emb and dL/d demb per atom
__global__ void __launch_bounds__(256)
k_adj_atoms(AdjointArgs a, const double *__restrict__ rho, const double *__restrict__ mu,
            double *__restrict__ nu, double *__restrict__ g_emb, double *__restrict__ g_demb) {
    extern __shared__ double sh[];
    const int nb = a.n + 1;
    double *he = sh, *hd = sh + nb;
    hist_clear(sh, 2 * nb);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nm; i += gridDim.x * blockDim.x) {
        double r = rho[i];
        double v = 0.0;
        if (r > 1e-40) {
            int q; double w0, w1;
            e_weights(a, r, q, w0, w1);
            // slopes of the interpolants; zero at and beyond rhomax
            double sde = q >= a.n ? 0.0 : (a.demb[q + 1] - a.demb[q]) * a.e_recipstep;
            double sem = q >= a.n ? 0.0 : (a.emb[q + 1] - a.emb[q]) * a.e_recipstep;
            v = mu[i] * sde + a.gE * sem;
            hist_add(he, q, a.n, a.gE, w0, w1);
            hist_add(hd, q, a.n, mu[i], w0, w1);
        }
        nu[i] = v;
    }
    hist_flush(he, g_emb, nb);
    hist_flush(hd, g_demb, nb);
}

// dL/d phi = nu_i + nu_j and dL/d vee = gE per pair
__global__ void __launch_bounds__(256)
k_adj_pairs_c(AdjointArgs a, const double4 *__restrict__ pos, const int32_t *__restrict__ nlist,
              const int32_t *__restrict__ numn, const BoxState *__restrict__ bs,
              const double *__restrict__ nu, double *__restrict__ g_vee, double *__restrict__ g_phi) {
    extern __shared__ double sh[];
    const int nb = a.n + 1;
    double *hv = sh, *hp = sh + nb;
    hist_clear(sh, 2 * nb);
    const Box bx = load_box(bs);
    const int nm = a.nm;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += gridDim.x * blockDim.x) {
        const double4 pi = pos[i];
        const double nui = nu[i];
        const int n = numn[i];
        for (int k = 0; k < n; ++k) {
            const int j = nlist[(size_t)i * a.nnbrs + k];
            double ux, uy, uz, r;
            pair_geom(a.ivol, bx, pi, pos[j], ux, uy, uz, r);
            int q; double w0, w1;
            r_weights(a, r, q, w0, w1);
            hist_add(hp, q, a.n, nui + nu[j], w0, w1);
            hist_add(hv, q, a.n, a.gE, w0, w1);
        }
    }
    hist_flush(hv, g_vee, nb);
    hist_flush(hp, g_phi, nb);
}

}  // namespace

size_t adjoint_smem_bytes(int nlookup) { return 2 * ((size_t)nlookup + 1) * sizeof(double); }

// Queues the backward pass.  grads receives 6*(n+1) table gradients in the
// order vee, dvee, phi, dphi, emb, demb (zeroed here); scr holds rho, F', mu,
// nu (nm each); gF (3*nm, device, x|y|z) is dL/dF of the real forces.
void launch_table_adjoint(const DeviceState &d, const AdjointArgs &a, double *grads, double *scr,
                          const double *gF, cudaStream_t s) {
    const int nb = a.n + 1, nm = a.nm;
    double *rho = scr, *fpr = scr + nm, *mu = scr + 2 * (size_t)nm, *nu = scr + 3 * (size_t)nm;
    const size_t smem = adjoint_smem_bytes(a.n);
    cudaMemsetAsync(grads, 0, 6 * (size_t)nb * sizeof(double), s);
    cudaMemsetAsync(rho, 0, (size_t)nm * sizeof(double), s);
    cudaMemsetAsync(mu, 0, (size_t)nm * sizeof(double), s);
    cudaFuncSetAttribute(k_adj_pairs_a, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_adj_atoms, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_adj_pairs_c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int g = grid_blocks(nm, kAtomThreads);
    // histogram kernels: at most two blocks per SM, so each flush serves many atoms
    const int gh = g < 2 * 148 ? g : 2 * 148;
    k_adj_density<<<g, kAtomThreads, 0, s>>>(a, d.pos, d.nlist, d.numn, d.box, rho);
    k_adj_embed<<<(nm + kAtomThreads - 1) / kAtomThreads, kAtomThreads, 0, s>>>(a, rho, d.dafrho, fpr);
    k_adj_pairs_a<<<gh, kAtomThreads, smem, s>>>(a, d.pos, d.nlist, d.numn, d.mass, d.box, fpr, gF, mu,
                                                 grads + 1 * nb, grads + 3 * nb);
    k_adj_atoms<<<gh, kAtomThreads, smem, s>>>(a, rho, mu, nu, grads + 4 * nb, grads + 5 * nb);
    k_adj_pairs_c<<<gh, kAtomThreads, smem, s>>>(a, d.pos, d.nlist, d.numn, d.box, nu, grads + 0 * nb,
                                                 grads + 2 * nb);
}

}  // namespace moldy
