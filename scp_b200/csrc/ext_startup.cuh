// ext_startup.cuh -- start-up and diagnostic kernels of the extension
// steppers (higgs_u1.cuh, fabrics.cuh): the Higgs start value and energy, the
// second Gauss law and its projection, the fabrics' EM charge density, Gauss
// residual, charges and the view of fabric L for the energy reductions.
// Host translation unit scp_gpu.cu only (the ring kernels live in kern_ext.cu).
#pragma once
#include "fabrics.cuh"
#include "gauss.cuh"
#include "higgs_u1.cuh"
#include "real6.cuh"
#include "reduce.cuh"

namespace scp {

// ---- Higgs condensate and second gauge
// Higgs start value (the reference's main, scp_sim.c:2802-2817): the vacuum
// value v, or with a cavity of radius rvoid, v (1 + tanh((r - rvoid)/0.6)) / 2
__global__ void hu_higgs_start_kernel(double *H, double *Hdot, HuConsts c, double rvoid) {
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < c.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        double h = c.hv;
        if (rvoid > 0.0) {
            int i, j, k;
            site_ijk(idx, c.N, &i, &j, &k);
            const double x = -c.L + i * c.dx, y = -c.L + j * c.dx, z = -c.L + k * c.dx;
            h = c.hv * 0.5 * (1.0 + tanh((sqrt(x * x + y * y + z * z) - rvoid) / 0.6));
        }
        H[idx] = h;
        Hdot[idx] = 0.0;
    }
}

// Higgs energy sum_x [Hdot^2/2 + |grad H|^2/2 + V_H] dV with central
// differences (the reference adds it to E_total, scp_sim.c:1970-1975, :2034)
__global__ void __launch_bounds__(kRedThreads) hu_higgs_energy_kernel(const double *X, const double *H,
                                                                      const double *Hdot, HuConsts c, double *part) {
    __shared__ double scratch[32];
    double S[1] = {0.0}, M[1] = {0.0};
    const int N = c.N;
    const long long NN = (long long)N * N, N3 = c.N3;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        site_ijk(idx, N, &i, &j, &k);
        double s = 1.0;
        for (int a = 0; a < 3; a++) {
            const double u = X[(FU + a) * N3 + idx], w = X[(FV + a) * N3 + idx];
            s *= u * u + w * w;
        }
        const long long row = (long long)i * NN + (long long)j * N;
        const double gx = (H[(long long)wrapi(i + 1, N) * NN + (long long)j * N + k] -
                           H[(long long)wrapi(i - 1, N) * NN + (long long)j * N + k]) * c.idx1;
        const double gy = (H[(long long)i * NN + (long long)wrapi(j + 1, N) * N + k] -
                           H[(long long)i * NN + (long long)wrapi(j - 1, N) * N + k]) * c.idx1;
        const double gz = (H[row + wrapi(k + 1, N)] - H[row + wrapi(k - 1, N)]) * c.idx1;
        const double h = H[idx], hd = Hdot[idx];
        const double dv = h * h - c.hv * c.hv;
        S[0] += (0.5 * hd * hd + 0.5 * (gx * gx + gy * gy + gz * gz) + 0.25 * c.hlam * dv * dv +
                 0.5 * c.hkap * s * h * h) * c.dV;
    }
    block_fold<1, 0>(S, M, scratch, part);
}

// residual of the second Gauss law, div E2 - g2 sum_a q_a rho_a (rho_a the
// Noether density of component a), and its partial sums (init_gauss2_project's
// right-hand side, scp_sim.c:2387-2396)
__global__ void __launch_bounds__(kRedThreads) hu_gauss2_rhs_kernel(const double *X, const double *P,
                                                                    const double *E2, HuConsts c, double *b,
                                                                    double *part) {
    __shared__ double scratch[32];
    double S[1] = {0.0}, M[1] = {0.0};
    const int N = c.N;
    const long long NN = (long long)N * N, N3 = c.N3;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        site_ijk(idx, N, &i, &j, &k);
        const double div = (E2[idx] - E2[(long long)wrapi(i - 1, N) * NN + (long long)j * N + k] +
                            E2[N3 + idx] - E2[N3 + (long long)i * NN + (long long)wrapi(j - 1, N) * N + k] +
                            E2[2 * N3 + idx] - E2[2 * N3 + (long long)i * NN + (long long)j * N + wrapi(k - 1, N)]) /
                           c.dx;
        double q = 0.0;
        for (int a = 0; a < 3; a++) {
            const double ra = X[(FU + a) * N3 + idx] * P[(FV + a) * N3 + idx] -
                              X[(FV + a) * N3 + idx] * P[(FU + a) * N3 + idx] +
                              X[(FTU + a) * N3 + idx] * P[(FTV + a) * N3 + idx] -
                              X[(FTV + a) * N3 + idx] * P[(FTU + a) * N3 + idx];
            q += c.q[a] * ra;
        }
        const double G = div - c.g2 * q;
        b[idx] = G;
        S[0] += G;
    }
    block_fold<1, 0>(S, M, scratch, part);
}

// E2_d += (chi(x + d) - chi(x)) / dx with chi = x - xbar (the CG's result)
__global__ void hu_gauss2_apply_kernel(double *E2, const double *chi, const double *cg, HuConsts c) {
    const int N = c.N;
    const long long NN = (long long)N * N, N3 = c.N3;
    const double xbar = cg[CG_XBAR];
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        site_ijk(idx, N, &i, &j, &k);
        const double c0 = chi[idx] - xbar;
        const long long up[3] = {(long long)wrapi(i + 1, N) * NN + (long long)j * N + k,
                                 (long long)i * NN + (long long)wrapi(j + 1, N) * N + k,
                                 (long long)i * NN + (long long)j * N + wrapi(k + 1, N)};
        for (int d = 0; d < 3; d++) E2[d * N3 + idx] += ((chi[up[d]] - xbar) - c0) / c.dx;
    }
}

// ---- three fabrics
// The three fabrics at one time: positions and momenta of C (15 arrays with
// the links and E), Q and L (12 each; Q is C when locked).
struct FabView {
    const double *XC, *PC, *XQ, *PQ, *XL, *PL;
    long long N3;
    double q[3];              // EM weights q_C, q_Q, q_L
};

// Noether density of one fabric at a site: sum_a Im[Phi_a^* dPhi_a] + Im[Theta_a^* dTheta_a]
__device__ __forceinline__ double fabric_rho(const double *X, const double *P, long long N3, long long idx) {
    double r = 0.0;
    for (int a = 0; a < 3; a++)
        r += X[(FU + a) * N3 + idx] * P[(FV + a) * N3 + idx] - X[(FV + a) * N3 + idx] * P[(FU + a) * N3 + idx] +
             X[(FTU + a) * N3 + idx] * P[(FTV + a) * N3 + idx] - X[(FTV + a) * N3 + idx] * P[(FTU + a) * N3 + idx];
    return r;
}

__device__ __forceinline__ double fabric_rho_em(const FabView &f, long long idx) {
    return f.q[0] * fabric_rho(f.XC, f.PC, f.N3, idx) + f.q[1] * fabric_rho(f.XQ, f.PQ, f.N3, idx) +
           f.q[2] * fabric_rho(f.XL, f.PL, f.N3, idx);
}

// Gauss residual div E - g rho_em at a site
__device__ __forceinline__ double fabric_gauss(const FabView &f, int N, double dx, double g, long long idx) {
    const long long NN = (long long)N * N, N3 = f.N3;
    int i, j, k;
    site_ijk(idx, N, &i, &j, &k);
    const double *E = f.PC + FTH * N3;
    const double div = (E[idx] - E[(long long)wrapi(i - 1, N) * NN + (long long)j * N + k] + E[N3 + idx] -
                        E[N3 + (long long)i * NN + (long long)wrapi(j - 1, N) * N + k] + E[2 * N3 + idx] -
                        E[2 * N3 + (long long)i * NN + (long long)j * N + wrapi(k - 1, N)]) / dx;
    return div - g * fabric_rho_em(f, idx);
}

// sums of rho_em dV and |rho_em| dV (net_charge_check with rho_em)
__global__ void __launch_bounds__(kRedThreads) fabric_net_charge_kernel(FabView f, double dV, double *part) {
    __shared__ double scratch[2 * 32];
    double S[2] = {0.0, 0.0}, M[1] = {0.0};
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < f.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        const double r = fabric_rho_em(f, idx);
        S[0] += r * dV;
        S[1] += fabs(r) * dV;
    }
    block_fold<2, 0>(S, M, scratch, part);
}

// b = Gauss residual (when b is given) and the partial sums of it
__global__ void __launch_bounds__(kRedThreads) fabric_gauss_kernel(FabView f, int N, double dx, double g, double *b,
                                                                   double *part) {
    __shared__ double scratch[32];
    double S[1] = {0.0}, M[1] = {0.0};
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < f.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        const double G = fabric_gauss(f, N, dx, g, idx);
        if (b) b[idx] = G;
        S[0] += G;
    }
    block_fold<1, 0>(S, M, scratch, part);
}

// Gauss norm over the interior |x| < Rint with rho_em (compute_gauss) and the
// per-fabric charges (compute_mf_charges).  Sums: (G - OFF)^2, interior
// count, rho_C, rho_Q, rho_L, rho_em; maximum: |G - OFF| over the interior.
enum : int { FS_GL2 = 0, FS_NIN, FS_QC, FS_QQ, FS_QL, FS_QEM, FS_NSUM };
__global__ void __launch_bounds__(kRedThreads) fabric_diag_kernel(FabView f, int N, double L, double dx, double g,
                                                                  double Rint2, double G_offset, double *part) {
    __shared__ double scratch[(FS_NSUM + 1) * 32];
    double S[FS_NSUM], M[1] = {0.0};
    for (int q = 0; q < FS_NSUM; q++) S[q] = 0.0;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < f.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        site_ijk(idx, N, &i, &j, &k);
        const double x = -L + i * dx, y = -L + j * dx, z = -L + k * dx;
        const double rc = fabric_rho(f.XC, f.PC, f.N3, idx), rq = fabric_rho(f.XQ, f.PQ, f.N3, idx);
        const double rl = fabric_rho(f.XL, f.PL, f.N3, idx);
        if (x * x + y * y + z * z < Rint2) {
            const double dG = fabric_gauss(f, N, dx, g, idx) - G_offset;
            M[0] = fmax(M[0], fabs(dG));
            S[FS_GL2] += dG * dG;
            S[FS_NIN] += 1.0;
        }
        S[FS_QC] += rc;
        S[FS_QQ] += rq;
        S[FS_QL] += rl;
        S[FS_QEM] += f.q[0] * rc + f.q[1] * rq + f.q[2] * rl;
    }
    block_fold<FS_NSUM, 1>(S, M, scratch, part);
}

// Fabric L seen through the diagnostics' state view: its 12 matter fields
// with C's links and E (the reference's energy of L uses the unit-charge
// links, compute_energy_complex_gauge :1977-2028)
struct ViewFabric {
    const double *XF, *PF, *XC, *PC;
    long long N3;
    __device__ __forceinline__ double q(int f, long long i) const { return f < 12 ? XF[f * N3 + i] : XC[f * N3 + i]; }
    __device__ __forceinline__ double p(int f, long long i) const { return f < 12 ? PF[f * N3 + i] : PC[f * N3 + i]; }
};

// ---- real mode with the optional terms
// Energy terms of the real mode (compute_energy with the optional terms) and
// P_integrated, theta^2 for theta_rms.  Sums in the order of the diagnostics
// slots; maxima |phi_a| and |P|.
enum : int { R6_EPK = 0, R6_ETK, R6_EG, R6_EM, R6_EP, R6_ETG, R6_ETM, R6_EC, R6_PINT, R6_TH2, R6_NSUM };
enum : int { R6_PHIMAX = 0, R6_PMAX, R6_NMAX };

__global__ void __launch_bounds__(256) r6_energy_kernel(const double *X, const double *V, R6Consts c, double *part) {
    __shared__ double scratch[(R6_NSUM + R6_NMAX) * 32];
    double S[R6_NSUM], M[R6_NMAX];
    for (int q = 0; q < R6_NSUM; q++) S[q] = 0.0;
    for (int q = 0; q < R6_NMAX; q++) M[q] = 0.0;
    const int N = c.N;
    const long long NN = (long long)N * N, N3 = c.N3;
    const double dV = c.dV;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        site_ijk(idx, N, &i, &j, &k);
        // neighbour offsets +d and -d along i, j, k
        const long long nbp[3] = {(long long)wrapi(i + 1, N) * NN + (long long)j * N + k,
                                  (long long)i * NN + (long long)wrapi(j + 1, N) * N + k,
                                  (long long)i * NN + (long long)j * N + wrapi(k + 1, N)};
        const long long nbm[3] = {(long long)wrapi(i - 1, N) * NN + (long long)j * N + k,
                                  (long long)i * NN + (long long)wrapi(j - 1, N) * N + k,
                                  (long long)i * NN + (long long)j * N + wrapi(k - 1, N)};
        auto grad = [&](const double *F, int d) { return (F[nbp[d]] - F[nbm[d]]) * c.idx1; };
        auto curl = [&](const double *F, int a) {
            const int b = (a + 1) % 3, e = (a + 2) % 3;
            return grad(F + e * N3, b) - grad(F + b * N3, e);
        };
        const double *phi = X, *th = X + 3 * N3;
        double p[3], t[3];
        for (int a = 0; a < 3; a++) { p[a] = phi[a * N3 + idx]; t[a] = th[a * N3 + idx]; }
        const double sig = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        const double m2e = (c.mode == 1) ? c.ia / (1.0 + c.ib * sig) : c.m2;
        const double ke = (c.mode == 3) ? c.kappa / (1.0 + c.kg * sig) : c.kappa;
        for (int a = 0; a < 3; a++) {
            const double vp = V[a * N3 + idx], vt = V[(3 + a) * N3 + idx];
            S[R6_EPK] += 0.5 * vp * vp * dV;
            S[R6_ETK] += 0.5 * vt * vt * dV;
            const double gx = grad(phi + a * N3, 0), gy = grad(phi + a * N3, 1), gz = grad(phi + a * N3, 2);
            S[R6_EG] += 0.5 * (gx * gx + gy * gy + gz * gz) * dV;
            S[R6_EM] += 0.5 * m2e * p[a] * p[a] * dV;
            const double hx = grad(th + a * N3, 0), hy = grad(th + a * N3, 1), hz = grad(th + a * N3, 2);
            S[R6_ETG] += 0.5 * (hx * hx + hy * hy + hz * hz) * dV;
            S[R6_ETM] += 0.5 * c.mtheta2 * t[a] * t[a] * dV;
            M[R6_PHIMAX] = fmax(M[R6_PHIMAX], fabs(p[a]));
            S[R6_TH2] += t[a] * t[a];
        }
        const double P = p[0] * p[1] * p[2], P2 = P * P;
        if (c.mode == 3) {
            const double D = 1.0 + c.kg * sig + c.kappa * P2;
            S[R6_EP] += (c.mu / 2.0) * P2 * (1.0 + c.kg * sig) / D * dV;
        } else {
            S[R6_EP] += (c.mu / 2.0) * P2 / (1.0 + ke * P2) * dV;
        }
        M[R6_PMAX] = fmax(M[R6_PMAX], fabs(P));
        S[R6_PINT] += fabs(P) * dV;
        if (c.alpha != 0 || c.beta != 0 || c.kh != 0) {
            double cp[3];
            for (int a = 0; a < 3; a++) cp[a] = curl(phi, a);
            if (c.alpha != 0) {
                double m = 0.0;
                for (int a = 0; a < 3; a++) {
                    const double ca = cp[a] * 0.5 - t[a];
                    m += ca * ca;
                }
                S[R6_EP] += c.alpha * m * dV;
            }
            if (c.beta != 0)
                S[R6_EP] += 0.5 * c.beta * (t[0] * t[0] + t[1] * t[1] + t[2] * t[2]) *
                            (cp[0] * cp[0] + cp[1] * cp[1] + cp[2] * cp[2]) * dV;
            if (c.kh != 0) S[R6_EP] += c.kh * P2 * (p[0] * cp[0] + p[1] * cp[1] + p[2] * cp[2]) * dV;
        }
        for (int a = 0; a < 3; a++) S[R6_EC] -= c.eta * p[a] * curl(th, a) * dV;
    }
    block_fold<R6_NSUM, R6_NMAX>(S, M, scratch, part);
}

}  // namespace scp
