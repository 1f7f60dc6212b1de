// diag.cuh -- FP64 diagnostics of the complex / gauged lattice state:
// energies (compute_energy_complex / _gauge, sfa/sim/scp_sim.c:1823-2036),
// theta_rms and P_int (:2041-2061), Noether charges and core diagnostics
// (compute_charges, :2074-2169) and the Gauss-law residual (compute_gauss,
// :2186-2243).  Per-site terms are written in the reference's operation
// order; sums are folded deterministically (reduce.cuh).
#pragma once
#include "reduce.cuh"
#include "trig.cuh"

namespace scp {

// Read-only view of a state: positions (u v tu tv th) and synchronous momenta
// (du dv dtu dtv E).  The FP32-compensated layout provides its own view.
struct ViewF64 {
    const double *X, *S;
    long long N3;
    __device__ __forceinline__ double q(int f, long long i) const { return X[f * N3 + i]; }
    __device__ __forceinline__ double p(int f, long long i) const { return S[f * N3 + i]; }
};

struct DiagConsts {
    int N;
    long long N3;
    double L, dx, dV, idx1;
    double m2, mtheta2, eta, mu, kappa;
    int gauged;               // covariant energy, plaquette energy (g != 0)
    int links;                // th / E columns present: Gauss residual, E_em, Q_flux
    int real;                 // real 6-field mode (imaginary sector zero): theta_rms over 3 components
    double g, bpre;           // bpre = 1/(g^2 dx^4)
    double R2;                // qdiag_radius^2
    double Rcube;             // qdiag_radius (Q_flux cube half width)
    double Rint2;             // interior radius^2 of the Gauss norm
    double G_offset;
};

// pass-1 slots
enum : int {
    DS_EPK = 0, DS_ETK, DS_EG, DS_EM, DS_EP, DS_ETG, DS_ETM, DS_EC, DS_EEM, DS_PINT, DS_TRS,
    DS_QP, DS_QT, DS_M0, DS_CX, DS_CY, DS_CZ, DS_QC, DS_QP0, DS_QP1, DS_QP2,
    DS_GL2, DS_NOM, DS_FSUM, DS_NC,
    DS_NSUM,
    DM_PM = 0, DM_PMAX, DM_SMAX, DM_GMAX, DM_NMAX
};
constexpr int kDiag1Q = DS_NSUM + DM_NMAX;

// per-thread sums and maxima of the pass-1 slots
struct DiagSums {
    double S[DS_NSUM], M[DM_NMAX];
    __device__ __forceinline__ void clear() {
#pragma unroll
        for (int q = 0; q < DS_NSUM; q++) S[q] = 0.0;
#pragma unroll
        for (int q = 0; q < DM_NMAX; q++) M[q] = 0.0;
    }
};

template <class View>
__global__ void __launch_bounds__(kRedThreads) diag_pass1_kernel(View V, DiagConsts c, double *part) {
    __shared__ double scratch[kDiag1Q * 32];
    double S[DS_NSUM], M[DM_NMAX];
    #pragma unroll
    for (int q = 0; q < DS_NSUM; q++) S[q] = 0.0;
    #pragma unroll
    for (int q = 0; q < DM_NMAX; q++) M[q] = 0.0;
    const int N = c.N;
    const long long NN = (long long)N * N;
    const double dV = c.dV, idx1 = c.idx1;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < c.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        site_ijk(idx, N, &i, &j, &k);
        const long long np[3] = {(long long)wrapi(i + 1, N) * NN + (long long)j * N + k,
                                 (long long)i * NN + (long long)wrapi(j + 1, N) * N + k,
                                 (long long)i * NN + (long long)j * N + wrapi(k + 1, N)};
        const long long nm[3] = {(long long)wrapi(i - 1, N) * NN + (long long)j * N + k,
                                 (long long)i * NN + (long long)wrapi(j - 1, N) * N + k,
                                 (long long)i * NN + (long long)j * N + wrapi(k - 1, N)};
        double fu[6], fv[6];
        #pragma unroll
        for (int a = 0; a < 3; a++) {
            fu[a] = V.q(FU + a, idx);  fv[a] = V.q(FV + a, idx);
            fu[3 + a] = V.q(FTU + a, idx); fv[3 + a] = V.q(FTV + a, idx);
        }
        // ---- energies
        double DcU[3][6], DcV[3][6];
        #pragma unroll
        for (int d = 0; d < 3; d++) {
            double cP = 1.0, sP = 0.0, cM = 1.0, sM = 0.0;
            if (c.gauged) {
                sincos_any(V.q(FTH + d, idx), &sP, &cP);
                sincos_any(V.q(FTH + d, nm[d]), &sM, &cM);
            }
            #pragma unroll
            for (int q = 0; q < 6; q++) {
                const int fre = q < 3 ? FU + q : FTU + q - 3, fim = q < 3 ? FV + q : FTV + q - 3;
                const double upn = V.q(fre, np[d]), vpn = V.q(fim, np[d]);
                const double umn = V.q(fre, nm[d]), vmn = V.q(fim, nm[d]);
                if (c.gauged) {
                    DcU[d][q] = ((cP * upn - sP * vpn) - (cM * umn + sM * vmn)) * idx1;
                    DcV[d][q] = ((cP * vpn + sP * upn) - (cM * vmn - sM * umn)) * idx1;
                } else {
                    DcU[d][q] = (upn - umn) * idx1;
                    DcV[d][q] = (vpn - vmn) * idx1;
                }
            }
        }
        double s2[3];
        #pragma unroll
        for (int a = 0; a < 3; a++) {
            s2[a] = fu[a] * fu[a] + fv[a] * fv[a];
            const double pu = V.p(FU + a, idx), pv = V.p(FV + a, idx);
            const double ptu = V.p(FTU + a, idx), ptv = V.p(FTV + a, idx);
            S[DS_EPK] += 0.5 * (pu * pu + pv * pv) * dV;
            S[DS_ETK] += 0.5 * (ptu * ptu + ptv * ptv) * dV;
            S[DS_EG] += 0.5 * (DcU[0][a] * DcU[0][a] + DcU[1][a] * DcU[1][a] + DcU[2][a] * DcU[2][a]
                               + DcV[0][a] * DcV[0][a] + DcV[1][a] * DcV[1][a] + DcV[2][a] * DcV[2][a]) * dV;
            S[DS_EM] += 0.5 * c.m2 * s2[a] * dV;
            S[DS_ETG] += 0.5 * (DcU[0][3 + a] * DcU[0][3 + a] + DcU[1][3 + a] * DcU[1][3 + a]
                                + DcU[2][3 + a] * DcU[2][3 + a] + DcV[0][3 + a] * DcV[0][3 + a]
                                + DcV[1][3 + a] * DcV[1][3 + a] + DcV[2][3 + a] * DcV[2][3 + a]) * dV;
            S[DS_ETM] += 0.5 * c.mtheta2 * (fu[3 + a] * fu[3 + a] + fv[3 + a] * fv[3 + a]) * dV;
            M[DM_PM] = fmax(M[DM_PM], sqrt(s2[a]));
            const int d1 = (a + 1) % 3, d2 = (a + 2) % 3;
            double reDxT, imDxT;
            if (c.gauged) {   // transported curls (scp_sim.c:1950-1953)
                reDxT = DcU[d1][3 + d2] - DcU[d2][3 + d1];
                imDxT = DcV[d1][3 + d2] - DcV[d2][3 + d1];
            } else {          // curl_component of theta (scp_sim.c:409-415, :1868-1870)
                const int fa = FTU + d2, fb = FTU + d1, ga = FTV + d2, gb = FTV + d1;
                reDxT = (V.q(fa, np[d1]) - V.q(fa, nm[d1]) - V.q(fb, np[d2]) + V.q(fb, nm[d2])) * idx1;
                imDxT = (V.q(ga, np[d1]) - V.q(ga, nm[d1]) - V.q(gb, np[d2]) + V.q(gb, nm[d2])) * idx1;
            }
            S[DS_EC] -= c.eta * (fu[a] * reDxT + fv[a] * imDxT) * dV;
        }
        const double s = s2[0] * s2[1] * s2[2];
        S[DS_EP] += (c.mu / 2.0) * s / (1.0 + c.kappa * s) * dV;
        M[DM_PMAX] = fmax(M[DM_PMAX], sqrt(s));
        S[DS_PINT] += sqrt(s) * dV;
        #pragma unroll
        for (int a = 0; a < 3; a++) S[DS_TRS] += fu[3 + a] * fu[3 + a] + fv[3 + a] * fv[3 + a];
        // ---- charges
        const double x = -c.L + i * c.dx, y = -c.L + j * c.dx, z = -c.L + k * c.dx;
        double rho2 = 0.0, qpv = 0.0, qtv = 0.0, sprod = 1.0;
        #pragma unroll
        for (int a = 0; a < 3; a++) {
            const double u = fu[a], v = fv[a];
            const double ud = V.p(FU + a, idx), vd = V.p(FV + a, idx);
            const double tu = fu[3 + a], tv = fv[3 + a];
            const double tud = V.p(FTU + a, idx), tvd = V.p(FTV + a, idx);
            const double qa = u * vd - v * ud;
            qpv += qa;
            S[DS_QP0 + a] += qa;
            qtv += tu * tvd - tv * tud;
            const double s2a = u * u + v * v;
            rho2 += s2a;
            sprod *= s2a;
        }
        S[DS_QP] += qpv;
        S[DS_QT] += qtv;
        if (x * x + y * y + z * z <= c.R2) S[DS_QC] += qpv + qtv;
        M[DM_SMAX] = fmax(M[DM_SMAX], sprod);
        S[DS_M0] += rho2;
        S[DS_CX] += x * rho2; S[DS_CY] += y * rho2; S[DS_CZ] += z * rho2;
        // ---- Gauss law and E_em (compute_gauss: also with g = 0, where the
        //      links are carried unchanged and only 1/2 E^2 enters E_em)
        if (c.links) {
            const double E0 = V.p(FTH + 0, idx), E1 = V.p(FTH + 1, idx), E2 = V.p(FTH + 2, idx);
            const double divE = (E0 - V.p(FTH + 0, nm[0]) + E1 - V.p(FTH + 1, nm[1])
                                 + E2 - V.p(FTH + 2, nm[2])) / c.dx;
            double rho = 0.0;
            #pragma unroll
            for (int a = 0; a < 3; a++)
                rho += fu[a] * V.p(FV + a, idx) - fv[a] * V.p(FU + a, idx)
                     + fu[3 + a] * V.p(FTV + a, idx) - fv[3 + a] * V.p(FTU + a, idx);
            const double G = divE - c.g * rho;
            if (x * x + y * y + z * z < c.Rint2) {
                M[DM_GMAX] = fmax(M[DM_GMAX], fabs(G - c.G_offset));
                S[DS_GL2] += (G - c.G_offset) * (G - c.G_offset);
                S[DS_NOM] += 1.0;
            }
            double ee = 0.5 * (E0 * E0 + E1 * E1 + E2 * E2);
            if (c.gauged) {
                const double th0 = V.q(FTH + 0, idx), th1 = V.q(FTH + 1, idx), th2 = V.q(FTH + 2, idx);
                double bb = 0.0, sn, cs;
                sincos_any(th0 + V.q(FTH + 1, np[0]) - V.q(FTH + 0, np[1]) - th1, &sn, &cs);
                bb += 1.0 - cs;
                sincos_any(th1 + V.q(FTH + 2, np[1]) - V.q(FTH + 1, np[2]) - th2, &sn, &cs);
                bb += 1.0 - cs;
                sincos_any(th2 + V.q(FTH + 0, np[2]) - V.q(FTH + 2, np[0]) - th0, &sn, &cs);
                bb += 1.0 - cs;
                ee += c.bpre * bb;
            }
            S[DS_EEM] += ee * dV;
            if (fabs(x) <= c.Rcube && fabs(y) <= c.Rcube && fabs(z) <= c.Rcube) {
                S[DS_FSUM] += divE * dV;
                S[DS_NC] += 1.0;
            }
        }
    }
    block_fold<DS_NSUM, DM_NMAX>(S, M, scratch, part + 0);
}

// Pass 2: r_core second moment about the centroid and the lowest site index
// with s >= smax*(1-1e-12) (scp_sim.c:2118-2139, :2155-2168).
// fin1: folded pass-1 values.  part2 per CTA: [rsum, -min_idx] as sums/max.
template <class View>
__global__ void __launch_bounds__(kRedThreads) diag_pass2_kernel(View V, DiagConsts c, const double *fin1,
                                                                 double *part) {
    __shared__ double scratch[2 * 32];
    const double M0 = fin1[DS_M0] * c.dV;
    const double cx = M0 < 1e-30 ? 0.0 : fin1[DS_CX] * c.dV / M0;
    const double cy = M0 < 1e-30 ? 0.0 : fin1[DS_CY] * c.dV / M0;
    const double cz = M0 < 1e-30 ? 0.0 : fin1[DS_CZ] * c.dV / M0;
    const double sthr = fin1[DS_NSUM + DM_SMAX] * (1.0 - 1e-12);
    const int N = c.N;
    double S[1] = {0.0}, M[1] = {-INFINITY};   // M holds -(lowest qualifying index)
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < c.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        site_ijk(idx, N, &i, &j, &k);
        const double x = -c.L + i * c.dx, y = -c.L + j * c.dx, z = -c.L + k * c.dx;
        double rho2 = 0.0, sp = 1.0;
        for (int a = 0; a < 3; a++) {
            const double u = V.q(FU + a, idx), v = V.q(FV + a, idx);
            rho2 += u * u + v * v;
            sp *= u * u + v * v;
        }
        S[0] += ((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz)) * rho2;
        if (sp >= sthr) M[0] = fmax(M[0], -(double)idx);
    }
    block_fold<1, 1>(S, M, scratch, part);
}

// Pass 2 after a synchronous step launch that summed pass 1 itself (step.cuh,
// StepIO::dpart): r_core and the argmax site as diag_pass2_kernel, and the
// Gauss-law slots of pass 1 (compute_gauss, scp_sim.c:2186-2243), which need
// E_{n+1} of the neighbouring sites, from the charge density the launch
// stored (rho, N^3; links only).
// part per CTA: sums [rsum, GL2, NOM, FSUM, NC], maxima [-min_idx, GMAX].
template <class View>
__global__ void __launch_bounds__(kRedThreads) diag_pass2g_kernel(View V, DiagConsts c, const double *fin1,
                                                                  const double *rho, double *part) {
    __shared__ double scratch[7 * 32];
    const double M0 = fin1[DS_M0] * c.dV;
    const double cx = M0 < 1e-30 ? 0.0 : fin1[DS_CX] * c.dV / M0;
    const double cy = M0 < 1e-30 ? 0.0 : fin1[DS_CY] * c.dV / M0;
    const double cz = M0 < 1e-30 ? 0.0 : fin1[DS_CZ] * c.dV / M0;
    const double sthr = fin1[DS_NSUM + DM_SMAX] * (1.0 - 1e-12);
    const int N = c.N;
    const long long NN = (long long)N * N;
    double S[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, M[2] = {-INFINITY, 0.0};
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < c.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        site_ijk(idx, N, &i, &j, &k);
        const double x = -c.L + i * c.dx, y = -c.L + j * c.dx, z = -c.L + k * c.dx;
        double rho2 = 0.0, sp = 1.0;
        for (int a = 0; a < 3; a++) {
            const double u = V.q(FU + a, idx), v = V.q(FV + a, idx);
            rho2 += u * u + v * v;
            sp *= u * u + v * v;
        }
        S[0] += ((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz)) * rho2;
        if (sp >= sthr) M[0] = fmax(M[0], -(double)idx);
        if (c.links) {
            const long long im = (long long)wrapi(i - 1, N) * NN + (long long)j * N + k;
            const long long jm = (long long)i * NN + (long long)wrapi(j - 1, N) * N + k;
            const long long km = (long long)i * NN + (long long)j * N + wrapi(k - 1, N);
            const double E0 = V.p(FTH, idx), E1 = V.p(FTH + 1, idx), E2 = V.p(FTH + 2, idx);
            const double divE = (E0 - V.p(FTH, im) + E1 - V.p(FTH + 1, jm) + E2 - V.p(FTH + 2, km)) / c.dx;
            const double G = divE - c.g * rho[idx];
            if (x * x + y * y + z * z < c.Rint2) {
                M[1] = fmax(M[1], fabs(G - c.G_offset));
                S[1] += (G - c.G_offset) * (G - c.G_offset);
                S[2] += 1.0;
            }
            if (fabs(x) <= c.Rcube && fabs(y) <= c.Rcube && fabs(z) <= c.Rcube) {
                S[3] += divE * c.dV;
                S[4] += 1.0;
            }
        }
    }
    block_fold<5, 2>(S, M, scratch, part);
}

// Final scalar reads: omega_core at the argmax-s site and the two theta probes.
// out[0]=omega_core out[1..4]=thp1u thp1v thp2u thp2v
// negidx_p: the folded -(lowest qualifying site index).
template <class View>
__global__ void diag_point_kernel(View V, DiagConsts c, const double *negidx_p, double probe1, double probe2,
                                  double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int N = c.N;
    const long long NN = (long long)N * N;
    out[0] = 0.0;
    const double negidx = *negidx_p;
    if (isfinite(negidx)) {
        const long long idx = (long long)(-negidx);
        const double u0 = V.q(FU, idx), v0 = V.q(FV, idx), ud0 = V.p(FU, idx), vd0 = V.p(FV, idx);
        const double den = u0 * u0 + v0 * v0;
        if (den >= 1e-20) out[0] = (u0 * vd0 - v0 * ud0) / den;
    }
    int jc = (int)llround(c.L / c.dx);
    jc = jc < 0 ? 0 : (jc > N - 1 ? N - 1 : jc);
    int i1 = (int)llround((probe1 + c.L) / c.dx);
    i1 = i1 < 0 ? 0 : (i1 > N - 1 ? N - 1 : i1);
    int i2 = (int)llround((probe2 + c.L) / c.dx);
    i2 = i2 < 0 ? 0 : (i2 > N - 1 ? N - 1 : i2);
    const long long p1 = (long long)i1 * NN + (long long)jc * N + jc;
    const long long p2 = (long long)i2 * NN + (long long)jc * N + jc;
    out[1] = V.q(FTU + 1, p1); out[2] = V.q(FTV + 1, p1);
    out[3] = V.q(FTU + 1, p2); out[4] = V.q(FTV + 1, p2);
}

}  // namespace scp
