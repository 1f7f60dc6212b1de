// diag_ring.cuh -- the first diagnostics reduction (energies, charges,
// centroid moments, Gauss residual, E_em; the pass-1 slots of diag.cuh) for
// FP64 states, on the plane ring: every stencil value comes from shared
// memory, each field is read once, and every thread keeps its sums over all
// the sites it walks before one block fold at the end.  The per-site terms
// are those of diag_pass1_kernel (compute_energy_complex[_gauge],
// compute_charges, compute_gauss, sfa/sim/scp_sim.c:1823-2243); only the
// order in which the sites are summed differs (fixed by the tile plan, so
// the result is still the same from run to run).
#pragma once
#include "diag.cuh"
#include "ring.cuh"

namespace scp {

// One instantiation per GAUGED: states with and without links run the same
// machine code (the links are a runtime flag, c.links), so a g = 0 run that
// carries links sums exactly as the run without them.  Without links the
// th / E slots of the ring are staged from matter arrays and never read.
template <bool GAUGED>
struct DiagRing {
    static constexpr int NR = 18;                // matter positions, th, E
    static constexpr int TH = 12, EF = 15;
    static constexpr int MIN_CTAS = 1;
    struct Args {
        RingSrc<NR> src;
        int N;
        DiagConsts c;
        const double *mom;   // the 12 matter momenta (N^3 arrays)
    };
    struct Carry {
        double cm0, sm0;   // cos / sin of link 0 at x - i (gauged)
    };
    __device__ static void prefetch(const Args &A, long long idx) {
#pragma unroll
        for (int f = 0; f < 12; f++) prefetch_l2(A.mom + f * A.c.N3 + idx);
    }

    template <class V>
    __device__ static void site(const Args &A, const V &v, int i, int j, int k, long long idx, Carry &cy,
                                bool first_plane, DiagSums &acc) {
        const DiagConsts &c = A.c;
        const long long N3 = c.N3;
        const double dV = c.dV, idx1 = c.idx1;
        double* S = acc.S;
        double* M = acc.M;
        double mu_[12];   // matter momenta at this site, loaded first (latency under the stencil)
#pragma unroll
        for (int f = 0; f < 12; f++) mu_[f] = A.mom[f * N3 + idx];
        double fu[6], fv[6];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            fu[a] = v(FU + a); fv[a] = v(FV + a);
            fu[3 + a] = v(FTU + a); fv[3 + a] = v(FTV + a);
        }
        // central differences, transported by the links when gauged, summed
        // into the gradient energies as the directions come in; the curl of
        // Theta (D_{a+1} Theta_{a+2} - D_{a+2} Theta_{a+1}) is built the same way
        double eg = 0.0, etg = 0.0, cr[3], ci[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double cP = 1.0, sP = 0.0, cM = 1.0, sM = 0.0;
            if (GAUGED) {
                sincos_any(v(TH + d), &sP, &cP);
                if (d == 0) {   // link 0 at x - i: this thread's value from the previous plane
                    if (first_plane) sincos_any(nb(v, TH, 0, -1), &cy.sm0, &cy.cm0);
                    sM = cy.sm0; cM = cy.cm0;
                    cy.sm0 = sP; cy.cm0 = cP;
                } else {
                    sincos_any(nb(v, TH + d, d, -1), &sM, &cM);
                }
            }
#pragma unroll
            for (int q = 0; q < 6; q++) {
                const int fre = q < 3 ? FU + q : FTU + q - 3, fim = q < 3 ? FV + q : FTV + q - 3;
                const double up = nb(v, fre, d, 1), vp = nb(v, fim, d, 1);
                const double um = nb(v, fre, d, -1), vm = nb(v, fim, d, -1);
                double DR, DI;
                if (GAUGED) {
                    DR = ((cP * up - sP * vp) - (cM * um + sM * vm)) * idx1;
                    DI = ((cP * vp + sP * up) - (cM * vm - sM * um)) * idx1;
                } else {
                    DR = (up - um) * idx1;
                    DI = (vp - vm) * idx1;
                }
                if (q < 3) eg += DR * DR + DI * DI;
                else etg += DR * DR + DI * DI;
                const int qa = q - 3;
                if (GAUGED && q >= 3 && qa != d) {
                    if (qa == (d + 1) % 3) {            // plus term of component a = d + 2
                        const int a = (d + 2) % 3;
                        if (d < (a + 2) % 3) { cr[a] = DR; ci[a] = DI; }
                        else { cr[a] = DR - cr[a]; ci[a] = DI - ci[a]; }
                    } else {                            // minus term of component a = d + 1
                        const int a = (d + 1) % 3;
                        if (d < (a + 1) % 3) { cr[a] = DR; ci[a] = DI; }
                        else { cr[a] = cr[a] - DR; ci[a] = ci[a] - DI; }
                    }
                }
            }
        }
        S[DS_EG] += 0.5 * eg * dV;
        S[DS_ETG] += 0.5 * etg * dV;
        double s2[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            s2[a] = fu[a] * fu[a] + fv[a] * fv[a];
            const double pu = mu_[FU + a], pv = mu_[FV + a], ptu = mu_[FTU + a], ptv = mu_[FTV + a];
            S[DS_EPK] += 0.5 * (pu * pu + pv * pv) * dV;
            S[DS_ETK] += 0.5 * (ptu * ptu + ptv * ptv) * dV;
            S[DS_EM] += 0.5 * c.m2 * s2[a] * dV;
            S[DS_ETM] += 0.5 * c.mtheta2 * (fu[3 + a] * fu[3 + a] + fv[3 + a] * fv[3 + a]) * dV;
            M[DM_PM] = fmax(M[DM_PM], sqrt(s2[a]));
            if (!GAUGED) {   // curl_component of theta (scp_sim.c:409-415, :1868-1870)
                const int d1 = (a + 1) % 3, d2 = (a + 2) % 3;
                const int fa = FTU + d2, fb = FTU + d1, ga = FTV + d2, gb = FTV + d1;
                cr[a] = (nb(v, fa, d1, 1) - nb(v, fa, d1, -1) - nb(v, fb, d2, 1) + nb(v, fb, d2, -1)) * idx1;
                ci[a] = (nb(v, ga, d1, 1) - nb(v, ga, d1, -1) - nb(v, gb, d2, 1) + nb(v, gb, d2, -1)) * idx1;
            }
            S[DS_EC] -= c.eta * (fu[a] * cr[a] + fv[a] * ci[a]) * dV;
        }
        const double s = s2[0] * s2[1] * s2[2];
        S[DS_EP] += (c.mu / 2.0) * s / (1.0 + c.kappa * s) * dV;
        M[DM_PMAX] = fmax(M[DM_PMAX], sqrt(s));
        S[DS_PINT] += sqrt(s) * dV;
#pragma unroll
        for (int a = 0; a < 3; a++) S[DS_TRS] += fu[3 + a] * fu[3 + a] + fv[3 + a] * fv[3 + a];
        // Noether charges, core and centroid moments
        const double x = -c.L + i * c.dx, y = -c.L + j * c.dx, z = -c.L + k * c.dx;
        double rho2 = 0.0, qp = 0.0, qt = 0.0, sprod = 1.0;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const double qa = fu[a] * mu_[FV + a] - fv[a] * mu_[FU + a];
            qp += qa;
            S[DS_QP0 + a] += qa;
            qt += fu[3 + a] * mu_[FTV + a] - fv[3 + a] * mu_[FTU + a];
            const double s2a = fu[a] * fu[a] + fv[a] * fv[a];
            rho2 += s2a;
            sprod *= s2a;
        }
        S[DS_QP] += qp;
        S[DS_QT] += qt;
        if (x * x + y * y + z * z <= c.R2) S[DS_QC] += qp + qt;
        M[DM_SMAX] = fmax(M[DM_SMAX], sprod);
        S[DS_M0] += rho2;
        S[DS_CX] += x * rho2;
        S[DS_CY] += y * rho2;
        S[DS_CZ] += z * rho2;
        if (c.links) {   // Gauss law and E_em (also with g = 0: then only E^2/2)
            const double E0 = v(EF), E1 = v(EF + 1), E2 = v(EF + 2);
            const double divE = (E0 - v.at(EF, -1, 0, 0) + E1 - v.at(EF + 1, 0, -1, 0) + E2 - v.at(EF + 2, 0, 0, -1)) / c.dx;
            double rho = 0.0;
#pragma unroll
            for (int a = 0; a < 3; a++)
                rho += fu[a] * mu_[FV + a] - fv[a] * mu_[FU + a] + fu[3 + a] * mu_[FTV + a] - fv[3 + a] * mu_[FTU + a];
            const double G = divE - c.g * rho;
            if (x * x + y * y + z * z < c.Rint2) {
                M[DM_GMAX] = fmax(M[DM_GMAX], fabs(G - c.G_offset));
                S[DS_GL2] += (G - c.G_offset) * (G - c.G_offset);
                S[DS_NOM] += 1.0;
            }
            double ee = 0.5 * (E0 * E0 + E1 * E1 + E2 * E2);
            if (GAUGED) {
                const double t0 = v(TH), t1 = v(TH + 1), t2 = v(TH + 2);
                double bb = 0.0, sn, cs;
                sincos_any(t0 + v.at(TH + 1, 1, 0, 0) - v.at(TH, 0, 1, 0) - t1, &sn, &cs);
                bb += 1.0 - cs;
                sincos_any(t1 + v.at(TH + 2, 0, 1, 0) - v.at(TH + 1, 0, 0, 1) - t2, &sn, &cs);
                bb += 1.0 - cs;
                sincos_any(t2 + v.at(TH, 0, 0, 1) - v.at(TH + 2, 1, 0, 0) - t0, &sn, &cs);
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
};

template <bool GAUGED, int TX, int TY>
__global__ void __launch_bounds__(TX *TY, 1) diag_ring_kernel(typename DiagRing<GAUGED>::Args a, TileGrid tg,
                                                              double *part) {
    extern __shared__ __align__(16) double ring[];
    __shared__ double scratch[kDiag1Q * 32];
    DiagSums acc;
#pragma unroll
    for (int q = 0; q < DS_NSUM; q++) acc.S[q] = 0.0;
#pragma unroll
    for (int q = 0; q < DM_NMAX; q++) acc.M[q] = 0.0;
    for_each_piece(tg, a.N, [&](const Piece &pc) { ring_item<DiagRing<GAUGED>, TX, TY>(a, pc, ring, acc); });
    block_fold<DS_NSUM, DM_NMAX>(acc.S, acc.M, scratch, part);
}

}  // namespace scp
