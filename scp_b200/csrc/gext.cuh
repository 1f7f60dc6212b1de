// gext.cuh -- the gauged stepper with the reference's v71 extensions: the
// Higgs condensate H (scalar, self-coupling lambda, matter coupling kappa_H:
// V_H = (lambda/4)(H^2 - v^2)^2 + (kappa_H/2) s H^2) and the second compact
// U(1) gauge field (links th2, field E2, coupling g2, per-component charges
// q_a; matter transported by th + q_a th2).  compute_forces_complex_gauge,
// sfa/sim/scp_sim.c:1053-1263; verlet_step, :1583-1716; Higgs energy,
// :1970-1975; second Gauss projection, :2400-2458.
//
// These runs use per-site kernels over global memory in the reference's
// arithmetic order, three sweeps per step (kick + drift, link cos/sin and
// plaquette sines, forces) and a closing kick after the last step of a call,
// with the state in the packed layout of the fused kernels (X: u v tu tv th,
// S: du dv dtu dtv E, synchronous between calls) so that the diagnostics and
// snapshots are shared.  Gauged runs without these extensions take the fused
// kernels.
#pragma once
#include "common.cuh"
#include "gauss.cuh"
#include "reduce.cuh"
#include "trig.cuh"

namespace scp {

struct GextConsts {
    int N;
    long long N3;
    double L, dx, dV, idx1, idx2, inva, hdt, dt;
    double mu, kappa, m2, mtheta2, eta;
    double g, stp, gad;                // gauge 1: coupling, 1/(g dx^3), -g dx dt
    int g2on;
    double g2, stp2, gad2, q[3];       // gauge 2
    int higgs;
    double hv, hlam, hkap;
    int damp;
    double damp_width, damp_rate;
};

struct GextState {
    double *X, *S, *A;                 // packed 15-field positions, momenta, accelerations (A: 12 + E_acc)
    double *T2, *E2, *K2;              // second gauge: links, field, field kick (3 each)
    double *H, *HV, *HA;               // Higgs field, velocity, acceleration
    double *LC, *LS, *PS, *PS2;        // scratch: gauge-1 link cos / sin, plaquette sines (both gauges)
};

__device__ __forceinline__ void gext_nb(long long idx, int N, long long np[3], long long nm[3]) {
    const long long NN = (long long)N * N;
    int i, j, k;
    site_ijk(idx, N, &i, &j, &k);
    np[0] = (long long)wrapi(i + 1, N) * NN + (long long)j * N + k;
    nm[0] = (long long)wrapi(i - 1, N) * NN + (long long)j * N + k;
    np[1] = (long long)i * NN + (long long)wrapi(j + 1, N) * N + k;
    nm[1] = (long long)i * NN + (long long)wrapi(j - 1, N) * N + k;
    np[2] = (long long)i * NN + (long long)j * N + wrapi(k + 1, N);
    nm[2] = (long long)i * NN + (long long)j * N + wrapi(k - 1, N);
}

// pass A (:1072-1079, gauge-1 link cos/sin) and pass B (:1090-1109,
// plaquette sines of planes (0,1) (1,2) (2,0) for both gauges) in one sweep
__global__ void __launch_bounds__(kRedThreads) gext_links_plaq_kernel(GextState s, GextConsts c) {
    const long long N3 = c.N3;
    const double *th = s.X + FTH * N3;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double sn, cs;
            sincos_any(th[d * N3 + idx], &sn, &cs);
            s.LC[d * N3 + idx] = cs;
            s.LS[d * N3 + idx] = sn;
        }
        long long np[3], nm[3];
        gext_nb(idx, c.N, np, nm);
        const int pa[3] = {0, 1, 2}, pb[3] = {1, 2, 0};
#pragma unroll
        for (int p = 0; p < 3; p++) {
            const int a = pa[p], b = pb[p];
            double sn, cs;
            const double ang = th[a * N3 + idx] + th[b * N3 + np[a]] - th[a * N3 + np[b]] - th[b * N3 + idx];
            sincos_any(ang, &sn, &cs);
            s.PS[p * N3 + idx] = sn;
            if (c.g2on) {
                const double *t2 = s.T2;
                const double ang2 = t2[a * N3 + idx] + t2[b * N3 + np[a]] - t2[a * N3 + np[b]] - t2[b * N3 + idx];
                sincos_any(ang2, &sn, &cs);
                s.PS2[p * N3 + idx] = sn;
            }
        }
    }
}

// pass C (:1112-1262): matter accelerations, Higgs acceleration, E kicks
__global__ void __launch_bounds__(kRedThreads) gext_force_kernel(GextState s, GextConsts c) {
    const long long N3 = c.N3;
    const double *X = s.X;
    auto Q = [&](int f, long long y) { return X[f * N3 + y]; };
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        long long np[3], nm[3];
        gext_nb(idx, c.N, np, nm);
        double fu[6], fv[6];
        #pragma unroll
        for (int a = 0; a < 3; a++) {
            fu[a] = Q(FU + a, idx); fv[a] = Q(FV + a, idx);
            fu[3 + a] = Q(FTU + a, idx); fv[3 + a] = Q(FTV + a, idx);
        }
        double TRp[3][6], TIp[3][6], TRm[3][6], TIm[3][6];
        double tup[3][3], tvp[3][3];
        #pragma unroll
        for (int d = 0; d < 3; d++) {
            #pragma unroll
            for (int a = 0; a < 3; a++) {
                double cP, sP, cM, sM;
                if (c.g2on) {   // combined link th + q_a th2 for component a
                    const double php = Q(FTH + d, idx) + c.q[a] * s.T2[d * N3 + idx];
                    const double phm = Q(FTH + d, nm[d]) + c.q[a] * s.T2[d * N3 + nm[d]];
                    sincos_any(php, &sP, &cP);
                    sincos_any(phm, &sM, &cM);
                } else {
                    cP = s.LC[d * N3 + idx]; sP = s.LS[d * N3 + idx];
                    cM = s.LC[d * N3 + nm[d]]; sM = s.LS[d * N3 + nm[d]];
                }
                const double upn = Q(FU + a, np[d]), vpn = Q(FV + a, np[d]);
                const double umn = Q(FU + a, nm[d]), vmn = Q(FV + a, nm[d]);
                const double tpn = Q(FTU + a, np[d]), wpn = Q(FTV + a, np[d]);
                const double tmn = Q(FTU + a, nm[d]), wmn = Q(FTV + a, nm[d]);
                TRp[d][a] = cP * upn - sP * vpn;     TIp[d][a] = cP * vpn + sP * upn;
                TRm[d][a] = cM * umn + sM * vmn;     TIm[d][a] = cM * vmn - sM * umn;
                TRp[d][3 + a] = cP * tpn - sP * wpn; TIp[d][3 + a] = cP * wpn + sP * tpn;
                TRm[d][3 + a] = cM * tmn + sM * wmn; TIm[d][3 + a] = cM * wmn - sM * tmn;
                tup[d][a] = tpn; tvp[d][a] = wpn;
            }
        }
        const double s2_0 = fu[0] * fu[0] + fv[0] * fv[0];
        const double s2_1 = fu[1] * fu[1] + fv[1] * fv[1];
        const double s2_2 = fu[2] * fu[2] + fv[2] * fv[2];
        const double sp = s2_0 * s2_1 * s2_2;
        const double den = 1.0 + c.kappa * sp;
        const double Vp = 0.5 * c.mu / (den * den);
        const double prod_rest[3] = {s2_1 * s2_2, s2_0 * s2_2, s2_0 * s2_1};
        const double hh = c.higgs ? s.H[idx] * s.H[idx] : 0.0;
        double DcU[3][6], DcV[3][6];
        #pragma unroll
        for (int d = 0; d < 3; d++)
            #pragma unroll
            for (int f = 0; f < 6; f++) {
                DcU[d][f] = (TRp[d][f] - TRm[d][f]) * c.idx1;
                DcV[d][f] = (TIp[d][f] - TIm[d][f]) * c.idx1;
            }
        const int ci1[3] = {1, 2, 0}, ci2[3] = {2, 0, 1};
        #pragma unroll
        for (int a = 0; a < 3; a++) {
            const int d1 = ci1[a], d2 = ci2[a];
            const double reDxT = DcU[d1][3 + ci2[a]] - DcU[d2][3 + ci1[a]];
            const double imDxT = DcV[d1][3 + ci2[a]] - DcV[d2][3 + ci1[a]];
            const double reDxP = DcU[d1][ci2[a]] - DcU[d2][ci1[a]];
            const double imDxP = DcV[d1][ci2[a]] - DcV[d2][ci1[a]];
            const double lapU_P = (TRp[0][a] + TRm[0][a] + TRp[1][a] + TRm[1][a] + TRp[2][a] + TRm[2][a] - 6.0 * fu[a]) * c.idx2;
            const double lapV_P = (TIp[0][a] + TIm[0][a] + TIp[1][a] + TIm[1][a] + TIp[2][a] + TIm[2][a] - 6.0 * fv[a]) * c.idx2;
            const double lapU_T = (TRp[0][3 + a] + TRm[0][3 + a] + TRp[1][3 + a] + TRm[1][3 + a] + TRp[2][3 + a] +
                                   TRm[2][3 + a] - 6.0 * fu[3 + a]) * c.idx2;
            const double lapV_T = (TIp[0][3 + a] + TIm[0][3 + a] + TIp[1][3 + a] + TIm[1][3 + a] + TIp[2][3 + a] +
                                   TIm[2][3 + a] - 6.0 * fv[3 + a]) * c.idx2;
            s.A[(FU + a) * N3 + idx] = lapU_P - c.m2 * fu[a] - 2.0 * Vp * fu[a] * prod_rest[a] + c.eta * reDxT -
                                       c.hkap * hh * fu[a] * prod_rest[a];
            s.A[(FV + a) * N3 + idx] = lapV_P - c.m2 * fv[a] - 2.0 * Vp * fv[a] * prod_rest[a] + c.eta * imDxT -
                                       c.hkap * hh * fv[a] * prod_rest[a];
            s.A[(FTU + a) * N3 + idx] = lapU_T - c.mtheta2 * fu[3 + a] + c.eta * reDxP;
            s.A[(FTV + a) * N3 + idx] = lapV_T - c.mtheta2 * fv[3 + a] + c.eta * imDxP;
        }
        if (c.higgs) {
            const double *H = s.H;
            const double lapH = (H[np[0]] + H[nm[0]] + H[np[1]] + H[nm[1]] + H[np[2]] + H[nm[2]] - 6.0 * H[idx]) * c.idx2;
            const double h = H[idx];
            s.HA[idx] = lapH - c.hlam * h * (h * h - c.hv * c.hv) - c.hkap * sp * h;
        }
        const double *PS = s.PS;
        double st[3];
        st[0] = (PS[0 * N3 + idx] - PS[0 * N3 + nm[1]]) - (PS[2 * N3 + idx] - PS[2 * N3 + nm[2]]);
        st[1] = -(PS[0 * N3 + idx] - PS[0 * N3 + nm[0]]) + (PS[1 * N3 + idx] - PS[1 * N3 + nm[2]]);
        st[2] = (PS[2 * N3 + idx] - PS[2 * N3 + nm[0]]) - (PS[1 * N3 + idx] - PS[1 * N3 + nm[1]]);
        double st2[3] = {0, 0, 0};
        if (c.g2on) {
            const double *P2 = s.PS2;
            st2[0] = (P2[0 * N3 + idx] - P2[0 * N3 + nm[1]]) - (P2[2 * N3 + idx] - P2[2 * N3 + nm[2]]);
            st2[1] = -(P2[0 * N3 + idx] - P2[0 * N3 + nm[0]]) + (P2[1 * N3 + idx] - P2[1 * N3 + nm[2]]);
            st2[2] = (P2[2 * N3 + idx] - P2[2 * N3 + nm[0]]) - (P2[1 * N3 + idx] - P2[1 * N3 + nm[1]]);
        }
        #pragma unroll
        for (int d = 0; d < 3; d++) {
            const double cP = s.LC[d * N3 + idx], sP = s.LS[d * N3 + idx];
            double Jg = 0.0;
            #pragma unroll
            for (int a = 0; a < 3; a++) {
                Jg += fu[a] * TIp[d][a] - fv[a] * TRp[d][a];
                Jg += fu[3 + a] * TIp[d][3 + a] - fv[3 + a] * TRp[d][3 + a];
            }
            const int d1 = ci1[d], d2 = ci2[d];
            const double WpR1 = cP * fu[d2] + sP * fv[d2], WpI1 = cP * fv[d2] - sP * fu[d2];
            const double WpR2 = cP * fu[d1] + sP * fv[d1], WpI2 = cP * fv[d1] - sP * fu[d1];
            const double T12 = (fu[3 + d1] * TIp[d][d2] - fv[3 + d1] * TRp[d][d2]) + (tup[d][d1] * WpI1 - tvp[d][d1] * WpR1);
            const double T21 = (fu[3 + d2] * TIp[d][d1] - fv[3 + d2] * TRp[d][d1]) + (tup[d][d2] * WpI2 - tvp[d][d2] * WpR2);
            const double Jlat = c.inva * Jg - 0.5 * c.eta * (T12 - T21);
            s.A[(FTH + d) * N3 + idx] = c.stp * st[d] + c.g * Jlat;
            if (c.g2on) {
                double Jg2 = 0.0;
                #pragma unroll
                for (int a = 0; a < 3; a++) {
                    Jg2 += c.q[a] * (fu[a] * TIp[d][a] - fv[a] * TRp[d][a]);
                    Jg2 += c.q[a] * (fu[3 + a] * TIp[d][3 + a] - fv[3 + a] * TRp[d][3 + a]);
                }
                s.K2[d * N3 + idx] = c.stp2 * st2[d] + c.g2 * c.inva * Jg2;
            }
        }
    }
}

// sponge factor of apply_damping at a site (1 outside the sponge)
__device__ __forceinline__ double sponge_factor(int N, double L, double dx, double width, double rate, long long idx) {
    int i, j, k;
    site_ijk(idx, N, &i, &j, &k);
    const double x = -L + i * dx, y = -L + j * dx, z = -L + k * dx;
    const double r = sqrt(x * x + y * y + z * z);
    const double Rd = L - width;
    if (!(r > Rd)) return 1.0;
    double sc = (r - Rd) / width;
    if (sc > 1) sc = 1;
    return 1.0 - rate * sc * sc;
}

// stage 4 kick: momenta, E, E2, Hdot += dt/2 * accelerations; then stage 5
// (apply_damping, :1440-1473): the matter momenta and E are damped in the
// sponge (not E2, not Hdot)
__global__ void __launch_bounds__(kRedThreads) gext_kick_damp_kernel(GextState s, GextConsts c) {
    const long long N3 = c.N3;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int f = 0; f < 15; f++) s.S[f * N3 + idx] += c.hdt * s.A[f * N3 + idx];
        if (c.g2on)
#pragma unroll
            for (int d = 0; d < 3; d++) s.E2[d * N3 + idx] += c.hdt * s.K2[d * N3 + idx];
        if (c.higgs) s.HV[idx] += c.hdt * s.HA[idx];
        if (c.damp) {
            const double dmp = sponge_factor(c.N, c.L, c.dx, c.damp_width, c.damp_rate, idx);
            if (dmp != 1.0)
#pragma unroll
                for (int f = 0; f < 15; f++) s.S[f * N3 + idx] *= dmp;
        }
    }
}

// stage 1 kick and stage 2 drift of the matter, the wrapped links of both
// gauges, and H, in one sweep (each site's drift needs only its own kicked
// momenta, kept in registers).  PREV: the previous step's stage 4 kick and
// stage 5 sponge come first, with the same accelerations, in the same
// operation order as two separate sweeps.
template <bool PREV>
__global__ void __launch_bounds__(kRedThreads) gext_kick_drift_kernel(GextState s, GextConsts c) {
    const long long N3 = c.N3;
    const double twopi = 2.0 * 3.14159265358979323846;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        double v[15];
        const double dmp = (PREV && c.damp) ? sponge_factor(c.N, c.L, c.dx, c.damp_width, c.damp_rate, idx) : 1.0;
#pragma unroll
        for (int f = 0; f < 15; f++) {
            const double a = s.A[f * N3 + idx];
            double w = s.S[f * N3 + idx];
            if (PREV) {
                w = w + c.hdt * a;
                if (dmp != 1.0) w *= dmp;
            }
            v[f] = w + c.hdt * a;
            s.S[f * N3 + idx] = v[f];
        }
#pragma unroll
        for (int f = 0; f < 12; f++) s.X[f * N3 + idx] += c.dt * v[f];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double w = s.X[(FTH + d) * N3 + idx] + c.gad * v[FTH + d];
            s.X[(FTH + d) * N3 + idx] = w - twopi * rint(w / twopi);
        }
        if (c.g2on) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const double k2 = s.K2[d * N3 + idx];
                double e2 = s.E2[d * N3 + idx];
                if (PREV) e2 = e2 + c.hdt * k2;
                e2 = e2 + c.hdt * k2;
                s.E2[d * N3 + idx] = e2;
                const double w = s.T2[d * N3 + idx] + c.gad2 * e2;
                s.T2[d * N3 + idx] = w - twopi * rint(w / twopi);
            }
        }
        if (c.higgs) {
            const double ha = s.HA[idx];
            double hv = s.HV[idx];
            if (PREV) hv = hv + c.hdt * ha;
            hv = hv + c.hdt * ha;
            s.HV[idx] = hv;
            s.H[idx] += c.dt * hv;
        }
    }
}

// Higgs energy density (:1970-1975), summed into E_total by the reference
__global__ void __launch_bounds__(256) gext_higgs_energy_kernel(GextState s, GextConsts c, double *part) {
    __shared__ double scratch[32];
    double S[1] = {0.0}, M[1] = {0.0};
    const long long N3 = c.N3;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        long long np[3], nm[3];
        gext_nb(idx, c.N, np, nm);
        double sp = 1.0;
        for (int a = 0; a < 3; a++) {
            const double u = s.X[(FU + a) * N3 + idx], v = s.X[(FV + a) * N3 + idx];
            sp *= u * u + v * v;
        }
        const double *H = s.H;
        const double h = H[idx], hv = s.HV[idx];
        const double gx = (H[np[0]] - H[nm[0]]) * c.idx1, gy = (H[np[1]] - H[nm[1]]) * c.idx1;
        const double gz = (H[np[2]] - H[nm[2]]) * c.idx1;
        const double hd = h * h - c.hv * c.hv;
        S[0] += (0.5 * hv * hv + 0.5 * (gx * gx + gy * gy + gz * gz) + 0.25 * c.hlam * hd * hd + 0.5 * c.hkap * sp * h * h) *
                c.dV;
    }
    block_fold<1, 0>(S, M, scratch, part);
}

// Higgs start value (the reference's main, scp_sim.c:2802-2817): the VEV, or
// a central cavity of radius rvoid with a tanh wall of width 0.6
__global__ void gext_higgs_init_kernel(GextState s, GextConsts c, double rvoid) {
    const long long N3 = c.N3;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        double h = c.hv;
        if (rvoid > 0.0) {
            int i, j, k;
            site_ijk(idx, c.N, &i, &j, &k);
            const double x = -c.L + i * c.dx, y = -c.L + j * c.dx, z = -c.L + k * c.dx;
            const double r = sqrt(x * x + y * y + z * z);
            h = c.hv * 0.5 * (1.0 + tanh((r - rvoid) / 0.6));
        }
        s.H[idx] = h;
        s.HV[idx] = 0.0;
    }
}

// second-gauge Gauss residual div E2 - g2 sum_a q_a rho_a (:2387-2396) and
// the E2 correction of its projection (:2452-2455)
__global__ void __launch_bounds__(256) gext_gauss2_rhs_kernel(GextState s, GextConsts c, double *b, double *part) {
    __shared__ double scratch[32];
    double S[1] = {0.0}, M[1] = {0.0};
    const long long N3 = c.N3;
    const double *X = s.X, *V = s.S;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        long long np[3], nm[3];
        gext_nb(idx, c.N, np, nm);
        const double *E = s.E2;
        const double divE = (E[idx] - E[nm[0]] + E[N3 + idx] - E[N3 + nm[1]] + E[2 * N3 + idx] - E[2 * N3 + nm[2]]) / c.dx;
        double rho = 0;
        for (int a = 0; a < 3; a++)
            rho += c.q[a] * (X[(FU + a) * N3 + idx] * V[(FV + a) * N3 + idx] - X[(FV + a) * N3 + idx] * V[(FU + a) * N3 + idx] +
                             X[(FTU + a) * N3 + idx] * V[(FTV + a) * N3 + idx] -
                             X[(FTV + a) * N3 + idx] * V[(FTU + a) * N3 + idx]);
        const double G = divE - c.g2 * rho;
        b[idx] = G;
        S[0] += G;
    }
    block_fold<1, 0>(S, M, scratch, part);
}

__global__ void gext_gauss2_correct_kernel(GextState s, GextConsts c, const double *x, const double *cg) {
    const long long N3 = c.N3;
    const double xbar = cg[CG_XBAR];
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        long long np[3], nm[3];
        gext_nb(idx, c.N, np, nm);
        const double c0 = x[idx] - xbar;
        for (int d = 0; d < 3; d++) s.E2[d * N3 + idx] += ((x[np[d]] - xbar) - c0) / c.dx;
    }
}

}  // namespace scp
