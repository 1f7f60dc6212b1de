// mf.cuh -- the gauged stepper with three matter fabrics C, Q, L under one
// shared compact U(1) (the reference's multi-fabric "B1 shape beta"):
// every fabric is a full complex 12-field Cosserat multiplet with its own bag
// potential, transported by the charge-q_f links exp(i q_f th); the E kick
// is the staple term plus sum_f g q_f J_f (force_fabric_gauged_accum and
// compute_forces_complex_gauge_mf, sfa/sim/scp_sim.c:1274-1433); the Gauss
// law and the net-charge check use rho_em = sum_f q_f rho_f (em_rho_at,
// :184-197).  With the C-Q lock (mf_lock_CQ) Q is C at every step boundary
// (the reference copies C into Q after each force evaluation and kick,
// :169-172, :1680): here Q's arrays simply alias C's, which gives the same
// state, the same Q acceleration (the q_Q pass over C's fields writes C's
// acceleration last, as in the reference) and the same charges.
//
// FP64 per-site kernels over global memory in the reference's arithmetic
// order.  C holds the packed 15-field layout of the fused kernels (matter,
// then th / E), Q and L the first 12 fields of it.
#pragma once
#include "common.cuh"
#include "gauss.cuh"
#include "reduce.cuh"
#include "gext.cuh"
#include "trig.cuh"

namespace scp {

struct MfConsts {
    int N;
    long long N3;
    double L, dx, dV, idx1, idx2, inva, hdt, dt;
    double mu, kappa, m2, mtheta2, eta;
    double g, stp, gad;
    double q[3];           // EM weights q_C, q_Q, q_L
    int lock;              // Q aliases C
    int damp;
    double damp_width, damp_rate;
    double Rint2, G_offset;
};

struct MfState {
    double *XC, *SC, *AC;  // 15 fields each: C matter, th (X) / E (S) / E_acc (A)
    double *XQ, *SQ, *AQ;  // 12 fields each (= the C pointers when locked)
    double *XL, *SL, *AL;  // 12 fields each
    double *PS;            // plaquette sines, 3 planes
};

// Read-only diagnostic view of fabric L with the shared links of C
// (compute_energy_complex_gauge's L block, scp_sim.c:1977-2028, transports L
// with the unit-charge links)
struct ViewFab {
    const double *XF, *SF, *XC, *SC;
    long long N3;
    __device__ __forceinline__ double q(int f, long long i) const { return f < 12 ? XF[f * N3 + i] : XC[f * N3 + i]; }
    __device__ __forceinline__ double p(int f, long long i) const { return f < 12 ? SF[f * N3 + i] : SC[f * N3 + i]; }
};

__device__ __forceinline__ double mf_rho(const double *X, const double *S, long long N3, long long idx) {
    double r = 0.0;
    for (int a = 0; a < 3; a++)
        r += X[(FU + a) * N3 + idx] * S[(FV + a) * N3 + idx] - X[(FV + a) * N3 + idx] * S[(FU + a) * N3 + idx] +
             X[(FTU + a) * N3 + idx] * S[(FTV + a) * N3 + idx] - X[(FTV + a) * N3 + idx] * S[(FTU + a) * N3 + idx];
    return r;
}

__device__ __forceinline__ double mf_rho_em(const MfState &s, const MfConsts &c, long long idx) {
    return c.q[0] * mf_rho(s.XC, s.SC, c.N3, idx) + c.q[1] * mf_rho(s.XQ, s.SQ, c.N3, idx) +
           c.q[2] * mf_rho(s.XL, s.SL, c.N3, idx);
}

__device__ __forceinline__ double mf_gauss_at(const MfState &s, const MfConsts &c, long long idx, const long long nm[3]) {
    const double *E = s.SC + FTH * c.N3;
    const long long N3 = c.N3;
    const double divE = (E[idx] - E[nm[0]] + E[N3 + idx] - E[N3 + nm[1]] + E[2 * N3 + idx] - E[2 * N3 + nm[2]]) / c.dx;
    return divE - c.g * mf_rho_em(s, c, idx);
}

// One fabric's matter accelerations (written to A when A is not null) and
// its lattice current J_lat per direction, with charge-q links
// (force_fabric_gauged_accum's site body, scp_sim.c:1292-1381).
__device__ __forceinline__ void mf_fabric_site(const double *Xf, double *A, const double *th, double q, long long idx,
                                            const long long np[3], const long long nm[3], const MfConsts &c,
                                            double Jlat[3]) {
    const long long N3 = c.N3;
    double fu[6], fv[6];
    #pragma unroll
    for (int a = 0; a < 3; a++) {
        fu[a] = Xf[(FU + a) * N3 + idx]; fv[a] = Xf[(FV + a) * N3 + idx];
        fu[3 + a] = Xf[(FTU + a) * N3 + idx]; fv[3 + a] = Xf[(FTV + a) * N3 + idx];
    }
    double TRp[3][6], TIp[3][6], TRm[3][6], TIm[3][6];
    double tup[3][3], tvp[3][3], cPd[3], sPd[3];
    #pragma unroll
    for (int d = 0; d < 3; d++) {
        double cP, sP, cM, sM;
        sincos_any(q * th[d * N3 + idx], &sP, &cP);
        sincos_any(q * th[d * N3 + nm[d]], &sM, &cM);
        cPd[d] = cP; sPd[d] = sP;
        #pragma unroll
        for (int a = 0; a < 3; a++) {
            const double upn = Xf[(FU + a) * N3 + np[d]], vpn = Xf[(FV + a) * N3 + np[d]];
            const double umn = Xf[(FU + a) * N3 + nm[d]], vmn = Xf[(FV + a) * N3 + nm[d]];
            const double tpn = Xf[(FTU + a) * N3 + np[d]], wpn = Xf[(FTV + a) * N3 + np[d]];
            const double tmn = Xf[(FTU + a) * N3 + nm[d]], wmn = Xf[(FTV + a) * N3 + nm[d]];
            TRp[d][a] = cP * upn - sP * vpn;     TIp[d][a] = cP * vpn + sP * upn;
            TRm[d][a] = cM * umn + sM * vmn;     TIm[d][a] = cM * vmn - sM * umn;
            TRp[d][3 + a] = cP * tpn - sP * wpn; TIp[d][3 + a] = cP * wpn + sP * tpn;
            TRm[d][3 + a] = cM * tmn + sM * wmn; TIm[d][3 + a] = cM * wmn - sM * tmn;
            tup[d][a] = tpn; tvp[d][a] = wpn;
        }
    }
    const int ci1[3] = {1, 2, 0}, ci2[3] = {2, 0, 1};
    if (A) {
        const double s2_0 = fu[0] * fu[0] + fv[0] * fv[0];
        const double s2_1 = fu[1] * fu[1] + fv[1] * fv[1];
        const double s2_2 = fu[2] * fu[2] + fv[2] * fv[2];
        const double sp = s2_0 * s2_1 * s2_2;
        const double den = 1.0 + c.kappa * sp;
        const double Vp = 0.5 * c.mu / (den * den);
        const double prod_rest[3] = {s2_1 * s2_2, s2_0 * s2_2, s2_0 * s2_1};
        double DcU[3][6], DcV[3][6];
        #pragma unroll
        for (int d = 0; d < 3; d++)
            #pragma unroll
            for (int f = 0; f < 6; f++) {
                DcU[d][f] = (TRp[d][f] - TRm[d][f]) * c.idx1;
                DcV[d][f] = (TIp[d][f] - TIm[d][f]) * c.idx1;
            }
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
            A[(FU + a) * N3 + idx] = lapU_P - c.m2 * fu[a] - 2.0 * Vp * fu[a] * prod_rest[a] + c.eta * reDxT;
            A[(FV + a) * N3 + idx] = lapV_P - c.m2 * fv[a] - 2.0 * Vp * fv[a] * prod_rest[a] + c.eta * imDxT;
            A[(FTU + a) * N3 + idx] = lapU_T - c.mtheta2 * fu[3 + a] + c.eta * reDxP;
            A[(FTV + a) * N3 + idx] = lapV_T - c.mtheta2 * fv[3 + a] + c.eta * imDxP;
        }
    }
    #pragma unroll
    for (int d = 0; d < 3; d++) {
        const double cP = cPd[d], sP = sPd[d];
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
        Jlat[d] = c.inva * Jg - 0.5 * c.eta * (T12 - T21);
    }
}

// plaquette sines of the shared links (pass B, :1405-1416)
__global__ void __launch_bounds__(kRedThreads) mf_plaq_kernel(MfState s, MfConsts c) {
    const long long N3 = c.N3;
    const double *th = s.XC + FTH * N3;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        long long np[3], nm[3];
        gext_nb(idx, c.N, np, nm);
        const int pa[3] = {0, 1, 2}, pb[3] = {1, 2, 0};
        #pragma unroll
        for (int p = 0; p < 3; p++) {
            const int a = pa[p], b = pb[p];
            const double ang = th[a * N3 + idx] + th[b * N3 + np[a]] - th[a * N3 + np[b]] - th[b * N3 + idx];
            double sn, cs;
            sincos_any(ang, &sn, &cs);
            s.PS[p * N3 + idx] = sn;
        }
    }
}

// the three fabric passes and the E kick (:1418-1432): C with q_C sets
// E_acc = staples + g q_C J_C; Q (C's fields when locked) with q_Q and L with
// q_L add their currents.  When locked, the C pass's matter accelerations are
// not stored: the q_Q pass over the same fields overwrites them, as in the
// reference.
__global__ void __launch_bounds__(kRedThreads) mf_force_kernel(MfState s, MfConsts c) {
    const long long N3 = c.N3;
    const double *th = s.XC + FTH * N3;
    const double *PS = s.PS;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        long long np[3], nm[3];
        gext_nb(idx, c.N, np, nm);
        double st[3];
        st[0] = (PS[0 * N3 + idx] - PS[0 * N3 + nm[1]]) - (PS[2 * N3 + idx] - PS[2 * N3 + nm[2]]);
        st[1] = -(PS[0 * N3 + idx] - PS[0 * N3 + nm[0]]) + (PS[1 * N3 + idx] - PS[1 * N3 + nm[2]]);
        st[2] = (PS[2 * N3 + idx] - PS[2 * N3 + nm[0]]) - (PS[1 * N3 + idx] - PS[1 * N3 + nm[1]]);
        double E[3], J[3];
        if (c.lock && c.q[0] == 0.0) {
            // locked with q_C = 0 (the reference's default): the C pass stores
            // nothing (the q_Q pass overwrites C's accelerations) and adds
            // g*0*J_C, so for finite fields it leaves E = staples alone
#pragma unroll
            for (int d = 0; d < 3; d++) E[d] = c.stp * st[d];
        } else {
            mf_fabric_site(s.XC, c.lock ? nullptr : s.AC, th, c.q[0], idx, np, nm, c, J);
#pragma unroll
            for (int d = 0; d < 3; d++) E[d] = c.stp * st[d] + c.g * c.q[0] * J[d];
        }
        mf_fabric_site(s.XQ, s.AQ, th, c.q[1], idx, np, nm, c, J);
        for (int d = 0; d < 3; d++) E[d] += c.g * c.q[1] * J[d];
        mf_fabric_site(s.XL, s.AL, th, c.q[2], idx, np, nm, c, J);
        for (int d = 0; d < 3; d++) E[d] += c.g * c.q[2] * J[d];
        for (int d = 0; d < 3; d++) s.AC[(FTH + d) * N3 + idx] = E[d];
    }
}

// stage 4 kick of every fabric and E (Q skipped when locked), then the
// stage-5 damping of all matter momenta and E in the sponge (:1440-1473)
__global__ void __launch_bounds__(kRedThreads) mf_kick_damp_kernel(MfState s, MfConsts c) {
    const long long N3 = c.N3;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int f = 0; f < 15; f++) s.SC[f * N3 + idx] += c.hdt * s.AC[f * N3 + idx];
        if (!c.lock)
#pragma unroll
            for (int f = 0; f < 12; f++) s.SQ[f * N3 + idx] += c.hdt * s.AQ[f * N3 + idx];
#pragma unroll
        for (int f = 0; f < 12; f++) s.SL[f * N3 + idx] += c.hdt * s.AL[f * N3 + idx];
        if (c.damp) {
            const double dmp = sponge_factor(c.N, c.L, c.dx, c.damp_width, c.damp_rate, idx);
            if (dmp != 1.0) {
#pragma unroll
                for (int f = 0; f < 15; f++) s.SC[f * N3 + idx] *= dmp;
                if (!c.lock)
#pragma unroll
                    for (int f = 0; f < 12; f++) s.SQ[f * N3 + idx] *= dmp;
#pragma unroll
                for (int f = 0; f < 12; f++) s.SL[f * N3 + idx] *= dmp;
            }
        }
    }
}

// one fabric's stage 1 kick and stage 2 drift at one site; PREV: the
// previous step's stage 4 kick and sponge factor dmp first
template <bool PREV>
__device__ __forceinline__ void mf_kick_drift_fabric(double *X, double *S, const double *A, long long N3, long long idx,
                                                     double hdt, double dt, double dmp) {
#pragma unroll
    for (int f = 0; f < 12; f++) {
        const double a = A[f * N3 + idx];
        double w = S[f * N3 + idx];
        if (PREV) {
            w = w + hdt * a;
            if (dmp != 1.0) w *= dmp;
        }
        const double v = w + hdt * a;
        S[f * N3 + idx] = v;
        X[f * N3 + idx] += dt * v;
    }
}

// stage 1 kick and stage 2 drift of every fabric (Q skipped when locked),
// E and the wrapped links, in one sweep; PREV: the previous step's stage 4
// kick and stage 5 sponge first, in the operation order of separate sweeps
template <bool PREV>
__global__ void __launch_bounds__(kRedThreads) mf_kick_drift_kernel(MfState s, MfConsts c) {
    const long long N3 = c.N3;
    const double twopi = 2.0 * 3.14159265358979323846;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        const double dmp = (PREV && c.damp) ? sponge_factor(c.N, c.L, c.dx, c.damp_width, c.damp_rate, idx) : 1.0;
        mf_kick_drift_fabric<PREV>(s.XC, s.SC, s.AC, N3, idx, c.hdt, c.dt, dmp);
        if (!c.lock) mf_kick_drift_fabric<PREV>(s.XQ, s.SQ, s.AQ, N3, idx, c.hdt, c.dt, dmp);
        mf_kick_drift_fabric<PREV>(s.XL, s.SL, s.AL, N3, idx, c.hdt, c.dt, dmp);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double ea = s.AC[(FTH + d) * N3 + idx];
            double e = s.SC[(FTH + d) * N3 + idx];
            if (PREV) {
                e = e + c.hdt * ea;
                if (dmp != 1.0) e *= dmp;
            }
            e = e + c.hdt * ea;
            s.SC[(FTH + d) * N3 + idx] = e;
            const double w = s.XC[(FTH + d) * N3 + idx] + c.gad * e;
            s.XC[(FTH + d) * N3 + idx] = w - twopi * rint(w / twopi);
        }
    }
}

// net-charge sums of rho_em dV and |rho_em| dV (net_charge_check, :2264-2279)
__global__ void __launch_bounds__(kRedThreads) mf_net_charge_kernel(MfState s, MfConsts c, double *part) {
    __shared__ double scratch[2 * 32];
    double S[2] = {0.0, 0.0}, M[1] = {0.0};
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < c.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        const double r = mf_rho_em(s, c, idx);
        S[0] += r * c.dV;
        S[1] += fabs(r) * c.dV;
    }
    block_fold<2, 0>(S, M, scratch, part);
}

// b = G(x) with rho_em (init_gauss_project's right-hand side); partial sums of b
__global__ void __launch_bounds__(kRedThreads) mf_gauss_rhs_kernel(MfState s, MfConsts c, double *b, double *part) {
    __shared__ double scratch[32];
    double S[1] = {0.0}, M[1] = {0.0};
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < c.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        long long np[3], nm[3];
        gext_nb(idx, c.N, np, nm);
        const double G = mf_gauss_at(s, c, idx, nm);
        if (b) b[idx] = G;
        S[0] += G;
    }
    block_fold<1, 0>(S, M, scratch, part);
}

// multi-fabric diagnostics: Gauss norm over the interior with rho_em
// (compute_gauss, :2186-2240) and the per-fabric charges (compute_mf_charges,
// :2247-2261).  Sums: sum (G-OFF)^2, interior count, rho_C, rho_Q, rho_L,
// rho_em; maximum: |G - OFF| over the interior.
enum : int { MS_GL2 = 0, MS_NOM, MS_QC, MS_QQ, MS_QL, MS_QEM, MS_NSUM };
__global__ void __launch_bounds__(kRedThreads) mf_diag_kernel(MfState s, MfConsts c, double *part) {
    __shared__ double scratch[(MS_NSUM + 1) * 32];
    double S[MS_NSUM], M[1] = {0.0};
    for (int q = 0; q < MS_NSUM; q++) S[q] = 0.0;
    const long long N3 = c.N3;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        long long np[3], nm[3];
        gext_nb(idx, c.N, np, nm);
        int i, j, k;
        site_ijk(idx, c.N, &i, &j, &k);
        const double x = -c.L + i * c.dx, y = -c.L + j * c.dx, z = -c.L + k * c.dx;
        const double rc = mf_rho(s.XC, s.SC, N3, idx), rq = mf_rho(s.XQ, s.SQ, N3, idx);
        const double rl = mf_rho(s.XL, s.SL, N3, idx);
        if (x * x + y * y + z * z < c.Rint2) {
            const double G = mf_gauss_at(s, c, idx, nm);
            const double d = fabs(G - c.G_offset);
            if (d > M[0]) M[0] = d;
            S[MS_GL2] += (G - c.G_offset) * (G - c.G_offset);
            S[MS_NOM] += 1.0;
        }
        S[MS_QC] += rc;
        S[MS_QQ] += rq;
        S[MS_QL] += rl;
        S[MS_QEM] += c.q[0] * rc + c.q[1] * rq + c.q[2] * rl;
    }
    block_fold<MS_NSUM, 1>(S, M, scratch, part);
}

}  // namespace scp
