// real.cuh -- the real 6-field stepper with the reference's optional terms:
// mass modes 1 (inverse, m_eff^2 = inv_alpha/(1 + inv_beta*|phi|^2)) and 3
// (density-dependent kappa), Cosserat strain alpha_cs |curl(phi)/2 - theta|^2,
// curl-squared hardening (beta_h/2)|theta|^2 |curl phi|^2 and chiral helicity
// kappa_h P^2 phi.curl(phi) (compute_forces, sfa/sim/scp_sim.c:743-929;
// compute_energy, :1722-1801; theta_rms / P_integrated, :1803-1816).
//
// The terms in alpha_cs and beta_h take the curl of fields that contain
// curl(phi), i.e. a two-site stencil, which the reference evaluates in two
// passes over scratch arrays (mismatch M and hardening vector Q).  This path
// does the same with plain per-site kernels over global memory, in the
// reference's arithmetic order; one step is a kick+drift sweep, the scratch
// pass (when alpha_cs or beta_h is set), the force pass and a kick+sponge
// sweep.  The default-term real mode runs on the fused kernels instead.
//
// Field slots of the 6-field state: 0..2 phi_a, 3..5 theta_a (positions x,
// velocities v, accelerations a; scratch mq: 0..2 M_a, 3..5 Q_a).
#pragma once
#include "reduce.cuh"

namespace scp {

struct RealConsts {
    int N;
    long long N3;
    double L, dx, dV, idx1, idx2, hdt, dt;
    double mu, kappa, m2, mtheta2, eta;
    double kh, acs, bh, kg, ia, ib;
    int mode;
    int damp;
    double damp_width, damp_rate;
};

struct RealNb {
    long long ip, im, jp, jm, kp, km;
};

__device__ __forceinline__ RealNb real_nb(long long idx, int N, int *i_, int *j_, int *k_) {
    const long long NN = (long long)N * N;
    int i, j, k;
    site_ijk(idx, N, &i, &j, &k);
    RealNb n;
    n.ip = (long long)wrapi(i + 1, N) * NN + (long long)j * N + k;
    n.im = (long long)wrapi(i - 1, N) * NN + (long long)j * N + k;
    n.jp = (long long)i * NN + (long long)wrapi(j + 1, N) * N + k;
    n.jm = (long long)i * NN + (long long)wrapi(j - 1, N) * N + k;
    n.kp = (long long)i * NN + (long long)j * N + wrapi(k + 1, N);
    n.km = (long long)i * NN + (long long)j * N + wrapi(k - 1, N);
    *i_ = i; *j_ = j; *k_ = k;
    return n;
}

// curl component a of the 3-vector field F (F[c] at F + c*N3), central
// differences (curl_component, scp_sim.c:409-415)
__device__ __forceinline__ double real_curl(const double *F, long long N3, int a, const RealNb &n, double idx1) {
    const double *F0 = F, *F1 = F + N3, *F2 = F + 2 * N3;
    if (a == 0) return (F2[n.jp] - F2[n.jm] - F1[n.kp] + F1[n.km]) * idx1;
    if (a == 1) return (F0[n.kp] - F0[n.km] - F2[n.ip] + F2[n.im]) * idx1;
    return (F1[n.ip] - F1[n.im] - F0[n.jp] + F0[n.jm]) * idx1;
}

// pass 1: M_a = curl(phi)_a/2 - theta_a, Q_a = (beta/2)|theta|^2 curl(phi)_a
__global__ void real_pass1_kernel(const double *x, double *mq, RealConsts c) {
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < c.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        const RealNb n = real_nb(idx, c.N, &i, &j, &k);
        const double cp0 = real_curl(x, c.N3, 0, n, c.idx1);
        const double cp1 = real_curl(x, c.N3, 1, n, c.idx1);
        const double cp2 = real_curl(x, c.N3, 2, n, c.idx1);
        const double *th = x + 3 * c.N3;
        if (c.acs != 0) {
            mq[0 * c.N3 + idx] = cp0 * 0.5 - th[0 * c.N3 + idx];
            mq[1 * c.N3 + idx] = cp1 * 0.5 - th[1 * c.N3 + idx];
            mq[2 * c.N3 + idx] = cp2 * 0.5 - th[2 * c.N3 + idx];
        }
        if (c.bh != 0) {
            const double t0 = th[idx], t1 = th[c.N3 + idx], t2 = th[2 * c.N3 + idx];
            const double T2 = t0 * t0 + t1 * t1 + t2 * t2;
            const double coeff = 0.5 * c.bh * T2;
            mq[3 * c.N3 + idx] = coeff * cp0;
            mq[4 * c.N3 + idx] = coeff * cp1;
            mq[5 * c.N3 + idx] = coeff * cp2;
        }
    }
}

// pass 2: accelerations of phi and theta (scp_sim.c:789-925)
__global__ void real_force_kernel(const double *x, const double *mq, double *acc, RealConsts c) {
    const long long N3 = c.N3;
    const double *ph = x, *th = x + 3 * N3;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        const RealNb n = real_nb(idx, c.N, &i, &j, &k);
        const double p0 = ph[idx], p1 = ph[N3 + idx], p2 = ph[2 * N3 + idx];
        const double sig = p0 * p0 + p1 * p1 + p2 * p2;
        const double me2 = (c.mode == 1) ? c.ia / (1.0 + c.ib * sig) : c.m2;
        const double keff = (c.mode == 3) ? c.kappa / (1.0 + c.kg * sig) : c.kappa;
        const double P = p0 * p1 * p2, P2 = P * P;
        const double den = 1.0 + keff * P2;
        const double dVdP = c.mu * P / (den * den);
        double t2c = 0;
        if (c.mode == 3 && c.kg > 0) {
            const double D = 1.0 + c.kg * sig + c.kappa * P2;
            t2c = c.mu * c.kg * c.kappa * P2 * P2 / (D * D);
        }
        double curl_phi[3];
        for (int a = 0; a < 3; a++) curl_phi[a] = real_curl(ph, N3, a, n, c.idx1);
        const double h = p0 * curl_phi[0] + p1 * curl_phi[1] + p2 * curl_phi[2];
        double dP2dx = 0, dP2dy = 0, dP2dz = 0;
        if (c.kh != 0) {
            auto Pat = [&](long long y) { return ph[y] * ph[N3 + y] * ph[2 * N3 + y]; };
            const double Pip = Pat(n.ip), Pim = Pat(n.im), Pjp = Pat(n.jp), Pjm = Pat(n.jm);
            const double Pkp = Pat(n.kp), Pkm = Pat(n.km);
            dP2dx = (Pip * Pip - Pim * Pim) * c.idx1;
            dP2dy = (Pjp * Pjp - Pjm * Pjm) * c.idx1;
            dP2dz = (Pkp * Pkp - Pkm * Pkm) * c.idx1;
        }
        double curl_M[3] = {0, 0, 0}, curl_Q[3] = {0, 0, 0};
        if (c.acs != 0)
            for (int a = 0; a < 3; a++) curl_M[a] = real_curl(mq, N3, a, n, c.idx1);
        if (c.bh != 0)
            for (int a = 0; a < 3; a++) curl_Q[a] = real_curl(mq + 3 * N3, N3, a, n, c.idx1);
        const double curl_sq = curl_phi[0] * curl_phi[0] + curl_phi[1] * curl_phi[1] + curl_phi[2] * curl_phi[2];
        for (int a = 0; a < 3; a++) {
            const double *F = ph + a * N3;
            const double lap = (F[n.ip] + F[n.im] + F[n.jp] + F[n.jm] + F[n.kp] + F[n.km] - 6.0 * F[idx]) * c.idx2;
            const double dPda = (a == 0) ? p1 * p2 : (a == 1) ? p0 * p2 : p0 * p1;
            const double ct = real_curl(th, N3, a, n, c.idx1);
            double chiral = 0;
            if (c.kh != 0) {
                const double t1 = 2.0 * P * dPda * h;
                const double t2 = 2.0 * P2 * curl_phi[a];
                double t3;
                if (a == 0) t3 = -(dP2dz * p1 - dP2dy * p2);
                else if (a == 1) t3 = -(dP2dx * p2 - dP2dz * p0);
                else t3 = -(dP2dy * p0 - dP2dx * p1);
                chiral = c.kh * (t1 + t2 + t3);
            }
            const double cosserat_phi = -c.acs * curl_M[a];
            const double harden_phi = -2.0 * curl_Q[a];
            acc[a * N3 + idx] = lap - me2 * F[idx] - dVdP * dPda - t2c * F[idx] + c.eta * ct + chiral + cosserat_phi +
                                harden_phi;
        }
        for (int a = 0; a < 3; a++) {
            const double *T = th + a * N3;
            const double lapt = (T[n.ip] + T[n.im] + T[n.jp] + T[n.jm] + T[n.kp] + T[n.km] - 6.0 * T[idx]) * c.idx2;
            const double cp = curl_phi[a];
            const double cosserat_theta = (c.acs != 0) ? 2.0 * c.acs * mq[a * N3 + idx] : 0.0;
            const double harden_theta = -c.bh * curl_sq * T[idx];
            acc[(3 + a) * N3 + idx] = lapt - c.mtheta2 * T[idx] + c.eta * cp + cosserat_theta + harden_theta;
        }
    }
}

// stages 1-2 of verlet_step (scp_sim.c:1583-1640): v += dt/2 a, x += dt v
__global__ void real_kick_drift_kernel(double *x, double *v, const double *acc, RealConsts c) {
    const long long n = 6 * c.N3;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const double vv = v[q] + c.hdt * acc[q];
        v[q] = vv;
        x[q] = x[q] + c.dt * vv;
    }
}

// stages 4-5: v += dt/2 a, then the absorbing sponge (apply_damping, :1440-1473)
__global__ void real_kick_damp_kernel(double *v, const double *acc, RealConsts c) {
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < c.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        double d = 1.0;
        if (c.damp) {
            int i, j, k;
            site_ijk(idx, c.N, &i, &j, &k);
            const double xx = -c.L + i * c.dx, yy = -c.L + j * c.dx, zz = -c.L + k * c.dx;
            const double r = sqrt(xx * xx + yy * yy + zz * zz);
            const double Rd = c.L - c.damp_width;
            if (r > Rd) {
                double s = (r - Rd) / c.damp_width;
                if (s > 1) s = 1;
                d = 1.0 - c.damp_rate * s * s;
            }
        }
        for (int f = 0; f < 6; f++) {
            double vv = v[f * c.N3 + idx] + c.hdt * acc[f * c.N3 + idx];
            if (d != 1.0) vv *= d;
            v[f * c.N3 + idx] = vv;
        }
    }
}

// energy sums (compute_energy, :1722-1801), P_integrated and theta^2 for theta_rms
enum : int { RS_EPK = 0, RS_ETK, RS_EG, RS_EM, RS_EP, RS_ETG, RS_ETM, RS_EC, RS_PINT, RS_TH2, RS_NSUM };
enum : int { RM_PM = 0, RM_PMAX, RM_NMAX };

__global__ void __launch_bounds__(kRedThreads) real_energy_kernel(const double *x, const double *v, RealConsts c,
                                                                  double *part) {
    __shared__ double scratch[(RS_NSUM + RM_NMAX) * 32];
    double S[RS_NSUM], M[RM_NMAX];
    for (int q = 0; q < RS_NSUM; q++) S[q] = 0.0;
    for (int q = 0; q < RM_NMAX; q++) M[q] = 0.0;
    const long long N3 = c.N3;
    const double *ph = x, *th = x + 3 * N3;
    const double dV = c.dV;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        const RealNb n = real_nb(idx, c.N, &i, &j, &k);
        const double p0 = ph[idx], p1 = ph[N3 + idx], p2 = ph[2 * N3 + idx];
        const double sig = p0 * p0 + p1 * p1 + p2 * p2;
        const double me2 = (c.mode == 1) ? c.ia / (1.0 + c.ib * sig) : c.m2;
        const double keff = (c.mode == 3) ? c.kappa / (1.0 + c.kg * sig) : c.kappa;
        for (int a = 0; a < 3; a++) {
            const double *F = ph + a * N3, *T = th + a * N3;
            const double vp = v[a * N3 + idx], vt = v[(3 + a) * N3 + idx];
            S[RS_EPK] += 0.5 * vp * vp * dV;
            S[RS_ETK] += 0.5 * vt * vt * dV;
            const double gx = (F[n.ip] - F[n.im]) * c.idx1, gy = (F[n.jp] - F[n.jm]) * c.idx1;
            const double gz = (F[n.kp] - F[n.km]) * c.idx1;
            S[RS_EG] += 0.5 * (gx * gx + gy * gy + gz * gz) * dV;
            S[RS_EM] += 0.5 * me2 * F[idx] * F[idx] * dV;
            const double tgx = (T[n.ip] - T[n.im]) * c.idx1, tgy = (T[n.jp] - T[n.jm]) * c.idx1;
            const double tgz = (T[n.kp] - T[n.km]) * c.idx1;
            S[RS_ETG] += 0.5 * (tgx * tgx + tgy * tgy + tgz * tgz) * dV;
            S[RS_ETM] += 0.5 * c.mtheta2 * T[idx] * T[idx] * dV;
            M[RM_PM] = fmax(M[RM_PM], fabs(F[idx]));
            S[RS_TH2] += T[idx] * T[idx];
        }
        const double P = p0 * p1 * p2, P2 = P * P;
        if (c.mode == 3) {
            const double D = 1.0 + c.kg * sig + c.kappa * P2;
            S[RS_EP] += (c.mu / 2.0) * P2 * (1.0 + c.kg * sig) / D * dV;
        } else {
            S[RS_EP] += (c.mu / 2.0) * P2 / (1.0 + keff * P2) * dV;
        }
        M[RM_PMAX] = fmax(M[RM_PMAX], fabs(P));
        S[RS_PINT] += fabs(P) * dV;
        if (c.acs != 0 || c.bh != 0 || c.kh != 0) {
            const double cx0 = real_curl(ph, N3, 0, n, c.idx1), cx1 = real_curl(ph, N3, 1, n, c.idx1);
            const double cx2 = real_curl(ph, N3, 2, n, c.idx1);
            if (c.acs != 0) {
                const double m0 = cx0 * 0.5 - th[idx], m1 = cx1 * 0.5 - th[N3 + idx], m2c = cx2 * 0.5 - th[2 * N3 + idx];
                S[RS_EP] += c.acs * (m0 * m0 + m1 * m1 + m2c * m2c) * dV;
            }
            if (c.bh != 0) {
                const double csq = cx0 * cx0 + cx1 * cx1 + cx2 * cx2;
                const double T2 = th[idx] * th[idx] + th[N3 + idx] * th[N3 + idx] + th[2 * N3 + idx] * th[2 * N3 + idx];
                S[RS_EP] += 0.5 * c.bh * T2 * csq * dV;
            }
            if (c.kh != 0) {
                const double hel = p0 * cx0 + p1 * cx1 + p2 * cx2;
                S[RS_EP] += c.kh * P2 * hel * dV;
            }
        }
        for (int a = 0; a < 3; a++) {
            const double ct = real_curl(th, N3, a, n, c.idx1);
            S[RS_EC] -= c.eta * ph[a * N3 + idx] * ct * dV;
        }
    }
    block_fold<RS_NSUM, RM_NMAX>(S, M, scratch, part);
}

}  // namespace scp
