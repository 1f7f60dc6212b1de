// real6.cuh -- the real six-field stepper (phi_a, theta_a real) with the
// reference's optional terms (compute_forces, sfa/sim/scp_sim.c:743-929;
// compute_energy, :1722-1801; theta_rms and P_integrated, :1803-1816):
//
//   mass mode 1    m_eff^2 = inv_alpha / (1 + inv_beta |phi|^2)
//   mass mode 3    kappa_eff = kappa / (1 + kappa_gamma |phi|^2), which adds
//                  -mu kappa_gamma kappa P^4 / D^2 phi_a,  D = 1 + kappa_gamma |phi|^2 + kappa P^2
//   Cosserat strain  alpha |C|^2,  C = curl(phi)/2 - theta
//   hardening        (beta/2) |theta|^2 |curl phi|^2
//   chiral helicity  kappa_h P^2 phi . curl(phi)
// with P = phi_0 phi_1 phi_2.  Varying the strain and hardening energies gives
// -alpha curl(C) and -2 curl(B), B = (beta/2)|theta|^2 curl(phi), on phi: the
// curl of a field that itself holds a curl, a stencil two sites wide.
//
// Structure.  A step is one or two ring launches: when alpha or beta is set,
// an auxiliary launch stages phi and theta and writes C and B at every site;
// the step launch then stages phi, theta (and C, B), evaluates every force
// term at the site and advances the state with the fused leapfrog of the
// other steppers.  Buffers: positions X[0..1] and momenta W, S of 6 arrays
// (phi_0..2, theta_0..2), and 6 auxiliary arrays (C_0..2, B_0..2).
#pragma once
#include "ring.cuh"

namespace scp {

struct R6Consts {
    int N;
    long long N3;
    double L, dx, dV, idx1, idx2, hdt, dt;
    double mu, kappa, m2, mtheta2, eta;
    double kh, alpha, beta, kg, ia, ib;
    int mode;
    double damp_width, damp_rate;
};

// curl_a of the 3-vector held in ring fields f0..f0+2, central differences
template <class V>
__device__ __forceinline__ double ring_curl(const V &v, int f0, int a, double idx1) {
    // curl_a = d_{a+1} F_{a+2} - d_{a+2} F_{a+1}
    const int b = (a + 1) % 3, c = (a + 2) % 3;
    auto d = [&](int dir, int f) {
        return v.at(f0 + f, dir == 0, dir == 1, dir == 2) - v.at(f0 + f, -(dir == 0), -(dir == 1), -(dir == 2));
    };
    return (d(b, c) - d(c, b)) * idx1;
}

// phi_0 phi_1 phi_2 at a ring offset
template <class V>
__device__ __forceinline__ double ring_P(const V &v, int di, int dj, int dk) {
    return v.at(0, di, dj, dk) * v.at(1, di, dj, dk) * v.at(2, di, dj, dk);
}

// Auxiliary fields C = curl(phi)/2 - theta and B = (beta/2)|theta|^2 curl(phi).
struct R6Aux {
    static constexpr int NR = 6;
    static constexpr int MIN_CTAS = 2;
    struct Args {
        RingSrc<NR> src;
        int N;
        R6Consts c;
        double *aux;          // 6 arrays
    };
    struct Carry {};
    __device__ static void prefetch(const Args &, long long) {}
    template <class V>
    __device__ static void site(const Args &A, const V &v, int, int, int, long long idx, Carry &, bool) {
        const R6Consts &c = A.c;
        const long long N3 = c.N3;
        double cp[3];
#pragma unroll
        for (int a = 0; a < 3; a++) cp[a] = ring_curl(v, 0, a, c.idx1);
        const double t0 = v(3), t1 = v(4), t2 = v(5);
        if (c.alpha != 0.0) {
            A.aux[0 * N3 + idx] = cp[0] * 0.5 - t0;
            A.aux[1 * N3 + idx] = cp[1] * 0.5 - t1;
            A.aux[2 * N3 + idx] = cp[2] * 0.5 - t2;
        }
        if (c.beta != 0.0) {
            const double w = 0.5 * c.beta * (t0 * t0 + t1 * t1 + t2 * t2);
#pragma unroll
            for (int a = 0; a < 3; a++) A.aux[(3 + a) * N3 + idx] = w * cp[a];
        }
    }
};

template <bool AUX>
struct R6Step {
    static constexpr int NR = AUX ? 12 : 6;
    static constexpr int MIN_CTAS = 1;
    struct Args {
        RingSrc<NR> src;      // phi, theta, [C, B]
        int N;
        R6Consts c;
        const double *win;
        double *wout, *xout, *sout;
        int *flag;
        int first, sync, damp;
    };
    struct Carry {};
    __device__ static void prefetch(const Args &A, long long idx) {
#pragma unroll
        for (int f = 0; f < 6; f++) prefetch_l2(A.win + f * A.c.N3 + idx);
    }

    template <class V>
    __device__ static void site(const Args &A, const V &v, int i, int j, int k, long long idx, Carry &, bool) {
        const R6Consts &c = A.c;
        const long long N3 = c.N3;
        // momenta first: their latency passes under the stencil
        double wv[6];
#pragma unroll
        for (int f = 0; f < 6; f++) wv[f] = A.win[f * N3 + idx];
        const double p[3] = {v(0), v(1), v(2)}, t[3] = {v(3), v(4), v(5)};
        const double sig = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        const double m2e = (c.mode == 1) ? c.ia / (1.0 + c.ib * sig) : c.m2;
        const double ke = (c.mode == 3) ? c.kappa / (1.0 + c.kg * sig) : c.kappa;
        const double P = p[0] * p[1] * p[2], P2 = P * P;
        const double q = 1.0 + ke * P2;
        const double dVdP = c.mu * P / (q * q);
        double extra = 0.0;   // mode 3's additional -extra * phi_a
        if (c.mode == 3 && c.kg > 0) {
            const double D = 1.0 + c.kg * sig + c.kappa * P2;
            extra = c.mu * c.kg * c.kappa * P2 * P2 / (D * D);
        }
        double cp[3], ct[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            cp[a] = ring_curl(v, 0, a, c.idx1);
            ct[a] = ring_curl(v, 3, a, c.idx1);
        }
        const double hel = p[0] * cp[0] + p[1] * cp[1] + p[2] * cp[2];
        const double cp2 = cp[0] * cp[0] + cp[1] * cp[1] + cp[2] * cp[2];
        double gP2[3] = {0.0, 0.0, 0.0};   // gradient of P^2
        if (c.kh != 0.0) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const double Pp = ring_P(v, d == 0, d == 1, d == 2), Pm = ring_P(v, -(d == 0), -(d == 1), -(d == 2));
                gP2[d] = (Pp * Pp - Pm * Pm) * c.idx1;
            }
        }
        double acc[6];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const int b = (a + 1) % 3, e = (a + 2) % 3;
            const double lap = (v.at(a, 1, 0, 0) + v.at(a, -1, 0, 0) + v.at(a, 0, 1, 0) + v.at(a, 0, -1, 0) +
                                v.at(a, 0, 0, 1) + v.at(a, 0, 0, -1) - 6.0 * p[a]) * c.idx2;
            const double dPa = p[b] * p[e];   // dP / dphi_a
            double chiral = 0.0;
            if (c.kh != 0.0) {
                // kappa_h [2 P dP/dphi_a (phi.curl phi) + 2 P^2 curl_a phi + (grad P^2 x phi)_a]
                const double cross = gP2[b] * p[e] - gP2[e] * p[b];
                chiral = c.kh * (2.0 * P * dPa * hel + 2.0 * P2 * cp[a] + cross);
            }
            double f = lap - m2e * p[a] - dVdP * dPa - extra * p[a] + c.eta * ct[a] + chiral;
            if (AUX) {
                const double strain = -c.alpha * ring_curl(v, 6, a, c.idx1);
                const double hard = -2.0 * ring_curl(v, 9, a, c.idx1);
                f = f + strain + hard;
            }
            acc[a] = f;
            const double lapt = (v.at(3 + a, 1, 0, 0) + v.at(3 + a, -1, 0, 0) + v.at(3 + a, 0, 1, 0) +
                                 v.at(3 + a, 0, -1, 0) + v.at(3 + a, 0, 0, 1) + v.at(3 + a, 0, 0, -1) - 6.0 * t[a]) *
                                c.idx2;
            const double strain_t = (AUX && c.alpha != 0.0) ? 2.0 * c.alpha * v(6 + a) : 0.0;
            acc[3 + a] = lapt - c.mtheta2 * t[a] + c.eta * cp[a] + strain_t + -c.beta * cp2 * t[a];
        }
        const Leap leap{c.hdt, c.dt, A.first != 0};
        const double dmp = (A.damp && !A.first) ? sponge_at(i, j, k, c.L, c.dx, c.damp_width, c.damp_rate) : 1.0;
        bool bad = false;
#pragma unroll
        for (int f = 0; f < 6; f++) {
            double vv, wn;
            leap(wv[f], acc[f], dmp, &vv, &wn);
            const double x = (f < 3 ? p[f] : t[f - 3]) + c.dt * wn;
            st_cs(A.xout + f * N3 + idx, x);
            A.wout[f * N3 + idx] = wn;
            if (A.sync) {
                st_cs(A.sout + f * N3 + idx, vv);
                bad |= !isfinite(x) || !isfinite(vv);
            }
        }
        if (A.sync && bad) atomicOr(A.flag, 1);
    }
};

}  // namespace scp
