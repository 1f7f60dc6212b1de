// higgs_u1.cuh -- the gauged stepper with the Higgs condensate and/or the
// second compact U(1) (the reference's v71 extensions of the gauged force,
// sfa/sim/scp_sim.c:1053-1263; its energy :1970-1975; the second Gauss
// projection :2400-2458), as one fused ring kernel per time step.
//
// Physics.  The Higgs field H is a real scalar with
//     V_H = (lambda/4)(H^2 - v^2)^2 + (kappa_H/2) s H^2,   s = prod_a |Phi_a|^2,
// so it pushes the matter with -kappa_H H^2 Phi_a prod_{b!=a} |Phi_b|^2 and
// feels lap H - lambda H (H^2 - v^2) - kappa_H s H.  The second gauge has its
// own links th2, field E2, coupling g2, and per-component charges q_a: the
// matter component a is transported by the phase th_d + q_a th2_d, the E2
// kick is its plaquette term plus g2 sum_a q_a Im[f_a^* T+_a] / dx, and the
// E kick keeps the first gauge's plaquette term and current (whose cross term
// pairs the Theta and Phi components through the first gauge's link alone).
// The sponge damps the matter momenta and E, not E2 or dH/dt.
//
// Layout.  Position buffers (two, alternating) and momentum buffers hold, as
// N^3 arrays: the 12 matter fields and th (the 15-field order of the fused
// step, so diagnostics and snapshots read them the same way), then th2 (3)
// with the second gauge, then H with the Higgs field; the momenta follow the
// same order (matter, E, [E2], [dH/dt]).  One launch per step reads every
// position of the resident planes through the ring, so each word moves once
// per step.
#pragma once
#include "multiplet.cuh"
#include "ring.cuh"

namespace scp {

struct HuConsts {
    int N;
    long long N3;
    double L, dx, dV, idx1, idx2, inva, hdt, dt;
    double mu, kappa, m2, mtheta2, eta;
    double g, stp, gad;               // first gauge: coupling, 1/(g dx^3), -g dx dt
    double g2, stp2, gad2, q[3];      // second gauge
    double hv, hlam, hkap;            // Higgs
    double damp_width, damp_rate;
};

template <bool HIGGS, bool G2>
struct HiggsU1 {
    static constexpr int TH = 12;                        // first gauge links
    static constexpr int TH2 = 15;                       // second gauge links
    static constexpr int HF = G2 ? 18 : 15;              // the Higgs field
    static constexpr int NR = 15 + (G2 ? 3 : 0) + (HIGGS ? 1 : 0);
    static constexpr int MIN_CTAS = 1;

    struct Args {
        RingSrc<NR> src;      // positions x_{n+1}
        int N;
        HuConsts c;
        const double *win;    // momenta w_n (v_0 on the first launch), NR arrays
        double *wout;         // w_{n+1} (may alias win)
        double *xout;         // x_{n+2}
        double *sout;         // v_{n+1} (synchronous launches)
        int *flag;
        int first, sync, damp;
    };

    struct Carry {
        double cm[G2 ? 3 : 1], sm[G2 ? 3 : 1];   // link phase along i at x - i (per component with G2)
        double pm[2], pm2[2];                    // plaquette sines (0,1), (2,0) at x - i, both gauges
    };

    __device__ static void prefetch(const Args &A, long long idx) {
#pragma unroll
        for (int f = 0; f < NR; f++) prefetch_l2(A.win + f * A.c.N3 + idx);
    }

    template <class V>
    __device__ static void site(const Args &A, const V &v, int i, int j, int k, long long idx, Carry &cy,
                                bool first_plane) {
        const HuConsts &c = A.c;
        const long long N3 = c.N3;
        // the matter momenta are loaded first, so their latency passes under
        // the stencil instead of stalling the kicks
        double wv[NR];
#pragma unroll
        for (int f = 0; f < NR; f++) wv[f] = A.win[f * N3 + idx];
        double own[12];
#pragma unroll
        for (int f = 0; f < 12; f++) own[f] = v(f);
        constexpr int NC = G2 ? 3 : 1;
        if (first_plane) {   // the values carried from plane i-1, computed from the ring once
#pragma unroll
            for (int a = 0; a < NC; a++) {
                const double ph = G2 ? v.at(TH, -1, 0, 0) + c.q[a] * v.at(TH2, -1, 0, 0) : v.at(TH, -1, 0, 0);
                sincos_any(ph, &cy.sm[a], &cy.cm[a]);
            }
            cy.pm[0] = plaquette_sin(v, TH, 0, -1, 0, 0);
            cy.pm[1] = plaquette_sin(v, TH, 2, -1, 0, 0);
            if (G2) {
                cy.pm2[0] = plaquette_sin(v, TH2, 0, -1, 0, 0);
                cy.pm2[1] = plaquette_sin(v, TH2, 2, -1, 0, 0);
            }
        }
        // link phases of direction d: forward at x, backward at x - d; the
        // first gauge's own phase at x for the cross term
        auto links = [&](int d, double cP[3], double sP[3], double cM[3], double sM[3], double &cW, double &sW) {
            const double t1 = v(TH + d);
            sincos_bounded(t1, &sW, &cW);
            if (G2) {
                const double t2 = v(TH2 + d);
                const double t1m = nb(v, TH + d, d, -1), t2m = nb(v, TH2 + d, d, -1);
                // components of equal charge share their phase (the default
                // charges 1, 1, -2): the same angle, so the same cos / sin
                const bool same10 = c.q[1] == c.q[0], same20 = c.q[2] == c.q[0], same21 = c.q[2] == c.q[1];
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const int src = (a == 1 && same10) ? 0 : (a == 2 && same20) ? 0 : (a == 2 && same21) ? 1 : a;
                    if (src == a) {
                        sincos_any(t1 + c.q[a] * t2, &sP[a], &cP[a]);
                        if (d != 0) sincos_any(t1m + c.q[a] * t2m, &sM[a], &cM[a]);
                    } else if (src == 0) {
                        sP[a] = sP[0]; cP[a] = cP[0];
                        if (d != 0) { sM[a] = sM[0]; cM[a] = cM[0]; }
                    } else {
                        sP[a] = sP[1]; cP[a] = cP[1];
                        if (d != 0) { sM[a] = sM[1]; cM[a] = cM[1]; }
                    }
                    if (d == 0) {
                        cM[a] = cy.cm[a]; sM[a] = cy.sm[a];
                        cy.cm[a] = cP[a]; cy.sm[a] = sP[a];
                    }
                }
            } else {
                double cm, sm;
                if (d == 0) { cm = cy.cm[0]; sm = cy.sm[0]; cy.cm[0] = cW; cy.sm[0] = sW; }
                else sincos_bounded(nb(v, TH + d, d, -1), &sm, &cm);
#pragma unroll
                for (int a = 0; a < 3; a++) { cP[a] = cW; sP[a] = sW; cM[a] = cm; sM[a] = sm; }
            }
        };
        MultipletOut o;
        covariant_multiplet<G2>(v, 0, own, links, c.q, c.idx1, c.inva, c.eta, o);

        // potential: s_a = |Phi_a|^2, V'(s) = (mu/2)/(1 + kappa s)^2 with s = prod s_a
        double sa[3];
#pragma unroll
        for (int a = 0; a < 3; a++) sa[a] = own[MU + a] * own[MU + a] + own[MV + a] * own[MV + a];
        const double s = sa[0] * sa[1] * sa[2];
        const double den = 1.0 + c.kappa * s;
        const double Vp = 0.5 * c.mu / (den * den);
        const double h = HIGGS ? v(HF) : 0.0;
        const double hh = h * h;
        double acc[12];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const double others = sa[(a + 1) % 3] * sa[(a + 2) % 3];
            const double u = own[MU + a], w = own[MV + a], tu = own[MTU + a], tw = own[MTV + a];
            double au = (o.lsum[MU + a] - 6.0 * u) * c.idx2 - c.m2 * u - 2.0 * Vp * u * others + c.eta * o.curlT[a];
            double aw = (o.lsum[MV + a] - 6.0 * w) * c.idx2 - c.m2 * w - 2.0 * Vp * w * others + c.eta * o.curlT[3 + a];
            if (HIGGS) {
                au = au - c.hkap * hh * u * others;
                aw = aw - c.hkap * hh * w * others;
            }
            acc[MU + a] = au;
            acc[MV + a] = aw;
            acc[MTU + a] = (o.lsum[MTU + a] - 6.0 * tu) * c.idx2 - c.mtheta2 * tu + c.eta * o.curlP[a];
            acc[MTV + a] = (o.lsum[MTV + a] - 6.0 * tw) * c.idx2 - c.mtheta2 * tw + c.eta * o.curlP[3 + a];
        }
        double accH = 0.0;
        if (HIGGS) {
            const double lapH = (v.at(HF, 1, 0, 0) + v.at(HF, -1, 0, 0) + v.at(HF, 0, 1, 0) + v.at(HF, 0, -1, 0) +
                                 v.at(HF, 0, 0, 1) + v.at(HF, 0, 0, -1) - 6.0 * h) * c.idx2;
            accH = lapH - c.hlam * h * (h * h - c.hv * c.hv) - c.hkap * s * h;
        }
        // field kicks: plaquette terms plus currents
        double st[3], pat[2], K[3];
        staples(v, TH, cy.pm, st, pat);
        cy.pm[0] = pat[0]; cy.pm[1] = pat[1];
#pragma unroll
        for (int d = 0; d < 3; d++) K[d] = c.stp * st[d] + c.g * o.jlat[d];
        double K2[3] = {0.0, 0.0, 0.0};
        if (G2) {
            double st2[3];
            staples(v, TH2, cy.pm2, st2, pat);
            cy.pm2[0] = pat[0]; cy.pm2[1] = pat[1];
#pragma unroll
            for (int d = 0; d < 3; d++) K2[d] = c.stp2 * st2[d] + c.g2 * c.inva * o.jw[d];
        }

        // leapfrog (fused kick / sponge / kick / drift, see ring.cuh)
        const Leap leap{c.hdt, c.dt, A.first != 0};
        const double dmp = (A.damp && !A.first) ? sponge_at(i, j, k, c.L, c.dx, c.damp_width, c.damp_rate) : 1.0;
        bool bad = false;
        auto put = [&](int f, double x, double vv, double wn) {
            st_cs(A.xout + f * N3 + idx, x);
            A.wout[f * N3 + idx] = wn;
            if (A.sync) {
                st_cs(A.sout + f * N3 + idx, vv);
                bad |= !isfinite(x) || !isfinite(vv);
            }
        };
#pragma unroll
        for (int f = 0; f < 12; f++) {
            double vv, wn;
            leap(wv[f], acc[f], dmp, &vv, &wn);
            put(f, own[f] + c.dt * wn, vv, wn);
        }
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double E, Eh;
            leap(wv[TH + d], K[d], dmp, &E, &Eh);
            put(TH + d, wrap_angle(v(TH + d) + c.gad * Eh), E, Eh);
        }
        if (G2) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                double E2, E2h;
                leap(wv[TH2 + d], K2[d], 1.0, &E2, &E2h);
                put(TH2 + d, wrap_angle(v(TH2 + d) + c.gad2 * E2h), E2, E2h);
            }
        }
        if (HIGGS) {
            double hd, hdh;
            leap(wv[HF], accH, 1.0, &hd, &hdh);
            put(HF, h + c.dt * hdh, hd, hdh);
        }
        if (A.sync && bad) atomicOr(A.flag, 1);
    }
};

}  // namespace scp
